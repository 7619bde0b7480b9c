"""Build recipe of the native library ``libreno_b200.so`` (sm_100a only).

Every ``csrc/*.cu`` file is compiled by nvcc for ``-gencode
arch=compute_100a,code=sm_100a`` and linked into one shared library that sits
next to this file, so it travels with the source tree.  Run
``python -m renormalizer_b200.build`` (or call :func:`build_library`).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR / "csrc"
LIB_PATH = PKG_DIR / "libreno_b200.so"
BUILD_DIR = PKG_DIR / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I" + str(PKG_DIR.parent / "include")]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the B200 sweep engine needs the CUDA toolkit to build")
    return cand


def _sources():
    return sorted(CSRC.glob("*.cu"))


def _needs_rebuild() -> bool:
    if not LIB_PATH.exists():
        return True
    t = LIB_PATH.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list((PKG_DIR.parent / "include").glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build_library(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compile csrc/*.cu for sm_100a into libreno_b200.so (incremental)."""
    if not force and not _needs_rebuild():
        return LIB_PATH
    nvcc = _nvcc()
    BUILD_DIR.mkdir(exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []

    def compile_one(src: Path) -> Path:
        obj = BUILD_DIR / (src.stem + ".o")
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}")
        if verbose or ptxas_verbose:
            sys.stderr.write(r.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, _sources()))
    tmp = LIB_PATH.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stderr}")
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_library(force=force, verbose=True, ptxas_verbose="--ptxas" in sys.argv))
