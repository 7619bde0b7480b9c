"""ctypes binding of libreno_b200.so (include/reno_b200.h).

The library is the only compute path: if it is missing, or no CUDA device is
present, every entry point raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path
from typing import Optional

import torch

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libreno_b200.so"

RENO_OK, RENO_ERR_INVALID, RENO_ERR_OOM, RENO_ERR_CUDA, RENO_ERR_WORKSPACE, RENO_ERR_NONFINITE, \
    RENO_ERR_UNSUPPORTED = range(7)
RENO_F64, RENO_C128 = 0, 1
PREC = {"fp64": 0, "bf16x3": 1, "tf32x3": 2}

_c_int, _c_i64, _c_sz, _vp, _dp = ctypes.c_int, ctypes.c_int64, ctypes.c_size_t, ctypes.c_void_p, \
    ctypes.POINTER(ctypes.c_double)


class HeffDesc(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in
                ("nsite", "ml", "mr", "wl", "wm", "wr", "d1", "d2", "psi_dtype", "env_dtype", "mpo_dtype", "prec")]


class QrBlock(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int32), ("k", ctypes.c_int32), ("dtype", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("a", _vp), ("q", _vp), ("r", _vp)]


QR_MAX_BLOCKS = 16


class TruncDesc(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_int32), ("cols", ctypes.c_int32), ("qn_size", ctypes.c_int32),
                ("dtype", ctypes.c_int32), ("keep_left", ctypes.c_int32), ("mode", ctypes.c_int32),
                ("m_max", ctypes.c_int32), ("nsectors", ctypes.c_int32), ("threshold", ctypes.c_double),
                ("qn_rows", _vp), ("qn_cols", _vp), ("qntot", _vp), ("sectors", _vp)]


class HeevProblem(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("kt", ctypes.c_int32), ("a", _vp), ("d", _vp), ("e", _vp), ("tau", _vp),
                ("w", _vp), ("z", _vp), ("k", _vp)]


HEEV_MAX_BATCH = 32


class VecItem(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("dtype", ctypes.c_int32), ("j", ctypes.c_int32), ("x", _vp), ("y", _vp),
                ("out", _vp), ("scalars", _vp), ("s", _vp), ("ldv", ctypes.c_int64)]


VEC_GROUP_MAX = 128
VOP_NORM, VOP_ALPHA, VOP_ORTH, VOP_SCALE_INV, VOP_LINCOMB, VOP_ALLCLOSE = range(6)


class EnvDesc(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in
                ("side", "d", "w_in", "w_out", "mk_in", "mk_out", "mb_in", "mb_out", "env_dtype", "ket_dtype",
                 "bra_dtype", "mpo_dtype", "prec")]


# name -> (restype, argtypes)
_SIGS = {
    "reno_version": (_c_int, []),
    "reno_ctx_create": (_c_int, [_c_int, ctypes.POINTER(_vp)]),
    "reno_ctx_destroy": (_c_int, [_vp]),
    "reno_ctx_set_stream": (_c_int, [_vp, _vp]),
    "reno_last_error": (ctypes.c_char_p, [_vp]),
    "reno_ctx_synchronize": (_c_int, [_vp]),
    "reno_launch_count": (_c_int, [ctypes.POINTER(ctypes.c_longlong)]),
    "reno_heff_workspace_bytes": (_c_int, [ctypes.POINTER(HeffDesc), ctypes.POINTER(_c_sz)]),
    "reno_heff_apply": (_c_int, [_vp, ctypes.POINTER(HeffDesc), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_sz]),
    "reno_gemm_workspace_bytes": (_c_int, [_c_int, _c_int, _c_int, _c_int, _c_int, _c_int, ctypes.POINTER(_c_sz)]),
    "reno_gemm": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp, _c_int, _c_i64, _c_i64, _c_int, _vp, _c_int, _c_i64,
                           _c_i64, _c_int, _vp, _c_i64, _c_int, _vp, _c_sz]),
    "reno_device_error": (_c_int, [_vp, ctypes.POINTER(ctypes.c_int32)]),
    "reno_lanczos_workspace_bytes": (_c_int, [ctypes.POINTER(HeffDesc), _c_int, ctypes.POINTER(_c_sz)]),
    "reno_lanczos_expm": (_c_int, [_vp, ctypes.POINTER(HeffDesc), _vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_double,
                                   _vp, _c_int, ctypes.POINTER(ctypes.c_int32), _vp, _c_sz]),
    "reno_qn_svd_truncate_workspace_bytes": (_c_int, [ctypes.POINTER(TruncDesc), ctypes.POINTER(_c_sz)]),
    "reno_qn_svd_truncate": (_c_int, [_vp, ctypes.POINTER(TruncDesc), _vp, _vp, _vp, _c_int, _vp, _vp,
                                      ctypes.POINTER(ctypes.c_int32), _vp, _c_sz]),
    "reno_set_wait_limit_ns": (_c_int, [ctypes.c_uint64]),
    "reno_set_split_accumulation_chunk": (_c_int, [ctypes.c_int32]),
    "reno_test_skip_arrival": (_c_int, [ctypes.c_int32, ctypes.c_int32]),
    "reno_heff_apply_noalloc": (_c_int, [_vp, ctypes.POINTER(HeffDesc), _vp, _vp, _vp, _vp, _vp, _vp]),
    "reno_heff_diag": (_c_int, [_vp, ctypes.POINTER(HeffDesc), _vp, _vp, _vp, _vp, _vp]),
    "reno_heff_grouped_workspace_bytes": (_c_int, [_c_int, ctypes.POINTER(HeffDesc), ctypes.POINTER(_c_sz)]),
    "reno_heff_apply_grouped": (_c_int, [_vp, _c_int, ctypes.POINTER(HeffDesc), ctypes.POINTER(_vp),
                                         ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                         ctypes.POINTER(_vp), ctypes.POINTER(_vp), _vp, _c_sz]),
    "reno_heev_workspace_bytes": (_c_int, [_c_int, _c_int, ctypes.POINTER(_c_sz)]),
    "reno_heev_top": (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _c_sz]),
    "reno_heev_backtransform": (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _vp, _vp, _c_sz]),
    "reno_heev_status_offset": (_c_int, [ctypes.POINTER(_c_sz)]),
    "reno_heev_batched_workspace_bytes": (_c_int, [_c_int, ctypes.POINTER(HeevProblem), ctypes.POINTER(_c_sz)]),
    "reno_heev_top_batched": (_c_int, [_vp, _c_int, ctypes.POINTER(HeevProblem), _vp, _vp, _c_sz]),
    "reno_heev_backtransform_batched": (_c_int, [_vp, _c_int, ctypes.POINTER(HeevProblem), _vp, _c_sz]),
    "reno_qr_workspace_bytes": (_c_int, [_c_int, ctypes.POINTER(QrBlock), ctypes.POINTER(_c_sz)]),
    "reno_qr_blocks": (_c_int, [_vp, _c_int, ctypes.POINTER(QrBlock), _vp, _c_sz]),
    "reno_heff_backward_workspace_bytes": (_c_int, [ctypes.POINTER(HeffDesc), ctypes.POINTER(_c_sz)]),
    "reno_heff_backward": (_c_int, [_vp, ctypes.POINTER(HeffDesc), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                    _vp, _vp, _c_sz]),
    "reno_env_workspace_bytes": (_c_int, [ctypes.POINTER(EnvDesc), ctypes.POINTER(_c_sz)]),
    "reno_env_update": (_c_int, [_vp, ctypes.POINTER(EnvDesc), _vp, _vp, _vp, _vp, _vp, _vp, _c_sz]),
    "reno_vec_workspace_bytes": (_c_int, [_c_i64, ctypes.POINTER(_c_sz)]),
    "reno_vec_dotc": (_c_int, [_vp, _c_i64, _c_int, _vp, _vp, _vp, _vp, _c_sz]),
    "reno_vec_norm": (_c_int, [_vp, _c_i64, _c_int, _vp, _vp, _vp, _c_sz]),
    "reno_krylov_orth": (_c_int, [_vp, _c_i64, _c_int, _vp, _vp, _vp, _vp, _c_int, _vp, _c_sz]),
    "reno_krylov_alpha": (_c_int, [_vp, _c_i64, _c_int, _vp, _vp, _vp, _c_int, _vp, _c_sz]),
    "reno_vec_scale_inv": (_c_int, [_vp, _c_i64, _c_int, _vp, _vp, _vp]),
    "reno_vec_lincomb": (_c_int, [_vp, _c_i64, _c_int, _c_int, _vp, _c_i64, _vp, _vp]),
    "reno_vec_allclose": (_c_int, [_vp, _c_i64, _c_int, _vp, _vp, ctypes.c_double, ctypes.c_double, _vp, _vp,
                                   _c_sz]),
    "reno_vec_axpy": (_c_int, [_vp, _c_i64, _c_int, _vp, _vp, _vp, ctypes.c_double]),
    "reno_vec_precond": (_c_int, [_vp, _c_i64, _c_int, _vp, _vp, _vp, ctypes.c_double, _vp]),
    "reno_vec_grouped_workspace_bytes": (_c_int, [_c_int, ctypes.POINTER(_c_sz)]),
    "reno_vec_grouped": (_c_int, [_vp, _c_int, _c_int, ctypes.POINTER(VecItem), ctypes.c_double, ctypes.c_double,
                                  _vp, _c_sz]),
    "reno_qn_gather": (_c_int, [_vp, _c_int, _vp, _c_i64, _vp, _c_i64, _vp, _c_i64, _vp]),
    "reno_qn_scatter": (_c_int, [_vp, _c_int, _vp, _c_i64, _c_i64, _vp, _c_i64, _vp, _vp, _c_i64, _vp, _vp, _c_i64,
                                 _c_i64]),
}

_lib = None
_lib_lock = threading.Lock()


def launch_count() -> int:
    """Kernels launched by libreno_b200 in this process so far."""
    n = ctypes.c_longlong(0)
    load_library().reno_launch_count(ctypes.byref(n))
    return int(n.value)


def exported_symbols():
    return list(_SIGS)


def load_library(path: Optional[Path] = None):
    """Load libreno_b200.so and declare every entry point (no GPU needed)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            p = Path(path) if path else LIB_PATH
            if not p.exists():
                raise RuntimeError(f"{p} is missing: build it with `python -m renormalizer_b200.build` "
                                   "(the sweep engine has no CPU fallback)")
            lib = ctypes.CDLL(str(p))
            for name, (res, args) in _SIGS.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def _raise(status: int, msg: str):
    if status in (RENO_ERR_OOM, RENO_ERR_WORKSPACE):
        raise MemoryError(msg)
    if status == RENO_ERR_INVALID:
        raise AssertionError(msg)
    if status == RENO_ERR_NONFINITE:
        raise FloatingPointError(msg)
    if status == RENO_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(msg)


def dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.complex128:
        return RENO_C128
    if t.dtype == torch.float64:
        return RENO_F64
    raise TypeError(f"the sweep engine works on float64/complex128 tensors, got {t.dtype}")


def ptr(t: Optional[torch.Tensor]):
    if t is None:
        return None
    assert t.is_cuda, "sweep-engine tensors live on the GPU"
    assert t.is_contiguous(), "sweep-engine tensors are C-contiguous"
    # torch's lazy conjugate / negative views keep unconjugated memory behind a flag
    assert not (t.is_conj() or t.is_neg()), "resolve_conj()/resolve_neg() before passing a view to the engine"
    return ctypes.c_void_p(t.data_ptr())


def h2d(arr, device, dtype=None) -> torch.Tensor:
    """Host array -> device tensor through pinned memory without a stream sync
    (torch's caching host allocator keeps the staging block alive until the
    copy has run)."""
    import numpy as np
    a = np.ascontiguousarray(arr if dtype is None else np.asarray(arr, dtype=dtype))
    src = torch.from_numpy(a)
    pinned = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
    pinned.copy_(src)
    return pinned.to(device, non_blocking=True)


def raw_view(t: torch.Tensor) -> torch.Tensor:
    """A tensor whose memory holds the values it denotes (no lazy conj/neg bit)."""
    if t.is_conj():
        t = t.resolve_conj()
    if t.is_neg():
        t = t.resolve_neg()
    return t


class Engine:
    """One C-ABI context per CUDA device plus a growable device workspace.

    The workspace is allocated outside the hot calls (torch's caching
    allocator) and handed to the kernels, which never allocate."""

    _engines = {}

    def __init__(self, device: int):
        if not torch.cuda.is_available():
            raise RuntimeError("renormalizer_b200 needs a CUDA device (B200, sm_100a); none is visible")
        self.lib = load_library()
        self.device = device
        ctx = _vp()
        with torch.cuda.device(device):
            st = self.lib.reno_ctx_create(device, ctypes.byref(ctx))
        if st != RENO_OK:
            raise RuntimeError(f"reno_ctx_create failed on device {device} (status {st})")
        self.ctx = ctx
        self._stream_handle = None
        self._ws = None
        self._vec_ws = None
        self._vec_gws = None
        self.scalars = torch.zeros(4096, dtype=torch.float64, device=f"cuda:{device}")
        self.launches = 0

    @classmethod
    def get(cls, device=None) -> "Engine":
        if device is None:
            device = torch.cuda.current_device()
        if isinstance(device, torch.device):
            device = device.index if device.index is not None else torch.cuda.current_device()
        eng = cls._engines.get(device)
        if eng is None:
            eng = cls(device)
            cls._engines[device] = eng
        eng.sync_stream()
        return eng

    def sync_stream(self):
        h = torch.cuda.current_stream(self.device).cuda_stream
        if h != self._stream_handle:
            self.lib.reno_ctx_set_stream(self.ctx, _vp(h))
            self._stream_handle = h

    def check(self, status: int, what: str):
        if status != RENO_OK:
            msg = self.lib.reno_last_error(self.ctx)
            _raise(status, f"{what}: {msg.decode() if msg else 'error'}")

    def workspace(self, nbytes: int) -> torch.Tensor:
        if self._ws is None or self._ws.numel() < nbytes:
            grow = max(int(nbytes), int(1.25 * (self._ws.numel() if self._ws is not None else 0)), 1 << 20)
            self._ws = None
            self._ws = torch.empty(grow, dtype=torch.uint8, device=f"cuda:{self.device}")
        return self._ws

    def vec_workspace(self) -> torch.Tensor:
        if self._vec_ws is None:
            n = _c_sz()
            self.check(self.lib.reno_vec_workspace_bytes(0, ctypes.byref(n)), "reno_vec_workspace_bytes")
            self._vec_ws = torch.empty(int(n.value), dtype=torch.uint8, device=f"cuda:{self.device}")
        return self._vec_ws

    # ------------------------------------------------------------ wrappers
    def heff_apply(self, desc: HeffDesc, L, W1, W2, R, psi, y):
        n = _c_sz()
        self.check(self.lib.reno_heff_workspace_bytes(ctypes.byref(desc), ctypes.byref(n)), "reno_heff_workspace_bytes")
        ws = self.workspace(int(n.value))
        self.check(self.lib.reno_heff_apply(self.ctx, ctypes.byref(desc), ptr(L), ptr(W1), ptr(W2), ptr(R), ptr(psi),
                                            ptr(y), ptr(ws), ws.numel()), "reno_heff_apply")
        self.launches += 1

    def heff_backward(self, desc: HeffDesc, L, W1, W2, R, psi, gy, gpsi, gL, gW1, gW2, gR):
        """reno_heff_backward: any output may be None (not computed)."""
        n = _c_sz()
        self.check(self.lib.reno_heff_backward_workspace_bytes(ctypes.byref(desc), ctypes.byref(n)),
                   "reno_heff_backward_workspace_bytes")
        ws = self.workspace(int(n.value))
        opt = lambda t: ptr(t) if t is not None else None
        self.check(self.lib.reno_heff_backward(self.ctx, ctypes.byref(desc), ptr(L), opt(W1), opt(W2), ptr(R), ptr(psi),
                                               ptr(gy), opt(gpsi), opt(gL), opt(gW1), opt(gW2), opt(gR), ptr(ws),
                                               ws.numel()), "reno_heff_backward")

    def heev_batched(self, probs, status, ws, stage):
        """reno_heev_top_batched (stage "top") or reno_heev_backtransform_batched
        (stage "back") on a list of HeevProblem; ws sized by heev_batched_bytes"""
        arr = (HeevProblem * len(probs))(*probs)
        if stage == "top":
            self.check(self.lib.reno_heev_top_batched(self.ctx, len(probs), arr, ptr(status), ptr(ws), ws.numel()),
                       "reno_heev_top_batched")
        else:
            self.check(self.lib.reno_heev_backtransform_batched(self.ctx, len(probs), arr, ptr(ws), ws.numel()),
                       "reno_heev_backtransform_batched")

    def heev_batched_bytes(self, probs) -> int:
        arr = (HeevProblem * len(probs))(*probs)
        n = _c_sz()
        self.check(self.lib.reno_heev_batched_workspace_bytes(len(probs), arr, ctypes.byref(n)),
                   "reno_heev_batched_workspace_bytes")
        return int(n.value)

    def qr_blocks(self, mats):
        """Economic Householder QR of every matrix of ``mats`` (2-D device
        tensors of one dtype; not modified): lists Q (m x min(m,k)) and R
        (min(m,k) x k) with LAPACK's signs (reno_qr_blocks)."""
        Qs, Rs = [], []
        for i0 in range(0, len(mats), QR_MAX_BLOCKS):
            part = mats[i0:i0 + QR_MAX_BLOCKS]
            blocks, keep = [], []
            for a in part:
                m, k = a.shape
                kq = min(m, k)
                work = a.contiguous().clone()
                q = torch.empty((m, kq), dtype=a.dtype, device=a.device)
                r = torch.empty((kq, k), dtype=a.dtype, device=a.device)
                keep += [work, q, r]
                blocks.append(QrBlock(m, k, dtype_code(a), 0, _vp(work.data_ptr()), _vp(q.data_ptr()),
                                      _vp(r.data_ptr())))
                Qs.append(q)
                Rs.append(r)
            arr = (QrBlock * len(blocks))(*blocks)
            n = _c_sz()
            self.check(self.lib.reno_qr_workspace_bytes(len(blocks), arr, ctypes.byref(n)), "reno_qr_workspace_bytes")
            ws = self.workspace(int(n.value))
            self.check(self.lib.reno_qr_blocks(self.ctx, len(blocks), arr, ptr(ws), ws.numel()), "reno_qr_blocks")
        return Qs, Rs

    def device_error(self) -> int:
        """first timed-out wait of the tensor-core kernels since the last call (0 = none)"""
        c = ctypes.c_int32(0)
        self.check(self.lib.reno_device_error(self.ctx, ctypes.byref(c)), "reno_device_error")
        return int(c.value)

    def heff_apply_grouped(self, descs, Ls, W1s, W2s, Rs, psis, ys):
        """reno_heff_apply_grouped (FP64): lists of equal length; W1s / W2s
        entries None below one / two active sites"""
        m = len(descs)
        arr = (HeffDesc * m)(*descs)
        n = _c_sz()
        self.check(self.lib.reno_heff_grouped_workspace_bytes(m, arr, ctypes.byref(n)),
                   "reno_heff_grouped_workspace_bytes")
        ws = self.workspace(int(n.value))
        pa = lambda ts: (_vp * m)(*[_vp(t.data_ptr()) if t is not None else None for t in ts])
        for t in list(Ls) + list(Rs) + list(psis) + list(ys) + [w for w in list(W1s) + list(W2s) if w is not None]:
            ptr(t)  # contiguity / lazy-view checks
        self.check(self.lib.reno_heff_apply_grouped(self.ctx, m, arr, pa(Ls), pa(W1s), pa(W2s), pa(Rs), pa(psis),
                                                    pa(ys), ptr(ws), ws.numel()), "reno_heff_apply_grouped")
        self.launches += 1

    def heev_top(self, A, d, e, tau, w, Z, ws):
        """reno_heev_top: tridiagonal reduction of A (overwritten), top eigenvalues
        w (ascending) and tridiagonal eigenvectors Z (n x kt); ws from heev_workspace"""
        n, kt = A.shape[0], w.numel()
        self.check(self.lib.reno_heev_top(self.ctx, n, kt, ptr(A), ptr(d), ptr(e), ptr(tau), ptr(w), ptr(Z), ptr(ws),
                                          ws.numel()), "reno_heev_top")
        self.launches += 1

    def heev_workspace(self, n: int, kt: int) -> torch.Tensor:
        b = _c_sz()
        self.check(self.lib.reno_heev_workspace_bytes(n, kt, ctypes.byref(b)), "reno_heev_workspace_bytes")
        return torch.empty(int(b.value), dtype=torch.uint8, device=f"cuda:{self.device}")

    def heev_status_offset(self) -> int:
        o = _c_sz()
        self.check(self.lib.reno_heev_status_offset(ctypes.byref(o)), "reno_heev_status_offset")
        return int(o.value)

    def heev_backtransform(self, A, tau, K, ws):
        """K <- Q K for the reflectors of the last heev_top on A (cleaned in place)"""
        self.check(self.lib.reno_heev_backtransform(self.ctx, A.shape[0], K.shape[1], ptr(A), ptr(tau), ptr(K),
                                                    ptr(ws), ws.numel()), "reno_heev_backtransform")
        self.launches += 1

    def heff_diag(self, desc: HeffDesc, L, W1, W2, R, out):
        self.check(self.lib.reno_heff_diag(self.ctx, ctypes.byref(desc), ptr(L), ptr(W1), ptr(W2), ptr(R), ptr(out)),
                   "reno_heff_diag")

    def matmul(self, A: torch.Tensor, B: torch.Tensor, conj_a=False, conj_b=False, prec="fp64") -> torch.Tensor:
        """C = op(A) @ op(B) for 2-D device tensors (any strides) on the engine's GEMM."""
        assert A.dim() == 2 and B.dim() == 2 and A.shape[1] == B.shape[0]
        # a lazy conj view is the raw memory of the conjugate: fold it into the kernel's conj flag
        if A.is_conj():
            A, conj_a = A.conj(), not conj_a
        if B.is_conj():
            B, conj_b = B.conj(), not conj_b
        A, B = raw_view(A), raw_view(B)
        cplx = A.is_complex() or B.is_complex()
        C = torch.empty((A.shape[0], B.shape[1]), dtype=torch.complex128 if cplx else torch.float64, device=A.device)
        code = PREC[prec]
        wsp, wsn = None, 0
        if code:
            n = _c_sz()
            self.check(self.lib.reno_gemm_workspace_bytes(A.shape[0], B.shape[1], A.shape[1], dtype_code(A),
                                                          dtype_code(B), code, ctypes.byref(n)), "reno_gemm_workspace")
            ws = self.workspace(int(n.value))
            wsp, wsn = ptr(ws), ws.numel()
        self.check(self.lib.reno_gemm(self.ctx, A.shape[0], B.shape[1], A.shape[1], _vp(A.data_ptr()), dtype_code(A),
                                      A.stride(0), A.stride(1), int(conj_a), _vp(B.data_ptr()), dtype_code(B),
                                      B.stride(0), B.stride(1), int(conj_b), _vp(C.data_ptr()), C.stride(0), code,
                                      wsp, wsn), "reno_gemm")
        self.launches += 1
        return C

    def env_update(self, desc: EnvDesc, E, W, ket, bra, out):
        n = _c_sz()
        self.check(self.lib.reno_env_workspace_bytes(ctypes.byref(desc), ctypes.byref(n)), "reno_env_workspace_bytes")
        ws = self.workspace(int(n.value))
        self.check(self.lib.reno_env_update(self.ctx, ctypes.byref(desc), ptr(E), ptr(W), ptr(ket), ptr(bra),
                                            ptr(out), ptr(ws), ws.numel()), "reno_env_update")
        self.launches += 1

    # vector kernels (krylov.py / davidson.py algebra); scalars live in device arrays
    def _vws(self):
        ws = self.vec_workspace()
        return ptr(ws), ws.numel()

    def vec_norm(self, x, out):
        w, n = self._vws()
        self.check(self.lib.reno_vec_norm(self.ctx, x.numel(), dtype_code(x), ptr(x), ptr(out), w, n), "reno_vec_norm")

    def vec_dotc(self, x, y, out):
        w, n = self._vws()
        self.check(self.lib.reno_vec_dotc(self.ctx, x.numel(), dtype_code(x), ptr(x), ptr(y), ptr(out), w, n),
                   "reno_vec_dotc")

    def krylov_alpha(self, w_vec, v, ab, j):
        w, n = self._vws()
        self.check(self.lib.reno_krylov_alpha(self.ctx, v.numel(), dtype_code(v), ptr(w_vec), ptr(v), ptr(ab), j, w,
                                              n), "reno_krylov_alpha")

    def krylov_orth(self, w_vec, v, vprev, ab, j):
        w, n = self._vws()
        self.check(self.lib.reno_krylov_orth(self.ctx, v.numel(), dtype_code(v), ptr(w_vec), ptr(v), ptr(vprev),
                                             ptr(ab), j, w, n), "reno_krylov_orth")

    def scale_inv(self, x, s, out):
        self.check(self.lib.reno_vec_scale_inv(self.ctx, x.numel(), dtype_code(x), ptr(x), ptr(s), ptr(out)),
                   "reno_vec_scale_inv")

    def lincomb(self, V, k, coef, out):
        n = V.shape[1]
        self.check(self.lib.reno_vec_lincomb(self.ctx, n, k, dtype_code(V), ptr(V), n, ptr(coef), ptr(out)),
                   "reno_vec_lincomb")

    def allclose(self, a, b, rtol, atol, flag):
        w, n = self._vws()
        self.check(self.lib.reno_vec_allclose(self.ctx, a.numel(), dtype_code(a), ptr(a), ptr(b), rtol, atol,
                                              ptr(flag), w, n), "reno_vec_allclose")

    def axpy(self, y, x, c, sign=1.0):
        self.check(self.lib.reno_vec_axpy(self.ctx, y.numel(), dtype_code(y), ptr(y), ptr(x), ptr(c), sign),
                   "reno_vec_axpy")

    def precond(self, r, hdiag, e, shift, out):
        self.check(self.lib.reno_vec_precond(self.ctx, r.numel(), dtype_code(r), ptr(r), ptr(hdiag), ptr(e), shift,
                                             ptr(out)), "reno_vec_precond")

    def vec_grouped(self, op, items, rtol=0.0, atol=0.0):
        """One vector operation on many problems (reno_vec_grouped), in chunks
        of VEC_GROUP_MAX.  items: tuples (n, dtype, j, x, y, out, scalars, s,
        ldv) of sizes and tensors (None where the operation has no operand)."""
        for c0 in range(0, len(items), VEC_GROUP_MAX):
            chunk = items[c0:c0 + VEC_GROUP_MAX]
            arr = (VecItem * len(chunk))()
            for k, (n, dt, j, x, y, out, sc, sv, ldv) in enumerate(chunk):
                arr[k] = VecItem(n, dt, j, ptr(x), ptr(y), ptr(out), ptr(sc), ptr(sv), ldv)
            nbytes = _c_sz()
            self.check(self.lib.reno_vec_grouped_workspace_bytes(len(chunk), ctypes.byref(nbytes)),
                       "reno_vec_grouped_workspace_bytes")
            if self._vec_gws is None or self._vec_gws.numel() < nbytes.value:
                self._vec_gws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=f"cuda:{self.device}")
            self.check(self.lib.reno_vec_grouped(self.ctx, op, len(chunk), arr, rtol, atol, ptr(self._vec_gws),
                                                 self._vec_gws.numel()), "reno_vec_grouped")

    # quantum-number block movers
    def qn_gather(self, mat, rows, cols, out):
        """out[i, j] = mat[rows[i], cols[j]] for a C-contiguous 2-D mat"""
        self.check(self.lib.reno_qn_gather(self.ctx, dtype_code(mat), ptr(mat), mat.shape[1], ptr(rows),
                                           rows.numel(), ptr(cols), cols.numel(), ptr(out)), "reno_qn_gather")

    def qn_scatter(self, src, rows, scols, dcols, sigma, dst, dst_rs, dst_cs):
        """dst[rows[i]*dst_rs + dcols[j]*dst_cs] = sigma_j * src[i, scols[j]] for a 2-D view src"""
        src = raw_view(src)
        if src.dtype != dst.dtype:
            src = src.to(dst.dtype)
        self.check(self.lib.reno_qn_scatter(self.ctx, dtype_code(dst), _vp(src.data_ptr()), src.stride(0),
                                            src.stride(1), ptr(rows), rows.numel(), ptr(scols), ptr(dcols),
                                            dcols.numel(), ptr(sigma) if sigma is not None else None, ptr(dst),
                                            dst_rs, dst_cs), "reno_qn_scatter")
