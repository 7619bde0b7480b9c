"""Model description consumed by the sweep engine: local bases, symbolic
operator products and the Holstein / spin-boson Hamiltonians.

Mirrors the reference's model layer as far as the sweep path consumes it:
  Quantity               renormalizer/utils/quantity.py:30-103
  BasisSHO               renormalizer/model/basis.py:110-340 (second-quantised x, p, x^2, p^2)
  BasisSimpleElectron    renormalizer/model/basis.py:882-930
  BasisHalfSpin          renormalizer/model/basis.py:932-997
  Op                     renormalizer/model/op.py (products of one-dof symbols)
  Model / HolsteinModel / SpinBosonModel   renormalizer/model/model.py:18-439
  Mol / Phonon           renormalizer/model/mol.py:13-60, phonon.py:22-154
  SpectralDensityFunction (Ohmic, Wang1 / trapz)  renormalizer/sbm/lib.py:38-136
The operator matrices are built analytically in the truncated basis exactly
as the reference does (x^2 and p^2 from ladder-operator sums, not x @ x).
"""
from __future__ import annotations

from collections import Counter
from typing import Dict, List, Sequence, Union

import numpy as np

# ---------------------------------------------------------------- units
_AU2EV = 27.211386245988
_AU2CM = 219474.6313632
_AU2K = 315775.02480407
_AU2FS = 0.02418884326585747
_RATIO = {"a.u.": 1.0, "au": 1.0, "eV": _AU2EV, "ev": _AU2EV, "meV": _AU2EV * 1e3, "mev": _AU2EV * 1e3,
          "cm^{-1}": _AU2CM, "cm-1": _AU2CM, "K": _AU2K, "k": _AU2K, "fs": _AU2FS}


class Quantity:
    def __init__(self, value, unit="a.u."):
        if unit not in _RATIO:
            raise ValueError(f"Unit not in {sorted(_RATIO)}, got {unit}.")
        self.value = float(value)
        self.unit = unit

    def as_au(self) -> float:
        return self.value / _RATIO[self.unit]

    def to_beta(self) -> float:
        """quantity.py:53-56: 1 / (k_B T) in atomic units for a temperature"""
        return np.inf if self.value == 0 else 1.0 / self.as_au()

    def __repr__(self):
        return f"Quantity({self.value}, {self.unit!r})"


def _au(v):
    return v.as_au() if isinstance(v, Quantity) else float(v)


# ---------------------------------------------------------------- bases
class BasisSet:
    is_electron = False
    is_phonon = False
    is_spin = False
    multi_dof = False

    def __init__(self, dof, nbas: int, sigmaqn: Sequence):
        self.dof = dof
        assert type(nbas) is int
        self.nbas = nbas
        self.sigmaqn = np.array([np.atleast_1d(np.asarray(q, dtype=int)) for q in sigmaqn])

    @property
    def dofs(self):
        return [self.dof]

    def op_mat(self, symbol: str) -> np.ndarray:
        raise NotImplementedError

    def __repr__(self):
        return f"{self.__class__.__name__}(dof: {self.dof}, nbas: {self.nbas})"


class BasisSHO(BasisSet):
    is_phonon = True

    def __init__(self, dof, omega, nbas, x0=0.0):
        self.omega = float(omega)
        self.x0 = float(x0)
        super().__init__(dof, nbas, [0] * nbas)

    def _b(self):
        return np.diag(np.sqrt(np.arange(1, self.nbas)), k=1)

    def _bd(self):
        return np.diag(np.sqrt(np.arange(1, self.nbas)), k=-1)

    def _bb(self):
        if self.nbas == 1:
            return np.zeros((1, 1))
        return np.diag(np.sqrt(np.arange(1, self.nbas - 1) * np.arange(2, self.nbas)), k=2)

    def _bdbd(self):
        if self.nbas == 1:
            return np.zeros((1, 1))
        return np.diag(np.sqrt(np.arange(1, self.nbas - 1) * np.arange(2, self.nbas)), k=-2)

    def op_mat(self, symbol: str) -> np.ndarray:
        n = self.nbas
        s = symbol.replace(r"b^\dagger + b", r"b^\dagger+b")
        if s == "I":
            return np.eye(n)
        if s == "b":
            return self._b()
        if s == r"b^\dagger":
            return self._bd()
        if s == "b b":
            return self._bb()
        if s == r"b^\dagger b^\dagger":
            return self._bdbd()
        if s == r"b^\dagger+b":
            return self._bd() + self._b()
        if s == r"b^\dagger-b":
            return self._bd() - self._b()
        if s in (r"b^\dagger b", "n"):
            return np.diag(np.arange(n, dtype=float))
        if s == r"b b^\dagger":
            return np.diag(np.arange(n, dtype=float) + 1)
        if s == "x":
            return np.sqrt(0.5 / self.omega) * (self._bd() + self._b()) + np.eye(n) * self.x0
        if s == "x^2":
            m = np.eye(n) * self.x0 ** 2
            m = m + 2 * self.x0 * np.sqrt(0.5 / self.omega) * (self._bd() + self._b())
            m = m + 0.5 / self.omega * (self._bdbd() + np.diag(np.arange(n, dtype=float))
                                        + np.diag(np.arange(n, dtype=float) + 1) + self._bb())
            return m
        if s == "p":
            return 1j * np.sqrt(self.omega / 2) * (self._bd() - self._b())
        if s == "p^2":
            return -self.omega / 2 * (self._bdbd() - np.diag(np.arange(n, dtype=float))
                                      - np.diag(np.arange(n, dtype=float) + 1) + self._bb())
        raise ValueError(f"op_symbol:{symbol} is not supported by BasisSHO in the sweep engine")


class BasisSimpleElectron(BasisSet):
    is_electron = True

    def __init__(self, dof, sigmaqn=None):
        super().__init__(dof, 2, [0, 1] if sigmaqn is None else sigmaqn)

    def op_mat(self, symbol: str) -> np.ndarray:
        m = np.zeros((2, 2))
        if symbol == r"a^\dagger":
            m[1, 0] = 1.0
        elif symbol == "a":
            m[0, 1] = 1.0
        elif symbol == r"a^\dagger a":
            m[1, 1] = 1.0
        elif symbol == "I":
            m = np.eye(2)
        else:
            raise ValueError(f"op_symbol:{symbol} is not supported")
        return m


class BasisHalfSpin(BasisSet):
    is_spin = True

    def __init__(self, dof, sigmaqn=None):
        super().__init__(dof, 2, [0, 0] if sigmaqn is None else sigmaqn)

    def op_mat(self, symbol: str) -> np.ndarray:
        parts = symbol.split(" ")
        if len(parts) > 1:
            m = np.eye(2)
            for p in parts:
                m = m @ self.op_mat(p)
            return m
        s = parts[0]
        if s == "I":
            return np.eye(2)
        if s in ("sigma_x", "X", "x"):
            return np.array([[0.0, 1.0], [1.0, 0.0]])
        if s in ("sigma_y", "Y", "y"):
            return np.array([[0.0, -1.0j], [1.0j, 0.0]])
        if s in ("isigma_y", "iY", "iy"):
            return np.array([[0.0, 1.0], [-1.0, 0.0]])
        if s in ("sigma_z", "Z", "z"):
            return np.diag([1.0, -1.0])
        if s in ("sigma_-", "-"):
            return np.array([[0.0, 0.0], [1.0, 0.0]])
        if s in ("sigma_+", "+"):
            return np.array([[0.0, 1.0], [0.0, 0.0]])
        raise ValueError(f"op_symbol:{symbol} is not supported")


# ---------------------------------------------------------------- operators
class Op:
    """A product of one-dof symbols with a prefactor (op.py semantics: a
    single dof is shared by every simple symbol; a list gives one dof each)."""

    def __init__(self, symbol: str, dof, factor=1.0):
        self.symbol = symbol
        self.split_symbol = symbol.replace(r"b^\dagger + b", r"b^\dagger+b").split(" ")
        if isinstance(dof, list):
            assert len(dof) == len(self.split_symbol), "one dof per simple symbol"
            self.dofs = list(dof)
        else:
            self.dofs = [dof] * len(self.split_symbol)
        self.factor = _au(factor) if isinstance(factor, Quantity) else factor

    def __mul__(self, other):
        if isinstance(other, Op):
            return Op(" ".join(self.split_symbol + other.split_symbol), self.dofs + other.dofs,
                      self.factor * other.factor)
        return Op(self.symbol, list(self.dofs), self.factor * other)

    __rmul__ = __mul__

    def local_mats(self, model: "Model") -> Dict[int, np.ndarray]:
        """{site index: matrix} with the symbols on the same site multiplied in order."""
        per_site: Dict[int, List[str]] = {}
        order = []
        for sym, dof in zip(self.split_symbol, self.dofs):
            site = model.dof_to_siteidx[dof]
            if site not in per_site:
                per_site[site] = []
                order.append(site)
            per_site[site].append(sym)
        out = {}
        for site in order:
            basis = model.basis[site]
            syms = per_site[site]
            joined = " ".join(syms)
            try:
                mat = basis.op_mat(joined)
            except ValueError:
                mat = np.eye(basis.nbas)
                for s in syms:
                    mat = mat @ basis.op_mat(s)
            out[site] = np.asarray(mat)
        return out

    def __repr__(self):
        return f"Op({self.symbol!r}, {self.dofs}, {self.factor})"


# ---------------------------------------------------------------- models
class Model:
    def __init__(self, basis: List[BasisSet], ham_terms: List[Op], dipole=None):
        if not isinstance(basis, list) or len(basis) == 0:
            raise TypeError("Basis should be a non-empty list")
        all_dofs = [d for b in basis for d in b.dofs]
        if len(all_dofs) != len(set(all_dofs)):
            dup = [k for k, v in Counter(all_dofs).items() if v > 1]
            raise ValueError(f"Duplicate DoF definition found in the basis list: {dup}")
        self.basis = basis
        qs = {b.sigmaqn.shape[1] for b in basis}
        if len(qs) != 1:
            raise ValueError(f"Inconsistent quantum number size: {qs}")
        self.qn_size = qs.pop()
        self.dof_to_siteidx = {}
        for i, b in enumerate(basis):
            for d in b.dofs:
                self.dof_to_siteidx[d] = i
        self.ham_terms = [t for t in ham_terms if t.factor != 0]
        self.dipole = dipole
        self.mpos = {}
        self.pbond_list = [b.nbas for b in basis]

    @property
    def nsite(self):
        return len(self.basis)

    @property
    def e_dofs(self):
        return [b.dof for b in self.basis if b.is_electron]

    @property
    def v_dofs(self):
        return [b.dof for b in self.basis if b.is_phonon]

    @property
    def n_edofs(self):
        return len(self.e_dofs)

    def copy(self):
        new = self.__class__.__new__(self.__class__)
        new.__dict__ = self.__dict__.copy()
        new.mpos = dict(self.mpos)
        return new


class Phonon:
    def __init__(self, omega, displacement, n_phys_dim: int = None):
        self.omega = [_au(o) for o in omega]
        self.dis = [_au(d) for d in displacement]
        self.n_phys_dim = n_phys_dim

    @classmethod
    def simple_phonon(cls, omega, displacement, n_phys_dim):
        return cls([omega, omega], [Quantity(0), displacement], n_phys_dim)

    @property
    def is_simple(self):
        return self.omega[0] == self.omega[1]

    @property
    def reorganization_energy(self):
        return 0.5 * (self.dis[1] - self.dis[0]) ** 2 * self.omega[1] ** 2

    @property
    def coupling_constant(self):
        return float(np.sqrt(self.reorganization_energy / self.omega[0]))


class Mol:
    def __init__(self, elocalex, ph_list: List[Phonon], dipole=None):
        if len(ph_list) == 0:
            raise ValueError("No phonon mode in phonon list")
        self.elocalex = _au(elocalex)
        self.ph_list = ph_list
        self.dipole = dipole
        self.e0 = sum(ph.reorganization_energy for ph in ph_list)

    @property
    def gs_zpe(self):
        return sum(ph.omega[0] for ph in self.ph_list) / 2


def construct_j_matrix(mol_num, j_constant, periodic=False):
    j = np.ones(mol_num - 1) * _au(j_constant)
    m = np.diag(j, k=-1) + np.diag(j, k=1)
    if periodic:
        m[-1, 0] = m[0, -1] = _au(j_constant)
    return m


class HolsteinModel(Model):
    """model.py:231-349 with scheme 1-3 basis order [e_0, ph_0_*, e_1, ph_1_*, ...]:
    H = sum_ij J_ij a+_i a_j + sum_i (elocalex + e0) n_i + sum (p^2 + w^2 x^2)/2
        - sum w^2 D n_i x_i  (+ the x^2 shift when the two PES frequencies differ)."""

    def __init__(self, mol_list: List[Mol], j_matrix, scheme: int = 2, periodic: bool = False):
        n = len(mol_list)
        if isinstance(j_matrix, Quantity):
            j_matrix = construct_j_matrix(n, j_matrix, periodic)
        j_matrix = np.asarray(j_matrix, dtype=float)
        assert j_matrix.shape == (n, n)
        if scheme == 4:
            raise NotImplementedError("scheme 4 (multi-electron basis) is outside the sweep engine")
        self.mol_list = mol_list
        self.j_matrix = j_matrix
        self.scheme = scheme
        basis, ham = [], []
        for imol, mol in enumerate(mol_list):
            basis.append(BasisSimpleElectron(imol))
            for iph, ph in enumerate(mol.ph_list):
                basis.append(BasisSHO((imol, iph), ph.omega[0], ph.n_phys_dim))
        for i in range(n):
            for j in range(n):
                f = mol_list[i].elocalex + mol_list[i].e0 if i == j else j_matrix[i, j]
                ham.append(Op(r"a^\dagger a", [i, j], f))
        for imol, mol in enumerate(mol_list):
            for iph, ph in enumerate(mol.ph_list):
                ham.extend([Op("p^2", (imol, iph), 0.5), Op("x^2", (imol, iph), 0.5 * ph.omega[0] ** 2)])
        for imol, mol in enumerate(mol_list):
            for iph, ph in enumerate(mol.ph_list):
                if np.allclose(ph.omega[0], ph.omega[1]):
                    ham.append(Op(r"a^\dagger a", imol) * Op("x", (imol, iph)) * (-ph.omega[1] ** 2 * ph.dis[1]))
                else:
                    ham.append(Op(r"a^\dagger a", imol) * Op("x^2", (imol, iph))
                               * (0.5 * (ph.omega[1] ** 2 - ph.omega[0] ** 2)))
                    ham.append(Op(r"a^\dagger a", imol) * Op("x", (imol, iph)) * (-ph.omega[1] ** 2 * ph.dis[1]))
        super().__init__(basis, ham, dipole={i: m.dipole for i, m in enumerate(mol_list)})
        self.mol_num = n

    @property
    def gs_zpe(self):
        return sum(m.gs_zpe for m in self.mol_list)


class SpinBosonModel(Model):
    """model.py:408-439: eps sigma_z + Delta sigma_x + sum (p^2 + w^2 q^2)/2 + sigma_z sum c_i q_i."""

    def __init__(self, epsilon, delta, ph_list: List[Phonon], dipole: float = None):
        self.epsilon = _au(epsilon)
        self.delta = _au(delta)
        self.ph_list = ph_list
        basis = [BasisHalfSpin("spin")]
        for iph, ph in enumerate(ph_list):
            basis.append(BasisSHO(iph, ph.omega[0], ph.n_phys_dim))
        ham = [Op("sigma_z", "spin", self.epsilon), Op("sigma_x", "spin", self.delta)]
        for iph, ph in enumerate(ph_list):
            assert ph.is_simple
            ham.extend([Op("p^2", iph, 0.5), Op("x^2", iph, 0.5 * ph.omega[0] ** 2)])
            ham.append(Op("sigma_z", "spin") * Op("x", iph) * (-ph.omega[1] ** 2 * ph.dis[1]))
        super().__init__(basis, ham, dipole={"spin": 0 if dipole is None else dipole})


class SpectralDensityFunction:
    """Ohmic J(w) = pi/2 alpha w^s w_c^(1-s) exp(-w/w_c) (sbm/lib.py:38-136)."""

    def __init__(self, alpha: float, omega_c, s: float = 1):
        self.alpha = alpha
        self.omega_c = _au(omega_c)
        self.s = s

    def func(self, w):
        return np.pi / 2.0 * self.alpha * w ** self.s * self.omega_c ** (1 - self.s) * np.exp(-w / self.omega_c)

    def _dos_Wang1(self, nb, w):
        return (nb + 1) / self.omega_c * np.exp(-w / self.omega_c)

    def Wang1(self, nb):
        w = np.array([-np.log(-float(j) / (nb + 1) + 1.0) * self.omega_c for j in range(1, nb + 1)])
        c2 = 2.0 / np.pi * w * self.func(w) / self._dos_Wang1(nb, w)
        return w, c2

    def trapz(self, nb, x0, x1):
        dw = (x1 - x0) / float(nb)
        xs = [x0 + i * dw for i in range(nb + 1)]
        w = np.array([(xs[i] + xs[i + 1]) / 2.0 for i in range(nb)])
        c2 = np.array([(self.func(xs[i]) + self.func(xs[i + 1])) / 2 for i in range(nb)]) * 2.0 / np.pi * w * dw
        return w, c2

    @staticmethod
    def post_process(w, c2, ifsort=True):
        dis = np.sqrt(c2) / w ** 2
        idx = np.argsort(c2 / w)[::-1] if ifsort else np.arange(len(w))
        return [Quantity(w[i]) for i in idx], [Quantity(dis[i]) for i in idx]
