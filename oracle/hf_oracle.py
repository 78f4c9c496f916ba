"""
ORACLE (test infrastructure only): CPU restatement of the reference's
Hartree-Fock path (Nathan-W123/Ab-Initio-MD, ``aimd/qc``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference
arm of ``bench.py`` import this module; the product never does. It is the
checker that the CUDA path is compared with, at every size (including sizes
the reference cannot run, because it stores the ERI tensor).

* integral kernels: ``md_oracle.c`` (C + OpenMP), one function per reference
  kernel, loaded with ctypes from ``oracle/_build/libmd_oracle.so``;
* SCF algebra, SAD guess, DIIS and gradient assembly: numpy below, each
  function citing the reference lines it restates.

Pinning: tests/golden holds fixtures produced by the reference itself
(tests/golden/make_golden.py); tests/test_oracle_golden.py checks this
restatement against them. The basis arrays come from the product's basis
builder, which tests/test_basis.py pins bitwise to the reference's.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
import sys
from typing import Any, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libmd_oracle.so")
sys.path.insert(0, os.path.join(os.path.dirname(_HERE), "ab-initio-md_b200"))
from aimd_b200.basis import BasisSet, build_basis  # noqa: E402  (input layout only)

DEFAULT_SCHWARZ = 1e-12        # aimd/qc/integrals.py:114
DEFAULT_SCHWARZ_GRAD = 1e-14   # aimd/qc/integrals.py:119
PRIM_CUTOFF = 50.0             # aimd/qc/integrals.py:510

_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)
_lib = None


def build() -> str:
    """Compile the C restatement (make in oracle/); returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
    return _lib


def _p(a: np.ndarray):
    if a.dtype == np.int64:
        return a.ctypes.data_as(_i64p)
    return a.ctypes.data_as(_f64p)


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ============================================================ pair data

class Pairs:
    """aimd/qc/integrals.py:525-627 (_build_pairs, _Pairs), cached per BasisSet."""

    def __init__(self, basis: BasisSet) -> None:
        L = lib()
        nb = basis.nblock
        npair = nb * (nb + 1) // 2
        self.basis = basis
        self.pair_pp = np.zeros(npair + 1, dtype=np.int64)
        self.pair_blocks = np.zeros((npair, 2), dtype=np.int64)
        blk_atom = np.ascontiguousarray(basis.blk_atom)
        blk_prim = np.ascontiguousarray(basis.blk_prim)
        blk_exp = np.ascontiguousarray(basis.blk_exp)
        pos = np.ascontiguousarray(basis.positions)
        L.orc_count_pairs.restype = ctypes.c_int64
        npp = int(L.orc_count_pairs(ctypes.c_int64(nb), _p(blk_atom), _p(blk_prim), _p(blk_exp), _p(pos),
                                    _p(self.pair_pp), _p(self.pair_blocks)))
        self.lmax = int(basis.lmax)
        self.maxcon = int(basis.blk_coef.shape[1])
        L1, T1 = self.lmax + 2, 2 * self.lmax + 4
        self.pp_ab = np.zeros((npp, 2))
        self.pp_P = np.zeros((npp, 3))
        self.pp_E = np.zeros((npp, 3, L1, L1, T1))
        self.pp_C = np.zeros((npp, self.maxcon * self.maxcon))
        self.blk_l = np.ascontiguousarray(basis.blk_l)
        self.blk_ncon = np.ascontiguousarray(basis.blk_ncon)
        self.blk_ao = np.ascontiguousarray(basis.blk_ao)
        self.blk_atom = blk_atom
        L.orc_fill_pairs(ctypes.c_int64(nb), ctypes.c_int64(self.lmax), ctypes.c_int64(self.maxcon),
                         _p(blk_atom), _p(self.blk_l), _p(blk_prim), _p(blk_exp),
                         _p(np.ascontiguousarray(basis.blk_coef)), _p(self.blk_ncon), _p(pos),
                         _p(self.pp_ab), _p(self.pp_P), _p(self.pp_E), _p(self.pp_C))
        self.npair, self.npp, self.nb = npair, npp, nb
        npp_per = np.diff(self.pair_pp)
        self.maxpp = max(int(npp_per.max()), 1) if npair else 1
        i, j = self.pair_blocks.T
        nc = (self.blk_l + 1) * (self.blk_l + 2) // 2
        rows = self.blk_ncon[i] * self.blk_ncon[j] * nc[i] * nc[j]
        self.maxrow = max(int(rows.max()), 1) if npair else 1

    def args(self):
        return (ctypes.c_int64(self.nb), ctypes.c_int64(self.npp), ctypes.c_int64(self.lmax),
                ctypes.c_int64(self.maxcon), ctypes.c_int64(self.maxpp), ctypes.c_int64(self.maxrow),
                _p(self.blk_l), _p(self.blk_ncon), _p(self.blk_ao), _p(self.blk_atom), _p(self.pair_pp),
                _p(self.pair_blocks), _p(self.pp_ab), _p(self.pp_P), _p(self.pp_E), _p(self.pp_C))


def pairs(basis: BasisSet) -> Pairs:
    p = basis._cache.get("oracle_pairs")
    if p is None:
        p = basis._cache["oracle_pairs"] = Pairs(basis)
    return p


# ============================================================ two-electron

def boys(nmax: int, x: float) -> np.ndarray:
    """aimd/qc/boys.py:143-151"""
    out = np.zeros(nmax + 1)
    lib().orc_boys(ctypes.c_int(nmax), ctypes.c_double(x), _p(out))
    return out


def schwarz_bounds(basis: BasisSet) -> np.ndarray:
    """aimd/qc/integrals.py:970-983"""
    Q = basis._cache.get("oracle_schwarz")
    if Q is None:
        pr = pairs(basis)
        Q = np.zeros(pr.npair)
        lib().orc_schwarz(*pr.args(), _p(Q))
        basis._cache["oracle_schwarz"] = Q
    return Q


def eri_tensor(basis: BasisSet, schwarz_threshold: float = DEFAULT_SCHWARZ) -> np.ndarray:
    """aimd/qc/integrals.py:986-1006 (no size cap: callers keep nao small)."""
    pr = pairs(basis)
    Q = schwarz_bounds(basis)
    n = basis.nao
    eri = np.zeros((n, n, n, n))
    lib().orc_eri_tensor(*pr.args(), _p(Q), ctypes.c_double(schwarz_threshold), ctypes.c_int64(n), _p(eri))
    return eri


def jk_direct(basis: BasisSet, densities: np.ndarray, schwarz_threshold: float = DEFAULT_SCHWARZ,
              stride: int = 1, offset: int = 0):
    """
    J, K of aimd/qc/integrals.py:1031-1044 (jk_from_eri of the screened
    tensor) without storing the tensor. Densities may be non-symmetric:
    J depends on the symmetric part only, K = A(D) + A(D^T)^T.
    stride > 1 evaluates only the quartets of bra pairs p1 = offset (mod
    stride): a timing sample, not J/K.
    """
    D = np.asarray(densities, dtype=float)
    single = D.ndim == 2
    D3 = np.ascontiguousarray(D[None] if single else D)
    sym = np.array_equal(D3, D3.transpose(0, 2, 1))
    Din = D3 if sym else np.ascontiguousarray(np.concatenate([D3, D3.transpose(0, 2, 1)]))
    pr = pairs(basis)
    Q = schwarz_bounds(basis)
    n = basis.nao
    Ja = np.zeros_like(Din)
    Ka = np.zeros_like(Din)
    lib().orc_jk_direct_strided(*pr.args(), _p(Q), ctypes.c_double(schwarz_threshold), ctypes.c_int64(n),
                                ctypes.c_int64(Din.shape[0]), _p(Din), _p(Ja), _p(Ka), ctypes.c_int64(stride),
                                ctypes.c_int64(offset))
    if sym:
        J = Ja + Ja.transpose(0, 2, 1)
        K = Ka + Ka.transpose(0, 2, 1)
    else:
        m = D3.shape[0]
        Jh = Ja + Ja.transpose(0, 2, 1)
        J = 0.5 * (Jh[:m] + Jh[m:])
        K = Ka[:m] + Ka[m:].transpose(0, 2, 1)
    return (J[0], K[0]) if single else (J, K)


def _sym(D, nao, what):
    D = np.asarray(D, dtype=float)
    if D.shape != (nao, nao):
        raise ValueError(f"{what} must have shape ({nao}, {nao}), got {D.shape}")
    return np.ascontiguousarray(0.5 * (D + D.T))


def two_electron_gradient(basis: BasisSet, D_coulomb, D_exchange_list, k_factor,
                          schwarz_threshold: float = DEFAULT_SCHWARZ_GRAD, stride: int = 1,
                          offset: int = 0) -> np.ndarray:
    """aimd/qc/integrals.py:1498-1520 (stride > 1: bra pairs offset mod stride only, a timing sample)"""
    n = basis.nao
    Dc = _sym(D_coulomb, n, "D_coulomb")
    Dx = np.ascontiguousarray(np.array([_sym(d, n, "D_exchange") for d in D_exchange_list]).reshape(-1, n, n))
    pr = pairs(basis)
    Q = schwarz_bounds(basis)
    g = np.zeros((basis.natm, 3))
    lib().orc_grad2e_strided(*pr.args(), _p(Q), ctypes.c_double(schwarz_threshold), ctypes.c_int64(n),
                             ctypes.c_int64(basis.natm), _p(Dc), ctypes.c_int64(Dx.shape[0]), _p(Dx),
                             ctypes.c_double(k_factor), _p(g), ctypes.c_int64(stride), ctypes.c_int64(offset))
    return g


# ============================================================ one-electron

def _shell_args(b: BasisSet):
    return (ctypes.c_int64(b.nshell), _p(np.ascontiguousarray(b.shell_atom)), _p(np.ascontiguousarray(b.shell_l)),
            _p(np.ascontiguousarray(b.shell_prim)), _p(np.ascontiguousarray(b.shell_ao)),
            _p(np.ascontiguousarray(b.prim_exp)), _p(np.ascontiguousarray(b.prim_coef)),
            _p(np.ascontiguousarray(b.positions)))


def overlap_type(basis: BasisSet, origin=None):
    """aimd/qc/integrals.py:1374-1383 (S, T, dipole integrals)"""
    n = basis.nao
    S, T, M = np.zeros((n, n)), np.zeros((n, n)), np.zeros((3, n, n))
    o = np.zeros(3) if origin is None else np.asarray(origin, dtype=float).reshape(3).copy()
    lib().orc_overlap_type(*_shell_args(basis), ctypes.c_int64(n), _p(o), _p(S), _p(T), _p(M))
    return S, T, M


def nuclear_attraction_matrix(basis: BasisSet, charges=None) -> np.ndarray:
    """aimd/qc/integrals.py:1406-1411"""
    q = basis.nuclear_charges.copy() if charges is None else np.asarray(charges, dtype=float).copy()
    V = np.zeros((basis.nao, basis.nao))
    lib().orc_nuclear(*_shell_args(basis), ctypes.c_int64(basis.nao), ctypes.c_int64(basis.natm), _p(q),
                      _p(np.ascontiguousarray(basis.positions)), _p(V))
    return V


def one_electron_matrices(basis: BasisSet):
    S, T, _ = overlap_type(basis)
    return S, T, nuclear_attraction_matrix(basis)


def dipole_integrals(basis: BasisSet, origin=None) -> np.ndarray:
    return overlap_type(basis, origin)[2]


def nuclear_repulsion_energy(charges, positions) -> float:
    """aimd/qc/integrals.py:1421-1426"""
    q = np.asarray(charges, dtype=float).reshape(-1)
    x = np.asarray(positions, dtype=float).reshape(-1, 3)
    i, j = np.triu_indices(len(q), k=1)
    return float(np.sum(q[i] * q[j] / np.linalg.norm(x[i] - x[j], axis=1)))


def nuclear_repulsion_gradient(charges, positions) -> np.ndarray:
    """aimd/qc/integrals.py:1429-1440"""
    q = np.asarray(charges, dtype=float).reshape(-1)
    x = np.asarray(positions, dtype=float).reshape(-1, 3)
    i, j = np.triu_indices(len(q), k=1)
    d = x[i] - x[j]
    r = np.linalg.norm(d, axis=1)
    pair = -(q[i] * q[j] / r ** 3)[:, None] * d
    g = np.zeros_like(x)
    np.add.at(g, i, pair)
    np.add.at(g, j, -pair)
    return g


def nuclear_dipole(charges, positions, origin=None) -> np.ndarray:
    q = np.asarray(charges, dtype=float).reshape(-1)
    x = np.asarray(positions, dtype=float).reshape(-1, 3)
    o = np.zeros(3) if origin is None else np.asarray(origin, dtype=float).reshape(3)
    return q @ (x - o)


def one_electron_gradient(basis: BasisSet, D, W) -> np.ndarray:
    """aimd/qc/integrals.py:1483-1495"""
    n = basis.nao
    D = _sym(D, n, "D")
    W = _sym(W, n, "W")
    g = np.zeros((basis.natm, 3))
    lib().orc_ovlp_kin_grad(*_shell_args(basis), ctypes.c_int64(n), _p(np.ascontiguousarray(-W)), _p(D), _p(g))
    lib().orc_nuclear_grad(*_shell_args(basis), ctypes.c_int64(n), ctypes.c_int64(basis.natm),
                           _p(basis.nuclear_charges.copy()), _p(D), _p(g))
    return g


# ============================================================ SCF (numpy)

LINDEP_THRESHOLD = 1e-7


def orthogonalizer(S, method="auto", threshold=LINDEP_THRESHOLD):
    """aimd/qc/scf.py:284-303"""
    s, U = np.linalg.eigh(S)
    keep = s >= threshold
    if method == "symmetric" or (method == "auto" and keep.all()):
        if not keep.all():
            raise ValueError("basis nearly linearly dependent")
        return (U * s ** -0.5) @ U.T, 0, float(s[0])
    return U[:, keep] * s[keep] ** -0.5, int((~keep).sum()), float(s[0])


_MADELUNG = sorted(((n, l) for n in range(1, 8) for l in range(n)), key=lambda t: (t[0] + t[1], t[0]))


def ground_state_l_counts(Z: int) -> list[int]:
    """aimd/qc/scf.py:365-380"""
    counts, left = [0, 0, 0, 0], int(Z)
    for _n, l in _MADELUNG:
        if left <= 0:
            break
        k = min(left, 2 * (2 * l + 1))
        counts[l] += k
        left -= k
    return counts


def _atomic_occupations(eps, l_counts, tol=1e-6):
    """aimd/qc/scf.py:396-427"""
    groups, i = [], 0
    while i < len(eps):
        j = i + 1
        while j < len(eps) and eps[j] - eps[j - 1] < tol:
            j += 1
        groups.append((i, j))
        i = j
    occ = np.zeros(len(eps))
    left = list(l_counts) + [0] * (5 - len(l_counts))
    ok = True
    for i, j in groups:
        g = j - i
        if g % 2 == 0 or g > 9:
            ok = False
            break
        l = (g - 1) // 2
        k = min(left[l], 2 * g)
        occ[i:j] = k / g
        left[l] -= k
    if ok and not any(left):
        return occ
    occ[:] = 0.0
    n = float(sum(l_counts))
    for i, j in groups:
        k = min(n, 2.0 * (j - i))
        occ[i:j] = k / (j - i)
        n -= k
    return occ


class DIIS:
    """aimd/qc/scf.py:516-568 (anchored least squares solved by SVD, numpy lstsq)."""

    def __init__(self, space=8, max_coefficient=1e4):
        self.space, self.max_coefficient = int(space), float(max_coefficient)
        self.focks, self.errors = [], []

    def __len__(self):
        return len(self.focks)

    def reset(self):
        self.focks.clear()
        self.errors.clear()

    def push(self, fock, error):
        self.focks.append(np.array(fock, dtype=float))
        self.errors.append(np.array(error, dtype=float))
        while len(self.focks) > self.space:
            self.focks.pop(0)
            self.errors.pop(0)

    def coefficients(self):
        last = self.errors[-1].ravel()
        if len(self.errors) == 1:
            return np.ones(1)
        delta = np.stack([e.ravel() - last for e in self.errors[:-1]], axis=1)
        x = np.linalg.lstsq(delta, -last, rcond=None)[0]
        return np.append(x, 1.0 - x.sum())

    def extrapolate(self):
        while len(self.focks) > 1:
            c = self.coefficients()
            if np.all(np.isfinite(c)) and np.abs(c).max() <= self.max_coefficient:
                return sum(ci * Fi for ci, Fi in zip(c, self.focks))
            self.focks.pop(0)
            self.errors.pop(0)
        return self.focks[-1].copy()


_ATOM_CACHE: dict = {}


def atom_basis(basis: BasisSet, atom: int) -> BasisSet:
    """aimd/qc/scf.py:489-499"""
    sh = np.flatnonzero(basis.shell_atom == atom)
    k0 = [basis.shell_prim[s] for s in sh]
    k1 = [basis.shell_prim[s + 1] for s in sh]
    prim = np.concatenate([np.arange(a, b) for a, b in zip(k0, k1)]) if len(sh) else np.zeros(0, int)
    shell_prim = np.concatenate([[0], np.cumsum([b - a for a, b in zip(k0, k1)])])
    return BasisSet(basis.name, [basis.symbols[atom]], np.zeros((1, 3)), np.zeros(len(sh), dtype=np.int64),
                    basis.shell_l[sh], shell_prim, basis.prim_exp[prim], basis.prim_coef[prim])


def atomic_hf(ab: BasisSet, max_iter: int = 200):
    """aimd/qc/scf.py:433-482 (spherically averaged fractional-occupation atom)"""
    key = (int(ab.atomic_numbers[0]), ab.shell_l.tobytes(), ab.prim_exp.tobytes(), ab.prim_coef.tobytes())
    if key in _ATOM_CACHE:
        return _ATOM_CACHE[key]
    Z = int(ab.atomic_numbers[0])
    lc = ground_state_l_counts(Z)
    S, T, _ = overlap_type(ab)
    H = T + nuclear_attraction_matrix(ab)
    X, _, _ = orthogonalizer(S, "canonical")
    if Z == 1:
        eps, Cp = np.linalg.eigh(X.T @ H @ X)
        c = X @ Cp[:, 0]
        _ATOM_CACHE[key] = np.outer(c, c)
        return _ATOM_CACHE[key]
    eri = eri_tensor(ab)

    def density(Fo):
        eps, Cp = np.linalg.eigh(Fo)
        C = X @ Cp
        return (C * _atomic_occupations(eps, lc)) @ C.T

    D = density(X.T @ H @ X)
    diis = DIIS(8)
    e_old = np.inf
    for _ in range(max_iter):
        J = np.einsum("ijkl,kl->ij", eri, D)
        K = np.einsum("ikjl,kl->ij", eri, D)
        F = H + J - 0.5 * K
        F = 0.5 * (F + F.T)
        e = 0.5 * float(np.vdot(D, H + F))
        err = X.T @ (F @ D @ S - S @ D @ F) @ X
        if abs(e - e_old) < 1e-11 and np.abs(err).max() < 1e-8:
            break
        e_old = e
        diis.push((X.T @ F @ X)[None], err[None])
        D = density(diis.extrapolate()[0])
    _ATOM_CACHE[key] = 0.5 * (D + D.T)
    return _ATOM_CACHE[key]


def sad_density(basis: BasisSet) -> np.ndarray:
    """aimd/qc/scf.py:502-511"""
    P = np.zeros((basis.nao, basis.nao))
    for a in range(basis.natm):
        i, j = basis.atom_ao[a]
        if j > i:
            P[i:j, i:j] = atomic_hf(atom_basis(basis, a))
    return P


def electron_counts(nuclear_charge, charge, multiplicity):
    n = int(nuclear_charge) - int(charge)
    m = int(multiplicity)
    return (n + m - 1) // 2, (n - m + 1) // 2


def run_scf(symbols: Sequence[str], positions, basis: str, charge: int = 0, multiplicity: int = 1,
            reference: str | None = None, guess: Any = "sad", conv_energy: float = 1e-10,
            conv_commutator: float = 1e-7, max_iter: int = 100, diis_space: int = 8,
            diis_restart: int = 12, schwarz_threshold: float = DEFAULT_SCHWARZ) -> dict:
    """
    aimd/qc/scf.py:830-965 (SCFSolver._run/_iterate/_result) with the J/K of
    the stored tensor replaced by the integral-direct jk_direct above.
    Returns a dict with the SCFResult fields the tests use.
    """
    b = build_basis(symbols, np.asarray(positions, dtype=float), basis)
    ref = reference or ("rhf" if multiplicity == 1 else "uhf")
    na, nb = electron_counts(b.atomic_numbers.sum(), charge, multiplicity)
    nspin = 1 if ref == "rhf" else 2
    nocc = (na,) if nspin == 1 else (na, nb)
    S, T, _ = overlap_type(b)
    H = T + nuclear_attraction_matrix(b)
    X, n_removed, _ = orthogonalizer(S)
    enuc = nuclear_repulsion_energy(b.nuclear_charges, b.positions)
    if isinstance(guess, str):
        if guess == "sad":
            Ds = np.repeat(0.5 * sad_density(b)[None], nspin, axis=0)
        else:
            F0 = H if guess == "core" else None
            if F0 is None:
                h = np.diag(H)
                F0 = 0.5 * 1.75 * S * (h[:, None] + h[None, :])
                np.fill_diagonal(F0, h)
            Ds = []
            for k in nocc:
                _, Cp = np.linalg.eigh(X.T @ F0 @ X)
                C = X @ Cp[:, :k]
                Ds.append(C @ C.T)
            Ds = np.array(Ds)
    else:
        D = np.array(guess, dtype=float)
        Ds = np.repeat(0.5 * D[None], nspin, axis=0) if D.ndim == 2 else (
            D.copy() if nspin == 2 else 0.5 * (D[0] + D[1])[None])
        Ds = 0.5 * (Ds + Ds.transpose(0, 2, 1))
    g = 2.0 / nspin
    diis = DIIS(diis_space)
    e_prev, best, since, conv = np.nan, np.inf, 0, False
    for it in range(1, max_iter + 1):
        J, K = jk_direct(b, Ds, schwarz_threshold)
        F = H + g * J.sum(axis=0) - K
        F = 0.5 * (F + F.transpose(0, 2, 1))
        e_el = 0.5 * g * float(sum(np.vdot(Ds[s], H + F[s]) for s in range(nspin)))
        FDS = F @ Ds @ S
        err = X.T @ (FDS - FDS.transpose(0, 2, 1)) @ X
        err_norm = float(np.abs(err).max())
        de = e_el - e_prev
        if abs(de) < conv_energy and err_norm < conv_commutator:
            conv = True
            break
        if it == max_iter:
            break
        Fo = X.T @ F @ X
        if err_norm < best:
            best, since = err_norm, 0
        else:
            since += 1
        if diis_restart and since >= diis_restart:
            diis.reset()
            best, since = err_norm, 0
        diis.push(Fo, err)
        Fo = diis.extrapolate()
        Dn = np.empty_like(Ds)
        for s in range(nspin):
            _, Cp = np.linalg.eigh(Fo[s])
            C = X @ Cp[:, :nocc[s]]
            Dn[s] = C @ C.T
        Ds = Dn
        e_prev = e_el
    spin = np.array([Ds[0], Ds[-1]])
    P = spin[0] + spin[1]
    M = overlap_type(b)[2]
    dip = -np.einsum("xmn,mn->x", M, P) + nuclear_dipole(b.nuclear_charges, b.positions)
    return {"basis": b, "energy": e_el + enuc, "electronic_energy": e_el, "nuclear_repulsion": enuc,
            "converged": conv, "iterations": it, "spin_densities": spin, "density": P,
            "fock": F[0] if nspin == 1 else F, "unrestricted": nspin == 2, "dipole": dip,
            "commutator_norm": err_norm, "energy_change": de}


def energy_weighted_density(spin_densities, fock):
    """aimd/qc/gradients.py:106-125"""
    D = np.asarray(spin_densities)
    F = np.asarray(fock)
    if F.ndim == 2:
        W = D[0] @ F @ D[0] + D[1] @ F @ D[1]
    else:
        W = D[0] @ F[0] @ D[0] + D[1] @ F[1] @ D[1]
    return 0.5 * (W + W.T)


def scf_gradient(res: dict, schwarz_threshold: float = DEFAULT_SCHWARZ_GRAD) -> np.ndarray:
    """aimd/qc/gradients.py:168-193"""
    b = res["basis"]
    P = res["density"]
    W = energy_weighted_density(res["spin_densities"], res["fock"])
    g = nuclear_repulsion_gradient(b.nuclear_charges, b.positions)
    g += one_electron_gradient(b, P, W)
    if res["unrestricted"]:
        Dx, k = [res["spin_densities"][0], res["spin_densities"][1]], 1.0
    else:
        Dx, k = [P], 0.5
    g += two_electron_gradient(b, P, Dx, k, schwarz_threshold)
    return g


def flop_model(basis: BasisSet, threshold: float = DEFAULT_SCHWARZ) -> dict:
    """
    FP64 flop model of one ERI pass (the algorithmic work unit): per
    primitive quartet with bra pair (L_ab, n_ab, n_bc) and ket pair
    (L_cd, n_cd, n_kc), L = L_ab + L_cd,
        2 sum_{n=0..L} NH(L-n) + 2 NH(L_ab) NH(L_cd) n_cd n_kc + 2 NH(L_ab) n_ab n_cd n_kc,
    over unique block quartets (p1 >= p2, p1 as bra) with Q1 Q2 >= threshold.
    Returns the total and the number of primitive quartets.
    """
    pr = pairs(basis)
    Q = schwarz_bounds(basis)
    i, j = pr.pair_blocks.T
    l = pr.blk_l
    Lp = l[i] + l[j]
    nc = (l + 1) * (l + 2) // 2
    nab = nc[i] * nc[j]
    ncon = pr.blk_ncon[i] * pr.blk_ncon[j]
    npp = np.diff(pr.pair_pp).astype(float)

    def NH(L):
        return (L + 1) * (L + 2) * (L + 3) // 6

    rtab = np.array([sum(NH(L0 - n) for n in range(L0 + 1)) for L0 in range(2 * int(l.max(initial=0)) * 2 + 1)])
    per_bra = np.zeros(pr.npair)
    nq = 0.0
    for p1 in range(pr.npair):
        p2 = np.arange(p1 + 1)
        keep = Q[p1] * Q[p2] >= threshold
        p2 = p2[keep]
        if p2.size == 0:
            continue
        Lb, Lk = Lp[p1], Lp[p2]
        rsum = rtab[Lb + Lk]
        per = 2 * rsum + 2 * NH(Lb) * NH(Lk) * nab[p2] * ncon[p2] + 2 * NH(Lb) * nab[p1] * nab[p2] * ncon[p2]
        w = npp[p1] * npp[p2]
        per_bra[p1] = float(np.sum(per * w))
        nq += float(np.sum(w))
    # per_bra[p1]: the flops of bra pair p1's quartets (the unit the strided
    # samples of jk_direct / two_electron_gradient select)
    return {"flop": float(per_bra.sum()), "prim_quartets": nq, "per_bra": per_bra}
