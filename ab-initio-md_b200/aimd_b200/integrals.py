"""
Molecular integrals on the GPU, with the reference's public API
(``aimd.qc.integrals``, aimd/qc/integrals.py:1374-1520):

  schwarz_bounds, eri_tensor, jk_from_eri, jk (integral-direct, new),
  overlap_matrix, kinetic_matrix, dipole_integrals,
  nuclear_attraction_matrix, one_electron_matrices,
  nuclear_repulsion_energy, nuclear_repulsion_gradient, nuclear_dipole,
  one_electron_gradient, two_electron_gradient

Hartree atomic units; AO matrices in the unit-normalised Cartesian AOs of
:mod:`aimd_b200.basis`. Functions that take numpy arrays return numpy
arrays (as the reference does); the ``*_device`` variants take and return
CUDA float64 tensors and are what the SCF uses. Every evaluation runs in
the native CUDA library; there is no CPU path.
"""

from __future__ import annotations

from typing import Sequence

import numpy as np
import torch

from .basis import BasisSet
from .engine import engine_for

DEFAULT_SCHWARZ = 1e-12        # strict bound on each dropped ERI
DEFAULT_SCHWARZ_GRAD = 1e-14   # gradient screening on Q1 Q2 max|Gamma|
MAX_NAO_ERI = 120              # eri_tensor refuses larger bases unless raised


def _t(x) -> torch.Tensor:
    return torch.as_tensor(np.asarray(x, dtype=float), device="cuda")


def _check_sym(D: np.ndarray, nao: int, what: str) -> np.ndarray:
    D = np.asarray(D, dtype=float)
    if D.shape != (nao, nao):
        raise ValueError(f"{what} must have shape ({nao}, {nao}), got {D.shape}")
    return 0.5 * (D + D.T)


# ---------------------------------------------------------------- two-electron

def schwarz_bounds(basis: BasisSet) -> np.ndarray:
    """
    Q_P = max_ab |(ab|ab)|^(1/2) per block pair P = i(i+1)/2 + j (i >= j) of
    the basis's blocks (aimd/qc/integrals.py:970). Blocks whose general
    contraction the device splits are mapped back: the Q of a block pair is
    the maximum over its device sub-pairs.
    """
    eng = engine_for(basis)
    Qd = eng.schwarz().cpu().numpy()
    if not eng.split:
        return Qd
    orig = eng.blocks["orig"]
    nd = len(orig)
    i, j = np.tril_indices(nd)                      # device pair index i(i+1)/2 + j in row-major order
    I_, J_ = orig[i], orig[j]
    P = I_ * (I_ + 1) // 2 + J_
    Q = np.zeros(basis.nblock * (basis.nblock + 1) // 2)
    np.maximum.at(Q, P, Qd[i * (i + 1) // 2 + j])
    return Q


def eri_tensor(basis: BasisSet, schwarz_threshold: float = DEFAULT_SCHWARZ, max_nao: int = MAX_NAO_ERI) -> np.ndarray:
    """Full (mn|ls) tensor, (nao,)*4 (test and debug sizes; 8 nao^4 bytes)."""
    n = basis.nao
    if n > max_nao:
        raise MemoryError(f"ERI tensor for nao = {n} needs {8 * n ** 4 / 1e9:.1f} GB; "
                          f"raise max_nao (currently {max_nao}) if you really want it")
    return engine_for(basis).eri_tensor(schwarz_threshold).cpu().numpy()


def jk_from_eri(eri, densities):
    """J_mn = sum (mn|ls) D_ls, K_mn = sum (ml|ns) D_ls from a stored tensor (any D)."""
    E = torch.as_tensor(np.asarray(eri, dtype=float), device="cuda")
    D = torch.as_tensor(np.asarray(densities, dtype=float), device="cuda")
    single = D.dim() == 2
    D3 = D[None] if single else D
    J = torch.einsum("ijkl,skl->sij", E, D3)
    K = torch.einsum("ikjl,skl->sij", E, D3)
    J, K = J.cpu().numpy(), K.cpu().numpy()
    return (J[0], K[0]) if single else (J, K)


def jk_device(basis: BasisSet, D: torch.Tensor, schwarz_threshold: float = DEFAULT_SCHWARZ,
              symmetric: bool | None = None, fp32_cutoff: float = 0.0) -> tuple[torch.Tensor, torch.Tensor]:
    """
    Integral-direct J, K for a stack D[nset, n, n] (CUDA float64). Symmetric
    densities take one pass; otherwise J uses the symmetric part and
    K = A(D) + A(D^T)^T from a pass over [D, D^T]. Quartets with
    Q1 Q2 < fp32_cutoff are evaluated in FP32 (0: all FP64).
    """
    eng = engine_for(basis)
    if symmetric is None:
        symmetric = bool(torch.equal(D, D.transpose(1, 2)))
    if symmetric:
        Ja, Ka = eng.jk_acc(D, schwarz_threshold, fp32_cutoff)
        return Ja + Ja.transpose(1, 2), Ka + Ka.transpose(1, 2)
    m = D.shape[0]
    Ja, Ka = eng.jk_acc(torch.cat([D, D.transpose(1, 2)]).contiguous(), schwarz_threshold, fp32_cutoff)
    Jh = Ja + Ja.transpose(1, 2)
    return 0.5 * (Jh[:m] + Jh[m:]), Ka[:m] + Ka[m:].transpose(1, 2)


def jk(basis: BasisSet, densities, schwarz_threshold: float = DEFAULT_SCHWARZ):
    """J, K of ``densities`` ((n, n) or (nset, n, n)) without storing ERIs; numpy in, numpy out."""
    D = np.asarray(densities, dtype=float)
    single = D.ndim == 2
    J, K = jk_device(basis, _t(D[None] if single else D), schwarz_threshold)
    J, K = J.cpu().numpy(), K.cpu().numpy()
    return (J[0], K[0]) if single else (J, K)


def gamma_bound(Dc: torch.Tensor, Dx: torch.Tensor, k_factor: float) -> float:
    """An upper bound of max|Gamma| over all quartets (degeneracy <= 4)."""
    dc = float(Dc.abs().max())
    dx = float(Dx.abs().amax(dim=(1, 2)).pow(2).sum()) if Dx.shape[0] else 0.0
    return max(4.0 * (dc * dc + abs(k_factor) * dx), 1e-300)


def two_electron_gradient_device(basis: BasisSet, Dc: torch.Tensor, Dx: torch.Tensor, k_factor: float,
                                 schwarz_threshold: float = DEFAULT_SCHWARZ_GRAD,
                                 fp32_cutoff: float = 0.0) -> torch.Tensor:
    """d/dR of 1/2 sum Gamma (mn|ls) at fixed symmetric densities, (natm, 3) on the device."""
    eng = engine_for(basis)
    return eng.grad2e(Dc, Dx, k_factor, schwarz_threshold, gamma_bound(Dc, Dx, k_factor), fp32_cutoff)


def two_electron_gradient(basis: BasisSet, D_coulomb, D_exchange_list: Sequence, k_factor: float,
                          schwarz_threshold: float = DEFAULT_SCHWARZ_GRAD) -> np.ndarray:
    """
    d/dR of E2 = 1/2 sum Dc_mn Dc_ls (mn|ls) - k/2 sum_s sum Ds_ml Ds_ns (mn|ls)
    (RHF: Dc = P, [P], k = 1/2; UHF: Dc = Pa + Pb, [Pa, Pb], k = 1).
    """
    n = basis.nao
    Dc = _t(_check_sym(D_coulomb, n, "D_coulomb"))
    Dx = _t(np.array([_check_sym(d, n, "D_exchange_list entry") for d in D_exchange_list]).reshape(-1, n, n))
    return two_electron_gradient_device(basis, Dc, Dx, k_factor, schwarz_threshold).cpu().numpy()


# ---------------------------------------------------------------- one-electron

def one_electron_device(basis: BasisSet, origin=None):
    """(S, T, M, V) on the device; M is the (3, n, n) dipole <m|r - O|n>."""
    return engine_for(basis).onee(origin)


def overlap_matrix(basis: BasisSet) -> np.ndarray:
    return one_electron_device(basis)[0].cpu().numpy()


def kinetic_matrix(basis: BasisSet) -> np.ndarray:
    return one_electron_device(basis)[1].cpu().numpy()


def dipole_integrals(basis: BasisSet, origin: Sequence[float] | None = None) -> np.ndarray:
    return one_electron_device(basis, origin)[2].cpu().numpy()


def nuclear_attraction_matrix(basis: BasisSet) -> np.ndarray:
    return one_electron_device(basis)[3].cpu().numpy()


def one_electron_matrices(basis: BasisSet):
    S, T, _, V = one_electron_device(basis)
    return S.cpu().numpy(), T.cpu().numpy(), V.cpu().numpy()


def one_electron_gradient_device(basis: BasisSet, D: torch.Tensor, W: torch.Tensor) -> torch.Tensor:
    """d/dR [sum D (T + V)] - d/dR [sum W S] for symmetric D, W on the device."""
    return engine_for(basis).onee_grad(-W, D)


def one_electron_gradient(basis: BasisSet, D, W) -> np.ndarray:
    n = basis.nao
    return one_electron_gradient_device(basis, _t(_check_sym(D, n, "D")), _t(_check_sym(W, n, "W"))).cpu().numpy()


# ---------------------------------------------------------------- nuclei

def nuclear_repulsion_energy(charges, positions) -> float:
    """E_nuc = sum_{A<B} Z_A Z_B / R_AB."""
    q = np.asarray(charges, dtype=float).reshape(-1)
    x = np.asarray(positions, dtype=float).reshape(-1, 3)
    i, j = np.triu_indices(len(q), k=1)
    return float(np.sum(q[i] * q[j] / np.linalg.norm(x[i] - x[j], axis=1)))


def nuclear_repulsion_gradient(charges, positions) -> np.ndarray:
    """dE_nuc/dR_A = -sum_B Z_A Z_B (R_A - R_B) / R_AB^3."""
    q = np.asarray(charges, dtype=float).reshape(-1)
    x = np.asarray(positions, dtype=float).reshape(-1, 3)
    i, j = np.triu_indices(len(q), k=1)
    d = x[i] - x[j]
    pair = -(q[i] * q[j] / np.linalg.norm(d, axis=1) ** 3)[:, None] * d
    g = np.zeros_like(x)
    np.add.at(g, i, pair)
    np.add.at(g, j, -pair)
    return g


def nuclear_dipole(charges, positions, origin=None) -> np.ndarray:
    q = np.asarray(charges, dtype=float).reshape(-1)
    x = np.asarray(positions, dtype=float).reshape(-1, 3)
    o = np.zeros(3) if origin is None else np.asarray(origin, dtype=float).reshape(3)
    return q @ (x - o)
