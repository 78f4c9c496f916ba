"""
Analytic RHF/UHF nuclear gradients on the GPU, with the reference's API
(``aimd.qc.gradients``, aimd/qc/gradients.py:106-238):

    dE/dR = dE_nuc/dR + sum P d(T+V)/dR + 1/2 sum Gamma d(mn|ls)/dR - sum W dS/dR

with W = sum_s D_s F_s D_s formed from the SCF's last density and Fock
matrix (the convention of aimd/qc/gradients.py:106-125). The one- and
two-electron contractions run in the native kernels; nothing is stored.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import integrals as I
from .scf import SCFResult


def energy_weighted_density(spin_densities, fock):
    """W = sum_s D_s F_s D_s, symmetrised; numpy or torch in, same type out."""
    is_t = isinstance(spin_densities, torch.Tensor)
    D = spin_densities if is_t else np.asarray(spin_densities, dtype=float)
    F = fock if is_t else np.asarray(fock, dtype=float)
    if D.ndim != 3 or D.shape[0] != 2 or D.shape[1] != D.shape[2]:
        raise ValueError(f"spin_densities must have shape (2, nao, nao), got {tuple(D.shape)}")
    n = D.shape[1]
    if tuple(F.shape) == (n, n):
        W = D[0] @ F @ D[0] + D[1] @ F @ D[1]
    elif tuple(F.shape) == (2, n, n):
        W = D[0] @ F[0] @ D[0] + D[1] @ F[1] @ D[1]
    else:
        raise ValueError(f"fock must have shape ({n}, {n}) or (2, {n}, {n}), got {tuple(F.shape)}")
    return 0.5 * (W + W.T)


@dataclass(frozen=True)
class GradientTerms:
    """nuclear repulsion, one-electron (kinetic + nuclear attraction - W dS) and two-electron parts."""
    nuclear_repulsion: np.ndarray
    one_electron: np.ndarray
    two_electron: np.ndarray
    timings: dict[str, float] = field(default_factory=dict)

    @property
    def total(self) -> np.ndarray:
        return self.nuclear_repulsion + self.one_electron + self.two_electron


def _check(result: SCFResult, require_converged: bool) -> None:
    if not isinstance(result, SCFResult):
        raise TypeError(f"expected an SCFResult, got {type(result).__name__}")
    if require_converged and not result.converged:
        raise ValueError(f"SCF not converged ({result.iterations} iterations, commutator "
                         f"{result.commutator_norm:.2e}); its analytic gradient is not dE/dR")


def _device_terms(result: SCFResult, schwarz_threshold: float, fp32_cutoff: float = 0.0):
    b = result.basis
    dev = result.device
    if dev:
        spin, F = dev["spin"], dev["F"]
    else:
        spin = torch.as_tensor(result.spin_densities, device="cuda")
        F = torch.as_tensor(np.asarray(result.fock).reshape(-1, b.nao, b.nao), device="cuda")
    P = spin[0] + spin[1]
    Fm = F[0] if F.shape[0] == 1 else F
    W = energy_weighted_density(spin, Fm)
    g1 = I.one_electron_gradient_device(b, P, W)
    if result.unrestricted:
        Dx, k = spin, 1.0
    else:
        Dx, k = P[None], 0.5
    g2 = I.two_electron_gradient_device(b, P, Dx.contiguous(), k, schwarz_threshold, fp32_cutoff)
    return g1, g2


def scf_gradient_device(state, schwarz_threshold: float = I.DEFAULT_SCHWARZ_GRAD,
                        fp32_cutoff: float = 0.0) -> torch.Tensor:
    """
    Analytic gradient of a DeviceSCFState as a device tensor (nuclear term
    included); quartets with Q1 Q2 < fp32_cutoff in FP32 (0: all FP64).
    """
    b = state.basis
    spin, F = state.spin, state.fock
    P = spin[0] + spin[1]
    W = energy_weighted_density(spin, F[0] if F.shape[0] == 1 else F)
    g = I.one_electron_gradient_device(b, P, W)
    if state.unrestricted:
        Dx, k = spin, 1.0
    else:
        Dx, k = P[None], 0.5
    g = g + I.two_electron_gradient_device(b, P, Dx.contiguous(), k, schwarz_threshold, fp32_cutoff)
    gn = torch.as_tensor(I.nuclear_repulsion_gradient(b.nuclear_charges, b.positions), device=g.device)
    return g + gn


def scf_gradient(result: SCFResult, schwarz_threshold: float = I.DEFAULT_SCHWARZ_GRAD,
                 require_converged: bool = False, blas_threads: int | None = 1,
                 fp32_cutoff: float = 0.0) -> np.ndarray:
    """
    Analytic dE/dR (Eh/bohr, (natm, 3)) of an RHF or UHF SCF result
    (aimd/qc/gradients.py:168-193); ``fp32_cutoff`` > 0 evaluates the
    two-electron quartets with Q1 Q2 below it in FP32 (mixed precision).
    """
    _check(result, require_converged)
    b = result.basis
    g1, g2 = _device_terms(result, schwarz_threshold, fp32_cutoff)
    g = I.nuclear_repulsion_gradient(b.nuclear_charges, b.positions)
    return g + (g1 + g2).cpu().numpy()


def gradient_terms(result: SCFResult, schwarz_threshold: float = I.DEFAULT_SCHWARZ_GRAD,
                   require_converged: bool = False, blas_threads: int | None = 1) -> GradientTerms:
    """The gradient split into its parts, with timings (aimd/qc/gradients.py:196-223)."""
    _check(result, require_converged)
    b = result.basis
    t0 = time.perf_counter()
    gn = I.nuclear_repulsion_gradient(b.nuclear_charges, b.positions)
    t1 = time.perf_counter()
    g1, g2 = _device_terms(result, schwarz_threshold)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    return GradientTerms(gn, g1.cpu().numpy(), g2.cpu().numpy(),
                         {"nuclear": t1 - t0, "electronic": t2 - t1, "total": t2 - t0})


def invariance_residuals(positions, gradient):
    """(net force, net torque about the centroid) of a gradient (aimd/qc/gradients.py:226-238)."""
    x = np.asarray(positions, dtype=float).reshape(-1, 3)
    g = np.asarray(gradient, dtype=float).reshape(-1, 3)
    if x.shape != g.shape:
        raise ValueError(f"positions {x.shape} and gradient {g.shape} differ in shape")
    return g.sum(axis=0), np.cross(x - x.mean(axis=0), g).sum(axis=0)
