"""
The SCF energy as a differentiable function of the nuclear positions.

``scf_energy(positions, solver)`` returns E(R) (Eh) as a 0-d torch tensor;
``E.backward()`` fills ``positions.grad`` with dE/dR (Eh/bohr). The backward
pass recomputes every integral it needs instead of storing anything from the
forward pass: it is the analytic gradient of a converged SCF,

  dE/dR = sum P dh/dR - sum W dS/dR + 1/2 sum Gamma d(mn|ls)/dR + dV_nn/dR,

with the Pulay term W = sum_s D_s F_s D_s (aimd/qc/gradients.py:106-193),
evaluated by the integral-direct derivative kernels of this package
(one-electron: onee_grad_kernel; two-electron: grad2e_bra_kernel).

Only first derivatives are provided (a second backward raises). The energy
is stationary in the orbitals, so no response equations are needed; the
gradient is exact to the SCF convergence of the forward pass.
"""

from __future__ import annotations

import numpy as np
import torch

from .gradients import scf_gradient_device
from .integrals import DEFAULT_SCHWARZ_GRAD
from .scf import DeviceSCFState, SCFSolver, run_device


class SCFEnergyFunction(torch.autograd.Function):
    """E(R) forward by the device SCF, dE/dR backward by the gradient kernels."""

    @staticmethod
    def forward(ctx, positions: torch.Tensor, solver: SCFSolver, guess, holder: dict, screening: float):
        x = positions.detach().to("cpu", torch.float64).numpy().reshape(-1, 3)
        state = run_device(solver, x, guess)
        holder["state"] = state
        ctx.state = state
        ctx.fp32_cutoff = solver.options.fp32_cutoff
        ctx.screening = screening
        return torch.tensor(state.energy, dtype=torch.float64, device=positions.device)

    @staticmethod
    def backward(ctx, grad_energy: torch.Tensor):
        if ctx.state is None:
            raise RuntimeError("scf_energy: backward called twice (only first derivatives are available)")
        g = scf_gradient_device(ctx.state, ctx.screening, fp32_cutoff=ctx.fp32_cutoff)
        ctx.state = None
        return grad_energy * g.to(grad_energy.device, torch.float64), None, None, None, None


def scf_energy(positions: torch.Tensor, solver: SCFSolver, guess: torch.Tensor | None = None,
               holder: dict | None = None, gradient_screening: float = DEFAULT_SCHWARZ_GRAD) -> torch.Tensor:
    """
    SCF energy (Eh, 0-d float64 tensor) at ``positions`` ((natm, 3) bohr,
    any device), differentiable with respect to ``positions``. ``guess``: a
    device density to start from (as run_device); ``holder``, if given,
    receives the converged DeviceSCFState under "state";
    ``gradient_screening``: the backward pass's threshold on
    Q1 Q2 max|Gamma| (the reference's two-electron gradient screening).
    """
    if not isinstance(positions, torch.Tensor):
        raise TypeError("positions must be a torch.Tensor")
    if positions.dim() != 2 or positions.shape[1] != 3:
        raise ValueError(f"positions must have shape (natm, 3), got {tuple(positions.shape)}")
    return SCFEnergyFunction.apply(positions, solver, guess, {} if holder is None else holder,
                                   float(gradient_screening))


class HFEnergy:
    """
    E(R) of one molecule as a callable: ``HFEnergy(symbols, basis)(R)``
    returns a differentiable energy and reuses the previous converged
    density as the next starting guess (as the reference's backend does
    with ``reuse_density``).
    """

    def __init__(self, symbols, basis: str = "sto-3g", charge: int = 0, multiplicity: int = 1,
                 reference: str | None = None, options=None, **overrides) -> None:
        self.solver = SCFSolver(symbols, basis, charge=charge, multiplicity=multiplicity, reference=reference,
                                options=options, **overrides)
        self.last_state: DeviceSCFState | None = None

    def __call__(self, positions: torch.Tensor) -> torch.Tensor:
        guess = None
        if self.last_state is not None:
            sp = self.last_state.spin
            guess = sp if self.solver.unrestricted else sp[0] + sp[1]
        holder: dict = {}
        e = scf_energy(positions, self.solver, guess, holder)
        self.last_state = holder["state"]
        return e

    def energy_and_forces(self, positions) -> tuple[float, np.ndarray]:
        """(E, -dE/dR) as host values, through one forward and one backward pass."""
        x = torch.as_tensor(np.asarray(positions, dtype=float)).requires_grad_(True)
        e = self(x)
        (g,) = torch.autograd.grad(e, x)
        return float(e), -g.numpy()
