"""
Minimal MD drivers around the GPU backend, for the benchmark workloads:
velocity Verlet, the CSVR thermostat (Bussi, Donadio & Parrinello 2007) and
XL-BOMD with dissipation (Niklasson et al., J. Chem. Phys. 130, 214109
(2009), Table I coefficients). They follow the reference's callers
(aimd/integrators.py:215-232, aimd/thermostats.py:162-231,
aimd/xlbomd.py:78-145) step for step; the integrators themselves are not
part of the GPU hot path, they only call ``backend.compute`` and
``backend.set_density_guess``.
"""

from __future__ import annotations

import math

import numpy as np

from .elements import ATOMIC_MASSES_AMU
from .units import AMU_TO_AU, FS_TO_AU_TIME, KB_AU

# K: (kappa, alpha, c_0..c_K) from Niklasson et al. (2009), Table I
XL_COEFFICIENTS = {
    3: (1.69, 150e-3, (-2, 3, 0, -1)),
    4: (1.75, 57e-3, (-3, 6, -2, -2, 1)),
    5: (1.82, 18e-3, (-6, 14, -8, -3, 4, -1)),
    6: (1.84, 5.5e-3, (-14, 36, -27, -2, 12, -6, 1)),
    7: (1.86, 1.6e-3, (-36, 99, -88, 11, 32, -25, 8, -1)),
}


def masses_au(symbols) -> np.ndarray:
    return np.array([ATOMIC_MASSES_AMU[s] for s in symbols]) * AMU_TO_AU


def maxwell_boltzmann(symbols, temperature_k: float, seed: int) -> np.ndarray:
    """Velocities at T with the centre-of-mass motion removed, rescaled to T exactly (3N - 3 DOF)."""
    rng = np.random.default_rng(seed)
    m = masses_au(symbols)
    v = rng.normal(size=(len(m), 3)) * np.sqrt(KB_AU * temperature_k / m)[:, None]
    v -= (m[:, None] * v).sum(axis=0) / m.sum()
    t_now = (m[:, None] * v * v).sum() / ((3 * len(m) - 3) * KB_AU)
    return v * math.sqrt(temperature_k / t_now) if t_now > 0 else v


class AuxiliaryDensity:
    """P(t+dt) = 2P - P_prev + kappa (D - P) + alpha sum_k c_k P(t - k dt)."""

    def __init__(self, k: int = 5) -> None:
        self.kappa, self.alpha, c = XL_COEFFICIENTS[k]
        self.c = np.array(c, dtype=float)
        self.k = k
        self.history = None

    def reset(self, D) -> None:
        self.history = [D.copy() for _ in range(self.k + 1)]

    def propagate(self, D):
        h = self.history
        diss = self.c[0] * h[0]
        for ck, pk in zip(self.c[1:], h[1:]):
            diss = diss + ck * pk
        p_next = 2.0 * h[0] - h[1] + self.kappa * (D - h[0]) + self.alpha * diss
        self.history = [p_next] + h[:-1]
        return p_next.copy()


class CSVR:
    """Stochastic velocity rescaling applied for dt/2 before and after each step."""

    def __init__(self, temperature_k: float, tau_fs: float, seed: int, n_dof: int) -> None:
        self.kT = KB_AU * temperature_k
        self.tau = tau_fs * FS_TO_AU_TIME
        self.rng = np.random.default_rng(seed)
        self.n_dof = n_dof
        self.heat = 0.0

    def rescale(self, v: np.ndarray, m: np.ndarray, t: float) -> np.ndarray:
        ekin = 0.5 * float((m[:, None] * v * v).sum())
        if ekin <= 0.0:
            return v
        c = math.exp(-t / self.tau)
        q = (1.0 - c) * 0.5 * self.kT / ekin
        r1 = float(self.rng.standard_normal())
        s = 2.0 * float(self.rng.standard_gamma(0.5 * (self.n_dof - 1))) if self.n_dof > 1 else 0.0
        along = math.sqrt(c) + r1 * math.sqrt(q)
        a2 = along * along + q * s
        self.heat += ekin * (a2 - 1.0)
        return v * math.copysign(math.sqrt(a2), along)


class XLBOMDRun:
    """
    Velocity Verlet (NVE, or NVT with CSVR) with the XL-BOMD density guess,
    driving any backend with the density-guess protocol.
    """

    def __init__(self, backend, symbols, positions, velocities, timestep_fs: float, k: int = 5,
                 thermostat: CSVR | None = None, xl: bool = True) -> None:
        self.backend = backend
        self.m = masses_au(symbols)
        self.x = np.array(positions, dtype=float)
        self.v = np.array(velocities, dtype=float)
        self.dt = timestep_fs * FS_TO_AU_TIME
        self.thermo = thermostat
        self.aux = AuxiliaryDensity(k) if xl else None
        self.result = backend.compute(self.x)
        if self.aux is not None:
            self.aux.reset(self.result.density)

    def _accel(self) -> np.ndarray:
        return -self.result.gradient / self.m[:, None]

    def step(self):
        dt = self.dt
        if self.thermo is not None:
            self.v = self.thermo.rescale(self.v, self.m, 0.5 * dt)
        self.v += 0.5 * dt * self._accel()
        self.x += dt * self.v
        if self.aux is not None:
            self.backend.set_density_guess(self.aux.propagate(self.result.density))
        self.result = self.backend.compute(self.x)
        self.v += 0.5 * dt * self._accel()
        if self.thermo is not None:
            self.v = self.thermo.rescale(self.v, self.m, 0.5 * dt)
        return self.result

    def conserved_energy(self) -> float:
        ekin = 0.5 * float((self.m[:, None] * self.v * self.v).sum())
        heat = self.thermo.heat if self.thermo is not None else 0.0
        return self.result.energy + ekin - heat


class DeviceXLBOMD:
    """
    The same velocity Verlet + CSVR + XL-BOMD scheme with the auxiliary
    density history and the SCF densities kept on the device; only positions
    (natm x 3), forces and scalars cross to the host. Forces come from the
    differentiable SCF energy (aimd_b200.autograd.scf_energy): the forward
    pass is the device SCF from the XL-BOMD guess, the backward pass the
    derivative kernels (autograd=True, the default), or from the analytic
    gradient called directly (autograd=False; the same kernels).
    """

    def __init__(self, solver, symbols, positions, velocities, timestep_fs: float, k: int = 5,
                 thermostat: CSVR | None = None, gradient_screening: float = 1e-14, autograd: bool = True) -> None:
        import torch

        from .gradients import scf_gradient_device
        from .scf import run_device
        self._run, self._grad = run_device, scf_gradient_device
        self.torch = torch
        self.autograd = autograd
        self.phase_events = None
        self.solver = solver
        self.m = masses_au(symbols)
        self.x = np.array(positions, dtype=float)
        self.v = np.array(velocities, dtype=float)
        self.dt = timestep_fs * FS_TO_AU_TIME
        self.thermo = thermostat
        self.thr = gradient_screening
        self.fp32_cutoff = solver.options.fp32_cutoff
        kappa, alpha, c = XL_COEFFICIENTS[k]
        self.kappa, self.alpha, self.c = kappa, alpha, [float(v) for v in c]
        self.state, self.gradient = self._forces(None)
        D = self._density(self.state)
        self.history = [D.clone() for _ in range(k + 1)]
        self.iterations = [self.state.iterations]

    def _density(self, st):
        return st.spin if st.unrestricted else st.spin[0] + st.spin[1]

    def _event(self):
        ev = self.torch.cuda.Event(enable_timing=True)
        ev.record()
        return ev

    def _forces(self, guess):
        """
        (SCF state, dE/dR) at self.x from the device density ``guess``. With
        ``phase_events`` a list, appends CUDA events (start, SCF done,
        gradient done) of the call, for timing the two phases separately.
        """
        evs = self.phase_events
        e0 = self._event() if evs is not None else None
        if not self.autograd:
            st = self._run(self.solver, self.x, guess)
            e1 = self._event() if evs is not None else None
            g = self._grad(st, self.thr, self.fp32_cutoff)
        else:
            from .autograd import scf_energy
            x = self.torch.as_tensor(self.x).clone().requires_grad_(True)
            holder: dict = {}
            e = scf_energy(x, self.solver, guess, holder, gradient_screening=self.thr)
            e1 = self._event() if evs is not None else None
            (g,) = self.torch.autograd.grad(e, x)
            st = holder["state"]
        if evs is not None:
            evs.append((e0, e1, self._event()))
        return st, g

    def step(self):
        dt = self.dt
        if self.thermo is not None:
            self.v = self.thermo.rescale(self.v, self.m, 0.5 * dt)
        acc = -self.gradient.cpu().numpy() / self.m[:, None]
        self.v += 0.5 * dt * acc
        self.x += dt * self.v
        h = self.history
        D = self._density(self.state)
        diss = self.c[0] * h[0]
        for ck, pk in zip(self.c[1:], h[1:]):
            diss = diss + ck * pk
        guess = 2.0 * h[0] - h[1] + self.kappa * (D - h[0]) + self.alpha * diss
        self.history = [guess] + h[:-1]
        self.state, self.gradient = self._forces(guess)
        acc = -self.gradient.cpu().numpy() / self.m[:, None]
        self.v += 0.5 * dt * acc
        if self.thermo is not None:
            self.v = self.thermo.rescale(self.v, self.m, 0.5 * dt)
        self.iterations.append(self.state.iterations)
        return self.state

    def conserved_energy(self) -> float:
        ekin = 0.5 * float((self.m[:, None] * self.v * self.v).sum())
        heat = self.thermo.heat if self.thermo is not None else 0.0
        return self.state.energy + ekin - heat
