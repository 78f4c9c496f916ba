"""
MD observables against the reference's own trajectories. golden/nve_*.npz
were made by golden/make_md_golden.py with the reference's HF backend and
velocity-Verlet integrator from the same initial conditions; here the same
NVE runs use forces from the autograd path (HFEnergy: forward = device SCF,
backward = the derivative kernels) in a plain velocity-Verlet loop.

* water RHF/6-31G*, 300 K start, 1 ps at dt = 0.5 fs (2000 steps): the
  potential energy of every step within 1e-6 Eh of the reference's, and the
  energy-conservation figures within 10 % of the reference's: max
  |E_tot - E_tot(0)| and the fitted drift (a drift this far below the
  fluctuation is compared with an absolute floor of 1e-7 Eh/ps); the
  fluctuation at dt = 0.5 and 0.25 fs over 100 fs in the O(dt^2) ratio of
  velocity Verlet (3.5-4.5, the reference's own test bounds).
* methanol RHF/6-31G** (the 200-step NVE configuration): potential energy
  per step within 1e-6 Eh and max |E_tot - E_tot(0)| within 10 % of the
  reference's run.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _nve(sym, pos, vel, basis, dt_fs, nsteps):
    from aimd_b200.autograd import HFEnergy
    from aimd_b200.md import masses_au
    from aimd_b200.units import FS_TO_AU_TIME
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    f = HFEnergy([str(s) for s in sym], basis)
    m = masses_au([str(s) for s in sym])[:, None]
    x = np.array(pos, dtype=float)
    v = np.array(vel, dtype=float)
    dt = dt_fs * FS_TO_AU_TIME
    e, F = f.energy_and_forces(x)
    epot, etot = [e], [e + 0.5 * float((m * v * v).sum())]
    for _ in range(nsteps):
        v += 0.5 * dt * F / m
        x += dt * v
        e, F = f.energy_and_forces(x)
        v += 0.5 * dt * F / m
        epot.append(e)
        etot.append(e + 0.5 * float((m * v * v).sum()))
    return np.array(epot), np.array(etot)


def _drift(etot, dt_fs):
    t_ps = np.arange(len(etot)) * dt_fs * 1e-3
    return float(np.polyfit(t_ps, etot, 1)[0])


def _within(ours, ref, rel=0.10, floor=0.0):
    return abs(ours - ref) <= max(rel * abs(ref), floor)


def test_nve_water_matches_reference_energy_conservation(golden):
    g = golden("nve_water_631gs")
    epot, etot = _nve(g["symbols"], g["positions"], g["velocities"], str(g["basis"]), 0.5, 2000)
    assert np.abs(epot - g["dt05_epot"]).max() < 1e-6
    dev, dev_ref = np.abs(etot - etot[0]).max(), np.abs(g["dt05_etot"] - g["dt05_etot"][0]).max()
    drift, drift_ref = _drift(etot, 0.5), _drift(g["dt05_etot"], 0.5)
    print(f"water NVE 1 ps: max|E-E0| {dev:.3e} (reference {dev_ref:.3e}) Eh, "
          f"drift {drift:+.2e} (reference {drift_ref:+.2e}) Eh/ps")
    assert _within(dev, dev_ref)
    assert _within(drift, drift_ref, floor=1e-7)
    # O(dt^2): the fluctuation over the first 100 fs at half the step
    _, etot_h = _nve(g["symbols"], g["positions"], g["velocities"], str(g["basis"]), 0.25, 400)
    ratio = np.abs(etot[:201] - etot[0]).max() / np.abs(etot_h - etot_h[0]).max()
    ref_ratio = (np.abs(g["dt05_etot"][:201] - g["dt05_etot"][0]).max()
                 / np.abs(g["dt025_etot"][:401] - g["dt025_etot"][0]).max())
    assert 3.5 < ratio < 4.5, ratio
    assert _within(ratio, ref_ratio)


def test_nve_methanol_200_steps_matches_reference(golden):
    g = golden("nve_methanol_631gss")
    epot, etot = _nve(g["symbols"], g["positions"], g["velocities"], str(g["basis"]), 0.5, 200)
    assert np.abs(epot - g["dt05_epot"]).max() < 1e-6
    dev, dev_ref = np.abs(etot - etot[0]).max(), np.abs(g["dt05_etot"] - g["dt05_etot"][0]).max()
    print(f"methanol NVE 200 steps: max|E-E0| {dev:.3e} (reference {dev_ref:.3e}) Eh")
    assert _within(dev, dev_ref)
