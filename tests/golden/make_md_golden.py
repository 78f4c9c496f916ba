"""
MD fixtures from the REFERENCE (Nathan-W123/Ab-Initio-MD): NVE
velocity-Verlet trajectories driven by the reference's own HF backend and
integrator, from the same initial conditions the GPU tests use, so that the
energy conservation of the two codes can be compared step by step.

    NUMBA_CACHE_DIR=<writable dir> python tests/golden/make_md_golden.py <reference source tree>

  nve_water_631gs.npz     water RHF/6-31G*, 300 K Maxwell-Boltzmann start
                          (aimd_b200.md.maxwell_boltzmann, seed 7), 1 ps at
                          dt = 0.5 fs (2000 steps) and at dt = 0.25 fs (4000)
  nve_methanol_631gss.npz methanol RHF/6-31G** (50 AOs), 300 K start (seed 1),
                          200 steps at dt = 0.5 fs
Each holds the initial positions/velocities and, per step, the potential
and total energy (Eh).
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _run(ref_modules, sym, pos, vel, basis, dt_fs, nsteps):
    MolecularSystem, HFBackend, VelocityVerlet = ref_modules
    system = MolecularSystem(list(sym), np.array(pos, dtype=float), velocities=np.array(vel, dtype=float))
    integ = VelocityVerlet(HFBackend(list(sym), basis=basis), dt_fs)
    res = integ.initialize(system)
    epot = [res.energy]
    etot = [res.energy + system.kinetic_energy()]
    for _ in range(nsteps):
        res = integ.step(system)
        epot.append(res.energy)
        etot.append(res.energy + system.kinetic_energy())
    return np.array(epot), np.array(etot), system.positions.copy()


def main() -> None:
    if len(sys.argv) != 2:
        sys.exit("usage: make_md_golden.py <reference source tree>")
    sys.path.insert(0, sys.argv[1])
    sys.path.insert(0, os.path.join(REPO, "ab-initio-md_b200"))
    from aimd.backends.hf import HFBackend
    from aimd.integrators import VelocityVerlet
    from aimd.system import MolecularSystem
    from aimd_b200 import geometry as G
    from aimd_b200.md import maxwell_boltzmann
    mods = (MolecularSystem, HFBackend, VelocityVerlet)

    sym, pos = G.water()
    vel = maxwell_boltzmann(sym, 300.0, 7)
    out = {"symbols": np.array(sym), "positions": pos, "velocities": vel, "basis": np.array("6-31g*")}
    for dt, n, tag in ((0.5, 2000, "dt05"), (0.25, 4000, "dt025")):
        t0 = time.perf_counter()
        epot, etot, xf = _run(mods, sym, pos, vel, "6-31g*", dt, n)
        out[f"{tag}_epot"], out[f"{tag}_etot"], out[f"{tag}_final_positions"] = epot, etot, xf
        print(f"water dt {dt}: max|E-E0| {np.abs(etot - etot[0]).max():.3e} Eh ({time.perf_counter() - t0:.0f} s)",
              flush=True)
    np.savez_compressed(os.path.join(HERE, "nve_water_631gs.npz"), **out)

    sym, pos = G.methanol()
    vel = maxwell_boltzmann(sym, 300.0, 1)
    t0 = time.perf_counter()
    epot, etot, xf = _run(mods, sym, pos, vel, "6-31g**", 0.5, 200)
    print(f"methanol: max|E-E0| {np.abs(etot - etot[0]).max():.3e} Eh ({time.perf_counter() - t0:.0f} s)", flush=True)
    np.savez_compressed(os.path.join(HERE, "nve_methanol_631gss.npz"), symbols=np.array(sym), positions=pos,
                        velocities=vel, basis=np.array("6-31g**"), dt05_epot=epot, dt05_etot=etot,
                        dt05_final_positions=xf)


if __name__ == "__main__":
    main()
