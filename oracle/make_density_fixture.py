"""
Fixture for the CPU timing legs of bench.py (test and measurement
infrastructure, not the product): the converged RHF density of the bench
workload's starting geometry, (H2O)32 cc-pVDZ (800 AOs, water_cluster(32,
seed=1)), computed by the oracle's own SCF (hf_oracle.run_scf). The CPU
reference arm times the oracle's integral-direct Fock build and
two-electron gradient at this density, so that Schwarz/density screening
behaves as in the MD run. Stored as the packed upper triangle in float32
(timing needs realistic magnitudes, not 1e-10 accuracy).

    python oracle/make_density_fixture.py
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "ab-initio-md_b200"))

OUT = os.path.join(HERE, "data", "h2o32_ccpvdz_density.npz")


def main() -> None:
    from aimd_b200 import geometry as G
    from oracle import hf_oracle as O
    sym, pos = G.water_cluster(32, seed=1)
    t0 = time.perf_counter()
    res = O.run_scf(sym, pos, "cc-pvdz")
    P = res["density"]
    iu = np.triu_indices(P.shape[0])
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    np.savez_compressed(OUT, tri=P[iu].astype(np.float32), nao=P.shape[0], energy=res["energy"],
                        converged=res["converged"], iterations=res["iterations"])
    print(f"E = {res['energy']:.10f} Eh, {res['iterations']} iterations, converged {res['converged']}, "
          f"{time.perf_counter() - t0:.0f} s -> {OUT}")


def load() -> np.ndarray:
    """The fixture density as a symmetric float64 (nao, nao) array."""
    z = np.load(OUT)
    n = int(z["nao"])
    P = np.zeros((n, n))
    iu = np.triu_indices(n)
    P[iu] = z["tri"]
    return P + np.triu(P, 1).T


if __name__ == "__main__":
    main()
