"""
Batched SCF + gradient over molecules of uneven size (aimd_b200.batch):
concurrent workers on separate CUDA streams give the results of running each
molecule alone, and agree with the public backend on one of them.
"""

import numpy as np
import pytest

from aimd_b200 import geometry as G
from aimd_b200.backend import HFGPUBackend
from aimd_b200.batch import BatchSolver, default_multiplicity

pytestmark = pytest.mark.gpu


def _molecules(n, seed0=100):
    return [G.random_molecule(seed0 + k) for k in range(n)]


def test_batch_equals_one_at_a_time():
    mols = _molecules(6)
    conc = BatchSolver(mols, "6-31g*", workers=4).run()
    seq = BatchSolver(mols, "6-31g*", workers=1).run()
    for a, b in zip(conc, seq):
        assert a.converged and b.converged
        assert abs(a.energy - b.energy) < 1e-10
        np.testing.assert_allclose(a.gradient, b.gradient, atol=1e-9)
        np.testing.assert_allclose(a.dipole, b.dipole, atol=1e-8)


def test_batch_matches_backend_and_reruns():
    mols = _molecules(3, seed0=7)
    bs = BatchSolver(mols, "6-31g*", workers=3)
    res = bs.run()
    sym, pos = mols[1]
    r = HFGPUBackend(sym, basis="6-31g*", multiplicity=default_multiplicity(sym)).compute(pos)
    assert abs(res[1].energy - r.energy) < 1e-9
    np.testing.assert_allclose(res[1].gradient, r.gradient, atol=1e-7)
    np.testing.assert_allclose(res[1].dipole, r.dipole, atol=1e-6)
    moved = [p + 0.01 for _, p in mols]            # rigid shift: same energies
    res2 = bs.run(moved)
    for a, b in zip(res, res2):
        assert abs(a.energy - b.energy) < 1e-8
        # the dipole of a neutral molecule does not depend on the origin
        np.testing.assert_allclose(a.dipole, b.dipole, atol=1e-6)


def test_batch64_against_oracle():
    """
    The batched configuration at full size: 64 random H/C/N/O molecules of
    3-20 atoms in 6-31G* (RHF, or UHF for odd electron counts), SCF + gradient
    in one batch, each against the oracle's own SCF and gradient of that
    molecule (energies within 1e-9 Eh, forces within 1e-7 Eh/bohr, dipoles
    within 1e-6 e bohr).
    """
    from oracle import hf_oracle as O
    mols = _molecules(64, seed0=1000)
    res = BatchSolver(mols, "6-31g*", workers=8).run()
    assert len(res) == 64
    worst = (0.0, 0.0)
    for (sym, pos), r in zip(mols, res):
        assert r.converged
        ref = O.run_scf(sym, pos, "6-31g*", multiplicity=default_multiplicity(sym))
        assert ref["converged"]
        de = abs(r.energy - ref["energy"])
        df = float(np.abs(r.gradient - O.scf_gradient(ref)).max())
        worst = (max(worst[0], de), max(worst[1], df))
        assert de < 1e-9, (sym, de)
        assert df < 1e-7, (sym, df)
        np.testing.assert_allclose(r.dipole, ref["dipole"], atol=1e-6)
    print(f"batch64: max |dE| {worst[0]:.2e} Eh, max |dF| {worst[1]:.2e} Eh/bohr")
