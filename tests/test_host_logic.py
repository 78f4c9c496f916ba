"""Host-side logic that needs no GPU: basis layout, options, block splitting, geometry generators."""

import numpy as np
import pytest

from aimd_b200 import geometry as G
from aimd_b200.basis import build_basis, normalize_basis_name
from aimd_b200.engine import device_blocks
from aimd_b200.scf import SCFOptions, electron_counts, check_nuclear_separation


def test_basis_names_and_sizes():
    assert normalize_basis_name("6-31G*") == "6-31g*"
    assert normalize_basis_name(" 6-31G(d,p) ") == "6-31g**"
    assert normalize_basis_name("cc-pVDZ") == "cc-pvdz"
    with pytest.raises(ValueError):
        normalize_basis_name("def2-tzvp")
    sym, pos = G.water()
    assert build_basis(sym, pos, "6-31g*").nao == 19
    sym, pos = G.methanol()
    assert build_basis(sym, pos, "6-31g**").nao == 50
    sym, pos = G.water_cluster(8, seed=0)
    assert build_basis(sym, pos, "cc-pvdz").nao == 200


def test_basis_arrays_match_reference_fixture(golden):
    g = golden("water_ccpvdz")
    b = build_basis([str(s) for s in g["symbols"]], g["positions"], "cc-pvdz")
    assert b.nao == g["density"].shape[0]
    assert list(b.blk_ncon) == [2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1]


def test_device_blocks_split_over_cap_contractions():
    # Cl cc-pVDZ: s block with 3 contractions, p block with 2
    b = build_basis(["Cl"], np.zeros((1, 3)), "cc-pvdz")
    blk = device_blocks(b)
    assert blk["split"]
    assert all(n <= (2 if l == 0 else 1) for l, n in zip(blk["l"], blk["ncon"]))
    # every AO is covered exactly once
    covered = []
    for l, n, ao in zip(blk["l"], blk["ncon"], blk["ao"]):
        nc = (l + 1) * (l + 2) // 2
        covered.extend(range(ao, ao + n * nc))
    assert sorted(covered) == list(range(b.nao))
    # H/C/N/O bases need no split
    sym, pos = G.water()
    assert not device_blocks(build_basis(sym, pos, "cc-pvdz"))["split"]


def test_scf_options_and_electron_counts():
    with pytest.raises(ValueError):
        SCFOptions(conv_energy=0.0)
    with pytest.raises(ValueError):
        SCFOptions(damping=1.0)
    with pytest.raises(ValueError):
        SCFOptions(fock_rebuild=0)
    with pytest.raises(ValueError):
        SCFOptions(fp32_cutoff=-1.0)
    with pytest.raises(ValueError):
        SCFOptions(fp32_cutoff=float("inf"))
    assert SCFOptions().fp32_cutoff == 0.0
    assert SCFOptions().incremental_fock and SCFOptions(incremental_fock=False).fock_rebuild >= 1
    assert electron_counts(10, 0, 1, "rhf") == (5, 5)
    assert electron_counts(9, 0, 2) == (5, 4)
    with pytest.raises(ValueError):
        electron_counts(9, 0, 2, "rhf")
    with pytest.raises(ValueError):
        check_nuclear_separation(np.zeros((2, 3)), np.array([1, 1]))


def test_water_cluster_geometry():
    sym, pos = G.water_cluster(32, seed=1)
    assert sym.count("O") == 32 and len(sym) == 96
    o = pos[0::3] / 1.8897261254578281
    d = np.linalg.norm(o[:, None] - o[None], axis=-1) + np.eye(32) * 10
    assert d.min() >= 2.7 - 1e-12
    r = np.linalg.norm(pos[1::3] - pos[0::3], axis=1) / 1.8897261254578281
    np.testing.assert_allclose(r, 0.9572, atol=1e-12)


def test_random_molecules_are_valid():
    for seed in range(64):
        sym, pos = G.random_molecule(seed)
        assert 3 <= len(sym) <= 20
        assert set(sym) <= {"H", "C", "N", "O"}


def test_batch_default_multiplicity():
    from aimd_b200.batch import default_multiplicity
    assert default_multiplicity(["O", "H", "H"]) == 1
    assert default_multiplicity(["C", "H", "H", "H"]) == 2
    assert default_multiplicity(["C", "H", "H", "H"], charge=1) == 1


def test_autograd_and_batch_argument_checks():
    import torch
    from aimd_b200.autograd import scf_energy
    from aimd_b200.batch import BatchSolver
    with pytest.raises(TypeError):
        scf_energy(np.zeros((3, 3)), None)                     # not a tensor
    with pytest.raises(ValueError):
        scf_energy(torch.zeros(3, 2, dtype=torch.float64), None)   # not (natm, 3)
    with pytest.raises(ValueError):
        BatchSolver([], workers=0)
