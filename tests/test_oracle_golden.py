"""
Pin the oracle (oracle/: C + numpy restatement of the reference's path)
against fixtures produced by the reference itself (tests/golden). CPU only.
"""

import numpy as np
import pytest

from oracle import hf_oracle as O


def _basis(g):
    return O.build_basis([str(s) for s in g["symbols"]], g["positions"], str(g["basis"]))


def test_boys_matches_reference(golden):
    g = golden("boys")
    for x, F in zip(g["x"], g["F"]):
        np.testing.assert_allclose(O.boys(32, float(x)), F, rtol=1e-14, atol=1e-300)


@pytest.mark.parametrize("case", ["water_631gs", "water_ccpvdz", "methanol_631gss", "ch3_uhf_631gs", "h2s_631gs", "hcl_ccpvdz"])
def test_integrals_match_reference(golden, case):
    g = golden(case)
    b = _basis(g)
    np.testing.assert_allclose(O.schwarz_bounds(b), g["Q"], rtol=1e-13, atol=1e-14)
    eri = O.eri_tensor(b)
    i = g["eri_idx"]
    np.testing.assert_allclose(eri[i[:, 0], i[:, 1], i[:, 2], i[:, 3]], g["eri_val"], rtol=0, atol=1e-13)
    J, K = O.jk_direct(b, g["D_rand"])
    np.testing.assert_allclose(J, g["J_sym"], atol=1e-11)
    np.testing.assert_allclose(K, g["K_sym"], atol=1e-11)
    J, K = O.jk_direct(b, g["D_nonsym"])
    np.testing.assert_allclose(J, g["J_nonsym"], atol=1e-11)
    np.testing.assert_allclose(K, g["K_nonsym"], atol=1e-11)
    S, T, M = O.overlap_type(b, [0.3, -0.2, 0.5])
    np.testing.assert_allclose(S, g["S"], atol=1e-14)
    np.testing.assert_allclose(T, g["T"], atol=1e-13)
    np.testing.assert_allclose(M, g["M"], atol=1e-13)
    np.testing.assert_allclose(O.nuclear_attraction_matrix(b), g["V"], atol=1e-12)
    np.testing.assert_allclose(O.two_electron_gradient(b, g["D_rand"], [g["D_rand"]], 0.5), g["g2e_rhf"], atol=1e-11)
    np.testing.assert_allclose(O.two_electron_gradient(b, g["D_rand"], [g["D_rand"], g["W_rand"]], 1.0),
                               g["g2e_uhf"], atol=1e-11)
    np.testing.assert_allclose(O.one_electron_gradient(b, g["D_rand"], g["W_rand"]), g["g1e"], atol=1e-11)


@pytest.mark.parametrize("case", ["water_631gs", "water_ccpvdz", "methanol_631gss", "ch3_uhf_631gs", "h2s_631gs", "hcl_ccpvdz"])
def test_scf_energy_and_gradient_match_reference(golden, case):
    g = golden(case)
    sym = [str(s) for s in g["symbols"]]
    res = O.run_scf(sym, g["positions"], str(g["basis"]), charge=int(g["charge"]),
                    multiplicity=int(g["multiplicity"]))
    assert res["converged"]
    assert abs(res["energy"] - float(g["energy"])) < 1e-9
    np.testing.assert_allclose(O.scf_gradient(res), g["gradient"], atol=1e-8)
    np.testing.assert_allclose(res["dipole"], g["dipole"], atol=1e-7)


def test_flop_model_matches_reference(golden):
    for case in ["water_631gs", "methanol_631gss", "water_ccpvdz"]:
        g = golden(case)
        m = O.flop_model(_basis(g))
        assert m["flop"] == pytest.approx(float(g["flop_model"]), rel=1e-12)
        assert m["prim_quartets"] == pytest.approx(float(g["prim_quartets"]), rel=1e-12)
