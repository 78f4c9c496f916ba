"""
Parity of the CUDA path with the oracle and with the reference's own
outputs (golden fixtures), through the C ABI. Tolerances are those the
product promises for the plain FP64 path: <= 1e-10 Eh per ERI and per J/K
element, <= 1e-9 Eh in SCF energy, <= 1e-7 Eh/bohr in forces.
"""

import numpy as np
import pytest
import torch

from oracle import hf_oracle as O

pytestmark = pytest.mark.gpu

CASES = ["water_631gs", "water_ccpvdz", "methanol_631gss", "ch3_uhf_631gs", "h2s_631gs", "hcl_ccpvdz"]
ERI_TOL = 1e-10
E_TOL = 1e-9
F_TOL = 1e-7


def _basis(g):
    from aimd_b200.basis import build_basis
    return build_basis([str(s) for s in g["symbols"]], g["positions"], str(g["basis"]))


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from aimd_b200 import _lib
    _lib.load()          # fails loudly if the native library is missing


@pytest.mark.parametrize("case", CASES)
def test_schwarz_and_eri_tensor(golden, case):
    from aimd_b200 import integrals as I
    g = golden(case)
    b = _basis(g)
    np.testing.assert_allclose(I.schwarz_bounds(b), g["Q"], rtol=1e-12, atol=1e-13)
    eri = I.eri_tensor(b)
    ob = O.build_basis([str(s) for s in g["symbols"]], g["positions"], str(g["basis"]))
    np.testing.assert_allclose(eri, O.eri_tensor(ob), rtol=0, atol=ERI_TOL)
    i = g["eri_idx"]
    np.testing.assert_allclose(eri[i[:, 0], i[:, 1], i[:, 2], i[:, 3]], g["eri_val"], rtol=0, atol=ERI_TOL)


@pytest.mark.parametrize("case", CASES)
def test_integral_direct_jk(golden, case):
    from aimd_b200 import integrals as I
    g = golden(case)
    b = _basis(g)
    J, K = I.jk(b, g["D_rand"])
    np.testing.assert_allclose(J, g["J_sym"], rtol=0, atol=ERI_TOL * 10)
    np.testing.assert_allclose(K, g["K_sym"], rtol=0, atol=ERI_TOL * 10)
    J, K = I.jk(b, g["D_nonsym"])
    np.testing.assert_allclose(J, g["J_nonsym"], rtol=0, atol=ERI_TOL * 10)
    np.testing.assert_allclose(K, g["K_nonsym"], rtol=0, atol=ERI_TOL * 10)


@pytest.mark.parametrize("case", CASES)
def test_one_electron_integrals(golden, case):
    from aimd_b200 import integrals as I
    g = golden(case)
    b = _basis(g)
    S, T, M, V = (t.cpu().numpy() for t in I.one_electron_device(b, [0.3, -0.2, 0.5]))
    np.testing.assert_allclose(S, g["S"], atol=1e-13)
    np.testing.assert_allclose(T, g["T"], atol=1e-12)
    np.testing.assert_allclose(M, g["M"], atol=1e-12)
    np.testing.assert_allclose(V, g["V"], atol=1e-11)


@pytest.mark.parametrize("case", CASES)
def test_gradient_contractions(golden, case):
    from aimd_b200 import integrals as I
    g = golden(case)
    b = _basis(g)
    D, W = g["D_rand"], g["W_rand"]
    np.testing.assert_allclose(I.two_electron_gradient(b, D, [D], 0.5), g["g2e_rhf"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(I.two_electron_gradient(b, D, [D, W], 1.0), g["g2e_uhf"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(I.one_electron_gradient(b, D, W), g["g1e"], rtol=0, atol=1e-10)


@pytest.mark.parametrize("case", CASES + ["h2o8_ccpvdz"])
def test_scf_energy_gradient_dipole(golden, case):
    from aimd_b200.gradients import scf_gradient
    from aimd_b200.scf import run_scf
    g = golden(case)
    res = run_scf([str(s) for s in g["symbols"]], g["positions"], str(g["basis"]), charge=int(g["charge"]),
                  multiplicity=int(g["multiplicity"]))
    assert res.converged
    assert abs(res.energy - float(g["energy"])) < E_TOL
    np.testing.assert_allclose(scf_gradient(res), g["gradient"], rtol=0, atol=F_TOL)
    np.testing.assert_allclose(res.dipole, g["dipole"], rtol=0, atol=1e-6)


def test_jk_h2o8_against_oracle(golden):
    from aimd_b200 import integrals as I
    g = golden("h2o8_ccpvdz")
    b = _basis(g)
    P = g["density"]
    J, K = I.jk(b, P)
    ob = O.build_basis([str(s) for s in g["symbols"]], g["positions"], "cc-pvdz")
    Jo, Ko = O.jk_direct(ob, P)
    np.testing.assert_allclose(J, Jo, rtol=0, atol=ERI_TOL * 10)
    np.testing.assert_allclose(K, Ko, rtol=0, atol=ERI_TOL * 10)


def test_jk_is_linear_and_repeatable(golden):
    from aimd_b200 import integrals as I
    g = golden("methanol_631gss")
    b = _basis(g)
    D1, D2 = g["D_rand"], g["W_rand"]
    J1, K1 = I.jk(b, D1)
    J2, K2 = I.jk(b, D2)
    J12, K12 = I.jk(b, D1 + D2)
    np.testing.assert_allclose(J12, J1 + J2, atol=1e-11)
    np.testing.assert_allclose(K12, K1 + K2, atol=1e-11)
    Jr, Kr = I.jk(b, D1)
    np.testing.assert_allclose(Jr, J1, atol=1e-13)
    np.testing.assert_allclose(Kr, K1, atol=1e-13)


def test_eri_tensor_is_fp64_whatever_the_context_cutoff(golden):
    """
    C ABI: aimd_eri_tensor evaluates every quartet in FP64 even when the
    context carries an FP32 cutoff (here one above every Schwarz product, so
    a J/K call would run all quartets in FP32), and leaves the cutoff set.
    """
    import ctypes

    from aimd_b200 import _lib
    from aimd_b200.engine import engine_for
    g = golden("water_631gs")
    b = _basis(g)
    eng = engine_for(b)
    ref = eng.eri_tensor(1e-12)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(eng.lib.aimd_set_fp32_cutoff(eng.handle, ctypes.c_double(1e30)), "aimd_set_fp32_cutoff")
    try:
        out = torch.full_like(ref, float("nan"))
        _lib.check(eng.lib.aimd_eri_tensor(eng.handle, ctypes.c_void_p(out.data_ptr()), ctypes.c_double(1e-12),
                                           stream), "aimd_eri_tensor")
        torch.cuda.synchronize()
        assert float((out - ref).abs().max()) <= ERI_TOL
        # the cutoff is still in force for J/K: all-FP32 quartets differ from FP64
        D = torch.as_tensor(g["D_rand"], device="cuda")[None].contiguous()
        J32 = torch.empty_like(D)
        K32 = torch.empty_like(D)
        _lib.check(eng.lib.aimd_jk(eng.handle, 1, ctypes.c_void_p(D.data_ptr()), ctypes.c_void_p(J32.data_ptr()),
                                   ctypes.c_void_p(K32.data_ptr()), ctypes.c_double(1e-12), stream), "aimd_jk")
        eng._fp32_cutoff = 1e30
        J64, _ = eng.jk_acc(D, 1e-12, 0.0)
        assert float((J32 - J64).abs().max()) > 0.0
    finally:
        eng._precision(0.0)


@pytest.mark.parametrize("case", ["water_ccpvdz", "methanol_631gss"])
def test_jk_with_k_rows_in_global_memory(golden, case, monkeypatch):
    """
    The J/K path that large bases take when a CTA's shared K rows (NF x nao
    doubles) would not fit, forced here for every bra class with
    AIMD_JK_GLOBAL_K_ROWS=1 (read when the context is created).
    """
    from aimd_b200 import integrals as I
    monkeypatch.setenv("AIMD_JK_GLOBAL_K_ROWS", "1")
    g = golden(case)
    b = _basis(g)                      # a fresh basis object: a fresh native context
    J, K = I.jk(b, g["D_rand"])
    np.testing.assert_allclose(J, g["J_sym"], rtol=0, atol=ERI_TOL * 10)
    np.testing.assert_allclose(K, g["K_sym"], rtol=0, atol=ERI_TOL * 10)
