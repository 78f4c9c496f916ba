"""
The C-ABI device SCF driver (include/aimd_scf.h, aimd_scf_run) against the
reference's SCF energies (golden fixtures made by the reference itself) and
its status word: converged runs reach the reference energy within 1e-9 Eh
from the atomic guess and from the core-Hamiltonian guess; a run cut short
reports AIMD_SCF_MAX_ITER; a non-finite starting density is reported as
AIMD_SCF_NONFINITE without a fault; impossible options are refused.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

E_TOL = 1e-9


def _solver(g):
    from aimd_b200.scf import SCFSolver
    return SCFSolver([str(s) for s in g["symbols"]], str(g["basis"]), charge=int(g["charge"]),
                     multiplicity=int(g["multiplicity"]))


@pytest.mark.parametrize("case", ["water_631gs", "methanol_631gss", "ch3_uhf_631gs", "hcl_ccpvdz"])
def test_native_scf_matches_reference_energy(golden, case):
    from aimd_b200.scf import run_native
    g = golden(case)
    res = run_native(_solver(g), g["positions"], guess="sad")
    assert res.converged, res.status
    assert abs(res.energy - float(g["energy"])) < E_TOL
    P = (res.spin[0] + res.spin[-1]).cpu().numpy() if res.spin.shape[0] == 2 else 2 * res.spin[0].cpu().numpy()
    np.testing.assert_allclose(P, g["density"], atol=1e-5)
    F = res.fock.cpu().numpy()
    np.testing.assert_allclose(F, F.transpose(0, 2, 1), atol=1e-12)


def test_native_scf_core_guess_and_agreement_with_python_driver(golden):
    from aimd_b200.scf import run_native
    g = golden("water_ccpvdz")
    s = _solver(g)
    res = run_native(s, g["positions"], guess=None)
    assert res.converged and abs(res.energy - float(g["energy"])) < E_TOL
    ref = s.run(g["positions"])
    assert abs(res.energy - ref.energy) < E_TOL


def test_native_scf_status_max_iter_and_nonfinite(golden):
    from aimd_b200 import _lib
    from aimd_b200.scf import run_native
    g = golden("water_631gs")
    s = _solver(g)
    res = run_native(s, g["positions"], guess="sad", max_iter=2)
    assert res.status == _lib.AIMD_SCF_MAX_ITER and res.iterations == 2
    n = s.nao
    bad = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    res = run_native(s, g["positions"], guess=bad)
    assert res.status == _lib.AIMD_SCF_NONFINITE and res.iterations == 1
    # the context is still usable after the non-finite run
    res = run_native(s, g["positions"], guess="sad")
    assert res.converged and abs(res.energy - float(g["energy"])) < E_TOL


def test_native_scf_refuses_impossible_options(golden):
    import ctypes

    from aimd_b200 import _lib
    from aimd_b200.engine import engine_for
    g = golden("water_631gs")
    s = _solver(g)
    Ik = s.integrals(g["positions"])
    eng = engine_for(Ik.basis)
    lib = _lib.load_scf()
    opt = _lib.SCFOptions()
    lib.aimd_scf_default_options(ctypes.byref(opt))
    opt.n_alpha, opt.n_beta, opt.unrestricted = 5, 4, 0          # RHF needs n_alpha == n_beta
    n = Ik.nao
    D = torch.empty((1, n, n), dtype=torch.float64, device="cuda")
    e, it, st = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    r = lib.aimd_scf_run(eng.handle, ctypes.byref(opt), None, ctypes.c_void_p(D.data_ptr()),
                         ctypes.c_void_p(D.data_ptr()), ctypes.byref(e), ctypes.byref(it), ctypes.byref(st), None)
    assert r == _lib.AIMD_ERR_ARG
    assert "invalid options" in lib.aimd_scf_last_error().decode()
