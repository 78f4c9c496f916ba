"""
Mixed precision (quartets with Schwarz product Q1 Q2 below a cutoff in FP32,
FP64 accumulation) against the plain FP64 path on the same inputs. Bars:
energies within 1e-6 Eh and forces within 1e-5 Eh/bohr of FP64; a cutoff
of 0 is the FP64 path itself.
"""

import numpy as np
import pytest
import torch

from aimd_b200 import geometry as G
from aimd_b200 import integrals as I
from aimd_b200.basis import build_basis
from aimd_b200.engine import engine_for
from aimd_b200.gradients import scf_gradient_device
from aimd_b200.scf import SCFOptions, SCFSolver, run_device

pytestmark = pytest.mark.gpu

CUTOFF = 1e-7
E_TOL = 1e-6         # Eh
F_TOL = 1e-5         # Eh/bohr


def _density(nao, seed):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(nao, nao)) * 0.05
    return torch.as_tensor(d + d.T, device="cuda")[None].contiguous()


def test_jk_cutoff_zero_is_the_fp64_path():
    sym, pos = G.water_cluster(4, seed=3)
    b = build_basis(sym, pos, "cc-pvdz")
    D = _density(b.nao, 1)
    J0, K0 = I.jk_device(b, D, symmetric=True)
    J1, K1 = I.jk_device(b, D, symmetric=True, fp32_cutoff=0.0)
    assert float((J0 - J1).abs().max()) < 1e-12 and float((K0 - K1).abs().max()) < 1e-12


def test_mixed_jk_close_to_fp64_and_really_mixed():
    sym, pos = G.water_cluster(8, seed=1)
    b = build_basis(sym, pos, "cc-pvdz")
    D = _density(b.nao, 2)
    J0, K0 = I.jk_device(b, D, symmetric=True)
    Jm, Km = I.jk_device(b, D, symmetric=True, fp32_cutoff=CUTOFF)
    dj, dk = float((Jm - J0).abs().max()), float((Km - K0).abs().max())
    assert dj < 1e-7 and dk < 1e-7, (dj, dk)
    # the FP32 quartets did contribute: the result is not bitwise the FP64 one
    assert dj > 0.0 or dk > 0.0
    # everything in FP32 (cutoff above every Q1 Q2) is still close, but farther
    Ja, Ka = I.jk_device(b, D, symmetric=True, fp32_cutoff=1e30)
    assert float((Ja - J0).abs().max()) < 1e-3


def test_mixed_difference_build_matches_its_fp64_counterpart():
    sym, pos = G.water_cluster(4, seed=5)
    b = build_basis(sym, pos, "cc-pvdz")
    eng = engine_for(b)
    dD = _density(b.nao, 3) * 1e-3
    J0, K0 = eng.jk_delta_acc(dD, 1e-12, 1e-13)
    Jm, Km = eng.jk_delta_acc(dD, 1e-12, 1e-13, CUTOFF)
    assert float((Jm - J0).abs().max()) < 1e-9 and float((Km - K0).abs().max()) < 1e-9


@pytest.mark.parametrize("case", ["methanol", "h2o8"])
def test_mixed_scf_energy_and_forces_within_bars(case):
    if case == "methanol":
        sym, pos = G.methanol()
        basis = "6-31g**"
    else:
        sym, pos = G.water_cluster(8, seed=1)
        basis = "cc-pvdz"
    out = {}
    for cut in (0.0, CUTOFF):
        solver = SCFSolver(sym, basis, options=SCFOptions(fp32_cutoff=cut))
        st = run_device(solver, pos)
        assert st.converged
        g = scf_gradient_device(st, fp32_cutoff=cut)
        dip = torch.einsum("xmn,mn->x", st.dipole_ints, st.spin[0] + st.spin[1])
        out[cut] = (st.energy, g.cpu().numpy(), dip.cpu().numpy())
    (e0, g0, d0), (em, gm, dm) = out[0.0], out[CUTOFF]
    assert abs(em - e0) < E_TOL, em - e0
    assert np.abs(gm - g0).max() < F_TOL, np.abs(gm - g0).max()
    assert np.abs(dm - d0).max() < 1e-5


def test_mixed_gradient_cutoff_zero_is_the_fp64_path():
    sym, pos = G.methanol()
    st = run_device(SCFSolver(sym, "6-31g**"), pos)
    g0 = scf_gradient_device(st)
    g1 = scf_gradient_device(st, fp32_cutoff=0.0)
    assert float((g0 - g1).abs().max()) < 1e-12
