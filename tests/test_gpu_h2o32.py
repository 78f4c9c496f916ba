"""
Parity on the benchmark's own workload: (H2O)32 RHF/cc-pVDZ (800 AOs, the
seeded water cluster the bench runs), CUDA path against the oracle at the
converged density of the GPU SCF.

* FP64 J and K elementwise within 1e-9 of the oracle's integral-direct J/K.
* SCF energy: the oracle evaluates the RHF energy functional
  E(P) = E_nuc + tr(P h) + 1/2 tr(P (J - K/2)) with its own integrals at the
  GPU's converged density; the SCF energy is variational, so E(P) is the
  oracle's SCF energy to second order in the density error. Bar 1e-9 Eh.
* Forces: nuclear + one-electron (P, W) + two-electron (P) gradient of the
  oracle at the GPU's P and W, against the GPU's analytic gradient: 1e-7
  Eh/bohr for the FP64 path; the two-electron contraction alone likewise.
* Mixed precision at the bench's FP32 cutoff (quartets with Q1 Q2 < 1e-3 in
  FP32, FP64 accumulation): SCF energy within 1e-6 Eh and forces within
  1e-5 Eh/bohr of the FP64 oracle.
"""

import numpy as np
import pytest
import torch

from oracle import hf_oracle as O

pytestmark = pytest.mark.gpu

E_TOL, F_TOL = 1e-9, 1e-7                  # plain FP64 path
E_TOL_MIXED, F_TOL_MIXED = 1e-6, 1e-5      # mixed-precision path
JK_TOL = 1e-9                              # per J/K element
CUTOFF = 1e-3                              # the bench's FP32 cutoff


@pytest.fixture(scope="module")
def h2o32():
    if not torch.cuda.is_available():
        pytest.fail("gpu tests need a CUDA device")
    from aimd_b200 import geometry as G
    from aimd_b200.gradients import scf_gradient
    from aimd_b200.scf import SCFOptions, SCFSolver
    sym, pos = G.water_cluster(32, seed=1)
    res = SCFSolver(sym, "cc-pvdz").run(pos)
    assert res.converged and res.basis.nao == 800
    g = scf_gradient(res)
    res_m = SCFSolver(sym, "cc-pvdz", options=SCFOptions(fp32_cutoff=CUTOFF)).run(pos)
    assert res_m.converged
    g_m = scf_gradient(res_m, fp32_cutoff=CUTOFF)

    ob = O.build_basis(sym, pos, "cc-pvdz")
    P, W = res.density, res.energy_weighted_density
    J, K = O.jk_direct(ob, P)
    S, T, V = O.one_electron_matrices(ob)
    h = T + V
    enuc = O.nuclear_repulsion_energy(ob.nuclear_charges, ob.positions)
    e_oracle = enuc + float(np.vdot(P, h)) + 0.5 * float(np.vdot(P, J - 0.5 * K))
    g2 = O.two_electron_gradient(ob, P, [P], 0.5)
    g_oracle = (O.nuclear_repulsion_gradient(ob.nuclear_charges, ob.positions)
                + O.one_electron_gradient(ob, P, W) + g2)
    return {"basis": res.basis, "res": res, "g": g, "res_m": res_m, "g_m": g_m, "P": P, "J": J, "K": K,
            "e_oracle": e_oracle, "g2_oracle": g2, "g_oracle": g_oracle}


def test_h2o32_fp64_jk_against_oracle(h2o32):
    from aimd_b200 import integrals as I
    J, K = I.jk(h2o32["basis"], h2o32["P"])
    dj = np.abs(J - h2o32["J"]).max()
    dk = np.abs(K - h2o32["K"]).max()
    assert dj <= JK_TOL and dk <= JK_TOL, (dj, dk)


def test_h2o32_fp64_two_electron_gradient_against_oracle(h2o32):
    from aimd_b200 import integrals as I
    P = h2o32["P"]
    g2 = I.two_electron_gradient(h2o32["basis"], P, [P], 0.5)
    assert np.abs(g2 - h2o32["g2_oracle"]).max() <= F_TOL


def test_h2o32_fp64_energy_and_forces_against_oracle(h2o32):
    assert abs(h2o32["res"].energy - h2o32["e_oracle"]) <= E_TOL
    assert np.abs(h2o32["g"] - h2o32["g_oracle"]).max() <= F_TOL


def test_h2o32_mixed_energy_and_forces_against_fp64_oracle(h2o32):
    de = abs(h2o32["res_m"].energy - h2o32["e_oracle"])
    df = np.abs(h2o32["g_m"] - h2o32["g_oracle"]).max()
    assert de <= E_TOL_MIXED, de
    assert df <= F_TOL_MIXED, df
