"""
The differentiable SCF energy (aimd_b200.autograd): its backward pass (the
hand-written derivative kernels) against central finite differences of the
energy at h = 1e-4 bohr, and against the reference's analytic gradient
(golden fixture of water RHF/6-31G*).
"""

import numpy as np
import pytest
import torch

from aimd_b200 import geometry as G
from aimd_b200.autograd import HFEnergy, scf_energy
from aimd_b200.scf import SCFOptions, SCFSolver

pytestmark = pytest.mark.gpu


def test_backward_matches_reference_gradient(golden):
    g = golden("water_631gs")
    f = HFEnergy([str(s) for s in g["symbols"]], "6-31g*")
    x = torch.as_tensor(g["positions"]).clone().requires_grad_(True)
    e = f(x)
    e.backward()
    assert abs(float(e.detach()) - float(g["energy"])) < 1e-9
    np.testing.assert_allclose(x.grad.numpy(), g["gradient"], atol=1e-7)


def test_backward_matches_central_differences():
    sym, pos = G.methanol()
    f = HFEnergy(sym, "6-31g**", options=SCFOptions(conv_energy=1e-12, conv_commutator=1e-9))
    x = torch.as_tensor(pos).clone().requires_grad_(True)
    (grad,) = torch.autograd.grad(f(x), x)
    rng = np.random.default_rng(7)
    h = 1e-4
    for a in rng.choice(len(sym), size=3, replace=False):
        for k in range(3):
            xp, xm = pos.copy(), pos.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd = (float(f(torch.as_tensor(xp))) - float(f(torch.as_tensor(xm)))) / (2 * h)
            assert abs(fd - float(grad[a, k])) < 1e-6, (a, k, fd, float(grad[a, k]))


def test_chain_rule_and_single_backward():
    sym, pos = G.water()
    solver = SCFSolver(sym, "6-31g*")
    x = torch.as_tensor(pos).clone().requires_grad_(True)
    e = scf_energy(x, solver)
    (g1,) = torch.autograd.grad(3.0 * e, x, retain_graph=True)
    holder = {}
    e2 = scf_energy(x, solver, holder=holder)
    (g0,) = torch.autograd.grad(e2, x)
    np.testing.assert_allclose(g1.numpy(), 3.0 * g0.numpy(), rtol=1e-10, atol=1e-12)
    assert holder["state"].converged
    with pytest.raises(RuntimeError):
        torch.autograd.grad(e, x)          # the backward state was consumed by the first call
