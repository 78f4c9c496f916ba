"""
Launch-shape autotuner (Engine.autotune over aimd_set_launch_shape): the
shape only changes how the work of each class launch is cut into chunks and
how column items of many-primitive pairs are split, so J/K and the
two-electron gradient at every candidate shape agree with the default
shape to rounding (1e-10 per J/K element, 1e-9 Eh/bohr per gradient
component: the per-item fixed-point sums round differently when items
split differently); the tuner sets the fastest candidate, and shapes out of
range are refused with the context left unchanged.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup():
    from aimd_b200 import geometry as G
    from aimd_b200 import integrals as I
    from aimd_b200.basis import build_basis
    from aimd_b200.engine import engine_for
    sym, pos = G.water_cluster(4, seed=3)
    b = build_basis(sym, pos, "cc-pvdz")
    rng = np.random.default_rng(11)
    d = rng.normal(size=(b.nao, b.nao)) * 0.05
    D = torch.as_tensor(d + d.T, device="cuda")
    eng = engine_for(b)
    grad = (D, D[None].contiguous(), 0.5, I.DEFAULT_SCHWARZ_GRAD, I.gamma_bound(D, D[None], 0.5))
    return eng, D, grad


def test_autotune_picks_a_candidate_and_keeps_results():
    from aimd_b200 import integrals as I
    eng, D, grad = _setup()
    assert eng.launch_shape == (8, 32)
    J0, K0 = eng.jk_acc(D[None].contiguous(), I.DEFAULT_SCHWARZ)
    g0 = eng.grad2e(*grad)
    shapes = [(8, 32), (4, 16), (16, 64), (2, 8)]
    try:
        r = eng.autotune(D[None].contiguous(), I.DEFAULT_SCHWARZ, grad=grad, shapes=shapes, reps=1)
        assert r["shape"] in shapes and eng.launch_shape == r["shape"]
        assert [c["shape"] for c in r["candidates"]] == shapes
        assert all(c["jk_ms"] > 0 and c["grad_ms"] > 0 for c in r["candidates"])
        for shape in shapes:
            eng.set_launch_shape(*shape)
            J, K = eng.jk_acc(D[None].contiguous(), I.DEFAULT_SCHWARZ)
            assert float((J - J0).abs().max()) < 1e-10 and float((K - K0).abs().max()) < 1e-10
            assert float((eng.grad2e(*grad) - g0).abs().max()) < 1e-9
    finally:
        eng.set_launch_shape(8, 32)


def test_launch_shape_out_of_range_is_refused():
    from aimd_b200._lib import NativeError
    eng, _, _ = _setup()
    for bad in [(0, 32), (65, 32), (8, 3), (8, 5000)]:
        with pytest.raises(NativeError, match="aimd_set_launch_shape"):
            eng.set_launch_shape(*bad)
    assert eng.launch_shape == (8, 32)
