"""
aimd_eri_tensor_static (the entry point that allocates no device memory)
against aimd_eri_tensor, through the C ABI: two calls in a row must each give
the tensor of the allocating entry point, and sizes beyond the static scratch
are refused before any work.
"""

import ctypes

import pytest
import torch

from aimd_b200 import _lib, geometry as G
from aimd_b200.basis import build_basis
from aimd_b200.engine import engine_for

pytestmark = pytest.mark.gpu

THR = 1e-12
TOL = 1e-10          # per element, Eh; both paths run the same kernels, summation order aside


def _static_call(eng, out: torch.Tensor) -> int:
    return eng.lib.aimd_eri_tensor_static(eng.handle, ctypes.c_void_p(out.data_ptr()), THR,
                                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("case", [("water", "6-31g*"), ("methanol", "6-31g**")])
def test_static_scratch_matches_allocating_entry_point(case):
    mol, basis_name = case
    sym, pos = getattr(G, mol)()
    basis = build_basis(sym, pos, basis_name)
    eng = engine_for(basis)
    ref = eng.eri_tensor(THR)
    for _ in range(2):
        out = torch.full_like(ref, float("nan"))      # every element must be written
        _lib.check(_static_call(eng, out), "aimd_eri_tensor_static")
        torch.cuda.synchronize()
        assert torch.isfinite(out).all()
        assert float((out - ref).abs().max()) <= TOL


def test_static_scratch_refuses_sizes_beyond_its_limit():
    sym, pos = G.water_cluster(8, seed=1)
    basis = build_basis(sym, pos, "cc-pvdz")          # 200 AOs > 128
    eng = engine_for(basis)
    assert basis.nao > 128
    out = torch.empty(1, dtype=torch.float64, device="cuda")   # never written: refused first
    status = _static_call(eng, out)
    assert status == _lib.AIMD_ERR_ARG
    msg = eng.lib.aimd_last_error().decode()
    assert "static scratch limit of 128" in msg


def test_static_scratch_is_fp64_whatever_the_context_cutoff():
    """A context that carries an FP32 cutoff still gets the FP64 tensor."""
    sym, pos = G.water()
    basis = build_basis(sym, pos, "6-31g*")
    eng = engine_for(basis)
    ref = eng.eri_tensor(THR)
    _lib.check(eng.lib.aimd_set_fp32_cutoff(eng.handle, ctypes.c_double(1e30)), "aimd_set_fp32_cutoff")
    eng._fp32_cutoff = 1e30
    try:
        out = torch.full_like(ref, float("nan"))
        _lib.check(_static_call(eng, out), "aimd_eri_tensor_static")
        torch.cuda.synchronize()
        assert float((out - ref).abs().max()) <= TOL
    finally:
        eng._precision(0.0)
