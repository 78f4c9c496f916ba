"""
The host basis layout is bitwise the reference's: shell, primitive and
general-contraction block arrays (aimd/qc/basis.py:140-246) for the
molecules and basis sets stored in golden/basis_arrays.npz, which
golden/make_golden.py wrote by running the reference's build_basis.
Bitwise equality matters because the Schwarz bounds and the screening
decisions are per block pair and the AO order defines every matrix.
"""

import os

import numpy as np
import pytest

from aimd_b200.basis import build_basis

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "basis_arrays.npz")
ARRAYS = ("shell_atom", "shell_l", "shell_prim", "shell_ao", "prim_exp", "prim_coef", "blk_shell", "blk_atom",
          "blk_l", "blk_ncon", "blk_ao", "blk_prim", "blk_exp", "blk_coef", "ao_lxyz", "atom_ao")


def _cases():
    with np.load(GOLDEN) as z:
        return sorted({k.split("/")[0] for k in z.files})


@pytest.fixture(scope="module")
def fixture():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("case", _cases())
def test_basis_arrays_bitwise_equal_to_reference(fixture, case):
    sym = [str(s) for s in fixture[f"{case}/symbols"]]
    b = build_basis(sym, fixture[f"{case}/positions"], str(fixture[f"{case}/basis"]))
    for name in ARRAYS:
        ref = fixture[f"{case}/{name}"]
        ours = np.asarray(getattr(b, name))
        assert ours.shape == ref.shape, (case, name, ours.shape, ref.shape)
        if ref.dtype.kind == "f":
            # bitwise: compare the IEEE-754 bit patterns, not values
            assert np.array_equal(ours.astype(np.float64).view(np.int64), ref.astype(np.float64).view(np.int64)), \
                (case, name)
        else:
            assert np.array_equal(ours.astype(np.int64), ref.astype(np.int64)), (case, name)
