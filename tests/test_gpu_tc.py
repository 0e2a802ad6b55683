"""The tensor-core tile product (tcgen05.mma kind::tf32, three-term TF32 split) against FP64.

cf_tc_tile_product runs the building blocks the line patches' refresh uses for its 64 x 64 x 64
tile updates: operand split and canonical shared-memory layout, descriptors, the products, the
commit and the read-back from tensor memory.  The three-term split keeps ~22 bits of every
product, so the tile agrees with the FP64 product to a few FP32 roundings (bound 1e-5 of the
largest entry), where a single TF32 product would be off by ~1e-3.
"""
import ctypes

import numpy as np
import pytest

from cufcm_fil_b200 import _lib

pytestmark = pytest.mark.gpu


def _product(A, B):
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    D = np.zeros((64, 64), np.float32)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)
    _lib.call("cf_tc_tile_product", p(A), p(B), p(D), 0)
    return D


@pytest.mark.parametrize("seed", [0, 1])
def test_tile_product_matches_fp64(seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((64, 64)).astype(np.float32)
    B = rng.standard_normal((64, 64)).astype(np.float32)
    D = _product(A, B)
    ref = A.astype(np.float64).T @ B.astype(np.float64)
    err = np.abs(D - ref).max() / np.abs(ref).max()
    print(f"tile product, seed {seed}: max error {err:.2e} of the largest entry")
    assert err < 1e-5


def test_tile_layout_is_exact_on_integers():
    # small integers are exact in TF32: any misplaced row, column or K chunk shows as an exact mismatch
    rng = np.random.default_rng(7)
    A = rng.integers(-4, 5, (64, 64)).astype(np.float32)
    B = rng.integers(-4, 5, (64, 64)).astype(np.float32)
    np.testing.assert_array_equal(_product(A, B), (A.T @ B).astype(np.float32))
