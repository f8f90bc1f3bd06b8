"""The hand-written tcgen05 split-BF16 GEMM (tc_gemm.cuh) against the FP64 product.

out = A B^T with each FP64 operand split into BF16 hi + lo and hi hi + hi lo + lo hi accumulated in
FP32 in tensor memory. Each split value carries 16 significant bits (relative error <= 2^-17) and
the dropped lo lo term is 2^-16 of a product, so every entry is within ~3 * 2^-17 of |A| |B|^T
plus the FP32 accumulation; the bar below is 4e-5 |A| |B|^T + 1e-30. Shapes cover one tile, many
tiles, ragged edges in M, N and K (TMA zero fill, masked stores) and K below one 64-wide block.
"""
import ctypes

import numpy as np
import pytest

from pm3_rs import _lib

pytestmark = pytest.mark.gpu
F = ctypes.POINTER(ctypes.c_float)
D = ctypes.POINTER(ctypes.c_double)


def _gemm(ctx, a, b):
    m, k = a.shape
    n = b.shape[0]
    out = np.zeros((m, n), np.float32)
    rc = ctx.lib.pm3gpu_split_gemm(ctx.ptr, m, n, k, a.ctypes.data_as(D), a.shape[1], b.ctypes.data_as(D),
                                   b.shape[1], out.ctypes.data_as(F))
    assert rc == 0, ctx.last_error()
    return out


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (300, 520, 200), (1000, 777, 1501), (129, 257, 13), (64, 40, 8)])
def test_split_gemm_matches_fp64_product(m, n, k):
    ctx = _lib.default_context()
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a = rng.standard_normal((m, k)) * np.exp(rng.uniform(-3, 3, (m, 1)))
    b = rng.standard_normal((n, k))
    got = _gemm(ctx, a, b).astype(np.float64)
    ref = a @ b.T
    bound = 4e-5 * (np.abs(a) @ np.abs(b).T) + 1e-30
    err = np.abs(got - ref)
    assert np.all(err <= bound), float((err / bound).max())
    # far better than plain BF16 (2^-9 = 2e-3): the split is what gives FP32-level products
    assert np.median(err / (np.abs(a) @ np.abs(b).T)) < 4e-6


def test_split_gemm_symmetric_products_of_the_scf():
    """The two shapes the mixed SCF runs: F P with symmetric F, P (n x n) and X X^T (n x n_occ)."""
    ctx = _lib.default_context()
    rng = np.random.default_rng(4)
    n, occ = 700, 230
    f = rng.standard_normal((n, n))
    f = f + f.T
    p = rng.standard_normal((n, n))
    p = p + p.T
    fp = _gemm(ctx, f, p).astype(np.float64)  # F P^T = F P
    assert np.abs(fp - f @ p).max() <= 4e-5 * (np.abs(f) @ np.abs(p)).max()
    x = np.ascontiguousarray(rng.standard_normal((n, occ)))
    xx = _gemm(ctx, x, x).astype(np.float64)
    assert np.abs(xx - x @ x.T).max() <= 4e-5 * (np.abs(x) @ np.abs(x).T).max()
    assert np.abs(xx - xx.T).max() <= 1e-6 * np.abs(xx).max()
