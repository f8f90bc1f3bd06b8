"""The whole-GPU path's FP64 GEMM (pm3gpu_dgemm: the DMMA kernel that runs the commutator, the
density and the eigensolver's dense products) against numpy's FP64 product.

Every tile shape the kernel picks (128 x 128, 128 x 64 for K <= 128, 128 x 32 and 32 x 128 for
outputs one panel wide), every op combination, ragged edges, padded and odd leading dimensions
(8- and 16-byte copies), K = 0, and the deterministic split-K. Bound: the elementwise error of a
K-term FP64 dot product, |C - C_ref| <= 2 K eps (|alpha| |op(A)| |op(B)| + |beta C|).
"""
import ctypes

import numpy as np
import pytest

from pm3_rs import _lib

pytestmark = pytest.mark.gpu
D = ctypes.POINTER(ctypes.c_double)
EPS = np.finfo(np.float64).eps


def _run(ctx, ta, tb, m, n, k, alpha, beta, pad=0, seed=0):
    rng = np.random.default_rng(seed)
    ra, ca = (k, m) if ta else (m, k)
    rb, cb = (n, k) if tb else (k, n)
    lda, ldb, ldc = max(ra, 1) + pad, max(rb, 1) + pad, m + pad
    a = np.asfortranarray(rng.standard_normal((lda, max(ca, 1))))
    b = np.asfortranarray(rng.standard_normal((ldb, max(cb, 1))))
    c0 = np.asfortranarray(rng.standard_normal((ldc, n)))
    c = c0.copy(order="F")
    rc = ctx.lib.pm3gpu_dgemm(ctx.ptr, int(ta), int(tb), m, n, k, alpha, a.ctypes.data_as(D), lda,
                              b.ctypes.data_as(D), ldb, beta, c.ctypes.data_as(D), ldc)
    assert rc == _lib.OK, ctx.last_error()
    opa = a[:k, :m].T if ta else a[:m, :k]
    opb = b[:n, :k].T if tb else b[:k, :n]
    ref = alpha * (opa @ opb) + beta * c0[:m, :n]
    bound = 2 * max(k, 1) * EPS * (abs(alpha) * (np.abs(opa) @ np.abs(opb)) + abs(beta) * np.abs(c0[:m, :n])) + 1e-300
    err = np.abs(c[:m, :n] - ref)
    assert (err <= bound).all(), (ta, tb, m, n, k, float(err.max()), float((err / bound).max()))
    np.testing.assert_array_equal(c[m:, :], c0[m:, :])  # padding rows untouched
    return c[:m, :n].copy()


@pytest.fixture(scope="module")
def ctx():
    c = _lib.Context()
    yield c
    c.close()


@pytest.mark.parametrize("ta", [False, True])
@pytest.mark.parametrize("tb", [False, True])
def test_every_op_combination_on_ragged_sizes(ctx, ta, tb):
    _run(ctx, ta, tb, 300, 257, 333, -1.25, 0.5, pad=3, seed=1)  # 128 x 128 tiles, odd ld: 8-byte copies
    _run(ctx, ta, tb, 300, 190, 72, 1.0, 1.0, pad=2, seed=2)     # 128 x 64 tiles (low K), 16-byte copies
    _run(ctx, ta, tb, 333, 29, 61, 0.7, 0.0, seed=3)            # 128 x 32 tiles
    _run(ctx, ta, tb, 17, 333, 45, 0.7, -2.0, seed=4)           # 32 x 128 tiles


def test_split_k_is_exact_and_repeats_bit_for_bit(ctx):
    first = _run(ctx, False, True, 37, 29, 5000, 1.0, 0.0, seed=5)     # one tile, K split over the grid
    again = _run(ctx, False, True, 37, 29, 5000, 1.0, 0.0, seed=5)
    np.testing.assert_array_equal(first, again)
    _run(ctx, True, False, 700, 20, 2000, -1.0, 1.0, seed=6)
    _run(ctx, False, True, 256, 128, 4096, 1.0, 0.0, seed=7)             # 128 x 128 tiles, split


def test_degenerate_sizes(ctx):
    _run(ctx, False, False, 5, 3, 1, 2.0, 0.5, seed=8)
    _run(ctx, True, True, 1, 1, 7, 1.0, 0.0, seed=9)
    _run(ctx, False, False, 40, 50, 0, 1.0, 0.25, seed=10)  # K = 0: C = beta C
    assert ctx.lib.pm3gpu_dgemm(ctx.ptr, 0, 0, 10, 10, 10, 1.0, None, 10, None, 10, 0.0, None, 10) == _lib.INVALID_INPUT
