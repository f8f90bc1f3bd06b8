"""Mixed precision on the whole-GPU path (pm3gpu_set_precision): split-BF16 density and
commutator products while the density is far from converged, FP64 iterations to close.

The closing FP64 iterations make the result the FP64 fixed point, so the bars are the parity bars
of the GPU suite against the FP64 run of the same molecule (heat of formation 1e-6 kcal/mol,
Mulliken charges 1e-5 e, gradient components 1e-6 kcal/mol/A), far inside the 0.01 kcal/mol the
mixed mode is specified to. The per-iteration trace shows which iterations ran split-BF16 and how
close their products are to FP64.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from helpers import A2B
from pm3_rs import _lib, native, workloads

pytestmark = pytest.mark.gpu
HOF_TOL = 1e-6
Q_TOL = 1e-5
GRAD_TOL = 1e-6 * 0.0433641043 / 1.8897261246


def _trace(ctx):
    rows = ctx.lib.pm3gpu_last_large_trace(ctx.ptr, None, 0)
    out = np.zeros((max(rows, 1), 5))
    got = ctx.lib.pm3gpu_last_large_trace(ctx.ptr, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rows)
    assert got == rows
    return out[:rows]


def _solve(z, xyz, opts, mode, threshold=1, **kw):
    ctx = _lib.default_context()
    assert ctx.lib.pm3gpu_set_large_threshold(ctx.ptr, threshold) == 0
    assert ctx.lib.pm3gpu_set_precision(ctx.ptr, mode) == 0
    try:
        r = native.run(z, xyz, opts, **kw)
        return r, _trace(ctx)
    finally:
        assert ctx.lib.pm3gpu_set_precision(ctx.ptr, _lib.PRECISION_FP64) == 0
        assert ctx.lib.pm3gpu_set_large_threshold(ctx.ptr, 257) == 0


def _same(a, b):
    assert a["converged"] and b["converged"]
    assert abs(a["heat_of_formation_kcal"] - b["heat_of_formation_kcal"]) < HOF_TOL
    assert np.abs(np.asarray(a["charges"]) - np.asarray(b["charges"])).max() < Q_TOL
    assert a["unrestricted"] == b["unrestricted"]


def test_mode_is_validated():
    ctx = _lib.default_context()
    assert ctx.lib.pm3gpu_set_precision(ctx.ptr, 7) == _lib.INVALID_INPUT
    assert "precision" in ctx.last_error()


def test_water60_mixed_matches_fp64_and_oracle():
    z, xyz = workloads.water_cluster(60, grid=(5, 4, 3))
    opts = native.options(p_tol=1e-8)
    fp, tf = _solve(z, xyz * A2B, opts, _lib.PRECISION_FP64, threshold=257)
    mx, tm = _solve(z, xyz * A2B, opts, _lib.PRECISION_MIXED, threshold=257)
    _same(mx, fp)
    ref = O.single_point(z, xyz * A2B, p_tol=1e-8)
    _same(mx, ref)
    assert np.all(tf[:, 4] == 0)
    # split-BF16 iterations first, FP64 ones close the SCF
    modes = tm[:, 4]
    assert modes[0] == 1 and modes[-1] == 0
    assert np.all(np.diff(modes) <= 0)
    # the first iteration sees the same Fock matrix in both modes: its split-BF16 commutator norm
    # and density change agree with FP64 to the products' precision
    assert abs(tm[0, 3] - tf[0, 3]) < 1e-4 * tf[0, 3]
    assert abs(tm[0, 2] - tf[0, 2]) < 1e-4 * tf[0, 2]


def test_mixed_organics_uhf_and_gradient_match_fp64():
    # gradients move with the density at first order: both runs converge tightly, as in the FP64
    # gradient parity tests
    tight = dict(e_tol=1e-12, p_tol=1e-10)
    for n, seed in ((30, 7), (48, 6)):
        z, xyz = workloads.organic(n, seed)
        fp, _ = _solve(z, xyz * A2B, native.options(**tight), _lib.PRECISION_FP64, want_gradient=True)
        mx, tm = _solve(z, xyz * A2B, native.options(**tight), _lib.PRECISION_MIXED, want_gradient=True)
        _same(mx, fp)
        assert np.abs(mx["gradient"] - fp["gradient"]).max() < GRAD_TOL
        assert tm[0, 4] == 1
    z, xyz = workloads.radical(20, 11)
    opts = native.options(multiplicity=2, max_scf=1000)
    fp, _ = _solve(z, xyz * A2B, opts, _lib.PRECISION_FP64)
    mx, tm = _solve(z, xyz * A2B, opts, _lib.PRECISION_MIXED)
    _same(mx, fp)
    assert tm[0, 4] == 1 and tm[-1, 4] == 0


def test_per_cta_path_ignores_the_mode():
    z, xyz = workloads.organic(25, 9)
    ctx = _lib.default_context()
    a = native.run(z, xyz * A2B, native.options())
    assert ctx.lib.pm3gpu_set_precision(ctx.ptr, _lib.PRECISION_MIXED) == 0
    try:
        b = native.run(z, xyz * A2B, native.options())
    finally:
        assert ctx.lib.pm3gpu_set_precision(ctx.ptr, _lib.PRECISION_FP64) == 0
    # same FP64 path twice: equal up to the last bits of its reductions
    assert abs(a["heat_of_formation_kcal"] - b["heat_of_formation_kcal"]) < 1e-9
    assert a["iterations"] == b["iterations"]
