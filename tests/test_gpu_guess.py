"""Learned initial density (pm3gpu_guess_*): features and the BF16 network against a numpy
restatement, training on converged densities, and SCF results that do not depend on the start.

The SCF has the last word: starting from the learned density (or from an untrained network's
garbage) the converged heat of formation and charges must equal the standard-guess results
within the parity bars, because both runs converge to the same fixed point.
"""
import ctypes

import numpy as np
import pytest

import guess_mlp_ref as MLP
from helpers import A2B
from pm3_rs import _lib, native, workloads

pytestmark = pytest.mark.gpu
HOF_TOL = 1e-6
Q_TOL = 1e-5
NP = _lib.GUESS_PARAMS
F = ctypes.POINTER(ctypes.c_float)
I32 = ctypes.POINTER(ctypes.c_int32)
D = ctypes.POINTER(ctypes.c_double)


def _pack(mols):
    offs, z, xyz = workloads.pack(mols)
    return np.ascontiguousarray(offs, np.int32), np.ascontiguousarray(z, np.int32), np.ascontiguousarray(xyz * A2B)


def _rows(z, offs):
    return sum(n + n * (n - 1) // 2 for n in np.diff(offs))


def _predict(ctx, offs, z, xyz):
    rows = _rows(z, offs)
    feat = np.zeros((rows, 64), np.float32)
    out = np.zeros((rows, 8), np.float32)
    rc = ctx.lib.pm3gpu_guess_predict(ctx.ptr, len(offs) - 1, offs.ctypes.data_as(I32), z.ctypes.data_as(I32),
                                      xyz.ctypes.data_as(D), feat.ctypes.data_as(F), out.ctypes.data_as(F))
    assert rc == 0, ctx.last_error()
    return feat, out


def _bf16(a):
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16  # round to nearest even
    return (u.astype(np.uint32) << 16).view(np.float32)


def _numpy_forward(x, p):
    sizes = [(64, 256), (256, 256), (256, 256), (256, 8)]
    off, h = 0, _bf16(x)
    for li, (fi, fo) in enumerate(sizes):
        w = _bf16(p[off:off + fi * fo].reshape(fi, fo))
        off += fi * fo
        b = p[off:off + fo]
        off += fo
        zz = h.astype(np.float64) @ w.astype(np.float64) + b
        h = _bf16(zz / (1.0 + np.exp(-zz))) if li < 3 else zz
    return h


@pytest.fixture
def random_model():
    ctx = _lib.default_context()
    rng = np.random.default_rng(5)
    p = (rng.standard_normal(NP) * 0.05).astype(np.float32)
    assert ctx.lib.pm3gpu_guess_set_params(ctx.ptr, p.ctypes.data_as(F), NP) == 0
    return ctx, p


def test_features_and_bf16_network_match_numpy(random_model):
    ctx, p = random_model
    mols = [workloads.organic(9, 1), workloads.organic(14, 2)]
    offs, z, xyz = _pack(mols)
    feat, out = _predict(ctx, offs, z, xyz)
    # features of the first pair row of molecule 0 by hand
    n0 = offs[1] - offs[0]
    assert np.all(feat[:n0, 50] == 1.0) and np.all(feat[n0:n0 + n0 * (n0 - 1) // 2, 50] == 0.0)
    ref = _numpy_forward(feat, p)
    err = np.abs(out[:, :5] - ref[:, :5]).max()
    assert err < 2e-2 * max(1.0, np.abs(ref[:, :5]).max()), err


def test_learned_start_converges_to_the_standard_result(random_model):
    ctx, _ = random_model  # untrained: a poor start; the standard-guess backup may take over
    mols = [workloads.organic(n, 40 + n) for n in (8, 15, 23)]
    offs, z, xyz = _pack(mols)
    std = native.batch(offs, z, xyz, native.options())
    lrn = native.batch(offs, z, xyz, native.options(guess=_lib.GUESS_LEARNED))
    for m in range(len(mols)):
        assert lrn.status[m] == 0
        assert abs(lrn.heat_of_formation_kcal[m] - std.heat_of_formation_kcal[m]) < HOF_TOL
        assert np.abs(lrn.charges_of(m) - std.charges_of(m)).max() < Q_TOL


def test_training_lowers_the_loss_and_keeps_results():
    ctx = _lib.default_context()
    train = workloads.organic_batch(160, 5, 30, seed=77)
    offs, z, xyz = _pack(train)
    losses = np.zeros(6, np.float32)
    opts = native.options()
    rc = ctx.lib.pm3gpu_guess_train(ctx.ptr, len(train), offs.ctypes.data_as(I32), z.ctypes.data_as(I32),
                                    xyz.ctypes.data_as(D), ctypes.byref(opts), 6, 1024, 1e-3, 11,
                                    losses.ctypes.data_as(F))
    assert rc == 0, ctx.last_error()
    assert np.all(np.isfinite(losses)) and losses[-1] < 0.5 * losses[0], losses
    held = workloads.organic_batch(24, 10, 30, seed=78)
    offs, z, xyz = _pack(held)
    std = native.batch(offs, z, xyz, native.options())
    lrn = native.batch(offs, z, xyz, native.options(guess=_lib.GUESS_LEARNED))
    assert np.all(lrn.status == 0)
    assert np.abs(lrn.heat_of_formation_kcal - std.heat_of_formation_kcal).max() < HOF_TOL
    for m in range(len(held)):
        assert np.abs(lrn.charges_of(m) - std.charges_of(m)).max() < Q_TOL
    p = np.zeros(NP, np.float32)
    assert ctx.lib.pm3gpu_guess_get_params(ctx.ptr, p.ctypes.data_as(F), NP) == 0
    assert np.all(np.isfinite(p))


# ---------------------------------------------------------------- backward pass vs the restatement
BLOCKS = ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"]


def _blocks(g):
    out, off = {}, 0
    for li, (fi, fo) in enumerate(MLP.SIZES):
        out[f"W{li + 1}"] = g[off:off + fi * fo]
        off += fi * fo
        out[f"b{li + 1}"] = g[off:off + fo]
        off += fo
    return out


def test_backward_pass_matches_the_fp64_restatement(random_model):
    """Every dW / db of one hand-written BF16 backward pass (pm3gpu_guess_gradients) against the
    FP64 restatement in oracle/guess_mlp_ref.py, which rounds to BF16 at the same points: per
    block, relative Frobenius error below 2e-3 and largest entry error below 2e-2 of the block's
    largest entry (what is left is FP32 accumulation order and rare one-ulp BF16 flips)."""
    ctx, p = random_model
    mols = [workloads.organic(n, 90 + n) for n in (12, 19, 27)]
    offs, z, xyz = _pack(mols)
    feat, _ = _predict(ctx, offs, z, xyz)  # real feature rows (ragged count: not a multiple of 64)
    rng = np.random.default_rng(8)
    rows = feat.shape[0]
    tgt = rng.standard_normal((rows, 8)).astype(np.float32) * 0.3
    mask = (rng.random((rows, 8)) < 0.7).astype(np.float32)
    mask[:, 5:] = 0.0
    inv = np.float32(1.0 / (3.5 * rows))
    loss = np.zeros(1, np.float32)
    g = np.zeros(NP, np.float32)
    rc = ctx.lib.pm3gpu_guess_gradients(ctx.ptr, rows, feat.ctypes.data_as(F), tgt.ctypes.data_as(F),
                                        mask.ctypes.data_as(F), inv, loss.ctypes.data_as(F), g.ctypes.data_as(F))
    assert rc == 0, ctx.last_error()
    ref_loss, ref = MLP.loss_and_grad(p, feat, tgt, mask, float(inv))
    assert abs(loss[0] - ref_loss) <= 1e-4 * ref_loss
    got_b, ref_b = _blocks(g.astype(np.float64)), _blocks(ref)
    for name in BLOCKS:
        a, b = got_b[name], ref_b[name]
        assert np.linalg.norm(b) > 0.0, name
        assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b), (name, np.linalg.norm(a - b) / np.linalg.norm(b))
        assert np.abs(a - b).max() <= 2e-2 * np.abs(b).max(), name


def test_trained_network_cuts_scf_iterations():
    """What the trained network gains over the standard (SAD) start: trained on the plain SCF's
    own converged densities of 1024 organics, it lowers the mean SCF iteration count of 128
    held-out organics by at least 15%, every molecule converges, and the results equal the
    standard-guess ones within the parity bars (both runs reach the same fixed point)."""
    ctx = _lib.Context()
    try:
        train = workloads.organic_batch(1024, 5, 40, seed=501)
        offs, z, xyz = _pack(train)
        losses = np.zeros(8, np.float32)
        rc = ctx.lib.pm3gpu_guess_train(ctx.ptr, len(train), offs.ctypes.data_as(I32), z.ctypes.data_as(I32),
                                        xyz.ctypes.data_as(D), ctypes.byref(native.options()), 8, 1024, 1e-3, 3,
                                        losses.ctypes.data_as(F))
        assert rc == 0, ctx.last_error()
        held = workloads.organic_batch(128, 10, 40, seed=502)
        offs, z, xyz = _pack(held)
        std = native.batch(offs, z, xyz, native.options(), context=ctx)
        lrn = native.batch(offs, z, xyz, native.options(guess=_lib.GUESS_LEARNED), context=ctx)
        assert np.all(std.status == 0) and np.all(lrn.status == 0)
        assert np.abs(lrn.heat_of_formation_kcal - std.heat_of_formation_kcal).max() < HOF_TOL
        it_std, it_lrn = std.iterations.mean(), lrn.iterations.mean()
        print(f"mean SCF iterations: standard guess {it_std:.2f}, learned guess {it_lrn:.2f}")
        assert it_lrn <= 0.85 * it_std, (it_std, it_lrn)
    finally:
        ctx.close()
