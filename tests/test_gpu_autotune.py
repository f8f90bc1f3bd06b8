"""Autotuner (pm3gpu_autotune / pm3gpu_load_tuning / pm3gpu_tuning_choice).

The tuner times the two variants of each launch choice on a sample and keeps the faster per size
bucket. Both variants compute the same thing, so a batch solved under a loaded tuning file must
match the untuned context within the parity bars (heat of formation 1e-6 kcal/mol, charges
1e-5 e).
"""
import ctypes
import json

import numpy as np
import pytest

from helpers import A2B
from pm3_rs import _lib, native, workloads

pytestmark = pytest.mark.gpu
I32 = ctypes.POINTER(ctypes.c_int32)
D = ctypes.POINTER(ctypes.c_double)


def _pack(mols):
    offs, z, xyz = workloads.pack(mols)
    return (np.ascontiguousarray(offs, np.int32), np.ascontiguousarray(z, np.int32),
            np.ascontiguousarray(xyz * A2B))


def _batch(ctx, offs, z, xyz):
    n = len(offs) - 1
    res = (_lib.Result * n)()
    q = np.zeros(len(z))
    opts = native.options()
    rc = ctx.lib.pm3gpu_batch(ctx.ptr, n, offs.ctypes.data_as(I32), z.ctypes.data_as(I32), xyz.ctypes.data_as(D),
                              ctypes.byref(opts), 0, res, q.ctypes.data_as(D), None)
    assert rc == 0, ctx.last_error()
    return np.array([r.heat_of_formation_kcal for r in res]), q, np.array([r.status for r in res])


def test_autotune_writes_loads_and_keeps_results(tmp_path):
    organics = workloads.organic_batch(96, 5, 60, seed=91)
    sample = organics + [workloads.water_cluster(60, grid=(5, 4, 3))]
    offs, z, xyz = _pack(sample)
    path = tmp_path / "tuning.json"
    ctx = _lib.Context(0)
    try:
        opts = native.options()
        rc = ctx.lib.pm3gpu_autotune(ctx.ptr, len(sample), offs.ctypes.data_as(I32), z.ctypes.data_as(I32),
                                     xyz.ctypes.data_as(D), ctypes.byref(opts), str(path).encode())
        assert rc == 0, ctx.last_error()
        nmax = max(int(np.sum(np.where(np.asarray(zm) == 1, 1, 4))) for zm, _ in organics)
        batch_choice = ctx.lib.pm3gpu_tuning_choice(ctx.ptr, 0, nmax)
        large_choice = ctx.lib.pm3gpu_tuning_choice(ctx.ptr, 1, 360)
    finally:
        ctx.close()
    assert batch_choice in (1, 2)
    assert large_choice in (0, 1)
    table = json.loads(path.read_text())
    assert table["sms"] > 0
    (b,) = table["batch"]
    assert b["nmax_le"] >= nmax and b["ctas_per_sm"] == batch_choice
    assert b["ms_1cta"] > 0 and b["ms_2cta"] > 0
    assert b["ctas_per_sm"] == (2 if b["ms_2cta"] <= b["ms_1cta"] else 1)
    (lg,) = table["large"]
    assert lg["n_le"] == 512 and lg["coop"] == large_choice and lg["ms_coop"] > 0 and lg["ms_multi"] > 0

    offs, z, xyz = _pack(organics)
    ref = _lib.Context(0)
    tuned = _lib.Context(0)
    try:
        assert tuned.lib.pm3gpu_load_tuning(tuned.ptr, str(path).encode()) == 0
        assert tuned.lib.pm3gpu_tuning_choice(tuned.ptr, 0, nmax) == batch_choice
        assert ref.lib.pm3gpu_tuning_choice(ref.ptr, 0, nmax) == -1
        h0, q0, s0 = _batch(ref, offs, z, xyz)
        h1, q1, s1 = _batch(tuned, offs, z, xyz)
    finally:
        ref.close()
        tuned.close()
    assert np.all(s0 == 0) and np.all(s1 == 0)
    assert np.abs(h0 - h1).max() < 1e-6
    assert np.abs(q0 - q1).max() < 1e-5


def test_tuning_file_errors(tmp_path):
    ctx = _lib.Context(0)
    try:
        assert ctx.lib.pm3gpu_load_tuning(ctx.ptr, str(tmp_path / "missing.json").encode()) == _lib.INVALID_INPUT
        bad = tmp_path / "bad.json"
        bad.write_text('{"batch": [{"nmax_le": 128, "ctas_per_sm": 3}]}')
        assert ctx.lib.pm3gpu_load_tuning(ctx.ptr, str(bad).encode()) == _lib.INVALID_INPUT
        assert "ctas_per_sm" in ctx.last_error()
        assert ctx.lib.pm3gpu_tuning_choice(ctx.ptr, 0, 100) == -1
    finally:
        ctx.close()
