"""pm3gpu_single_point_noalloc (fixed device scratch, no allocation) against pm3gpu_single_point.

Both entry points run the same SCF kernel on the same inputs, so results agree to the parity
bars of the GPU suite: heat of formation within 1e-6 kcal/mol, Mulliken charges within 1e-5 e.
Every case makes two no-alloc calls in a row, so the second one runs on scratch the first left
behind. The file is named to be collected last and also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from helpers import A2B
from pm3_rs import _lib, native, workloads

pytestmark = pytest.mark.gpu
HOF_TOL = 1e-6
Q_TOL = 1e-5


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _call(name, z, xyz_bohr, opts):
    ctx = _lib.default_context()
    z = np.ascontiguousarray(z, dtype=np.int32)
    x = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(len(z), 3)
    res = _lib.Result()
    q = np.zeros(len(z))
    if name == "noalloc":
        rc = ctx.lib.pm3gpu_single_point_noalloc(ctx.ptr, len(z), _ip(z), _dp(x), ctypes.byref(opts),
                                                 ctypes.byref(res), _dp(q))
    else:
        rc = ctx.lib.pm3gpu_single_point(ctx.ptr, len(z), _ip(z), _dp(x), ctypes.byref(opts), ctypes.byref(res),
                                         _dp(q), None, None)
    return rc, res, q, ctx.last_error()


def _same(a, b):
    rc_a, ra, qa, _ = a
    rc_b, rb, qb, _ = b
    assert rc_a == rc_b == _lib.OK
    assert abs(ra.heat_of_formation_kcal - rb.heat_of_formation_kcal) <= HOF_TOL
    assert np.max(np.abs(qa - qb)) <= Q_TOL
    assert ra.converged == rb.converged == 1
    assert ra.unrestricted == rb.unrestricted
    assert ra.scf_paths_tried == rb.scf_paths_tried
    assert ra.iterations == rb.iterations
    assert ra.nao == rb.nao


def _molecules():
    mols = []
    for n, seed in ((12, 101), (40, 202)):
        z, xyz = workloads.organic(n, seed)
        mols.append((np.asarray(z), np.asarray(xyz) * A2B, native.options()))
    z, xyz = workloads.radical(15, 303)
    mols.append((np.asarray(z), np.asarray(xyz) * A2B, native.options(multiplicity=2, max_scf=1000)))
    return mols


def test_noalloc_matches_single_point_two_calls_in_a_row():
    mols = _molecules()
    ref = [_call("single_point", z, x, o) for z, x, o in mols]
    for rnd in range(2):
        for (z, x, o), r in zip(mols, ref):
            _same(_call("noalloc", z, x, o), r)


def test_noalloc_stability_rungs_two_calls_in_a_row():
    z, xyz = workloads.organic(20, 404)
    o = native.options(stability=2)  # PM3GPU_STABILITY_ALWAYS: the search runs whatever the first pass gives
    x = np.asarray(xyz) * A2B
    ref = _call("single_point", z, x, o)
    assert ref[1].scf_paths_tried > 1
    first = _call("noalloc", z, x, o)
    second = _call("noalloc", z, x, o)
    _same(first, ref)
    _same(second, ref)


def test_noalloc_rejects_molecule_beyond_scratch():
    # 204 basis functions: one workspace slot exceeds the scratch, and pm3gpu_single_point would
    # send this lone molecule to the whole-GPU path; either way the call refuses it
    z, xyz = workloads.water_cluster(34)
    rc, res, _, msg = _call("noalloc", z, np.asarray(xyz) * A2B, native.options())
    assert rc == _lib.RESOURCE_LIMIT
    assert res.status == _lib.RESOURCE_LIMIT
    assert "scratch" in msg or "whole-GPU" in msg
    # the context stays usable afterwards
    z, xyz = workloads.organic(12, 101)
    x = np.asarray(xyz) * A2B
    _same(_call("noalloc", z, x, native.options()), _call("single_point", z, x, native.options()))


def test_noalloc_has_no_post_scf_corrections():
    """The allocation-free entry runs plain PM3 only: a PM3-D3 request is refused, not ignored."""
    z, xyz = workloads.organic(8, 3)
    rc, _, _, msg = _call("noalloc", z, np.asarray(xyz) * A2B, native.options(variant=1))
    assert rc == _lib.INVALID_INPUT and "correction" in msg
