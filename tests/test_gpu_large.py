"""Whole-GPU path for large molecules (grid-wide integrals and Fock build, blocked eigensolver)
against the CPU oracle and against the per-CTA path on the same inputs.

Molecules below the default size threshold are sent to the whole-GPU path with
pm3gpu_set_large_threshold, so the two device paths and the oracle can be compared on the same
small systems; the 60-water cluster (360 basis functions) takes the whole-GPU path by size.
Bars as in the rest of the GPU suite: heat of formation 1e-6 kcal/mol, Mulliken charges 1e-5 e,
gradient components 1e-6 kcal/mol/A.
"""
import numpy as np
import pytest

import oracle as O
from helpers import A2B, GOLDEN, parse
from pm3_rs import _lib, native, workloads

pytestmark = pytest.mark.gpu
HOF_TOL = 1e-6
Q_TOL = 1e-5
GRAD_TOL = 1e-6 * 0.0433641043 / 1.8897261246


@pytest.fixture
def whole_gpu():
    ctx = _lib.default_context()
    assert ctx.lib.pm3gpu_set_large_threshold(ctx.ptr, 1) == 0
    yield ctx
    assert ctx.lib.pm3gpu_set_large_threshold(ctx.ptr, 257) == 0


def _cta(z, xyz, opts, **kw):
    ctx = _lib.default_context()
    assert ctx.lib.pm3gpu_set_large_threshold(ctx.ptr, 257) == 0
    r = native.run(z, xyz, opts, **kw)
    assert ctx.lib.pm3gpu_set_large_threshold(ctx.ptr, 1) == 0
    return r


def _close(got, ref, hof_tol=HOF_TOL):
    assert got["converged"] and ref["converged"]
    assert abs(got["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) < hof_tol
    assert np.abs(np.asarray(got["charges"]) - np.asarray(ref["charges"])).max() < Q_TOL
    assert np.abs(np.array(got["dipole_debye"]) - np.array(ref["dipole_debye"])).max() < 1e-5
    assert got["unrestricted"] == ref["unrestricted"]
    assert got["scf_paths_tried"] == ref["scf_paths_tried"]


@pytest.mark.parametrize("name", ["water", "formaldehyde", "h2s", "methyl_mopac"])
def test_golden_molecules_on_whole_gpu_path(whole_gpu, name):
    geom, charge, mult, hof = GOLDEN[name]
    z, xyz = parse(geom)
    opts = native.options(charge=charge, multiplicity=mult)
    got = native.run(z, xyz * A2B, opts)
    ref = O.single_point(z, xyz * A2B, charge=charge, multiplicity=mult)
    _close(got, ref)
    assert abs(got["heat_of_formation_kcal"] - hof) < 5e-3


def test_water34_whole_gpu_matches_cta_path_and_oracle(whole_gpu):
    z, xyz = workloads.water_cluster(34)
    opts = native.options(p_tol=1e-8)
    got = native.run(z, xyz * A2B, opts, want_mo_energies=True)
    cta = _cta(z, xyz * A2B, opts, want_mo_energies=True)
    ref = O.single_point(z, xyz * A2B, p_tol=1e-8)
    _close(got, ref)
    _close(got, cta)
    assert np.abs(got["mo_energies"] - cta["mo_energies"]).max() < 1e-7


def test_organics_with_adiis_history_match(whole_gpu):
    for n, seed in ((24, 5), (48, 6)):
        z, xyz = workloads.organic(n, seed)
        opts = native.options()
        got = native.run(z, xyz * A2B, opts)
        ref = O.single_point(z, xyz * A2B)
        _close(got, ref)
        cta = _cta(z, xyz * A2B, opts)
        assert got["iterations"] == cta["iterations"]


def test_radical_uhf_on_whole_gpu_path(whole_gpu):
    z, xyz = workloads.radical(20, 11)
    opts = native.options(multiplicity=2, max_scf=1000)
    got = native.run(z, xyz * A2B, opts)
    ref = O.single_point(z, xyz * A2B, multiplicity=2, max_scf=1000)
    _close(got, ref)


def test_stability_search_and_core_guess_on_whole_gpu_path(whole_gpu):
    z, xyz = workloads.organic(18, 21)
    for kw in (dict(stability=2), dict(guess=2)):
        opts = native.options(**kw)
        got = native.run(z, xyz * A2B, opts)
        cta = _cta(z, xyz * A2B, opts)
        _close(got, cta)
        ref = O.single_point(z, xyz * A2B, **kw)
        _close(got, ref)


def test_gradient_on_whole_gpu_path(whole_gpu):
    tight = dict(e_tol=1e-12, p_tol=1e-11)
    for geom, mult in (("O 0.0 0.0 0.0; H 1.05 0.0 0.0; H -0.30 1.02 0.0", 1),
                       ("C 0.0 0.0 0.05; H 1.12 0.0 0.0; H -0.55 0.95 0.0; H -0.55 -0.95 0.0", 2)):
        z, xyz = parse(geom)
        got = native.run(z, xyz * A2B, native.options(multiplicity=mult, **tight), want_gradient=True)
        ref = O.single_point(z, xyz * A2B, want_gradient=True, multiplicity=mult, **tight)
        assert np.abs(got["gradient"] - ref["gradient"]).max() < GRAD_TOL


def test_batch_mixes_cta_and_whole_gpu_molecules():
    mols = [workloads.organic(12, 3), workloads.water_cluster(60, grid=(5, 4, 3)), workloads.organic(30, 4)]
    offs, z, xyz = workloads.pack(mols)
    res = native.batch(offs, z, xyz * A2B)
    for m, (zm, xm) in enumerate(mols):
        ref = O.single_point(zm, xm * A2B)
        assert res.status[m] == 0
        assert abs(res.heat_of_formation_kcal[m] - ref["heat_of_formation_kcal"]) < HOF_TOL
        assert np.abs(res.charges_of(m) - ref["charges"]).max() < Q_TOL


def test_water60_beyond_one_cta_matches_oracle():
    z, xyz = workloads.water_cluster(60, grid=(5, 4, 3))
    assert O.nao(z) == 360
    got = native.run(z, xyz * A2B, native.options(p_tol=1e-8), want_density=True)
    ref = O.single_point(z, xyz * A2B, p_tol=1e-8, want_density=True)
    _close(got, ref)
    assert np.abs(got["density"] - ref["density"]).max() < 1e-6


def _single_point(ctx, z, xyz_bohr, opts):
    import ctypes

    z = np.ascontiguousarray(z, dtype=np.int32)
    x = np.ascontiguousarray(xyz_bohr, dtype=np.float64)
    res, q = _lib.Result(), np.zeros(len(z))
    mo = np.zeros(O.nao(z))
    D = ctypes.POINTER(ctypes.c_double)
    rc = ctx.lib.pm3gpu_single_point(ctx.ptr, len(z), z.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                     x.ctypes.data_as(D), ctypes.byref(opts), ctypes.byref(res), q.ctypes.data_as(D),
                                     None, mo.ctypes.data_as(D))
    assert rc == 0, ctx.last_error()
    return res, q, mo


def test_cooperative_and_multi_launch_reductions_agree(monkeypatch):
    """The Householder panels as one cooperative launch each (default) and as five launches per
    column (PM3GPU_COOP_PANELS=0) reduce the same matrices: equal results up to summation order."""
    z, xyz = workloads.water_cluster(34)
    opts = native.options(p_tol=1e-8)
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("PM3GPU_COOP_PANELS", flag)
        ctx = _lib.Context(0)
        try:
            assert ctx.lib.pm3gpu_set_large_threshold(ctx.ptr, 1) == 0
            out.append(_single_point(ctx, z, xyz * A2B, opts))
        finally:
            ctx.close()
    (ra, qa, ma), (rb, qb, mb) = out
    assert ra.converged and rb.converged and ra.iterations == rb.iterations
    assert abs(ra.heat_of_formation_kcal - rb.heat_of_formation_kcal) < 1e-8
    assert np.abs(qa - qb).max() < 1e-9
    assert np.abs(ma - mb).max() < 1e-9


def test_whole_gpu_path_is_reproducible(whole_gpu):
    """Every sum of the whole-GPU path runs in a fixed order (per-atom Coulomb and electron-core
    sums, fixed-order grid reductions, deterministic GEMMs): two solves agree to the last bit."""
    z, xyz = workloads.water_cluster(34)
    opts = native.options(p_tol=1e-8)
    a = native.run(z, xyz * A2B, opts, want_density=True)
    b = native.run(z, xyz * A2B, opts, want_density=True)
    assert a["heat_of_formation_kcal"] == b["heat_of_formation_kcal"]
    assert a["iterations"] == b["iterations"]
    assert np.array_equal(a["density"], b["density"])
