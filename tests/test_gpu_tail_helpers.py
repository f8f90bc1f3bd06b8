"""Two-CTA unrestricted jobs (pm3gpu_set_tail_helpers): CTAs left without work take the beta spin
of unaccelerated unrestricted jobs still running. The results equal the one-CTA results within the
parity bars of the GPU suite (the two runs differ only in the summation order of the electronic
energy), and the oracle's."""
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


def _two_ways(offs, z, xyz, opts, want_gradient=False):
    solo, duo = _lib.Context(), _lib.Context()
    try:
        assert duo.lib.pm3gpu_set_tail_helpers(duo.ptr, 1) == 0
        a = native.batch(offs, z, xyz, opts, want_gradient=want_gradient, context=solo)
        b = native.batch(offs, z, xyz, opts, want_gradient=want_gradient, context=duo)
        return a, b, duo.lib.pm3gpu_last_paired_jobs(duo.ptr), solo.lib.pm3gpu_last_paired_jobs(solo.ptr)
    finally:
        solo.close()
        duo.close()


def test_radicals_on_two_ctas_match_one_cta_and_the_oracle():
    # uneven sizes: the small radicals finish first and their CTAs take the large ones' beta spin
    mols = workloads.radical_batch(24, 6, 60, seed=61)
    offs, z, xyz = workloads.pack(mols)
    # tight thresholds, so that the gradient bar measures the gradient and not the convergence level
    tight = dict(multiplicity=2, e_tol=1e-12, p_tol=1e-11, max_scf=2000)
    opts = native.options(**tight)
    a, b, paired, paired_solo = _two_ways(offs, z, xyz * A2B, opts, want_gradient=True)
    assert paired >= 1 and paired_solo == 0
    assert np.array_equal(a.status, b.status)
    ok = a.status == 0
    assert ok.sum() >= 20
    assert np.abs(a.heat_of_formation_kcal[ok] - b.heat_of_formation_kcal[ok]).max() < HOF_TOL
    assert np.abs(a.gradients - b.gradients).max() < GRAD_TOL
    for m in range(len(mols)):
        if ok[m]:
            assert np.abs(a.charges_of(m) - b.charges_of(m)).max() < Q_TOL
            assert a.unrestricted[m] == b.unrestricted[m]
    for m in np.flatnonzero(ok)[:4]:  # and the oracle
        zz, xx = mols[m]
        ref = O.single_point(zz, xx * A2B, **tight)
        assert abs(b.heat_of_formation_kcal[m] - ref["heat_of_formation_kcal"]) < HOF_TOL


def test_unrestricted_rungs_of_closed_shells_on_two_ctas():
    """The stability search's unrestricted rung with a level shift and no accelerator
    (src/scf.rs:610-678) runs paired; the selected state and paths tried are unchanged."""
    mols = [workloads.organic(n, 700 + n) for n in (6, 9, 14, 22, 31, 40)]
    offs, z, xyz = workloads.pack(mols)
    opts = native.options(stability=2)
    a, b, paired, _ = _two_ways(offs, z, xyz * A2B, opts)
    assert paired >= 1
    assert np.array_equal(a.status, b.status) and np.array_equal(a.scf_paths_tried, b.scf_paths_tried)
    assert np.array_equal(a.unrestricted, b.unrestricted)
    assert np.abs(a.heat_of_formation_kcal - b.heat_of_formation_kcal).max() < HOF_TOL
