"""The D3 dispersion correction on the device (pm3gpu_d3_batch and the PM3-D3 variant of the single
point, batch and gradient) against the CPU restatement of the reference's d3.rs
(oracle/corrections_oracle.cpp), whose gradient comes from dual numbers rather than the kernels' analytic
derivatives.

Bars: D3 energies within 1e-12 eV and gradients within 1e-12 eV/Bohr of the oracle (FP64 on both
sides; the device's exp / pow and FMA contraction differ from the host's in the last bits); PM3-D3
single points at the SCF parity bars of the plain path (1e-6 kcal/mol, 1e-6 kcal/mol/A)."""
import numpy as np
import pytest

import oracle as O
from helpers import A2B, GOLDEN, parse
from pm3_rs import _lib, native, workloads

pytestmark = pytest.mark.gpu

E_TOL = 1.0e-12
G_TOL = 1.0e-12
HOF_TOL = 1e-6
GRAD_TOL = 1e-6 * 0.0433641043 / 1.8897261246
WATER_DIMER = ("O 0.0 0.0 0.0; H 0.96 0.0 0.0; H -0.24 0.93 0.0; O 2.9 0.0 0.0; H 3.2 0.9 0.0; H 3.2 -0.5 0.8")


def _mols():
    mols = [parse(GOLDEN[k][0]) for k in ("water", "ammonia", "formaldehyde", "methane", "h2s", "hcl")]
    mols.append(parse(WATER_DIMER))
    mols += workloads.organic_batch(40, 5, 60, seed=11)
    mols.append(workloads.water_cluster(34))
    return mols


@pytest.mark.parametrize("d3_set", [1, 2])
def test_d3_batch_matches_the_oracle(d3_set):
    mols = _mols()
    offs, z, xyz = workloads.pack(mols)
    got = native.d3_batch(offs, z, xyz * A2B, d3_set)
    worst_e = worst_g = 0.0
    for m, (zm, xm) in enumerate(mols):
        e, g, _ = O.d3(zm, xm * A2B, d3_set)
        worst_e = max(worst_e, abs(got["energy_ev"][m] - e))
        worst_g = max(worst_g, np.abs(got["gradient"][offs[m]:offs[m + 1]] - g).max())
    print(f"set {d3_set}: max |dE| {worst_e:.2e} eV, max |dg| {worst_g:.2e} eV/Bohr")
    assert worst_e < E_TOL and worst_g < G_TOL


def test_d3_batch_on_a_large_molecule_matches_oracle_energy_and_differences():
    """A 600-atom water box: the energy against the oracle's; the gradient of its 90-atom prefix
    against the oracle's dual-number gradient (O(n^3), slow at full size), and the full box's
    against central differences of the device's own energies and by translational invariance."""
    z, xyz = workloads.water_cluster(200, grid=(6, 6, 6))
    x = xyz * A2B
    sub = native.d3_batch(np.array([0, 90], np.int32), z[:90], x[:90], 1)
    ref_e, ref_g, _ = O.d3(z[:90], x[:90], 1)
    assert abs(sub["energy_ev"][0] - ref_e) < E_TOL and np.abs(sub["gradient"] - ref_g).max() < G_TOL
    offs = np.array([0, len(z)], np.int32)
    got = native.d3_batch(offs, z, x, 1)
    assert abs(got["energy_ev"][0] - O.d3(z, x, 1, want_gradient=False)[0]) < 10 * E_TOL
    g = got["gradient"]
    assert np.abs(g.sum(axis=0)).max() < 1e-10
    h = 1e-4
    for a, k in ((0, 0), (17, 1), (333, 2), (599, 0)):
        xp, xm = x.copy(), x.copy()
        xp[a, k] += h
        xm[a, k] -= h
        fd = (native.d3_batch(offs, z, xp, 1)["energy_ev"][0] - native.d3_batch(offs, z, xm, 1)["energy_ev"][0]) / (2 * h)
        assert abs(fd - g[a, k]) < 1e-8, (a, k, fd, g[a, k])


@pytest.mark.parametrize("name", ["water", "formaldehyde", "ammonia", "h2s"])
def test_pm3_d3_single_point_and_gradient_match_oracle(name):
    geom, charge, mult, _ = GOLDEN[name]
    z, xyz = parse(geom)
    got = native.run(z, xyz * A2B, native.options(charge, mult, variant=1), want_gradient=True)
    ref = O.single_point(z, xyz * A2B, want_gradient=True, charge=charge, multiplicity=mult, variant=1)
    plain = O.single_point(z, xyz * A2B, charge=charge, multiplicity=mult)
    assert ref["total_ev"] < plain["total_ev"]
    assert abs(got["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) < HOF_TOL
    assert np.abs(got["gradient"] - ref["gradient"]).max() < GRAD_TOL


def test_variants_mix_in_one_batch_and_through_the_python_api():
    """Per-molecule options: the PM3-D3 molecules get the correction, the plain ones do not; the
    water dimer of the reference's variant test (tests/api_surface.rs:38-70) is lowered by D3."""
    mols = workloads.organic_batch(12, 5, 30, seed=5) + [parse(WATER_DIMER)]
    offs, z, xyz = workloads.pack(mols)
    opts = [native.options(variant=m % 2) for m in range(len(mols))]
    res = native.batch(offs, z, xyz * A2B, opts, want_gradient=True)
    for m, (zm, xm) in enumerate(mols):
        ref = O.single_point(zm, xm * A2B, want_gradient=True, variant=m % 2)
        assert res.status[m] == 0
        assert abs(res.heat_of_formation_kcal[m] - ref["heat_of_formation_kcal"]) < HOF_TOL, m
        assert np.abs(res.gradients[offs[m]:offs[m + 1]] - ref["gradient"]).max() < GRAD_TOL, m
    zd, xd = parse(WATER_DIMER)
    plain = native.single_point(zd, xd)["energy_ev"]
    d3 = native.single_point(zd, xd, method="pm3-d3")["energy_ev"]
    assert d3 < plain
    e, _, _ = O.d3(zd, xd * A2B, 1)
    assert d3 - plain == pytest.approx(e, abs=1e-9)


def test_pm3_d3_on_the_whole_gpu_path_matches_oracle():
    """A water cluster sent to the whole-GPU path (threshold 1): the correction joins that path's
    results too."""
    z, xyz = workloads.water_cluster(26)
    ctx = _lib.Context()
    try:
        assert ctx.lib.pm3gpu_set_large_threshold(ctx.ptr, 1) == 0
        got = native.run(z, xyz * A2B, native.options(p_tol=1e-8, variant=1), want_gradient=True, context=ctx)
    finally:
        ctx.close()
    ref = O.single_point(z, xyz * A2B, want_gradient=True, p_tol=1e-8, variant=1)
    assert abs(got["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) < HOF_TOL
    assert np.abs(got["gradient"] - ref["gradient"]).max() < 10 * GRAD_TOL


def test_d3_batch_rejects_bad_arguments():
    offs = np.array([0, 3], np.int32)
    z = np.array([8, 1, 1], np.int32)
    with pytest.raises(ValueError):
        native.d3_batch(offs, z, np.zeros((3, 3)), 3)
    with pytest.raises(ValueError):
        native.d3_batch(offs, z, np.full((3, 3), np.nan), 1)
