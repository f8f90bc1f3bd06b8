"""GPU (pm3gpu through its C ABI) against the CPU oracle on the same inputs.

Bars: heat of formation within 1e-6 kcal/mol, Mulliken charges within
1e-5 e, analytic gradient components within 1e-6 kcal/mol/A; H_core and Fock elements within
1e-10 eV (same FP64 formulas, different summation order).
"""
import ctypes
import json
import os

import numpy as np
import pytest

import oracle as O
from helpers import A2B, GOLDEN, KCAL_A_TO_EV_BOHR, WATER_GRAD_GEOM, WATER_GRAD_MOPAC, parse
from pm3_rs import _lib, native, workloads

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
HOF_TOL = 1e-6
Q_TOL = 1e-5
GRAD_TOL = 1e-6 * 0.0433641043 / 1.8897261246  # 1e-6 kcal/mol/A in eV/Bohr


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def gpu_core(z, xyz_bohr):
    ctx = _lib.default_context()
    n = O.nao(z)
    h = np.zeros((n, n))
    ecc = ctypes.c_double()
    z = np.ascontiguousarray(z, dtype=np.int32)
    x = np.ascontiguousarray(xyz_bohr)
    rc = ctx.lib.pm3gpu_core_hamiltonian(ctx.ptr, len(z), _ip(z), _dp(x), _dp(h), ctypes.byref(ecc))
    assert rc == 0, ctx.last_error()
    return h, ecc.value


def gpu_fock(z, xyz_bohr, pt, pa=None, pb=None):
    ctx = _lib.default_context()
    z = np.ascontiguousarray(z, dtype=np.int32)
    x = np.ascontiguousarray(xyz_bohr)
    fa = np.zeros_like(pt)
    fb = np.zeros_like(pt) if pa is not None else None
    rc = ctx.lib.pm3gpu_fock(ctx.ptr, len(z), _ip(z), _dp(x), _dp(np.ascontiguousarray(pt)),
                             None if pa is None else _dp(np.ascontiguousarray(pa)),
                             None if pb is None else _dp(np.ascontiguousarray(pb)), _dp(fa),
                             None if fb is None else _dp(fb))
    assert rc == 0, ctx.last_error()
    return fa, fb


MIXED = ("O 0.0 0.0 0.0; H 0.96 0.0 0.0; H -0.24 0.93 0.0; C 2.4 0.3 -0.7; Cl 3.9 -0.8 0.6; H 2.2 1.3 -1.2;"
         " S -1.9 -1.1 0.4; N 1.1 2.4 0.9; H 1.6 3.2 1.2; F -0.5 2.1 -1.7; Na 4.1 2.6 -2.2; Si -3.2 1.4 1.9;"
         " P 0.4 -2.6 -2.1; Mg 3.0 -3.1 2.4; Li -2.6 3.4 -1.1; B 5.2 0.1 1.0; Be -4.4 -1.9 -1.6; Al 1.9 4.4 -2.9")


def test_core_hamiltonian_matches_oracle_elementwise():
    for geom in (GOLDEN["water"][0], GOLDEN["formaldehyde"][0], MIXED):
        z, xyz = parse(geom)
        h_gpu, ecc = gpu_core(z, xyz * A2B)
        h_ref = O.core_hamiltonian(z, xyz * A2B)
        assert np.abs(h_gpu - h_ref).max() < 1e-10
        assert abs(ecc - O.core_core(z, xyz * A2B)) < 1e-9


def test_axis_aligned_pairs_both_frame_branches():
    # v_x < 0 and v_x >= 0 branches of the frame rotation, plus exactly on-axis pairs
    z, xyz = parse("C 0.0 0.0 0.0; O 1.21 0.0 0.0; N -1.47 0.0 0.0; H 0.0 0.0 1.09; S 0.0 -1.82 0.0")
    h_gpu, _ = gpu_core(z, xyz * A2B)
    assert np.abs(h_gpu - O.core_hamiltonian(z, xyz * A2B)).max() < 1e-10


def test_fock_matches_oracle_rhf_and_uhf():
    z, xyz = parse(MIXED)
    n = O.nao(z)
    rng = np.random.default_rng(3)
    a = rng.normal(size=(n, n))
    pt = (a + a.T) * 0.1
    b = rng.normal(size=(n, n))
    pa = (b + b.T) * 0.05
    pb = pt - pa
    f_gpu, _ = gpu_fock(z, xyz * A2B, pt)
    assert np.abs(f_gpu - O.fock(z, xyz * A2B, pt)).max() < 1e-10
    fa, fb = gpu_fock(z, xyz * A2B, pt, pa, pb)
    assert np.abs(fa - O.fock(z, xyz * A2B, pt, pa)).max() < 1e-10
    assert np.abs(fb - O.fock(z, xyz * A2B, pt, pb)).max() < 1e-10


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_single_point_matches_oracle(name):
    geom, charge, mult, hof = GOLDEN[name]
    z, xyz = parse(geom)
    ref = O.single_point(z, xyz * A2B, charge=charge, multiplicity=mult)
    got = native.run(z, xyz * A2B, native.options(charge, mult), want_density=True, want_mo_energies=True)
    assert got["converged"]
    assert abs(got["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) < HOF_TOL
    assert abs(got["heat_of_formation_kcal"] - hof) < 5e-3
    assert np.abs(got["charges"] - ref["charges"]).max() < Q_TOL
    assert np.abs(np.array(got["dipole_debye"]) - np.array(ref["dipole_debye"])).max() < 1e-5
    assert got["unrestricted"] == ref["unrestricted"]
    assert got["scf_paths_tried"] == ref["scf_paths_tried"]
    assert abs(got["homo_ev"] - ref["homo_ev"]) < 1e-6 and abs(got["lumo_ev"] - ref["lumo_ev"]) < 1e-6
    # the Pm3Result arrays: every alpha MO energy of the last iteration (virtuals included, from the
    # saved tridiagonal) and the total density
    refd = O.single_point(z, xyz * A2B, want_density=True, charge=charge, multiplicity=mult)
    assert np.abs(got["mo_energies"] - ref["mo_energies"]).max() < 1e-6
    assert np.abs(got["density"] - refd["density"]).max() < 1e-6


def test_python_drop_in_keys_and_units():
    z, xyz = parse(GOLDEN["water"][0])
    out = native.single_point(z, xyz)
    assert set(out) == {"energy_hartree", "energy_ev", "heat_of_formation_kcal", "electronic_ev", "core_ev",
                        "charges", "dipole_debye", "homo_ev", "lumo_ev", "converged", "unrestricted"}
    assert abs(out["heat_of_formation_kcal"] - (-53.2301514568744)) < 5e-3
    assert abs(out["energy_hartree"] * 27.211386245988 - out["energy_ev"]) < 1e-9
    assert out["unrestricted"] is False
    g = native.gradient(z, xyz)
    f = native.forces(z, xyz)
    assert np.allclose(np.array(f["forces_ev_per_angstrom"]), -np.array(g["gradient_ev_per_angstrom"]), atol=1e-12)
    uhf = native.single_point(z, xyz, reference="uhf")
    assert uhf["unrestricted"] is True
    assert abs(uhf["heat_of_formation_kcal"] - out["heat_of_formation_kcal"]) < 1e-4
    with pytest.raises(ValueError):
        native.single_point(*parse(GOLDEN["methyl_mopac"][0]), multiplicity=2, reference="rhf")


def test_mopac_subset_batch_matches_oracle_and_mopac():
    data = json.load(open(os.path.join(HERE, "golden", "mopac_sp.json")))
    rows = data["rows"]
    mols = [(np.array(r["z"], dtype=np.int32), np.array(r["xyz_angstrom"]) * A2B) for r in rows]
    offs, z, xyz = workloads.pack(mols)
    opts = [native.options(r["charge"], r["multiplicity"], max_scf=2000) for r in rows]
    res = native.batch(offs, z, xyz, opts)
    for m, r in enumerate(rows):
        ref = O.single_point(r["z"], mols[m][1], charge=r["charge"], multiplicity=r["multiplicity"], max_scf=2000)
        assert res.status[m] == 0, r["name"]
        assert abs(res.heat_of_formation_kcal[m] - ref["heat_of_formation_kcal"]) < HOF_TOL, r["name"]
        assert np.abs(res.charges_of(m) - ref["charges"]).max() < Q_TOL, r["name"]
        assert abs(res.heat_of_formation_kcal[m] - r["hof_kcal"]) < data["tolerances"]["hof_kcal"], r["name"]
        assert res.scf_paths_tried[m] == ref["scf_paths_tried"], r["name"]


def test_generated_organics_batch_matches_oracle():
    mols = workloads.organic_batch(48, 5, 60, seed=99)
    offs, z, xyz = workloads.pack(mols)
    res = native.batch(offs, z, xyz * A2B)
    for m, (zz, xx) in enumerate(mols):
        ref = O.single_point(zz, xx * A2B)
        assert res.status[m] == 0
        assert abs(res.heat_of_formation_kcal[m] - ref["heat_of_formation_kcal"]) < HOF_TOL
        assert np.abs(res.charges_of(m) - ref["charges"]).max() < Q_TOL


def test_generated_radicals_batch_matches_oracle():
    # unrestricted doublets iterate without an accelerator (scf.rs:1369-1374): give them room
    mols = workloads.radical_batch(16, 10, 40, seed=5)
    offs, z, xyz = workloads.pack(mols)
    res = native.batch(offs, z, xyz * A2B, native.options(multiplicity=2, max_scf=1000))
    for m, (zz, xx) in enumerate(mols):
        try:
            ref = O.single_point(zz, xx * A2B, multiplicity=2, max_scf=1000)
        except O.OracleError as e:
            assert e.code == 4 and res.status[m] == _lib.SCF_NOT_CONVERGED
            continue
        assert res.status[m] == 0 and res.unrestricted[m]
        assert abs(res.heat_of_formation_kcal[m] - ref["heat_of_formation_kcal"]) < HOF_TOL
        assert np.abs(res.charges_of(m) - ref["charges"]).max() < Q_TOL


def test_large_molecules_in_a_two_cta_batch_match_oracle():
    """Molecules larger than the shared-memory eigen matrix of a two-CTA-per-SM launch: 30 small
    organics keep the launch at two CTAs per SM (over 90% of the batch fits), so the water
    clusters of 26, 34 and 42 molecules (n = 156, 204, 252) run their eigensolver on a packed
    matrix in global memory. Every molecule against the oracle."""
    small = workloads.organic_batch(30, 5, 15, seed=77)
    waters = [workloads.water_cluster(26), workloads.water_cluster(34), workloads.water_cluster(42, grid=(4, 4, 3))]
    mols = small + waters
    offs, z, xyz = workloads.pack(mols)
    o = native.options(p_tol=1e-8)
    ctx = _lib.Context()
    try:
        res = native.batch(offs, z, xyz * A2B, o, context=ctx)
        ctas, nsm = ctypes.c_int(), ctypes.c_int()
        assert ctx.lib.pm3gpu_last_launch_layout(ctx.ptr, ctypes.byref(ctas), ctypes.byref(nsm)) == _lib.OK
    finally:
        ctx.close()
    assert ctas.value == 2 and nsm.value < 156, (ctas.value, nsm.value)
    for m, (zz, xx) in enumerate(mols):
        ref = O.single_point(zz, xx * A2B, p_tol=1e-8)
        assert res.status[m] == 0
        assert abs(res.heat_of_formation_kcal[m] - ref["heat_of_formation_kcal"]) < HOF_TOL, m
        assert np.abs(res.charges_of(m) - ref["charges"]).max() < Q_TOL, m


def test_water_cluster_34_matches_oracle():
    z, xyz = workloads.water_cluster(34)
    ref = O.single_point(z, xyz * A2B, p_tol=1e-8)
    got = native.run(z, xyz * A2B, native.options(p_tol=1e-8))
    assert abs(got["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) < HOF_TOL
    assert np.abs(got["charges"] - ref["charges"]).max() < Q_TOL


def test_gradient_matches_oracle_and_mopac():
    tight = dict(e_tol=1e-12, p_tol=1e-11)
    for geom, mult in ((WATER_GRAD_GEOM, 1), ("C 0.0 0.0 0.0; O 0.03 0.0 1.25; H 0.95 0.02 -0.55; H -0.94 -0.03 -0.52", 1),
                       ("C 0.0 0.0 0.05; H 1.12 0.0 0.0; H -0.55 0.95 0.0; H -0.55 -0.95 0.0", 2), (MIXED_GRAD, 1)):
        z, xyz = parse(geom)
        ref = O.single_point(z, xyz * A2B, want_gradient=True, multiplicity=mult, **tight)
        got = native.run(z, xyz * A2B, native.options(multiplicity=mult, **tight), want_gradient=True)
        assert np.abs(got["gradient"] - ref["gradient"]).max() < GRAD_TOL
    z, xyz = parse(WATER_GRAD_GEOM)
    got = native.run(z, xyz * A2B, native.options(), want_gradient=True)
    assert np.abs(got["gradient"] - np.array(WATER_GRAD_MOPAC) * KCAL_A_TO_EV_BOHR).max() < 0.02 * KCAL_A_TO_EV_BOHR


MIXED_GRAD = "S 0.0 0.0 0.0; C 1.82 0.05 0.0; H 2.2 1.05 0.1; H 2.2 -0.5 0.9; O 2.4 -0.6 -1.1; H 3.3 -0.8 -1.0; H -0.2 1.33 0.1"


def test_batch_gradients_match_single_molecule_gradients():
    mols = workloads.organic_batch(6, 8, 24, seed=31)
    offs, z, xyz = workloads.pack(mols)
    res = native.batch(offs, z, xyz * A2B, want_gradient=True)
    for m, (zz, xx) in enumerate(mols):
        ref = O.single_point(zz, xx * A2B, want_gradient=True)
        g = res.gradients[offs[m]:offs[m + 1]]
        assert np.abs(g - ref["gradient"]).max() < 1e-6  # default convergence: density noise ~1e-7


def test_edge_cases_and_errors():
    lib = _lib.load()
    # a lone hydrogen atom: one AO, a UHF doublet
    r = native.run(np.array([1], np.int32), np.zeros((1, 3)), native.options(multiplicity=2))
    ref = O.single_point([1], np.zeros((1, 3)), multiplicity=2)
    assert abs(r["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) < HOF_TOL
    # OH with multiplicity 1: odd electron count -> invalid
    with pytest.raises(ValueError):
        native.run(np.array([8, 1], np.int32), np.array([[0, 0, 0], [1.8, 0, 0.0]]), native.options())
    with pytest.raises(ValueError):
        native.run(np.array([35, 1], np.int32), np.array([[0, 0, 0], [2.7, 0, 0.0]]), native.options())
    with pytest.raises(ValueError):
        native.run(np.array([1, 1], np.int32), np.array([[0, 0, 0], [np.nan, 0, 0.0]]), native.options())
    z, xyz = parse(GOLDEN["water"][0])
    with pytest.raises(ValueError, match="did not converge"):
        native.run(z, xyz * A2B, native.options(max_scf=1))
    # a batch with good and bad molecules: per-molecule status, the good ones still solved
    mols = [(z, xyz * A2B), (np.array([35], np.int32), np.zeros((1, 3))), (np.array([8, 1], np.int32),
             np.array([[0, 0, 0], [1.8, 0, 0.0]])), (z, xyz * A2B)]
    offs, zz, xx = workloads.pack(mols)
    res = native.batch(offs, zz, xx)
    assert list(res.status) == [0, _lib.UNSUPPORTED, _lib.INVALID_INPUT, 0]
    assert abs(res.heat_of_formation_kcal[0] - res.heat_of_formation_kcal[3]) < 1e-12
    # an empty batch
    res = native.batch(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros((0, 3)))
    assert len(res.status) == 0
    assert lib.pm3gpu_last_kernel_launches(_lib.default_context().ptr) == 0


def test_batched_radical_gradients_match_oracle_at_the_parity_bar():
    """The radicals configuration's path: UHF doublets solved in one batch with analytic gradients,
    each gradient component within 1e-6 kcal/mol/A of the oracle's analytic UHF gradient
    (src/gradient.rs:494-599) at tight SCF thresholds, so the bar measures the gradient and not
    the convergence level. The batch includes organics on both sides of the per-CTA sizes used
    elsewhere (10-40 atoms)."""
    tight = dict(multiplicity=2, e_tol=1e-12, p_tol=1e-11, max_scf=2000)
    mols = workloads.radical_batch(10, 10, 40, seed=17)
    offs, z, xyz = workloads.pack(mols)
    res = native.batch(offs, z, xyz * A2B, native.options(**tight), want_gradient=True)
    checked = 0
    for m, (zz, xx) in enumerate(mols):
        try:
            ref = O.single_point(zz, xx * A2B, want_gradient=True, **tight)
        except O.OracleError as e:
            assert e.code == 4 and res.status[m] == _lib.SCF_NOT_CONVERGED
            continue
        assert res.status[m] == 0 and res.unrestricted[m] == ref["unrestricted"]
        assert abs(res.heat_of_formation_kcal[m] - ref["heat_of_formation_kcal"]) < HOF_TOL
        g = res.gradients[offs[m]:offs[m + 1]]
        assert np.abs(g - ref["gradient"]).max() < GRAD_TOL, (m, np.abs(g - ref["gradient"]).max() / GRAD_TOL)
        checked += 1
    assert checked >= 8


def test_uhf_gradient_matches_central_differences_of_gpu_energies():
    """Radical gradient (UHF) against central differences of the GPU's own total energy, step
    1e-4 A as the radicals configuration asks; all 6N displaced geometries go through one batch.
    Tight SCF thresholds and no stability search, so every displaced solve stays on the same state.
    The bar, 1e-5 eV/A, sits between the O(h^2) truncation (~1e-8) and the reference's own
    finite-difference bound (5e-5 eV/Bohr, gradient.rs:733-759)."""
    z, xyz = workloads.radical(10, 7)
    z = np.asarray(z, dtype=np.int32)
    xyz = np.asarray(xyz, dtype=np.float64)  # Angstrom
    tight = dict(multiplicity=2, e_tol=1e-12, p_tol=1e-11, max_scf=1000, stability=0)
    g = native.run(z, xyz * A2B, native.options(**tight), want_gradient=True)["gradient"]  # eV/Bohr
    h = 1e-4
    mols = []
    for a in range(len(z)):
        for k in range(3):
            for sgn in (1.0, -1.0):
                x = xyz.copy()
                x[a, k] += sgn * h
                mols.append((z, x))
    offs, zz, xx = workloads.pack(mols)
    res = native.batch(offs, zz, xx * A2B, native.options(**tight))
    assert np.all(res.status == 0) and np.all(res.unrestricted)
    e = res.total_ev.reshape(len(z), 3, 2)
    fd = (e[:, :, 0] - e[:, :, 1]) / (2 * h)  # eV/A
    assert np.abs(fd - g.reshape(-1, 3) * A2B).max() < 1e-5
