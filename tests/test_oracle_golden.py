"""The CPU oracle against the reference's own known answers (CPU only).

Pins the oracle before it is trusted as the GPU checker: every golden number below is
quoted in pm3-rs's tests (tests/molecules.rs, tests/mopac_oracle.rs, src/scf.rs,
src/overlap.rs, src/gradient.rs, src/params.rs), with the reference's tolerances.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from helpers import A2B, GOLDEN, KCAL_A_TO_EV_BOHR, WATER_GRAD_GEOM, WATER_GRAD_MOPAC, parse

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_heat_of_formation_matches_reference_golden(name):
    geom, charge, mult, hof = GOLDEN[name]
    z, xyz = parse(geom)
    r = O.single_point(z, xyz * A2B, charge=charge, multiplicity=mult)
    assert r["converged"]
    assert abs(r["heat_of_formation_kcal"] - hof) < 5e-3  # tests/molecules.rs tolerance
    assert abs(r["charges"].sum() - charge) < 1e-6


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_heat_of_formation_matches_reference_golden_tightly(name):
    """The same known answers at the level the restatement reaches (largest error 2.5e-7
    kcal/mol, ammonia): a regression of 1e-6 kcal/mol, the GPU parity bar, fails here."""
    geom, charge, mult, hof = GOLDEN[name]
    z, xyz = parse(geom)
    r = O.single_point(z, xyz * A2B, charge=charge, multiplicity=mult)
    assert abs(r["heat_of_formation_kcal"] - hof) < 1e-6


def test_water_dipole_and_charges():
    z, xyz = parse(GOLDEN["water"][0])
    r = O.single_point(z, xyz * A2B)
    assert abs(np.linalg.norm(r["dipole_debye"]) - 1.762063533710513) < 2e-3  # scf.rs:1902
    assert r["charges"][0] < -0.3 and r["charges"][1] > 0.1


def test_methyl_radical_is_unrestricted_with_one_unpaired_electron():
    z, xyz = parse(GOLDEN["methyl_1079"][0])
    r = O.single_point(z, xyz * A2B, multiplicity=2)
    assert r["unrestricted"] and r["converged"]


def test_oh_overlap_matches_mopac():  # overlap.rs:688-705
    p = O.pair(8, 1, [1.05 * A2B, 0.0, 0.0])
    assert abs(p["s"][0, 0] - 0.2502982386931348) < 1e-10
    assert abs(p["s"][1, 0]) > 0.1
    assert abs(p["s"][2, 0]) < 1e-14 and abs(p["s"][3, 0]) < 1e-14


def test_parameters_match_mopac_table():  # params.rs:827-848
    h = O.element(1)
    assert abs(h["uss"] + 13.073321) < 1e-9 and abs(h["betas"] + 5.626512) < 1e-9
    assert abs(h["zs"] - 0.967807) < 1e-9 and abs(h["gss"] - 14.794208) < 1e-9
    assert h["n_orb"] == 1 and h["dd"] == 0.0
    c = O.element(6)
    assert abs(c["uss"] + 47.270320) < 1e-9
    assert c["dd"] > 0 and c["qq"] > 0 and c["rho1"] > 0 and c["rho2"] > 0


def test_ssss_integral_is_rotation_invariant():  # integrals.rs:584-594
    r = 2.6
    a = O.pair(6, 6, [r, 0.0, 0.0])
    v = np.array([0.3, -0.5, 0.8])
    b = O.pair(6, 6, r * v / np.linalg.norm(v))
    assert abs(a["w"][0, 0] - b["w"][0, 0]) < 1e-9
    rho0 = O.element(6)["rho0"]
    assert abs(a["w"][0, 0] - 27.211386245988 / np.sqrt(r * r + (2 * rho0) ** 2)) < 1e-9


def test_fock_is_symmetric():  # fock.rs:626-642
    z, xyz = parse("C 0.0 0.0 0.0; O 0.0 0.0 1.21; H 0.94 0.0 -0.54; H -0.94 0.0 -0.54")
    n = O.nao(z)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    p = 0.37 * ((np.maximum(i, j) * 7 + np.minimum(i, j) * 3) % 11) - 1.1
    f = O.fock(z, xyz * A2B, p)
    assert np.abs(f - f.T).max() < 1e-12


def test_water_gradient_matches_mopac():  # gradient.rs:648-679
    z, xyz = parse(WATER_GRAD_GEOM)
    r = O.single_point(z, xyz * A2B, want_gradient=True)
    ref = np.array(WATER_GRAD_MOPAC) * KCAL_A_TO_EV_BOHR
    assert np.abs(r["gradient"] - ref).max() < 0.02 * KCAL_A_TO_EV_BOHR


def test_gradient_matches_finite_difference_of_energy():  # gradient.rs:681-705
    z, xyz = parse("C 0.0 0.0 0.0; O 0.03 0.0 1.25; H 0.95 0.02 -0.55; H -0.94 -0.03 -0.52")
    x = xyz * A2B
    opts = dict(e_tol=1e-12, p_tol=1e-11)
    g = O.single_point(z, x, want_gradient=True, **opts)["gradient"]
    h = 1e-4
    for a in range(len(z)):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd = (O.single_point(z, xp, **opts)["total_ev"] - O.single_point(z, xm, **opts)["total_ev"]) / (2 * h)
            assert abs(g[a, k] - fd) < 5e-5


def test_uhf_gradient_matches_finite_difference():  # gradient.rs:733-759
    z, xyz = parse("C 0.0 0.0 0.05; H 1.12 0.0 0.0; H -0.55 0.95 0.0; H -0.55 -0.95 0.0")
    x = xyz * A2B
    opts = dict(multiplicity=2, e_tol=1e-12, p_tol=1e-11)
    g = O.single_point(z, x, want_gradient=True, **opts)["gradient"]
    h = 1e-4
    for a in range(len(z)):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd = (O.single_point(z, xp, **opts)["total_ev"] - O.single_point(z, xm, **opts)["total_ev"]) / (2 * h)
            assert abs(g[a, k] - fd) < 5e-5


def test_accelerators_agree():  # scf.rs:1937-1963
    z, xyz = parse("C 0.0 0.0 0.0; O 0.0 0.0 1.21; H 0.94 0.0 -0.54; H -0.94 0.0 -0.54")
    e = [O.single_point(z, xyz * A2B, accelerator=a)["total_ev"] for a in (2, 1, 0)]
    assert abs(e[0] - e[1]) < 1e-6 and abs(e[0] - e[2]) < 1e-6


def test_mopac_oracle_subset():
    """The s/p rows of tests/data/mopac_oracle.tsv at the tolerances of tests/mopac_oracle.rs."""
    data = json.load(open(os.path.join(HERE, "golden", "mopac_sp.json")))
    tol = data["tolerances"]
    assert len(data["rows"]) >= 100
    for row in data["rows"]:
        r = O.single_point(row["z"], np.array(row["xyz_angstrom"]) * A2B, charge=row["charge"],
                           multiplicity=row["multiplicity"], max_scf=2000)
        assert abs(r["heat_of_formation_kcal"] - row["hof_kcal"]) < tol["hof_kcal"], row["name"]
        # tighter than the reference's tolerance: what the restatement reaches against the table
        # (largest 1.4e-5 kcal/mol without silicon, 1.5e-4 with it; median 4e-7)
        tight = 2e-4 if 14 in row["z"] else 2e-5
        assert abs(r["heat_of_formation_kcal"] - row["hof_kcal"]) < tight, row["name"]
        if row["dipole_debye"] is not None:
            assert abs(np.linalg.norm(r["dipole_debye"]) - row["dipole_debye"]) < tol["dipole_debye"], row["name"]
        if row["charges"]:
            assert np.abs(r["charges"] - np.array(row["charges"])).max() < tol["charge_e"], row["name"]
        if row["ip_ev"] is not None and r["homo_ev"] is not None:
            assert abs(-r["homo_ev"] - row["ip_ev"]) < tol["ip_ev"], row["name"]


def test_stability_search_rescues_hard_cases():  # tests/mopac_oracle.rs:282-323
    data = json.load(open(os.path.join(HERE, "golden", "mopac_sp.json")))
    rows = {r["name"]: r for r in data["rows"]}
    for name in ("butyne", "ketene", "methyl_radical"):
        if name not in rows:
            continue
        row = rows[name]
        args = dict(charge=row["charge"], multiplicity=row["multiplicity"], max_scf=2000)
        on = O.single_point(row["z"], np.array(row["xyz_angstrom"]) * A2B, **args)
        off = O.single_point(row["z"], np.array(row["xyz_angstrom"]) * A2B, stability=0, **args)
        assert abs(on["heat_of_formation_kcal"] - row["hof_kcal"]) < 2e-3
        assert on["scf_paths_tried"] > 1 and on["scf_improvement_ev"] > 1e-3
        assert abs(off["heat_of_formation_kcal"] - row["hof_kcal"]) > 2e-3


def test_invalid_inputs_are_rejected():
    z, xyz = parse("O 0.0 0.0 0.0; H 0.9584 0.0 0.0")  # OH radical as a singlet: parity error
    with pytest.raises(O.OracleError) as e:
        O.single_point(z, xyz * A2B)
    assert e.value.code == 1
    with pytest.raises(O.OracleError) as e:
        O.single_point(np.array([35, 1]), np.array([[0, 0, 0], [1.4, 0, 0.0]]) * A2B)
    assert e.value.code == 2
    z, xyz = parse(GOLDEN["water"][0])
    with pytest.raises(O.OracleError) as e:
        O.single_point(z, xyz * A2B, max_scf=1)
    assert e.value.code == 4
