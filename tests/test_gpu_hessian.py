"""Batched gradient-difference Hessians (pm3gpu_numerical_hessian_batch) against the CPU
restatement of the reference's numerical_hessian (oracle/hessian_ref.py) driving the oracle's
gradients, and the frequencies built from them against the reference's MOPAC-pinned water test
(tests/molecules.rs:121-138).

Both sides difference gradients that agree to the gradient parity bar (about 1e-9 eV/Bohr under
the tightened SCF), divided by 2h = 2e-3 Bohr, so the Hessians agree to about 1e-6 eV/Bohr^2; the
bar is 1e-5 eV/Bohr^2 on entries of order 1-50."""
import numpy as np
import pytest

import hessian_ref
from helpers import A2B, GOLDEN, parse
from pm3_rs import native, workloads

pytestmark = pytest.mark.gpu

HESSIAN_ATOL = 1.0e-5  # eV/Bohr^2


def _molecules():
    mols = [parse(GOLDEN[k][0]) for k in ("water", "ammonia", "formaldehyde", "methane", "h2s", "hcl")]
    for seed in (1, 4, 5):
        z, xyz = workloads.organic(6, seed)
        mols.append((np.asarray(z), np.asarray(xyz)))
    return mols


def test_batched_hessians_match_the_restated_reference():
    mols = _molecules()
    offs, z, xyz = workloads.pack(mols)
    got = native.numerical_hessian_batch(offs, z, xyz * A2B)
    for m, (zm, xm) in enumerate(mols):
        ref = hessian_ref.numerical_hessian(zm, xm * A2B)
        h = got["hessians"][m]
        err = np.abs(h - ref).max()
        print(f"mol {m} ({len(zm)} atoms): max |dH| {err:.2e} eV/Bohr^2 of max |H| {np.abs(ref).max():.1f}")
        assert got["status"][m] == 0
        assert h.shape == (3 * len(zm), 3 * len(zm))
        assert np.array_equal(h, h.T)
        assert err < HESSIAN_ATOL


def test_frequencies_of_the_relaxed_water_match_mopac():
    z, xyz = parse(GOLDEN["water"][0])
    r = native.optimize(z, xyz)
    f = native.frequencies(z, r["positions_angstrom"])
    assert f["n_rigid"] == 6 and f["masses"] == native.atomic_masses(z)
    v = np.array(f["frequencies_cm"])
    assert np.count_nonzero(v == 0.0) == 6
    for got, want in zip(np.sort(v)[-3:], [1743.46, 3868.68, 3989.81]):
        assert abs(got - want) < 2.0, (got, want)
    h = native.hessian(z, r["positions_angstrom"])
    assert h["ndof"] == 9 and len(h["hessian_hartree_per_bohr2"]) == 9


def test_a_failing_molecule_keeps_its_own_status():
    """An element outside the path fails its own molecule only (its block stays zero); an empty
    molecule has an empty Hessian."""
    water = parse(GOLDEN["water"][0])
    iron = (np.array([26, 1], np.int32), np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.6]]))
    empty = (np.zeros(0, np.int32), np.zeros((0, 3)))
    offs, z, xyz = workloads.pack([water, iron, empty, water])
    got = native.numerical_hessian_batch(offs, z, xyz * A2B)
    assert got["status"][0] == 0 and got["status"][3] == 0 and got["status"][2] == 0
    assert got["status"][1] != 0 and not got["hessians"][1].any()
    assert got["hessians"][2].shape == (0, 0)
    assert np.abs(got["hessians"][0] - got["hessians"][3]).max() < 1.0e-6
    with pytest.raises(ValueError):
        native.numerical_hessian_batch(offs, z, xyz * A2B, step=0.0)


def test_open_shell_and_linear_molecules():
    """A doublet radical (UHF gradients through the batched launch) against the oracle, and a
    linear molecule, whose rigid subspace has rank five."""
    z, xyz = parse(GOLDEN["methyl_mopac"][0])
    got = native.numerical_hessian_batch(np.array([0, len(z)], np.int32), z, xyz * A2B,
                                         native.options(multiplicity=2))
    ref = hessian_ref.numerical_hessian(z, xyz * A2B, multiplicity=2)
    assert got["status"][0] == 0
    assert np.abs(got["hessians"][0] - ref).max() < HESSIAN_ATOL
    hcn_z = [1, 6, 7]
    hcn = [[0.0, 0.0, -1.07], [0.0, 0.0, 0.0], [0.0, 0.0, 1.16]]
    f = native.frequencies(hcn_z, hcn)
    assert f["n_rigid"] == 5 and np.count_nonzero(np.array(f["frequencies_cm"]) == 0.0) == 5


def test_documented_example_block():
    """The reference's documented example (tests/test_python_api.py:285-308): PM3-D3H4
    optimisation, frequencies at the minimum, and a cation's gradient."""
    numbers = [8, 1, 1]
    positions = np.array([[0.00, 0.00, 0.00], [0.96, 0.00, 0.00], [-0.24, 0.93, 0.00]])
    assert np.isfinite(native.single_point(numbers, positions)["heat_of_formation_kcal"])
    opt = native.optimize(numbers, positions, method="pm3-d3h4")
    assert opt["converged"]
    freqs = native.frequencies(numbers, opt["positions_angstrom"], method="pm3-d3h4")
    assert len(freqs["frequencies_cm"]) == 9
    assert min(freqs["frequencies_cm"]) >= 0.0  # a minimum: no imaginary mode
    nh4 = np.array([[0.0, 0.0, 0.0], [0.63, 0.63, 0.63], [-0.63, -0.63, 0.63], [-0.63, 0.63, -0.63],
                    [0.63, -0.63, -0.63]])
    g = native.gradient([7, 1, 1, 1, 1], nh4, charge=1, multiplicity=1)
    assert np.asarray(g["gradient_hartree_per_bohr"]).shape == (5, 3)


def test_hessian_with_corrections_matches_the_restated_reference():
    """PM3-D3H4X on a hydrogen-bonded and a halogen-bonded pair: the corrections' gradients enter
    every displaced evaluation on both sides."""
    mols = [parse("O 0.0 0.0 0.0; H 0.96 0.0 0.0; H -0.24 0.93 0.0; O 2.9 0.0 0.0; H 3.2 0.9 0.0; H 3.2 -0.5 0.8"),
            parse("C 0 0 0; Cl 1.78 0 0; H -0.36 1.03 0; H -0.36 -0.51 0.89; H -0.36 -0.51 -0.89; N 4.80 0 0;"
                  " H 5.18 0.94 0; H 5.18 -0.47 0.81; H 5.18 -0.47 -0.81")]
    offs, z, xyz = workloads.pack(mols)
    got = native.numerical_hessian_batch(offs, z, xyz * A2B, native.options(variant=3))
    for m, (zm, xm) in enumerate(mols):
        ref = hessian_ref.numerical_hessian(zm, xm * A2B, variant=3)
        assert got["status"][m] == 0
        assert np.abs(got["hessians"][m] - ref).max() < HESSIAN_ATOL
