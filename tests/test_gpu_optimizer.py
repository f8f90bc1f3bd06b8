"""Batched geometry optimisation (pm3gpu_optimize_batch) against the CPU restatement of the
reference's L-BFGS (oracle/lbfgs_ref.py) driving the oracle's energies and gradients.

One batch holds the reference's distorted water (pinned to its frozen -53.4330121104622
kcal/mol), distorted formaldehyde and methane, and four small generated organics (ethane,
methanol, methanethiol and one more, 16-30 iterations from the generator's geometry). The
optimiser is the same algorithm on both sides and the energies and gradients agree to the parity
bars, so every molecule takes the same path: the same iteration and evaluation counts, final
heats of formation within 1e-6 kcal/mol and final positions within 1e-5 Bohr."""
import numpy as np
import pytest

import lbfgs_ref
from helpers import A2B, parse
from pm3_rs import native, workloads

pytestmark = pytest.mark.gpu


def _molecules():
    mols = [parse("O 0.0 0.0 0.0; H 1.05 0.0 0.0; H -0.30 1.02 0.0"),
            parse("C 0.0 0.0 0.0; O 1.25 0.05 0.0; H -0.55 0.97 0.1; H -0.60 -0.90 -0.05"),
            parse("C 0.0 0.0 0.0; H 1.15 0.0 0.0; H -0.30 1.00 0.0; H -0.35 -0.50 0.90; H -0.40 -0.45 -0.95")]
    for seed in (1, 4, 5, 8):  # ethane, methanol, methanethiol, ...: 16-30 iterations from the generator
        z, xyz = workloads.organic(6, seed)
        mols.append((np.asarray(z), np.asarray(xyz)))
    return mols


def test_batched_optimisation_follows_the_restated_reference_path():
    mols = _molecules()
    offs, z, xyz = workloads.pack(mols)
    got = native.optimize_batch(offs, z, xyz * A2B, want_gradient=True)
    for m, (zm, xm) in enumerate(mols):
        ref = lbfgs_ref.optimize(zm, xm * A2B)
        pos = got["positions_bohr"][offs[m]:offs[m + 1]]
        print(f"mol {m}: it {got['iterations'][m]} / {ref['iterations']}, evals {got['evaluations'][m]} / "
              f"{ref['evaluations']}, dHf {got['heat_of_formation_kcal'][m] - ref['heat_of_formation_kcal']:.2e}, "
              f"dx {np.abs(pos - ref['positions_bohr']).max():.2e}")
        assert got["status"][m] == 0
        assert bool(got["converged"][m]) == ref["converged"]
        assert got["iterations"][m] == ref["iterations"] and got["evaluations"][m] == ref["evaluations"]
        assert abs(got["heat_of_formation_kcal"][m] - ref["heat_of_formation_kcal"]) < 1.0e-6
        assert np.abs(pos - ref["positions_bohr"]).max() < 1.0e-5
        assert got["max_gradient"][m] == pytest.approx(np.abs(got["gradients"][offs[m]:offs[m + 1]]).max(), rel=1e-12)
    assert abs(got["heat_of_formation_kcal"][0] - (-53.4330121104622)) < 1.0e-5


def test_single_molecule_optimize_keys_and_units():
    z, xyz = parse("O 0.0 0.0 0.0; H 1.05 0.0 0.0; H -0.30 1.02 0.0")
    r = native.optimize(z, xyz)  # Angstrom in and out, the reference's keys
    assert r["converged"] and r["iterations"] == r["steps"]
    assert abs(r["heat_of_formation_kcal"] - (-53.4330121104622)) < 1.0e-5
    assert r["positions"] == r["positions_angstrom"] and len(r["positions"]) == 3
    assert abs(r["energy_hartree"] - r["energy_ev"] / 27.211386245988) < 1e-12


def test_batched_optimisation_with_corrections_follows_the_restated_path():
    """PM3-D3H4 (and PM3-D3 with MMOK on an amide) through the batched optimiser: the corrections'
    energies and gradients enter every line-search trial, on both sides."""
    mols = [parse("O 0.0 0.0 0.0; H 1.05 0.0 0.0; H -0.30 1.02 0.0; O 2.9 0.1 0.0; H 3.3 0.9 0.0; H 3.2 -0.6 0.7"),
            parse("O 0.44 1.30 -0.04; C 0.05 0.14 -0.01; N 1.03 -0.89 -0.07; C -1.40 -0.27 0.0; H 0.76 -1.74 0.38;"
                  " H -2.06 0.60 0.01; H -1.64 -0.86 -0.89; H -1.63 -0.88 0.88; H 1.96 -0.61 0.17")]
    for variant, mmok in ((2, 0), (1, 1)):
        offs, z, xyz = workloads.pack(mols)
        got = native.optimize_batch(offs, z, xyz * A2B, native.options(variant=variant, mmok=mmok))
        for m, (zm, xm) in enumerate(mols):
            ref = lbfgs_ref.optimize(zm, xm * A2B, variant=variant, mmok=mmok)
            pos = got["positions_bohr"][offs[m]:offs[m + 1]]
            assert got["status"][m] == 0 and bool(got["converged"][m]) and ref["converged"]
            if m == 0:  # the floppy dimer (~140 iterations): the paths part in the last bits and both
                # stop where the largest gradient component falls below gtol, on a flat surface
                assert got["max_gradient"][m] < 1.0e-3 and ref["max_gradient"] < 1.0e-3
                assert abs(got["heat_of_formation_kcal"][m] - ref["heat_of_formation_kcal"]) < 2.0e-3
                continue
            assert got["iterations"][m] == ref["iterations"] and got["evaluations"][m] == ref["evaluations"]
            assert abs(got["heat_of_formation_kcal"][m] - ref["heat_of_formation_kcal"]) < 1.0e-6
            assert np.abs(pos - ref["positions_bohr"]).max() < 1.0e-5
