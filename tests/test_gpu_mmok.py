"""MOPAC's MMOK amide term on the device (the ``+mmok`` method suffix, ``pm3gpu_options.mmok``)
against the CPU restatement (oracle/corrections_oracle.cpp) and the reference's acetamide test
(tests/test_python_api.py:125-168: MOPAC v23.2.5 gives -51.032295890 kcal/mol with NOMM and
-48.705646220 by default; the reference asserts 2e-3). Bars: the SCF parity bars of the plain path
(1e-6 kcal/mol, 1e-6 kcal/mol/A)."""
import numpy as np
import pytest

import oracle as O
from helpers import A2B, GOLDEN, parse
from pm3_rs import native, workloads
from test_mmok_ref import ACETAMIDE_R, ACETAMIDE_Z

pytestmark = pytest.mark.gpu

HOF_TOL = 1e-6
GRAD_TOL = 1e-6 * 0.0433641043 / 1.8897261246
FORMAMIDE_TWISTED = "O 0 1.22 0; C 0 0 0; N 1.36 0 0; H 1.86 0.5 0.72; H 1.86 -0.4 -0.75; H -0.95 -0.55 0"


def test_acetamide_follows_the_reference_python_test():
    plain = native.single_point(ACETAMIDE_Z, ACETAMIDE_R, method="pm3")
    corrected = native.single_point(ACETAMIDE_Z, ACETAMIDE_R, method="pm3+mmok")
    assert abs(plain["heat_of_formation_kcal"] - (-51.032295890)) < 2e-3
    assert abs(corrected["heat_of_formation_kcal"] - (-48.705646220)) < 2e-3
    assert plain["electronic_ev"] == corrected["electronic_ev"]
    assert plain["homo_ev"] == corrected["homo_ev"] and plain["charges"] == corrected["charges"]
    assert native.single_point(ACETAMIDE_Z, ACETAMIDE_R, method="pm3-d3h4+mmok")["energy_ev"] != \
        native.single_point(ACETAMIDE_Z, ACETAMIDE_R, method="pm3-d3h4")["energy_ev"]
    wz, wx = parse(GOLDEN["water"][0])
    assert native.single_point(wz, wx, method="pm3+mmok")["energy_ev"] == native.single_point(wz, wx)["energy_ev"]
    g0 = np.asarray(native.gradient(ACETAMIDE_Z, ACETAMIDE_R, method="pm3")["gradient_ev_per_angstrom"])
    g1 = np.asarray(native.gradient(ACETAMIDE_Z, ACETAMIDE_R, method="pm3+mmok")["gradient_ev_per_angstrom"])
    assert np.abs(g1 - g0).max() > 1e-3


@pytest.mark.parametrize("variant", [0, 2])
def test_mmok_batches_match_oracle(variant):
    """Acetamide, a twisted formamide and generated organics, every other molecule with MMOK."""
    mols = [(np.array(ACETAMIDE_Z, np.int32), ACETAMIDE_R), parse(FORMAMIDE_TWISTED)] + \
        workloads.organic_batch(10, 5, 30, seed=3)
    offs, z, xyz = workloads.pack(mols)
    opts = [native.options(variant=variant, mmok=(m + 1) % 2) for m in range(len(mols))]
    res = native.batch(offs, z, xyz * A2B, opts, want_gradient=True)
    for m, (zm, xm) in enumerate(mols):
        ref = O.single_point(zm, xm * A2B, want_gradient=True, variant=variant, mmok=(m + 1) % 2)
        assert res.status[m] == 0
        assert abs(res.heat_of_formation_kcal[m] - ref["heat_of_formation_kcal"]) < HOF_TOL, m
        assert np.abs(res.gradients[offs[m]:offs[m + 1]] - ref["gradient"]).max() < GRAD_TOL, m
