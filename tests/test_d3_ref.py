"""The CPU restatement of the reference's D3 dispersion (oracle/corrections_oracle.cpp, the checker of the GPU
library's D3 kernels) pinned to the reference's own D3 tests (src/corrections/d3.rs:462-539): the
CN-interpolated C6 of H-H and O-O at isolated and bonded coordination numbers, the water-dimer
coordination numbers, attractive dispersion and the size of methane's D3H4 dispersion; plus the
dual-number gradient against central differences of the energy, and the variant's place in the
single point (scf.rs:740-743: added to total_ev and the heat of formation, gradient.rs:324-357: its
gradient added to the SCF gradient)."""
import numpy as np
import pytest

import oracle as O
from helpers import A2B, GOLDEN, parse
from pm3_rs import native

WATER_DIMER = ("O -1.551007 -0.114520 0.0; H -1.934259 0.762503 0.0; H -0.599677 0.040712 0.0;"
               " O 1.350625 0.111469 0.0; H 1.680398 -0.373741 -0.758561; H 1.680398 -0.373741 0.758561")
METHANE = "C 0 0 0; H 0.629 0.629 0.629; H -0.629 -0.629 0.629; H -0.629 0.629 -0.629; H 0.629 -0.629 -0.629"
EV_TO_KCAL = 23.06054783061903


def test_c6_is_cn_interpolated_as_the_reference_asserts():
    h_iso, h_bond = O.d3_c6(1, 1, 0.0, 0.0), O.d3_c6(1, 1, 1.0, 1.0)
    o_iso, o_bond = O.d3_c6(8, 8, 0.0, 0.0), O.d3_c6(8, 8, 2.0, 2.0)
    assert 7.0 < h_iso < 7.6 and 2.8 < h_bond < 3.3 and h_iso > h_bond
    assert 15.0 < o_iso < 15.6 and 10.0 < o_bond < 11.0 and o_iso > o_bond
    # the pair key is (max Z, min Z) with the coordination numbers aligned to it
    assert O.d3_c6(8, 1, 1.9, 0.9) == O.d3_c6(1, 8, 0.9, 1.9)


def test_water_dimer_components_are_sane():
    z, x = parse(WATER_DIMER)
    e, g, cn = O.d3(z, x * A2B, 1)
    assert abs(cn[0] - 2.0) < 0.1 and abs(cn[1] - 1.0) < 0.1
    assert O.d3_c6(8, 8, cn[0], cn[3]) > 10.0
    assert e < 0.0


def test_methane_d3h4_dispersion_is_small_and_negative():
    z, x = parse(METHANE)
    e, _, _ = O.d3(z, x * A2B, 2)
    assert -1.0 < e < 0.0


@pytest.mark.parametrize("d3_set", [1, 2])
def test_dual_number_gradient_matches_central_differences(d3_set):
    z, x = parse(WATER_DIMER)
    x = x * A2B
    _, g, _ = O.d3(z, x, d3_set)
    h = 1.0e-5
    fd = np.zeros_like(g)
    for a in range(len(z)):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd[a, k] = (O.d3(z, xp, d3_set)[0] - O.d3(z, xm, d3_set)[0]) / (2 * h)
    assert np.abs(fd - g).max() < 1e-9 * max(1.0, np.abs(g).max()) + 1e-11
    assert np.abs(g.sum(axis=0)).max() < 1e-14  # translation costs nothing


def test_pm3_d3_single_point_adds_the_dispersion_energy_and_gradient():
    z, x = parse(WATER_DIMER)
    x = x * A2B
    plain = O.single_point(z, x, want_gradient=True)
    d3 = O.single_point(z, x, want_gradient=True, variant=1)
    e, g, _ = O.d3(z, x, 1)
    assert d3["total_ev"] == pytest.approx(plain["total_ev"] + e, abs=1e-12)
    assert d3["heat_of_formation_kcal"] == pytest.approx(plain["heat_of_formation_kcal"] + e * EV_TO_KCAL, abs=1e-9)
    assert d3["total_ev"] < plain["total_ev"]  # dispersion is attractive (tests/api_surface.rs:38-70)
    assert np.abs(d3["gradient"] - (plain["gradient"] + g)).max() < 1e-12


def test_method_strings_parse_like_the_reference():
    """corrections::Variant::parse (src/corrections/mod.rs:180-191, tests/api_surface.rs:224-240)."""
    v = lambda m: native._check_method(m, None)["variant"]
    assert v("pm3") == 0 and v(" ") == 0
    assert v("PM3-D3") == 1 and v("pm3_d3") == 1
    assert v("pm3-d3h4") == 2 and v("PM3 D3H4X") == 3
    assert native._check_method("pm3-d3h4+mmok", None) == {"variant": 2, "mmok": 1}
    assert native._check_method("pm3+mmok", None) == {"variant": 0, "mmok": 1}
    assert native._check_method("pm3", None)["mmok"] == 0
    for bad in ("am1", "pm3-d3+mmok+mmok"):
        with pytest.raises(ValueError):
            native._check_method(bad, None)
    with pytest.raises(ValueError):
        native._check_method("pm3", [0.0, 0.0, 0.01])
