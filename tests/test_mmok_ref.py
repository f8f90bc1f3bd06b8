"""The CPU restatement of MOPAC's MMOK amide term (oracle/corrections_oracle.cpp, the checker of the
GPU library's MMOK kernel) pinned to the reference's tests: src/corrections/mmok.rs:150-224 (a planar
amide costs nothing and a perpendicular one the full constant; amines and N-H-free carbonyls do
not count; each amide hydrogen adds its own term) and tests/test_python_api.py:108-168 (acetamide:
MOPAC v23.2.5 gives -51.032295890 kcal/mol with NOMM and -48.705646220 by default, the reference
asserts 2e-3; the term moves the heat of formation, not the wavefunction, and reaches the
gradient)."""
import numpy as np
import pytest

import oracle as O
from helpers import A2B

K_EV = 7.185300 / 23.06054783061903
ACETAMIDE_Z = [8, 6, 7, 6, 1, 1, 1, 1, 1]
ACETAMIDE_R = np.array([
    [0.443779398, 1.296449633, -0.035323927], [0.052004373, 0.138591678, -0.005705918],
    [1.033082758, -0.888429398, -0.066016666], [-1.395111112, -0.272769730, -0.000022728],
    [0.760253342, -1.735205329, 0.378344955], [-2.061780078, 0.599727626, 0.013338598],
    [-1.639979626, -0.861723040, -0.894240325], [-1.632894254, -0.884590928, 0.880357946],
    [1.959783051, -0.608911632, 0.167787223]])


def _mmok(z, pos_bohr):
    return O.corrections(z, np.asarray(pos_bohr, float), 0, want_gradient=True, mmok=True)


def test_torsion_term_follows_the_reference_unit_tests():
    # coordinates are Bohr, as the reference's unit tests pass them
    planar = [[0.0, 1.22, 0.0], [0.0, 0.0, 0.0], [1.36, 0.0, 0.0], [1.86, 0.87, 0.0]]
    perp = [[0.0, 1.22, 0.0], [0.0, 0.0, 0.0], [1.36, 0.0, 0.0], [1.86, 0.0, 0.87]]
    assert abs(_mmok([8, 6, 7, 1], planar)[0]["mmok"]) < 1e-12
    assert abs(_mmok([8, 6, 7, 1], perp)[0]["mmok"] - K_EV) < 1e-9
    assert _mmok([7, 1, 6], [[0, 0, 0], [1.0, 0, 0], [0, 1.47, 0]])[0]["mmok"] == 0.0
    assert _mmok([8, 6, 7, 6], [[0, 1.22, 0], [0, 0, 0], [1.36, 0, 0], [1.86, 1.4, 0]])[0]["mmok"] == 0.0
    two = [[0.0, 1.22, 0.0], [0.0, 0.0, 0.0], [1.36, 0.0, 0.0], [1.86, 0.0, 0.87], [1.86, 0.0, -0.87]]
    assert abs(_mmok([8, 6, 7, 1, 1], two)[0]["mmok"] - 2 * K_EV) < 1e-9


def test_acetamide_matches_mopac_with_and_without_mmok():
    x = ACETAMIDE_R * A2B
    plain = O.single_point(ACETAMIDE_Z, x)
    mm = O.single_point(ACETAMIDE_Z, x, mmok=1)
    assert abs(plain["heat_of_formation_kcal"] - (-51.032295890)) < 2e-3
    assert abs(mm["heat_of_formation_kcal"] - (-48.705646220)) < 2e-3
    assert plain["electronic_ev"] == mm["electronic_ev"]
    assert np.array_equal(plain["charges"], mm["charges"])


def test_mmok_gradient_matches_central_differences():
    x = ACETAMIDE_R * A2B
    rng = np.random.default_rng(2)
    x = x + rng.normal(scale=0.05, size=x.shape)
    _, g = _mmok(ACETAMIDE_Z, x)
    assert np.abs(g).max() > 1e-4
    h = 1e-5
    for a in range(len(ACETAMIDE_Z)):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd = (_mmok(ACETAMIDE_Z, xp)[0]["mmok"] - _mmok(ACETAMIDE_Z, xm)[0]["mmok"]) / (2 * h)
            assert abs(fd - g[a, k]) < 1e-9
