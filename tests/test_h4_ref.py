"""The CPU restatement of the reference's H4, H-H and halogen-bond corrections
(oracle/corrections_oracle.cpp, the checker of the GPU library's H4 kernel) pinned to the reference's
own tests: h4.rs:391-418 (no bridging hydrogen, no H4; the water dimer's H4 is attractive; H-H at
1.2 Angstrom repels), hx.rs:91-117 (no halogen, no X; Cl...N at 3 Angstrom small, positive and
decaying) and tests/api_surface.rs:38-70 (on a halogen-free dimer PM3-D3H4 differs from PM3-D3 and
PM3-D3H4X equals PM3-D3H4); plus the dual-number gradients against central differences on systems
that switch on the water, NR4+ and carboxylate scale factors, and the variants' place in the single
point."""
import numpy as np
import pytest

import oracle as O
from helpers import A2B, parse

DIMER_H4 = "O 0.0 0.0 0.0; H 0.0 0.0 0.96; H 0.93 0.0 -0.24; O 0.0 0.0 2.90; H 0.0 0.76 3.15; H 0.0 -0.76 3.15"
DIMER_API = "O 0.0 0.0 0.0; H 0.96 0.0 0.0; H -0.24 0.93 0.0; O 2.9 0.0 0.0; H 3.2 0.9 0.0; H 3.2 -0.5 0.8"
AMMONIUM_WATER = ("N 0 0 0; H 0.6 0.6 0.6; H -0.6 -0.6 0.6; H -0.6 0.6 -0.6; H 0.6 -0.6 -0.6; O 1.65 1.65 1.65;"
                  " H 2.2 1.4 2.3; H 2.2 2.2 1.1")
ACETATE_WATER = ("C 0 0 0; C 1.52 0 0; O 2.15 1.08 0; O 2.15 -1.08 0; H -0.38 1.02 0; H -0.38 -0.51 0.88;"
                 " H -0.38 -0.51 -0.88; O 4.9 1.3 0; H 3.95 1.2 0; H 5.2 0.4 0")
CHLOROMETHANE_AMMONIA = ("C 0 0 0; Cl 1.78 0 0; H -0.36 1.03 0; H -0.36 -0.51 0.89; H -0.36 -0.51 -0.89;"
                         " N 4.80 0 0; H 5.18 0.94 0; H 5.18 -0.47 0.81; H 5.18 -0.47 -0.81")


def _parts(geom, variant, grad=False):
    z, x = parse(geom)
    p, g = O.corrections(z, x * A2B, variant, want_gradient=grad)
    return p, g


def test_h4_and_hx_follow_the_reference_unit_tests():
    assert _parts("N 0 0 0; N 0 0 1.1", 2)[0]["h4"] == 0.0
    assert _parts(DIMER_H4, 2)[0]["h4"] < 0.0
    assert _parts("H 0 0 0; H 0 0 1.2", 2)[0]["hh"] > 0.0
    assert _parts("H 0 0 0; H 0 0 0.74", 3)[0]["hx"] == 0.0
    near = _parts("Cl 0 0 0; N 0 0 3.0", 3)[0]["hx"]
    far = _parts("Cl 0 0 0; N 0 0 5.0", 3)[0]["hx"]
    assert np.isfinite(near) and 0.0 < near < 0.5 and far < near


def test_variants_on_the_api_surface_dimer():
    z, x = parse(DIMER_API)
    x = x * A2B
    e = {v: O.single_point(z, x, variant=v)["total_ev"] for v in (0, 1, 2, 3)}
    assert e[1] < e[0]
    assert e[2] != e[1]
    assert e[3] == e[2]  # no halogen: X contributes exactly nothing


def test_scale_factors_switch_on():
    """The contacts that switch on the NR4+ donor factor (ammonium, valence 4), the carboxylate
    acceptor factor (acetate) and the Cl...N halogen bond give H-bond attraction and X repulsion."""
    nh4, _ = _parts(AMMONIUM_WATER, 2)
    assert nh4["h4"] < 0.0
    ac, _ = _parts(ACETATE_WATER, 2)
    assert ac["h4"] < 0.0
    cl, _ = _parts(CHLOROMETHANE_AMMONIA, 3)
    assert cl["hx"] > 0.0


@pytest.mark.parametrize("geom", [DIMER_H4, AMMONIUM_WATER, ACETATE_WATER, CHLOROMETHANE_AMMONIA])
@pytest.mark.parametrize("seed", [0, 1])
def test_dual_number_gradients_match_central_differences(geom, seed):
    z, x = parse(geom)
    rng = np.random.default_rng(seed)
    x = (x + (rng.normal(scale=0.12, size=x.shape) if seed else 0.0)) * A2B
    _, g = O.corrections(z, x, 3)
    h = 1.0e-5
    fd = np.zeros_like(g)
    for a in range(len(z)):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd[a, k] = (sum(O.corrections(z, xp, 3, False)[0].values()) -
                        sum(O.corrections(z, xm, 3, False)[0].values())) / (2 * h)
    assert np.abs(fd - g).max() < 2e-8 * max(1.0, np.abs(g).max())
    assert np.abs(g.sum(axis=0)).max() < 1e-12


def test_d3h4_single_point_adds_the_parts():
    z, x = parse(DIMER_API)
    x = x * A2B
    plain = O.single_point(z, x, want_gradient=True)
    for v in (2, 3):
        r = O.single_point(z, x, want_gradient=True, variant=v)
        p, g = O.corrections(z, x, v)
        assert r["total_ev"] == pytest.approx(plain["total_ev"] + sum(p.values()), abs=1e-12)
        assert np.abs(r["gradient"] - (plain["gradient"] + g)).max() < 1e-12
        assert p["d3"] == pytest.approx(O.d3(z, x, 2, want_gradient=False)[0], abs=1e-15)
