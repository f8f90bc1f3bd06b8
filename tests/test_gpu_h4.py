"""The H4 hydrogen-bond, H-H repulsion and halogen-bond corrections on the device
(pm3gpu_corrections_batch and the PM3-D3H4 / PM3-D3H4X variants of the single point, batch and
gradient) against the CPU restatement of the reference's h4.rs / hx.rs
(oracle/corrections_oracle.cpp), whose gradients come from dual numbers rather than the kernel's
hand-derived adjoints.

Bars: each correction part within 1e-12 eV of the oracle; gradients within 1e-11 eV/Bohr (the H4
kernel accumulates its triples with FP64 atomics, so the order of those sums varies in the last
bits); PM3-D3H4 single points at the SCF parity bars (1e-6 kcal/mol, 1e-6 kcal/mol/A)."""
import numpy as np
import pytest

import oracle as O
from helpers import A2B, parse
from pm3_rs import native, workloads
from test_h4_ref import ACETATE_WATER, AMMONIUM_WATER, CHLOROMETHANE_AMMONIA, DIMER_API, DIMER_H4

pytestmark = pytest.mark.gpu

PART_TOL = 1.0e-12
G_TOL = 1.0e-11
HOF_TOL = 1e-6
GRAD_TOL = 1e-6 * 0.0433641043 / 1.8897261246
AMMONIA_WATER = ("N 0 0 0; H 0.0 0.94 0.38; H 0.81 -0.47 0.38; H -0.81 -0.47 0.38; O 0 0 -2.95;"
                 " H 0 0 -1.99; H 0.93 0 -3.2")
ACETIC_WATER = ("C 0 0 0; C 1.50 0 0; O 2.10 1.05 0; O 2.15 -1.15 0; H 3.10 -1.05 0; H -0.36 1.03 0;"
                " H -0.36 -0.51 0.89; H -0.36 -0.51 -0.89; O 3.0 3.65 0; H 2.686 2.742 0; H 3.9 3.9 0")
CHLOROMETHANE_WATER = ("C 0 0 0; Cl 1.78 0 0; H -0.36 1.03 0; H -0.36 -0.51 0.89; H -0.36 -0.51 -0.89;"
                       " O 4.70 0 0; H 5.0 0.9 0; H 5.0 -0.9 0")


def _systems():
    base = [parse(g) for g in (DIMER_H4, DIMER_API, AMMONIUM_WATER, ACETATE_WATER, CHLOROMETHANE_AMMONIA,
                               AMMONIA_WATER, ACETIC_WATER, CHLOROMETHANE_WATER)]
    rng = np.random.default_rng(7)
    jittered = [(z, x + rng.normal(scale=0.12, size=x.shape)) for z, x in base]
    return base + jittered + [workloads.water_cluster(12), workloads.water_cluster(26)] + \
        workloads.organic_batch(20, 5, 40, seed=21)


@pytest.mark.parametrize("variant", [2, 3])
def test_corrections_batch_matches_the_oracle(variant):
    mols = _systems()
    offs, z, xyz = workloads.pack(mols)
    method = {2: "pm3-d3h4", 3: "pm3-d3h4x"}[variant]
    got = native.corrections_batch(offs, z, xyz * A2B, method)
    worst = {"d3": 0.0, "h4": 0.0, "hh": 0.0, "hx": 0.0, "g": 0.0}
    for m, (zm, xm) in enumerate(mols):
        p, g = O.corrections(zm, xm * A2B, variant)
        for k in ("d3", "h4", "hh", "hx"):
            worst[k] = max(worst[k], abs(got[k + "_ev"][m] - p[k]))
        worst["g"] = max(worst["g"], np.abs(got["gradient"][offs[m]:offs[m + 1]] - g).max())
    print(variant, {k: f"{v:.1e}" for k, v in worst.items()})
    assert max(worst[k] for k in ("d3", "h4", "hh", "hx")) < PART_TOL
    assert worst["g"] < G_TOL


def test_corrections_on_a_large_water_box():
    """600 atoms: the parts against the oracle's energies; the gradient of a 120-atom prefix against
    the oracle's dual numbers, and the full box's by translational invariance and central
    differences of the device's own energies."""
    z, xyz = workloads.water_cluster(200, grid=(6, 6, 6))
    x = xyz * A2B
    offs = np.array([0, len(z)], np.int32)
    got = native.corrections_batch(offs, z, x, "pm3-d3h4")
    p, _ = O.corrections(z, x, 2, want_gradient=False)
    for k in ("d3", "h4", "hh"):
        assert abs(got[k + "_ev"][0] - p[k]) < 20 * PART_TOL, k
    sub = native.corrections_batch(np.array([0, 120], np.int32), z[:120], x[:120], "pm3-d3h4")
    _, gs = O.corrections(z[:120], x[:120], 2)
    assert np.abs(sub["gradient"] - gs).max() < G_TOL
    g = got["gradient"]
    assert np.abs(g.sum(axis=0)).max() < 1e-9
    h = 1e-4
    for a, k in ((0, 0), (1, 1), (301, 2), (598, 0)):
        xp, xm = x.copy(), x.copy()
        xp[a, k] += h
        xm[a, k] -= h
        ep = native.corrections_batch(offs, z, xp, "pm3-d3h4", want_gradient=False)["total_ev"][0]
        em = native.corrections_batch(offs, z, xm, "pm3-d3h4", want_gradient=False)["total_ev"][0]
        assert abs((ep - em) / (2 * h) - g[a, k]) < 1e-7, (a, k)


@pytest.mark.parametrize("geom,method", [(DIMER_API, "pm3-d3h4"), (AMMONIA_WATER, "pm3-d3h4"),
                                         (ACETIC_WATER, "pm3-d3h4"), (CHLOROMETHANE_AMMONIA, "pm3-d3h4x"),
                                         (CHLOROMETHANE_WATER, "pm3-d3h4x")])
def test_d3h4_single_points_and_gradients_match_oracle(geom, method):
    z, xyz = parse(geom)
    variant = native._check_method(method, None)["variant"]
    got = native.run(z, xyz * A2B, native.options(variant=variant), want_gradient=True)
    ref = O.single_point(z, xyz * A2B, want_gradient=True, variant=variant)
    assert abs(got["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) < HOF_TOL
    assert np.abs(got["gradient"] - ref["gradient"]).max() < GRAD_TOL


def test_method_strings_through_the_python_api():
    """The reference's variant checks (tests/test_python_api.py:97-105, tests/api_surface.rs:38-70):
    D3 lowers the energy, D3H4 differs from D3, and X adds nothing without a halogen."""
    zd, xd = parse(DIMER_API)
    e = {m: native.single_point(zd, xd, method=m)["energy_ev"] for m in ("pm3", "pm3-d3", "pm3-d3h4", "pm3-d3h4x")}
    assert e["pm3-d3"] < e["pm3"]
    assert e["pm3-d3h4"] != e["pm3-d3"]
    assert e["pm3-d3h4x"] == e["pm3-d3h4"]
    zc, xc = parse(CHLOROMETHANE_AMMONIA)
    gx = native.gradient(zc, xc, method="pm3-d3h4x")
    g4 = native.gradient(zc, xc, method="pm3-d3h4")
    assert gx["energy_ev"] > g4["energy_ev"]  # the halogen-bond term is repulsive here
    assert np.abs(np.asarray(gx["gradient_hartree_per_bohr"]) - np.asarray(g4["gradient_hartree_per_bohr"])).max() > 0


def test_correction_entries_refuse_elements_outside_the_tables():
    """The device tables hold the s/p elements; a bromine is refused rather than given numbers that
    would differ from the reference's."""
    offs = np.array([0, 2], np.int32)
    z = np.array([35, 1], np.int32)
    x = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 2.7]])
    with pytest.raises(ValueError, match="unsupported element"):
        native.corrections_batch(offs, z, x, "pm3-d3h4x")
    with pytest.raises(ValueError, match="unsupported element"):
        native.d3_batch(offs, z, x, 1)


def test_d3h4_on_the_whole_gpu_path_and_from_device_inputs():
    """The corrections join the whole-GPU path's results (threshold 1), and the batch entry whose
    coordinates are already on the device (the corrections read the caller's arrays there)."""
    import ctypes

    import torch

    from pm3_rs import _lib

    z, xyz = workloads.water_cluster(12)
    ctx = _lib.Context()
    try:
        assert ctx.lib.pm3gpu_set_large_threshold(ctx.ptr, 1) == 0
        got = native.run(z, xyz * A2B, native.options(p_tol=1e-8, variant=2), want_gradient=True, context=ctx)
    finally:
        ctx.close()
    ref = O.single_point(z, xyz * A2B, want_gradient=True, p_tol=1e-8, variant=2)
    assert abs(got["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) < HOF_TOL
    assert np.abs(got["gradient"] - ref["gradient"]).max() < 10 * GRAD_TOL

    mols = [parse(DIMER_API), parse(ACETIC_WATER), parse(CHLOROMETHANE_AMMONIA)]
    offs, zz, xx = workloads.pack(mols)
    host = native.batch(offs, zz, xx * A2B, native.options(variant=3), want_gradient=True)
    dz = torch.tensor(np.asarray(zz, np.int32), device="cuda")
    dx = torch.tensor(np.ascontiguousarray(xx * A2B), dtype=torch.float64, device="cuda")
    doffs = torch.tensor(np.asarray(offs, np.int32), device="cuda")
    ho = np.ascontiguousarray(offs, np.int32)
    hz = np.ascontiguousarray(zz, np.int32)
    res = (_lib.Result * len(mols))()
    q = np.zeros(len(zz))
    g = np.zeros((len(zz), 3))
    c = _lib.default_context()
    torch.cuda.synchronize()
    I32, D = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)
    o = native.options(variant=3)
    rc = c.lib.pm3gpu_batch_device_inputs(c.ptr, len(mols), ctypes.c_void_p(doffs.data_ptr()),
                                          ctypes.c_void_p(dz.data_ptr()), ctypes.c_void_p(dx.data_ptr()),
                                          ho.ctypes.data_as(I32), hz.ctypes.data_as(I32), ctypes.byref(o), res,
                                          q.ctypes.data_as(D), g.ctypes.data_as(D))
    assert rc == 0, c.last_error()
    for m in range(len(mols)):
        assert res[m].status == 0
        assert abs(res[m].heat_of_formation_kcal - host.heat_of_formation_kcal[m]) < 1e-9
    # the SCF and gradient kernels sum some atom terms with atomics: the two runs agree to rounding
    assert np.abs(g - host.gradients).max() < 1e-8
