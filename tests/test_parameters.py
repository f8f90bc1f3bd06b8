"""The &Pm3Parameters argument of run_pm3 (pm3-rs src/scf.rs:450-452) across the C ABI.

pm3gpu_standard_parameters is Pm3Parameters::standard() (src/params.rs:133-137) for the s/p path;
pm3gpu_set_parameters hands a caller's set to a context. The oracle takes the same structures
(oracle_set_parameters), so a perturbed set can be checked on both sides.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from helpers import A2B, GOLDEN, parse
from pm3_rs import _lib, native

WATER_Z, _w = parse(GOLDEN["water"][0])
WATER_XYZ = _w * A2B
FORMALDEHYDE_Z, _f = parse(GOLDEN["formaldehyde"][0])
FORMALDEHYDE_XYZ = _f * A2B


def _status(ctx, z, xyz):
    """pm3gpu_single_point's status code (native.run turns non-OK into ValueError)."""
    res, q = _lib.Result(), np.zeros(len(z))
    x = np.ascontiguousarray(xyz, dtype=np.float64)
    return ctx.lib.pm3gpu_single_point(ctx.ptr, len(z), z.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                       x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(native.options()),
                                       ctypes.byref(res), q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None, None)


def _by_z(elems):
    return {e.z: e for e in elems}


@pytest.fixture
def oracle_params():
    yield
    O.reset_parameters()


def test_standard_set_matches_the_oracle_derivation():
    """Raw and derived constants of every element equal the oracle's restatement of
    params.rs:155-343 (oracle_element: n_orb, uss, upp, zs, zp, betas, betap, gss, gsp, gpp, gp2,
    hsp, alpha, core, dd, qq, rho0, rho1, rho2, e_isol, eheat_ev, mass). Host-only call."""
    elems, pairs = _lib.standard_parameters()
    assert len(elems) == 15 and len(pairs) >= 1
    for e in elems:
        ref = np.zeros(22)
        assert O.lib().oracle_element(e.z, ref.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
        got = [e.n_orb, e.u_ss, e.u_pp, e.zeta_s, e.zeta_p, e.beta_s, e.beta_p, e.g_ss, e.g_sp, e.g_pp, e.g_p2,
               e.h_sp, e.alpha, e.core_charge, e.dd, e.qq, e.rho0, e.rho1, e.rho2, e.e_isol, e.eheat_ev, e.mass]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12, err_msg=f"Z={e.z}")
        assert e.po[9] == e.rho0 and e.po[1] == e.rho0
        if e.n_orb == 4:
            assert e.ddp[2] == e.dd and e.ddp[3] == pytest.approx(e.qq * np.sqrt(2.0), rel=1e-15)
    c = _by_z(elems)[6]
    assert c.u_ss == -47.27032 and c.beta_p == -9.802755  # src/params.rs:827-848


def test_oracle_takes_the_standard_set_unchanged(oracle_params):
    """The standard set handed back through oracle_set_parameters reproduces the built-in one
    bit for bit (water, src/scf.rs:1890-1906: -53.2301514568744 kcal/mol)."""
    base = O.single_point(WATER_Z, WATER_XYZ)
    elems, pairs = _lib.standard_parameters()
    O.set_parameters(elems, pairs)
    again = O.single_point(WATER_Z, WATER_XYZ)
    assert again["heat_of_formation_kcal"] == base["heat_of_formation_kcal"]
    assert abs(base["heat_of_formation_kcal"] - (-53.2301514568744)) < 1e-6


def test_oracle_uses_a_perturbed_parameter_and_reports_missing_elements(oracle_params):
    elems, pairs = _lib.standard_parameters()
    base = O.single_point(FORMALDEHYDE_Z, FORMALDEHYDE_XYZ)["heat_of_formation_kcal"]
    _by_z(elems)[6].beta_p += 0.5
    O.set_parameters(elems, pairs)
    moved = O.single_point(FORMALDEHYDE_Z, FORMALDEHYDE_XYZ)["heat_of_formation_kcal"]
    assert abs(moved - base) > 0.1
    without_c = (_lib.Element * (len(elems) - 1))(*[e for e in elems if e.z != 6])
    O.set_parameters(without_c, pairs)
    with pytest.raises(O.OracleError) as err:
        O.single_point(FORMALDEHYDE_Z, FORMALDEHYDE_XYZ)
    assert err.value.code == 2  # Pm3Error::MissingElement


def test_set_parameters_rejects_bad_entries_without_a_device():
    """Argument checks run before any CUDA call: a null context is rejected outright."""
    elems, pairs = _lib.standard_parameters()
    L = _lib.load()
    assert L.pm3gpu_set_parameters(None, elems, len(elems), pairs, len(pairs)) == _lib.INVALID_INPUT


@pytest.mark.gpu
def test_perturbed_parameters_match_the_oracle_fed_the_same_set(oracle_params):
    """One perturbed parameter (carbon beta_p + 0.5 eV, oxygen u_pp - 0.3 eV): GPU and oracle,
    both given the same set, agree within the parity bars (1e-6 kcal/mol, 1e-5 e); the standard
    set restores the standard answer; an element left out gives PM3GPU_MISSING_ELEMENT."""
    ctx = _lib.Context()
    try:
        std = native.run(FORMALDEHYDE_Z, FORMALDEHYDE_XYZ, native.options(), context=ctx)
        elems, pairs = _lib.standard_parameters()
        _by_z(elems)[6].beta_p += 0.5
        _by_z(elems)[8].u_pp -= 0.3
        assert ctx.lib.pm3gpu_set_parameters(ctx.ptr, elems, len(elems), pairs, len(pairs)) == _lib.OK
        O.set_parameters(elems, pairs)
        for z, xyz in ((FORMALDEHYDE_Z, FORMALDEHYDE_XYZ), (WATER_Z, WATER_XYZ)):
            got = native.run(z, xyz, native.options(), context=ctx)
            ref = O.single_point(z, xyz)
            assert abs(got["heat_of_formation_kcal"] - ref["heat_of_formation_kcal"]) < 1e-6
            assert np.abs(got["charges"] - ref["charges"]).max() < 1e-5
        moved = native.run(FORMALDEHYDE_Z, FORMALDEHYDE_XYZ, native.options(), context=ctx)
        assert abs(moved["heat_of_formation_kcal"] - std["heat_of_formation_kcal"]) > 0.1
        # back to the standard set
        elems, pairs = _lib.standard_parameters()
        assert ctx.lib.pm3gpu_set_parameters(ctx.ptr, elems, len(elems), pairs, len(pairs)) == _lib.OK
        back = native.run(FORMALDEHYDE_Z, FORMALDEHYDE_XYZ, native.options(), context=ctx)
        assert back["heat_of_formation_kcal"] == std["heat_of_formation_kcal"]
        # carbon left out: MissingElement, as Pm3Parameters::element reports it
        without_c = (_lib.Element * (len(elems) - 1))(*[e for e in elems if e.z != 6])
        assert ctx.lib.pm3gpu_set_parameters(ctx.ptr, without_c, len(without_c), pairs, len(pairs)) == _lib.OK
        assert _status(ctx, FORMALDEHYDE_Z, FORMALDEHYDE_XYZ) == _lib.MISSING_ELEMENT
        assert "Z=6" in ctx.last_error()
        # a non-finite entry is refused and leaves the set as it was
        bad, _ = _lib.standard_parameters()
        bad[0].u_ss = float("nan")
        assert ctx.lib.pm3gpu_set_parameters(ctx.ptr, bad, len(bad), pairs, len(pairs)) == _lib.INVALID_INPUT
        assert _status(ctx, FORMALDEHYDE_Z, FORMALDEHYDE_XYZ) == _lib.MISSING_ELEMENT
    finally:
        ctx.close()
