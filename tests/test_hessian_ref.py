"""The CPU restatement of the reference's gradient-difference Hessian (oracle/hessian_ref.py, the
checker of pm3gpu_numerical_hessian_batch) and the host-side vibrational analysis
(pm3_rs/vibrations.py), pinned to the reference's own test (tests/molecules.rs:121-138): water
relaxed to its PM3 minimum has its bend and two O-H stretches at MOPAC's FORCE frequencies
1743.46, 3868.68 and 3989.81 cm^-1 (the reference asserts 2 cm^-1)."""
import ctypes

import numpy as np
import pytest

import hessian_ref
import lbfgs_ref
import oracle as O
from helpers import A2B, GOLDEN, parse
from pm3_rs import _lib, vibrations
from pm3_rs.native import atomic_masses


@pytest.fixture(scope="module")
def relaxed_water():
    z, xyz = parse(GOLDEN["water"][0])
    r = lbfgs_ref.optimize(z, xyz * A2B)
    assert r["converged"]
    return z, r["positions_bohr"]


def test_restated_hessian_reproduces_the_mopac_water_frequencies(relaxed_water):
    z, x = relaxed_water
    h = hessian_ref.numerical_hessian(z, x)
    assert np.array_equal(h, h.T)
    masses = [O.element(int(v))["mass"] for v in z]
    assert masses == atomic_masses(z)
    vib = vibrations.vibrational_analysis(h, x, masses)
    assert vib["n_rigid"] == 6
    f = np.array(vib["frequencies_cm"])
    assert np.count_nonzero(f == 0.0) == 6
    top3 = np.sort(f)[-3:]
    for got, want in zip(top3, [1743.46, 3868.68, 3989.81]):
        assert abs(got - want) < 2.0, (got, want)
    # at a minimum the rigid directions carry almost nothing before projection
    assert vib["rigid_residual_cm"] < 50.0


def test_restated_hessian_obeys_translational_invariance(relaxed_water):
    """Moving every atom alike costs nothing: each row summed over the atoms, axis by axis, is zero
    up to the central difference's error."""
    z, x = relaxed_water
    h = hessian_ref.numerical_hessian(z, x)
    nat = len(z)
    sums = h.reshape(3 * nat, nat, 3).sum(axis=1)
    assert np.abs(sums).max() < 1.0e-4 * np.abs(h).max()


def test_rigid_basis_rank_follows_the_geometry():
    m = [12.011, 15.999, 15.999]
    linear = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 2.2], [0.0, 0.0, -2.2]])
    bent = np.array([[0.0, 0.0, 0.0], [0.0, 1.5, 1.5], [0.0, -1.5, 1.5]])
    assert len(vibrations.rigid_body_basis(linear, m)) == 5
    assert len(vibrations.rigid_body_basis(bent, m)) == 6
    assert len(vibrations.rigid_body_basis(np.zeros((1, 3)), [1.008])) == 3
    b = np.stack(vibrations.rigid_body_basis(bent, m), axis=1)
    assert np.allclose(b.T @ b, np.eye(6), atol=1e-12)


def test_projection_removes_the_rigid_subspace_from_both_sides():
    rng = np.random.default_rng(3)
    x = rng.normal(size=(4, 3))
    m = [12.0, 1.0, 1.0, 16.0]
    basis = vibrations.rigid_body_basis(x, m)
    a = rng.normal(size=(12, 12))
    a = a + a.T
    p = vibrations.project_out_symmetric(basis, a)
    b = np.stack(basis, axis=1)
    assert np.allclose(p, p.T, atol=1e-12)
    assert np.abs(p @ b).max() < 1e-10
    # the complement is untouched: (1-P) A (1-P) restricted there equals A
    q = np.eye(12) - b @ b.T
    assert np.allclose(p, q @ a @ q, atol=1e-12)


def test_signed_wavenumber_keeps_the_sign():
    assert vibrations.signed_wavenumber(4.0) == pytest.approx(2 * 521.4709)
    assert vibrations.signed_wavenumber(-4.0) == pytest.approx(-2 * 521.4709)
    assert vibrations.signed_wavenumber(0.0) == 0.0


def test_hessian_entry_rejects_bad_arguments_without_a_device():
    L = _lib.load()
    offs = np.array([0, 3], np.int32)
    z = np.array([8, 1, 1], np.int32)
    x = np.zeros(9)
    h = np.zeros(81)
    st = np.zeros(1, np.int32)
    I32, D = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)
    args = (offs.ctypes.data_as(I32), z.ctypes.data_as(I32), x.ctypes.data_as(D))
    assert L.pm3gpu_numerical_hessian_batch(None, 1, *args, None, 1e-3, h.ctypes.data_as(D),
                                            st.ctypes.data_as(I32)) == _lib.INVALID_INPUT
