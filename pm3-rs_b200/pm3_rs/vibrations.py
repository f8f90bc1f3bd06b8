"""Harmonic vibrational analysis of a Cartesian Hessian (host side): the post-processing of the
reference's vibrational_analysis (pm3-rs src/hessian.rs:327-415) and its rigid-body projector
(src/rigid.rs:59-300).

The Hessian (eV/Bohr^2) is mass-weighted to eV/(Angstrom^2 amu), massless sites leaving their rows
and columns at zero; the translations and rotations are built in closed form from the geometry and
the masses, orthonormalised by modified Gram-Schmidt (two passes, a candidate kept when its norm is
above 1e-6, so a linear molecule keeps five and an atom three), and projected out from both sides
before the matrix is diagonalised. The Rayleigh quotients of those directions before projection are
reported as ``rigid_residual_cm``; after diagonalisation the ``n_rigid`` eigenvectors with the most
weight in the rigid subspace get an eigenvalue of exactly zero. Frequencies carry the sign of the
eigenvalue (negative = imaginary).
"""
from __future__ import annotations

import numpy as np

# sqrt(eV / (Angstrom^2 amu)) -> cm^-1 (hessian.rs:110).
SQRT_EV_PER_ANG2_AMU_TO_CM = 521.4709
ANGSTROM_TO_BOHR = 1.0 / 0.529177210903


def signed_wavenumber(eigenvalue):
    """hessian.rs:116-122: sqrt of the magnitude, with the eigenvalue's sign."""
    lam = np.asarray(eigenvalue, dtype=np.float64)
    return np.where(lam >= 0.0, 1.0, -1.0) * SQRT_EV_PER_ANG2_AMU_TO_CM * np.sqrt(np.abs(lam))


def _orthonormalize(candidates):
    """rigid.rs:123-145: modified Gram-Schmidt, twice, dropping spanned directions."""
    basis = []
    for c in candidates:
        v = np.array(c, dtype=np.float64)
        for _ in range(2):
            for b in basis:
                v -= float(np.dot(v, b)) * b
        norm = float(np.sqrt(np.dot(v, v)))
        if norm > 1.0e-6:
            basis.append(v / norm)
    return basis


def rigid_body_basis(positions, masses, rotations: bool = True):
    """rigid.rs:59-119: translations (and rotations about the centre of mass) in mass-weighted
    coordinates, orthonormalised."""
    r = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    m = np.asarray(masses, dtype=np.float64)
    nat = len(m)
    total = float(m.sum())
    centre = (m[:, None] * r).sum(axis=0) / total if total > 0.0 else np.zeros(3)
    root = np.sqrt(m)
    cands = []
    for axis in range(3):
        v = np.zeros(3 * nat)
        v[axis::3] = root
        cands.append(v)
    if rotations:
        d = r - centre
        for axis in range(3):
            cross = np.zeros((nat, 3))
            if axis == 0:
                cross[:, 1], cross[:, 2] = -d[:, 2], d[:, 1]
            elif axis == 1:
                cross[:, 0], cross[:, 2] = d[:, 2], -d[:, 0]
            else:
                cross[:, 0], cross[:, 1] = -d[:, 1], d[:, 0]
            cands.append((root[:, None] * cross).reshape(-1))
    return _orthonormalize(cands)


def project_out_symmetric(basis, a):
    """rigid.rs:170-205: A <- (1 - P) A (1 - P), P the projector onto the basis."""
    if not basis:
        return a
    b = np.stack(basis, axis=1)
    w = a @ b
    inner = b.T @ w
    return a - b @ w.T - w @ b.T + b @ inner @ b.T


def rayleigh_quotients(basis, a):
    """rigid.rs:261-275: b^T A b per rigid direction."""
    return [float(bv @ a @ bv) for bv in basis]


def rigid_mode_indices(basis, modes):
    """rigid.rs:283-300: the len(basis) eigenvectors with the largest weight in the rigid subspace,
    chosen by rank (a stable descending sort), returned in ascending order."""
    if not basis:
        return []
    b = np.stack(basis, axis=1)
    weights = ((b.T @ modes) ** 2).sum(axis=0)
    order = sorted(range(modes.shape[1]), key=lambda k: -weights[k])
    return sorted(order[:len(basis)])


def vibrational_analysis(hessian_ev_bohr2, positions, masses) -> dict:
    """hessian.rs:327-415 from a Cartesian Hessian: frequencies_cm, eigenvalues (eV/(Angstrom^2 amu)),
    modes (mass-weighted, as columns), n_rigid, rigid_residual_cm and the unprojected hessian."""
    h = np.asarray(hessian_ev_bohr2, dtype=np.float64)
    m = np.asarray(masses, dtype=np.float64)
    md = np.repeat(m, 3)
    mij = np.sqrt(np.outer(md, md))
    a0_sq = ANGSTROM_TO_BOHR * ANGSTROM_TO_BOHR
    with np.errstate(divide="ignore", invalid="ignore"):
        mw = np.where(mij > 0.0, h * a0_sq / np.where(mij > 0.0, mij, 1.0), 0.0)
    rigid = rigid_body_basis(positions, m)
    rq = rayleigh_quotients(rigid, mw)
    residual = float(np.max(np.abs(signed_wavenumber(np.array(rq))))) if rq else 0.0
    mw = project_out_symmetric(rigid, mw)
    eigs, modes = np.linalg.eigh(mw)
    eigs = eigs.copy()
    for k in rigid_mode_indices(rigid, modes):
        eigs[k] = 0.0
    return {
        "hessian": h,
        "frequencies_cm": signed_wavenumber(eigs).tolist(),
        "eigenvalues": eigs.tolist(),
        "modes": modes,
        "n_rigid": len(rigid),
        "rigid_residual_cm": residual,
    }
