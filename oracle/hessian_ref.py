"""CPU restatement of the reference's gradient-difference Hessian (pm3-rs src/hessian.rs:268-319,
`numerical_hessian`), driving the oracle's run_pm3 analytic gradient.

Test infrastructure only (tests/ use it as the checker of pm3gpu_numerical_hessian_batch); the
product package never imports it. Same steps: the SCF tightened for second derivatives
(hessian.rs:169-175: e_tol <= 1e-12, p_tol <= 1e-11, max_scf >= 500), column j = 3 * atom + axis
from the central difference (g(x + h e_j) - g(x - h e_j)) / (2h), then the average with the
transpose (hessian.rs:86-95). Positions in Bohr, Hessian in eV/Bohr^2.
"""
import numpy as np

import oracle as O


def tightened(e_tol=1.0e-8, p_tol=1.0e-7, max_scf=200, **opts):
    opts = dict(opts)
    opts["e_tol"] = min(e_tol, 1.0e-12)
    opts["p_tol"] = min(p_tol, 1.0e-11)
    opts["max_scf"] = max(max_scf, 500)
    return opts


def numerical_hessian(z, xyz_bohr, step=1.0e-3, **scf_opts):
    x0 = np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    nat = len(x0)
    nd = 3 * nat
    opts = tightened(**scf_opts)
    h = np.zeros((nd, nd))
    for j in range(nd):
        a, k = divmod(j, 3)
        plus = x0.copy()
        minus = x0.copy()
        plus[a, k] += step
        minus[a, k] -= step
        gp = O.single_point(z, plus, want_gradient=True, **opts)["gradient"].reshape(-1)
        gm = O.single_point(z, minus, want_gradient=True, **opts)["gradient"].reshape(-1)
        h[:, j] = (gp - gm) / (2.0 * step)
    for i in range(nd):
        for j in range(i):
            v = 0.5 * (h[i, j] + h[j, i])
            h[i, j] = v
            h[j, i] = v
    return h


AU_DIPOLE_TO_DEBYE = 2.541746473  # constants.rs:64


def fixed_origin_dipole(z, x, charge, res):
    """The dipole about the coordinate origin (e Bohr) from a result's centre-of-mass dipole:
    mu_0 = mu_COM + Q R_COM."""
    m = np.array([O.element(int(v))["mass"] for v in z])
    com = (m[:, None] * np.asarray(x).reshape(-1, 3)).sum(axis=0) / m.sum()
    return np.asarray(res["dipole_debye"]) / AU_DIPOLE_TO_DEBYE + charge * com


def dipole_derivatives(z, xyz_bohr, step=1.0e-3, charge=0.0, **scf_opts):
    """d mu / d R (elementary charges, 3 x 3N) by central differences of the fixed-origin dipole
    under the tightened SCF: the quantity the reference's analytic dipole_derivatives
    (src/ir.rs:103-190) is checked against in its own tests (src/ir.rs:393-436)."""
    x0 = np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    nd = 3 * len(x0)
    opts = tightened(**scf_opts)
    out = np.zeros((3, nd))
    for j in range(nd):
        a, k = divmod(j, 3)
        mus = []
        for sign in (1.0, -1.0):
            x = x0.copy()
            x[a, k] += sign * step
            r = O.single_point(z, x, charge=charge, **opts)
            mus.append(fixed_origin_dipole(z, x, charge, r))
        out[:, j] = (mus[0] - mus[1]) / (2.0 * step)
    return out
