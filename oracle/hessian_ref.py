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
