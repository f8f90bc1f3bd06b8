"""CPU restatement of the reference's geometry optimiser (pm3-rs src/optimizer.rs:77-221, `drive`
behind `optimize`), driving the oracle's run_pm3 energy and analytic gradient.

Test infrastructure only (tests/ use it as the checker of pm3gpu_optimize_batch); the product
package never imports it. Same steps in the same order as `drive`: the two-loop recursion over the
last `history` pairs with the initial Hessian scaled by s.y / y.y (0.1 / max|g| before the first
pair), the uphill guard, the backtracking Armijo search (c1 = 1e-4, step halved down to 1e-8; a
trial whose SCF fails is rejected), the curvature filter s.y > 1e-10, and the loop's iteration
count and stopping rules. Dot products are sequential sums, as the reference's iterator sums are.
Positions in Bohr, energies in eV, gradients in eV/Bohr.
"""
import numpy as np

import oracle as O


def _dot(a, b):
    s = 0.0
    for x, y in zip(a.tolist(), b.tolist()):
        s += x * y
    return s


def optimize(z, xyz_bohr, max_iter=200, gtol=1.0e-3, history=8, **scf_opts):
    """Returns dict(positions_bohr, energy_ev, heat_of_formation_kcal, converged, iterations,
    max_gradient, evaluations)."""
    x = np.asarray(xyz_bohr, dtype=np.float64).reshape(-1).copy()
    nat = len(x) // 3

    def evaluate(xv):
        r = O.single_point(z, xv.reshape(nat, 3), want_gradient=True, **scf_opts)
        g = np.asarray(r["gradient"], dtype=np.float64).reshape(-1)
        return r["total_ev"], r["heat_of_formation_kcal"], g

    def energy_only(xv):
        try:
            return O.single_point(z, xv.reshape(nat, 3), **scf_opts)["total_ev"]
        except O.OracleError:
            return None

    evals = 1
    energy, heat, g = evaluate(x)
    max_grad = float(np.abs(g).max()) if len(g) else 0.0
    S, Y, R = [], [], []
    converged = max_grad < gtol
    iterations = 0
    for it in range(max_iter):
        iterations = it + 1
        if converged:
            break
        q = g.copy()
        m = len(S)
        alpha = [0.0] * m
        for i in range(m - 1, -1, -1):
            a = R[i] * _dot(S[i], q)
            alpha[i] = a
            q = q - a * Y[i]
        if m > 0:
            sy = _dot(S[m - 1], Y[m - 1])
            yy = _dot(Y[m - 1], Y[m - 1])
            gamma = sy / yy if yy > 0.0 else 1.0
        else:
            gamma = 0.1 / max(max_grad, 1.0e-6)
        q = q * gamma
        for i in range(m):
            beta = R[i] * _dot(Y[i], q)
            q = q + (alpha[i] - beta) * S[i]
        d = -q
        if _dot(d, g) > 0.0:
            d = -g
        g_dot_d = _dot(g, d)
        step = 1.0
        ok = False
        while True:
            x_new = x + step * d
            evals += 1
            trial = energy_only(x_new)
            if trial is not None and trial <= energy + 1.0e-4 * step * g_dot_d:
                ok = True
                break
            step *= 0.5
            if step < 1.0e-8:
                break
        if not ok:
            break
        energy, heat, g_new = evaluate(x_new)
        s = x_new - x
        y = g_new - g
        sy = _dot(s, y)
        if sy > 1.0e-10:
            S.append(s)
            Y.append(y)
            R.append(1.0 / sy)
            if len(S) > history:
                S.pop(0)
                Y.pop(0)
                R.pop(0)
        x = x_new
        g = g_new
        max_grad = float(np.abs(g).max())
        converged = max_grad < gtol
    return {"positions_bohr": x.reshape(nat, 3), "energy_ev": energy, "heat_of_formation_kcal": heat,
            "converged": converged, "iterations": iterations, "max_gradient": max_grad, "evaluations": evals}
