// Batched geometry optimisation (host side): the reference's L-BFGS (pm3-rs src/optimizer.rs:77-221,
// `drive` behind `optimize`) run for many molecules at once, every energy and gradient coming from
// the batched SCF + gradient launch. Included by pm3gpu.cu inside its private namespace, after
// run_batch.
//
// Per molecule the state machine follows `drive` line by line: the two-loop recursion over the
// last `history` pairs (s, y) with the initial Hessian scaled by s.y / y.y (0.1 / max|g| before the
// first pair), the uphill guard, the backtracking Armijo search (c1 = 1e-4, step halved until
// 1e-8; a geometry whose SCF does not converge is a rejected step), the curvature filter
// s.y > 1e-10, and the iteration count and stopping rules of its loop. A round evaluates every
// molecule's pending geometry (its start, or its current trial) in one batched call with
// gradients; an accepted trial keeps that gradient, which is what `drive` recomputes at the same
// geometry (the same deterministic SCF).
#pragma once
// (needs <deque>, included by pm3gpu.cu before its private namespace)

struct OptMol {
  int m = 0, na = 0, a0 = 0;
  std::vector<double> x, g, d, xn;
  std::deque<std::vector<double>> S, Y;
  std::deque<double> rho;
  double e = 0.0, hof = 0.0, maxg = 0.0, gd = 0.0, step = 1.0;
  int it = 0, iterations = 0, evals = 0, status = PM3GPU_OK;
  bool conv = false, done = false, first = true;
};

inline double opt_dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}
inline void opt_axpy(std::vector<double>& y, double a, const std::vector<double>& x) {
  for (size_t i = 0; i < y.size(); ++i) y[i] += a * x[i];
}
inline double opt_maxabs(const std::vector<double>& g) {
  double m = 0.0;
  for (double v : g) m = std::max(m, std::fabs(v));
  return m;
}

// `for iter in 0..max_iter { iterations = iter + 1; if converged { break } ... }`: start the next
// iteration (direction and first trial point) or finish.
inline void opt_start_iteration(OptMol& s, const pm3gpu_opt_options& o) {
  if (s.it >= o.max_iter) {
    s.done = true;
    return;
  }
  s.iterations = s.it + 1;
  ++s.it;
  if (s.conv) {
    s.done = true;
    return;
  }
  std::vector<double> q = s.g;
  const int mh = (int)s.S.size();
  std::vector<double> alpha(mh, 0.0);
  for (int i = mh - 1; i >= 0; --i) {
    const double a = s.rho[i] * opt_dot(s.S[i], q);
    alpha[i] = a;
    opt_axpy(q, -a, s.Y[i]);
  }
  double gamma;
  if (mh > 0) {
    const double sy = opt_dot(s.S[mh - 1], s.Y[mh - 1]);
    const double yy = opt_dot(s.Y[mh - 1], s.Y[mh - 1]);
    gamma = yy > 0.0 ? sy / yy : 1.0;
  } else {
    gamma = 0.1 / std::max(s.maxg, 1.0e-6);  // cautious first step
  }
  for (double& v : q) v *= gamma;
  for (int i = 0; i < mh; ++i) {
    const double beta = s.rho[i] * opt_dot(s.Y[i], q);
    opt_axpy(q, alpha[i] - beta, s.S[i]);
  }
  s.d.resize(q.size());
  for (size_t i = 0; i < q.size(); ++i) s.d[i] = -q[i];
  if (opt_dot(s.d, s.g) > 0.0)  // uphill guard
    for (size_t i = 0; i < q.size(); ++i) s.d[i] = -s.g[i];
  s.gd = opt_dot(s.g, s.d);
  s.step = 1.0;
  s.xn = s.x;
  opt_axpy(s.xn, s.step, s.d);
}

int optimize_batch(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, double* xyz,
                   const pm3gpu_options* opts, const pm3gpu_opt_options& o, pm3gpu_opt_result* out, double* gradients) {
  std::vector<OptMol> mols(n_mol);
  for (int m = 0; m < n_mol; ++m) {
    OptMol& s = mols[m];
    s.m = m;
    s.a0 = offs[m];
    s.na = offs[m + 1] - offs[m];
    s.x.assign(xyz + 3 * (size_t)s.a0, xyz + 3 * (size_t)(s.a0 + s.na));
    s.xn = s.x;
  }
  std::vector<int32_t> boff, bz;
  std::vector<double> bxyz, bq, bg;
  std::vector<pm3gpu_result> br;
  std::vector<int> pend;
  Want w;
  w.grad = true;
  for (;;) {
    pend.clear();
    for (int m = 0; m < n_mol; ++m)
      if (!mols[m].done && mols[m].na > 0) pend.push_back(m);
      else if (mols[m].na == 0) mols[m].done = true;
    if (pend.empty()) break;
    // one batched launch over every pending geometry
    boff.assign(1, 0);
    bz.clear();
    bxyz.clear();
    for (int m : pend) {
      const OptMol& s = mols[m];
      bz.insert(bz.end(), z + s.a0, z + s.a0 + s.na);
      bxyz.insert(bxyz.end(), s.xn.begin(), s.xn.end());
      boff.push_back(boff.back() + s.na);
    }
    const int np = (int)pend.size();
    br.assign(np, pm3gpu_result{});
    bq.assign(bz.size(), 0.0);
    bg.assign(3 * bz.size(), 0.0);
    const int rc = run_batch(c, np, boff.data(), bz.data(), bxyz.data(), nullptr, nullptr, opts, 0, w, br.data(),
                             bq.data(), bg.data(), nullptr, nullptr);
    if (rc == PM3GPU_CUDA_ERROR || rc == PM3GPU_INVALID_INPUT) return rc;  // not a molecule's failure
    if (rc != PM3GPU_OK && np == 1 && br[0].status == PM3GPU_OK) br[0].status = rc;  // one molecule: its own code
    for (int k = 0; k < np; ++k) {
      OptMol& s = mols[pend[k]];
      ++s.evals;
      const pm3gpu_result& r = br[k];
      const bool ok = r.status == PM3GPU_OK;
      std::vector<double> gn(bg.begin() + 3 * (size_t)boff[k], bg.begin() + 3 * (size_t)boff[k + 1]);
      if (s.first) {  // the start geometry must evaluate (`evaluate(&mol)?`)
        s.first = false;
        if (!ok) {
          s.status = r.status;
          s.done = true;
          continue;
        }
        s.g = gn;
        s.e = r.total_ev;
        s.hof = r.heat_of_formation_kcal;
        s.maxg = opt_maxabs(gn);
        s.conv = s.maxg < o.gtol;
        opt_start_iteration(s, o);
        continue;
      }
      if (ok && r.total_ev <= s.e + 1.0e-4 * s.step * s.gd) {  // Armijo: accept, update the memory
        std::vector<double> sv(s.x.size()), yv(s.x.size());
        for (size_t i = 0; i < sv.size(); ++i) {
          sv[i] = s.xn[i] - s.x[i];
          yv[i] = gn[i] - s.g[i];
        }
        const double sy = opt_dot(sv, yv);
        if (sy > 1.0e-10) {
          s.S.push_back(std::move(sv));
          s.Y.push_back(std::move(yv));
          s.rho.push_back(1.0 / sy);
          if ((int)s.S.size() > o.history) {
            s.S.pop_front();
            s.Y.pop_front();
            s.rho.pop_front();
          }
        }
        s.x = s.xn;
        s.g = std::move(gn);
        s.e = r.total_ev;
        s.hof = r.heat_of_formation_kcal;
        s.maxg = opt_maxabs(s.g);
        s.conv = s.maxg < o.gtol;
        opt_start_iteration(s, o);
      } else {  // backtrack
        s.step *= 0.5;
        if (s.step < 1.0e-8) {
          s.done = true;  // no progress: stop at the current point
        } else {
          s.xn = s.x;
          opt_axpy(s.xn, s.step, s.d);
        }
      }
    }
  }
  for (int m = 0; m < n_mol; ++m) {
    const OptMol& s = mols[m];
    pm3gpu_opt_result& r = out[m];
    r.status = s.status;
    r.converged = s.status == PM3GPU_OK && s.conv ? 1 : 0;
    r.iterations = s.iterations;
    r.evaluations = s.evals;
    r.energy_ev = s.e;
    r.heat_of_formation_kcal = s.hof;
    r.max_gradient = s.maxg;
    if (s.status == PM3GPU_OK) std::copy(s.x.begin(), s.x.end(), xyz + 3 * (size_t)s.a0);
    if (gradients && s.status == PM3GPU_OK) std::copy(s.g.begin(), s.g.end(), gradients + 3 * (size_t)s.a0);
  }
  return PM3GPU_OK;
}
