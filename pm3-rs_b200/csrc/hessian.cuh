// Batched Cartesian Hessians by central differences of the analytic gradient (host side): the
// reference's numerical_hessian (pm3-rs src/hessian.rs:268-319) for many molecules at once.
// Included by pm3gpu.cu inside its private namespace, after run_batch.
//
// Column j of molecule m's Hessian is (g(x + h e_j) - g(x - h e_j)) / (2h); the rows and columns are
// Cartesian degrees of freedom 3 * atom + axis, and the result is averaged with its transpose
// (hessian.rs:86-95). Every displaced geometry of every molecule is one entry of a batched SCF +
// gradient launch, so the 6N gradient evaluations of a molecule and those of all the other molecules
// run side by side on the device. The SCF is tightened first, as the reference does for second
// derivatives (hessian.rs:169-175: e_tol <= 1e-12, p_tol <= 1e-11, max_scf >= 500). A molecule whose
// displaced SCF fails takes the status of the first failing column in column order, the plus
// displacement before the minus one, which is the error the reference's `col?` loop returns.
#pragma once

inline pm3gpu_options tighten_for_hessian(const pm3gpu_options& o) {
  pm3gpu_options t = o;
  t.e_tol = std::min(t.e_tol, 1.0e-12);
  t.p_tol = std::min(t.p_tol, 1.0e-11);
  t.max_scf = std::max(t.max_scf, 500);
  return t;
}

// Displaced atoms per batched launch: bounds the host staging of one chunk of columns.
constexpr long long kHessianChunkAtoms = 1LL << 20;

int hessian_batch(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, const double* xyz,
                  const pm3gpu_options* opts, double step, double* hess, int* status) {
  const pm3gpu_options t = tighten_for_hessian(*opts);
  std::vector<size_t> hoff(n_mol + 1, 0);
  for (int m = 0; m < n_mol; ++m) {
    const size_t nd = 3 * (size_t)(offs[m + 1] - offs[m]);
    hoff[m + 1] = hoff[m] + nd * nd;
    status[m] = PM3GPU_OK;
  }
  std::fill(hess, hess + hoff[n_mol], 0.0);

  struct Column {
    int m, j;
  };
  std::vector<Column> cols;
  std::vector<int32_t> boff, bz;
  std::vector<double> bxyz, bq, bg;
  std::vector<pm3gpu_result> br;
  Want w;
  w.grad = true;
  const double inv2h = 1.0 / (2.0 * step);

  auto flush = [&]() -> int {
    const int np = (int)boff.size() - 1;
    if (np <= 0) return PM3GPU_OK;
    br.assign(np, pm3gpu_result{});
    bq.assign(bz.size(), 0.0);
    bg.assign(3 * bz.size(), 0.0);
    const int rc = run_batch(c, np, boff.data(), bz.data(), bxyz.data(), nullptr, nullptr, &t, 0, w, br.data(),
                             bq.data(), bg.data(), nullptr, nullptr);
    if (rc == PM3GPU_CUDA_ERROR || rc == PM3GPU_INVALID_INPUT) return rc;  // not a molecule's failure
    for (size_t k = 0; k < cols.size(); ++k) {
      const Column& col = cols[k];
      if (status[col.m] != PM3GPU_OK) continue;  // an earlier column already failed
      const pm3gpu_result& rp = br[2 * k];
      const pm3gpu_result& rm = br[2 * k + 1];
      if (rp.status != PM3GPU_OK) {
        status[col.m] = rp.status;
        continue;
      }
      if (rm.status != PM3GPU_OK) {
        status[col.m] = rm.status;
        continue;
      }
      const int nd = 3 * (offs[col.m + 1] - offs[col.m]);
      const double* gp = bg.data() + 3 * (size_t)boff[2 * k];
      const double* gm = bg.data() + 3 * (size_t)boff[2 * k + 1];
      double* h = hess + hoff[col.m];
      for (int i = 0; i < nd; ++i) h[(size_t)i * nd + col.j] = (gp[i] - gm[i]) * inv2h;
    }
    cols.clear();
    boff.assign(1, 0);
    bz.clear();
    bxyz.clear();
    return PM3GPU_OK;
  };

  boff.assign(1, 0);
  for (int m = 0; m < n_mol; ++m) {
    const int a0 = offs[m], na = offs[m + 1] - offs[m];
    const double* x0 = xyz + 3 * (size_t)a0;
    for (int j = 0; j < 3 * na; ++j) {
      if ((long long)bz.size() + 2LL * na > kHessianChunkAtoms) {
        const int rc = flush();
        if (rc != PM3GPU_OK) return rc;
      }
      cols.push_back({m, j});
      for (int sign = 1; sign >= -1; sign -= 2) {  // plus, then minus
        bz.insert(bz.end(), z + a0, z + a0 + na);
        const size_t at = bxyz.size();
        bxyz.insert(bxyz.end(), x0, x0 + 3 * (size_t)na);
        bxyz[at + j] += sign * step;
        boff.push_back(boff.back() + na);
      }
    }
  }
  const int rc = flush();
  if (rc != PM3GPU_OK) return rc;

  for (int m = 0; m < n_mol; ++m) {  // average with the transpose (hessian.rs:86-95)
    const int nd = 3 * (offs[m + 1] - offs[m]);
    double* h = hess + hoff[m];
    if (status[m] != PM3GPU_OK) {
      std::fill(h, h + (size_t)nd * nd, 0.0);
      continue;
    }
    for (int i = 0; i < nd; ++i)
      for (int j = 0; j < i; ++j) {
        const double v = 0.5 * (h[(size_t)i * nd + j] + h[(size_t)j * nd + i]);
        h[(size_t)i * nd + j] = v;
        h[(size_t)j * nd + i] = v;
      }
  }
  return PM3GPU_OK;
}
