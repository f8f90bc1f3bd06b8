// Host driver of the whole-GPU path for one large molecule: the run_job SCF loop (scf.rs:1179-1496)
// with the work spread over the device (large_scf.cuh kernels, the DMMA DGEMM of dgemm.cuh for
// the dense products). Included by pm3gpu.cu inside its private namespace, after the context
// definition.
//
// Matrices are row-major n x n FP64. The GEMM follows the column-major BLAS contract, which sees a
// row-major matrix as its transpose; every call below is written in that view (comments give the
// row-major product).
//
// Eigensolver for large n: blocked Householder tridiagonalisation (one cooperative launch per
// panel + one rank-64 DGEMM trailing update; five launches per column replayed from a CUDA graph
// where a cooperative launch cannot hold the matrix), division-free Sturm multisection for the
// lowest n_occ + 1
// eigenvalues (warm-started from the previous iteration), twisted-factorisation eigenvectors of
// the tridiagonal (one thread per vector), compact-WY back-transformation (DGEMM), then
// Newton-Schulz steps X <- X (3I - X^T X)/2 until the occupied vectors are orthonormal to
// 1e-13. Inside a cluster of close eigenvalues the twisted vectors are accurate only up to a
// rotation within the cluster, and the polar step fixes their orthogonality without leaving the
// cluster's invariant subspace, which is all the density P = w C_occ C_occ^T depends on.

// Mixed mode hands over to FP64 once the RMS density change is below max(100 p_tol, this floor),
// or when it stops falling. The split-BF16 density noise is ~2e-8 RMS at n = 12000 (water
// clusters); the switch keeps it a few tenths of a percent of the residuals that the DIIS history
// holds when the FP64 iterations take over. Switching near the noise (3.5e-7) was measured to
// derail the FP64 DIIS steps that follow (21 iterations instead of 14).
constexpr double kMixedFloor = 1.0e-5;

struct TriGraph {
  static constexpr int kKeys = 17;
  cudaGraphExec_t exec = nullptr;
  int n = 0, launches = 0;
  const void* key[kKeys] = {};
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    n = 0;
  }
};

struct LargeBufs {
  TriGraph tg;
  DevBuf gwork;  // split-K workspace of the DGEMMs
  DevBuf Vw;     // back-transformation block V (n x kWy)
  DevBuf ao, sprow, sroff;
  DevBuf H, W, hacc, dpk, jacc, part, part2, scal;
  DevBuf P[2], Q[2], Pt, F, G, hist, A;
  DevBuf d, e, e2, tau, lam, dlam, blk;
  DevBuf V, Wp, y, wtmp, ps, s64, vcol, tp, ctr, refl;
  DevBuf X, Xt, Dp, Lp, Um;
  DevBuf Gm, Mm, Tm, Z1, Z2, blocks, Gk;
  DevBuf mh[2], ml[2], c32;  // mixed mode: BF16 hi / lo parts of two operands, FP32 product
  DevBuf gsync, vw, wv;      // cooperative panels: grid barrier, X = [V | W] and Y = [W | V]
  DevBuf Fchk;               // eigen-residual check: the diagonalised matrix rebuilt
  DevBuf tcerr;              // error flag of the tcgen05 split-BF16 GEMM
  bool tcerr_zeroed = false;
  void release() {
    for (DevBuf* b : {&ao, &sprow, &sroff, &H, &W, &hacc, &dpk, &jacc, &part, &part2, &scal, &P[0], &P[1], &Q[0], &Q[1], &Pt,
                      &F, &G, &hist, &A, &d, &e, &e2, &tau, &lam, &dlam, &blk, &V, &Wp, &y, &wtmp, &ps, &s64, &vcol, &tp, &ctr, &refl, &X, &Xt,
                      &Dp, &Lp, &Um, &Gm, &Mm, &Tm, &Z1, &Z2, &blocks, &Gk, &mh[0], &mh[1], &ml[0], &ml[1], &c32, &gsync, &vw, &wv, &Fchk, &tcerr})
      b->release();
    tcerr_zeroed = false;
    gwork.release();
    Vw.release();
    tg.reset();
  }
};

// Result of one large SCF (one pass of run_pm3's driver).
struct LargeRun {
  JobOut o;
  bool uhf = false;
  std::vector<double> eps_a, eps_b;      // eigenvalues of the last iteration (n_occ + 1 each)
  std::vector<double> tri_a, tri_b;      // saved tridiagonals (d | e) of the last iteration
  std::vector<double> charges;
};

// Phases of the whole-GPU path (wall-clock ms when profiling).
enum LargePhase : int {
  kLgCore = 0, kLgFock, kLgDiis, kLgTridiag, kLgEigval, kLgEigvec, kLgBack, kLgOrth, kLgDensity, kLgPhases
};

#define GEMM_TRY(call)                 \
  do {                                 \
    const int rc_ = (call);            \
    if (rc_ != PM3GPU_OK) return rc_;  \
  } while (0)

inline int grid_for(size_t work, int per_block = large::kBlock, int cap = large::kRedBlocks) {
  const size_t g = (work + per_block - 1) / per_block;
  return (int)std::max<size_t>(1, std::min<size_t>(g, (size_t)cap));
}

// A-DIIS weights (scf.rs:1152-1172, 1637-1693), serial form (the device path runs the same
// iteration on one warp).
void adiis_host(int m, const double* mg, double* c) {
  const int last = m - 1;
  const double mnn = mg[last * kMaxDepth + last];
  double d[kMaxDepth], S[kMaxDepth * kMaxDepth];
  for (int i = 0; i < m; ++i) d[i] = mg[i * kMaxDepth + last] - mnn;
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j)
      S[i * kMaxDepth + j] = mg[i * kMaxDepth + j] - mg[i * kMaxDepth + last] - mg[last * kMaxDepth + j] + mnn;
  double L = 1.0e-12;
  for (int i = 0; i < m; ++i) {
    double row = 0.0;
    for (int j = 0; j < m; ++j) row += std::fabs(S[i * kMaxDepth + j] + S[j * kMaxDepth + i]);
    L = std::max(L, row);
  }
  const double lr = 1.0 / L;
  for (int i = 0; i < m; ++i) c[i] = i == last ? 1.0 : 0.0;
  for (int it = 0; it < 400; ++it) {
    double tr[kMaxDepth], u[kMaxDepth];
    for (int k = 0; k < m; ++k) {
      double g = 2.0 * d[k];
      for (int j = 0; j < m; ++j) g += (S[k * kMaxDepth + j] + S[j * kMaxDepth + k]) * c[j];
      tr[k] = c[k] - lr * g;
      u[k] = tr[k];
    }
    for (int i = 1; i < m; ++i) {  // descending, stable
      const double key = u[i];
      int j = i - 1;
      while (j >= 0 && u[j] < key) {
        u[j + 1] = u[j];
        --j;
      }
      u[j + 1] = key;
    }
    double css = 0.0, theta = 0.0;
    for (int j = 0; j < m; ++j) {
      css += u[j];
      const double t = (css - 1.0) / (double)(j + 1);
      if (u[j] - t > 0.0) theta = t;
    }
    double delta = 0.0;
    for (int i = 0; i < m; ++i) {
      const double p = std::max(tr[i] - theta, 0.0);
      delta += std::fabs(p - c[i]);
      c[i] = p;
    }
    if (delta < 1.0e-12) break;
  }
}

class LargeSolver {
 public:
  LargeSolver(pm3gpu_ctx* c, LargeBufs& B) : c_(c), B_(B) {}

  // Molecule setup: per-atom tables, H_core and the pair table. d_z / d_xyz: device copies.
  int setup(const int32_t* h_z, const int32_t* d_z, const double* d_xyz, int natom, int nao, double* ecc) {
    N_ = natom;
    n_ = nao;
    nn_ = (size_t)n_ * n_;
    std::vector<int> ao(N_), sprow(N_ + 1);
    std::vector<long long> sroff(N_);
    int off = 0, pr = 0;
    for (int a = 0; a < N_; ++a) {
      ao[a] = off;
      off += c_->h_elem[h_z[a]].norb;
      sprow[a] = pr;
      pr += c_->h_elem[h_z[a]].norb == 4 ? 10 : 1;
    }
    sprow[N_] = pr;
    long long ro = 0;
    for (int a = 0; a < N_; ++a) {
      sroff[a] = ro;
      ro += (long long)(sprow[a + 1] - sprow[a]) * (pr - sprow[a + 1]);
    }
    wcap_ = std::max<long long>(ro, 1);
    CUDA_TRY(c_, B_.ao.ensure(4 * (size_t)N_));
    CUDA_TRY(c_, B_.sprow.ensure(4 * (size_t)(N_ + 1)));
    CUDA_TRY(c_, B_.sroff.ensure(8 * (size_t)N_));
    CUDA_TRY(c_, cudaMemcpyAsync(B_.ao.p, ao.data(), 4 * (size_t)N_, cudaMemcpyHostToDevice, c_->stream));
    CUDA_TRY(c_, cudaMemcpyAsync(B_.sprow.p, sprow.data(), 4 * (size_t)(N_ + 1), cudaMemcpyHostToDevice, c_->stream));
    CUDA_TRY(c_, cudaMemcpyAsync(B_.sroff.p, sroff.data(), 8 * (size_t)N_, cudaMemcpyHostToDevice, c_->stream));
    m_.elem = c_->elem.as<ElemDev>();
    m_.pairs = c_->pairs.as<PairDev>();
    m_.z = d_z;
    m_.xyz = d_xyz;
    m_.ao = B_.ao.as<int>();
    m_.sprow = B_.sprow.as<int>();
    m_.sroff = B_.sroff.as<long long>();
    m_.N = N_;
    m_.n = n_;
    hz_ = h_z;
    CUDA_TRY(c_, B_.H.ensure(8 * nn_));
    CUDA_TRY(c_, B_.W.ensure(8 * (size_t)wcap_));
    CUDA_TRY(c_, B_.hacc.ensure(80 * (size_t)N_));
    CUDA_TRY(c_, B_.dpk.ensure(80 * (size_t)N_));
    CUDA_TRY(c_, B_.jacc.ensure(80 * (size_t)N_));
    CUDA_TRY(c_, B_.part.ensure(8 * (size_t)large::kRedBlocks));
    CUDA_TRY(c_, B_.part2.ensure(8 * (size_t)large::kRedBlocks));
    CUDA_TRY(c_, B_.scal.ensure(8 * 128));
    const long long np = (long long)N_ * (N_ - 1) / 2;
    const int gp = grid_for((size_t)std::max<long long>(np, 1));
    large::core_pairs_kernel<<<gp, large::kBlock, 0, c_->stream>>>(m_, B_.H.as<double>(), B_.W.as<double>(),
                                                                  B_.part.as<double>());
    ++c_->launches;
    large::core_atoms_kernel<<<(N_ + large::kBlock / 32 - 1) / (large::kBlock / 32), large::kBlock, 0, c_->stream>>>(
        m_, B_.hacc.as<double>());
    ++c_->launches;
    large::finish_sum<<<1, large::kBlock, 0, c_->stream>>>(B_.part.as<double>(), gp, B_.scal.as<double>());
    large::core_diag_kernel<<<grid_for((size_t)N_ * 16), large::kBlock, 0, c_->stream>>>(m_, B_.hacc.as<double>(),
                                                                                        B_.H.as<double>());
    c_->launches += 2;
    CUDA_TRY(c_, cudaGetLastError());
    CUDA_TRY(c_, cudaMemcpyAsync(ecc, B_.scal.p, 8, cudaMemcpyDeviceToHost, c_->stream));
    CUDA_TRY(c_, cudaStreamSynchronize(c_->stream));
    tick(kLgCore);
    return PM3GPU_OK;
  }

  // One SCF with job J (the first pass or a stability rung).
  int scf(const JobDesc& J, LargeRun& R) {
    const bool uhf = (J.flags & kJobUhf) != 0;
    const int na = J.n_alpha, nb = J.n_beta;
    const int n = n_;
    R.uhf = uhf;
    for (DevBuf* b : {&B_.P[0], &B_.P[1], &B_.F, &B_.A}) CUDA_TRY(c_, b->ensure(8 * nn_));
    if (uhf)
      for (DevBuf* b : {&B_.Q[0], &B_.Q[1], &B_.G, &B_.Pt}) CUDA_TRY(c_, b->ensure(8 * nn_));
    const int depth = J.depth < 2 ? 2 : (J.depth > kMaxDepth ? kMaxDepth : J.depth);
    const bool keep = (J.flags & kJobKeepDens) != 0;
    const int slot_mats = uhf ? 4 : (keep ? 3 : 2);
    if (J.accel != 0) CUDA_TRY(c_, B_.hist.ensure(8 * nn_ * (size_t)slot_mats * depth));
    int cur = 0;
    std::vector<double> lam_a, lam_b, dl_a, dl_b;
    // ------------------------------------------------------------- initial density
    double* Pa0 = B_.P[0].as<double>();
    double* Pb0 = uhf ? B_.Q[0].as<double>() : nullptr;
    if (J.guess == 2) {  // core-Hamiltonian orbitals (scf.rs:929-932, 969-975)
      int rc = copy(B_.H.as<double>(), work_matrix());
      if (rc) return rc;
      rc = eigensolve(work_matrix(), std::min(n, na + 1), na, lam_a, dl_a, false, nullptr);
      if (rc) return rc;
      rc = density_from_x(na, na, uhf ? 1.0 : 2.0, Pa0);
      if (rc) return rc;
      if (uhf) {
        rc = density_from_x(nb, na, 1.0, Pb0);
        if (rc) return rc;
      }
      lam_a.clear();
      dl_a.clear();
    } else {
      double fa = 1.0, fb = 0.0;
      if (uhf) {
        const double ne = (double)(na + nb);
        fa = ne > 0.0 ? na / ne : 0.5;
        fb = ne > 0.0 ? nb / ne : 0.5;
      }
      int tilt = -1;
      if (J.guess == 3) {
        double best = 0.0;
        for (int a = 0; a < N_; ++a) {
          const ElemDev& el = c_->h_elem[hz_[a]];
          if (el.norb == 4 && el.occ_p > best) {
            best = el.occ_p;
            tilt = a;
          }
        }
      }
      CUDA_TRY(c_, cudaMemsetAsync(Pa0, 0, 8 * nn_, c_->stream));
      large::sad_kernel<<<grid_for(N_), large::kBlock, 0, c_->stream>>>(m_, Pa0, fa, tilt);
      ++c_->launches;
      if (uhf) {
        CUDA_TRY(c_, cudaMemsetAsync(Pb0, 0, 8 * nn_, c_->stream));
        large::sad_kernel<<<grid_for(N_), large::kBlock, 0, c_->stream>>>(m_, Pb0, fb, tilt);
        ++c_->launches;
      }
    }
    // ------------------------------------------------------------- SCF iteration
    double bg[kMaxDepth * kMaxDepth] = {}, mg[kMaxDepth * kMaxDepth] = {}, coef[kMaxDepth + 1] = {};
    int len = 0, head = 0, iterations = 0;
    double e_old = 0.0, last_change = INFINITY;
    bool converged = false;
    const int kva = std::min(n, na + 1), kvb = std::min(n, nb + 1);
    // Mixed mode: the commutator and the density come from split-BF16 products until the density
    // settles (kMixedSwitch) or stops improving, then FP64 iterations close the SCF; only an FP64
    // iteration can satisfy the convergence test, so the result is the FP64 fixed point.
    bool lowp = c_->precision == PM3GPU_PRECISION_MIXED, prev_lowp = false;
    ++passes_;
    for (int iter = 0; iter < J.max_scf; ++iter) {
      iterations = iter + 1;
      const bool lowp_iter = lowp;
      double trace_err = 0.0;
      double* Pc = B_.P[cur].as<double>();
      double* Pn = B_.P[1 - cur].as<double>();
      double* Qc = uhf ? B_.Q[cur].as<double>() : nullptr;
      double* Qn = uhf ? B_.Q[1 - cur].as<double>() : nullptr;
      double* Fa = B_.F.as<double>();
      double* Fb = uhf ? B_.G.as<double>() : nullptr;
      double *Ea = nullptr, *Eb = nullptr, *Dh = nullptr;
      // First FP64 iteration after split-BF16 ones: the newest history entry's commutator is a
      // split-BF16 product. Its density (the previous iteration's input) is still in the other
      // buffer, so it is redone in FP64 and its Gram row refreshed before the history is used.
      if (prev_lowp && !lowp_iter && J.accel != 0 && len > 0 && (!uhf || J.damping == 0.0)) {
        const int l = len - 1;
        double* bl = slot(head, l, depth, slot_mats);
        int rc = commutator(bl, B_.P[1 - cur].as<double>(), bl + nn_);
        if (rc) return rc;
        if (uhf && (rc = commutator(bl + 2 * nn_, B_.Q[1 - cur].as<double>(), bl + 3 * nn_))) return rc;
        for (int k2 = 0; k2 < len; ++k2) {
          double* bk = slot(head, k2, depth, slot_mats);
          double v;
          if ((rc = dot(bk + nn_, bl + nn_, uhf ? bk + 3 * nn_ : nullptr, uhf ? bl + 3 * nn_ : nullptr, &v))) return rc;
          bg[k2 * kMaxDepth + l] = v;
          bg[l * kMaxDepth + k2] = v;
        }
      }
      prev_lowp = lowp_iter;
      if (J.accel != 0) {
        if (len == depth) {
          for (int i = 0; i + 1 < len; ++i)
            for (int j = 0; j + 1 < len; ++j) {
              bg[i * kMaxDepth + j] = bg[(i + 1) * kMaxDepth + j + 1];
              mg[i * kMaxDepth + j] = mg[(i + 1) * kMaxDepth + j + 1];
            }
          head = (head + 1) % depth;
          --len;
        }
        double* base = slot(head, len, depth, slot_mats);
        Fa = base;
        Ea = base + nn_;
        if (uhf) {
          Fb = base + 2 * nn_;
          Eb = base + 3 * nn_;
        } else if (keep) {
          Dh = base + 2 * nn_;
        }
      }
      double e_elec = 0.0;
      if (!uhf) {
        int rc = fock(Pc, nullptr, nullptr, Fa, nullptr);
        if (rc) return rc;
        double h1, h2;
        if ((rc = dot(Pc, B_.H.as<double>(), nullptr, nullptr, &h1)) || (rc = dot(Pc, Fa, nullptr, nullptr, &h2)))
          return rc;
        e_elec = 0.5 * (h1 + h2);
      } else {
        double* Pt = B_.Pt.as<double>();
        large::add_kernel<<<grid_for(nn_), large::kBlock, 0, c_->stream>>>(Pc, Qc, Pt, nn_);
        ++c_->launches;
        int rc = fock(Pt, Pc, Qc, Fa, Fb);
        if (rc) return rc;
        double h1, h2;
        if ((rc = dot(Pt, B_.H.as<double>(), nullptr, nullptr, &h1)) || (rc = dot(Pc, Fa, Qc, Fb, &h2))) return rc;
        e_elec = 0.5 * (h1 + h2);
      }
      tick(kLgFock);
      // ---- accelerator (scf.rs:1240-1259 RHF; 1398-1413 UHF)
      bool use_hist = false;
      if (J.accel != 0) {
        int rc = commutator(Fa, Pc, Ea, lowp_iter);
        if (rc) return rc;
        if (uhf && (rc = commutator(Fb, Qc, Eb, lowp_iter))) return rc;
        if (keep && (rc = copy(Pc, Dh))) return rc;
        double ee;
        if ((rc = dot(Ea, Ea, Eb, Eb, &ee))) return rc;
        double dnf = 0.0;
        if (keep && (rc = dot(Dh, Fa, nullptr, nullptr, &dnf))) return rc;
        for (int l = 0; l < len; ++l) {
          double* bl = slot(head, l, depth, slot_mats);
          double v;
          if ((rc = dot(bl + nn_, Ea, uhf ? bl + 3 * nn_ : nullptr, Eb, &v))) return rc;
          bg[l * kMaxDepth + len] = v;
          bg[len * kMaxDepth + l] = v;
          if (keep) {
            double a1, a2;
            if ((rc = dot(Dh, bl, nullptr, nullptr, &a1)) || (rc = dot(bl + 2 * nn_, Fa, nullptr, nullptr, &a2)))
              return rc;
            mg[len * kMaxDepth + l] = a1;  // <D_new, F_l>
            mg[l * kMaxDepth + len] = a2;  // <D_l, F_new>
          }
        }
        bg[len * kMaxDepth + len] = ee;
        mg[len * kMaxDepth + len] = dnf;
        const int m = len + 1;
        const double err = std::sqrt(ee);
        trace_err = err;
        bool ok;
        if (!uhf && J.accel == 2 && err > J.adiis_switch) {
          ok = keep && m >= 2;
          if (ok) adiis_host(m, mg, coef);
        } else {
          ok = cdiis_coeffs(m, bg, coef);
        }
        ++len;
        use_hist = ok;
        tick(kLgDiis);
      }
      // ---- diagonalise (level shift for UHF only, scf.rs:1416-1418) and rebuild densities
      double sq_a = 0.0, sq_b = 0.0;
      for (int spin = 0; spin < (uhf ? 2 : 1); ++spin) {
        large::Comb cb{};
        if (use_hist) {
          cb.len = len;
          for (int l = 0; l < len; ++l) {
            cb.m[l] = slot(head, l, depth, slot_mats) + (spin == 0 ? 0 : 2 * nn_);
            cb.c[l] = coef[l];
          }
        } else {
          cb.len = 1;
          cb.m[0] = spin == 0 ? Fa : Fb;
          cb.c[0] = 1.0;
        }
        const double shift = uhf ? J.shift : 0.0;
        large::combine_kernel<<<grid_for(nn_), large::kBlock, 0, c_->stream>>>(cb, spin == 0 ? Pc : Qc, shift, n,
                                                                              work_matrix());
        ++c_->launches;
        const int kv = spin == 0 ? kva : kvb, occ = spin == 0 ? na : nb;
        std::vector<double>& lam = spin == 0 ? lam_a : lam_b;
        std::vector<double>& dl = spin == 0 ? dl_a : dl_b;
        std::vector<double>& tri = spin == 0 ? R.tri_a : R.tri_b;
        int rc = eigensolve(work_matrix(), kv, occ, lam, dl, iter > 0, &tri);
        if (rc) return rc;
        double resid = NAN;
        if (c_->large_checks && occ > 0) {  // max |F X - X diag(lam)| of the occupied pairs
          CUDA_TRY(c_, B_.Fchk.ensure(8 * nn_));
          large::combine_kernel<<<grid_for(nn_), large::kBlock, 0, c_->stream>>>(cb, spin == 0 ? Pc : Qc, shift, n,
                                                                                B_.Fchk.as<double>());
          ++c_->launches;
          if ((rc = eigen_residual(B_.Fchk.as<double>(), occ, &resid))) return rc;
        }
        c_->lchecks.insert(c_->lchecks.end(), {(double)passes_, (double)iter, (double)spin, last_defect_, resid,
                                               (double)last_ns_steps_});
        double* Pold = spin == 0 ? Pc : Qc;
        double* Pnew = spin == 0 ? Pn : Qn;
        rc = density_from_x(occ, occ, uhf ? 1.0 : 2.0, Pnew, lowp_iter);
        if (rc) return rc;
        tick(kLgDensity);
        double sq;
        if ((rc = sqdiff(Pnew, Pold, &sq))) return rc;
        (spin == 0 ? sq_a : sq_b) = sq;
        const double damp = uhf ? J.damping : 0.0;
        if (damp > 0.0) {  // stored density (1 - lam) Pnew + lam Pold; the RMS used the undamped Pnew
          large::damp_kernel<<<grid_for(nn_), large::kBlock, 0, c_->stream>>>(Pnew, Pold, damp, nn_);
          ++c_->launches;
          if ((rc = copy(Pold, Pnew))) return rc;
        }
      }
      const double dp = uhf ? std::sqrt(sq_a / (double)nn_) + std::sqrt(sq_b / (double)nn_)
                            : std::sqrt(sq_a / (double)nn_);
      const double de = std::fabs(e_elec - e_old);
      c_->ltrace.insert(c_->ltrace.end(), {(double)passes_, iter > 0 ? de : INFINITY, dp, trace_err, lowp_iter ? 1.0 : 0.0});
      if (lowp && (dp < std::max(100.0 * J.p_tol, kMixedFloor) || (iter >= 2 && dp < 1.0e-3 && dp > 0.7 * last_change) ||
                   2 * iter >= J.max_scf))
        lowp = false;
      last_change = dp;
      e_old = e_elec;
      cur = 1 - cur;
      if (!lowp_iter && iter > 0 && de < J.e_tol && dp < J.p_tol) {
        converged = true;
        break;
      }
    }
    // ------------------------------------------------------------- closing energy
    double* Pf = B_.P[cur].as<double>();
    double* Qf = uhf ? B_.Q[cur].as<double>() : nullptr;
    double* Pt = Pf;
    JobOut& o = R.o;
    std::memset(&o, 0, sizeof(o));
    if (!uhf) {
      int rc = fock(Pf, nullptr, nullptr, B_.F.as<double>(), nullptr);
      if (rc) return rc;
      double h1, h2;
      if ((rc = dot(Pf, B_.H.as<double>(), nullptr, nullptr, &h1)) ||
          (rc = dot(Pf, B_.F.as<double>(), nullptr, nullptr, &h2)))
        return rc;
      o.electronic = 0.5 * (h1 + h2);
      o.spin_max = 0.0;
    } else {
      Pt = B_.Pt.as<double>();
      large::add_kernel<<<grid_for(nn_), large::kBlock, 0, c_->stream>>>(Pf, Qf, Pt, nn_);
      large::absdiff_max_kernel<<<large::kRedBlocks, large::kBlock, 0, c_->stream>>>(Pf, Qf, nn_, B_.part.as<double>());
      c_->launches += 2;
      std::vector<double> mx(large::kRedBlocks);
      CUDA_TRY(c_, cudaMemcpyAsync(mx.data(), B_.part.p, 8 * mx.size(), cudaMemcpyDeviceToHost, c_->stream));
      CUDA_TRY(c_, cudaStreamSynchronize(c_->stream));
      o.spin_max = 0.0;
      for (double v : mx) o.spin_max = std::max(o.spin_max, v);
      int rc = fock(Pt, Pf, Qf, B_.F.as<double>(), B_.G.as<double>());
      if (rc) return rc;
      double h1, h2;
      if ((rc = dot(Pt, B_.H.as<double>(), nullptr, nullptr, &h1)) ||
          (rc = dot(Pf, B_.F.as<double>(), Qf, B_.G.as<double>(), &h2)))
        return rc;
      o.electronic = 0.5 * (h1 + h2);
    }
    final_pt_ = Pt;
    final_pa_ = uhf ? Pf : nullptr;
    final_pb_ = Qf;
    o.converged = converged ? 1 : 0;
    o.iterations = iterations;
    o.last_change = last_change;
    o.status = converged ? 0 : 4;
    // frontier of the last iteration's orbitals (scf.rs:106-124, 804-822)
    o.has_homo_a = na >= 1;
    o.has_lumo_a = na < n;
    o.homo_a = na >= 1 ? lam_a[na - 1] : 0.0;
    o.lumo_a = na < n ? lam_a[na] : 0.0;
    o.homo = o.homo_a;
    o.lumo = o.lumo_a;
    o.has_homo = o.has_homo_a;
    o.has_lumo = o.has_lumo_a;
    if (uhf) {
      if (nb >= 1) {
        o.homo = o.has_homo ? std::max(o.homo, lam_b[nb - 1]) : lam_b[nb - 1];
        o.has_homo = 1;
      }
      if (nb < n) {
        o.lumo = o.has_lumo ? std::min(o.lumo, lam_b[nb]) : lam_b[nb];
        o.has_lumo = 1;
      }
    }
    o.gap = (o.has_homo && o.has_lumo) ? o.lumo - o.homo : INFINITY;
    R.eps_a = lam_a;
    R.eps_b = lam_b;
    return properties(Pt, R);
  }

  // Final densities of the last scf() call (device pointers into this solver's buffers).
  const double* final_pt() const { return final_pt_; }
  const double* final_pa() const { return final_pa_; }
  const double* final_pb() const { return final_pb_; }

  // All n eigenvalues of a saved tridiagonal (d | e) -- the MO energies output.
  int all_eigenvalues(const std::vector<double>& tri, std::vector<double>& out) {
    CUDA_TRY(c_, B_.d.ensure(8 * (size_t)n_));
    CUDA_TRY(c_, B_.e.ensure(8 * (size_t)n_));
    CUDA_TRY(c_, cudaMemcpyAsync(B_.d.p, tri.data(), 8 * (size_t)n_, cudaMemcpyHostToDevice, c_->stream));
    CUDA_TRY(c_, cudaMemcpyAsync(B_.e.p, tri.data() + n_, 8 * (size_t)n_, cudaMemcpyHostToDevice, c_->stream));
    std::vector<double> none;
    return eigenvalues(n_, out, none, false);
  }

  // Autotuner: device time of one Householder reduction of H_core with the cooperative panels
  // (coop = 1) or the multi-launch path (coop = 0); the second of two runs is timed.
  int time_reduction(int coop, double* ms) {
    int rc = prepare_reduction();
    if (rc) return rc;
    for (DevBuf* b : {&B_.P[0], &B_.P[1], &B_.F, &B_.A}) CUDA_TRY(c_, b->ensure(8 * nn_));
    c_->force_coop = coop;
    for (int rep = 0; rep < 2 && rc == PM3GPU_OK; ++rep) {
      if ((rc = copy(B_.H.as<double>(), work_matrix()))) break;
      CUDA_TRY(c_, cudaEventRecord(c_->kev[0], c_->stream));
      rc = run_tridiag(work_matrix());
      CUDA_TRY(c_, cudaEventRecord(c_->kev[1], c_->stream));
      CUDA_TRY(c_, cudaEventSynchronize(c_->kev[1]));
      float t = 0.0f;
      CUDA_TRY(c_, cudaEventElapsedTime(&t, c_->kev[0], c_->kev[1]));
      *ms = t;
      if (rc == PM3GPU_OK && coop_grid() > 0) {
        large::GridSync gsh{};
        CUDA_TRY(c_, cudaMemcpy(&gsh, B_.gsync.p, sizeof(gsh), cudaMemcpyDeviceToHost));
        if (gsh.err) rc = fail(c_, PM3GPU_CUDA_ERROR, "Householder panel: a grid barrier wait ran out");
      }
    }
    c_->force_coop = -1;
    return rc;
  }

 private:
  pm3gpu_ctx* c_;
  LargeBufs& B_;
  large::Mol m_{};
  const int32_t* hz_ = nullptr;
  int N_ = 0, n_ = 0;
  int coop_g_ = -1;  // cooperative panel grid for this device (-1: not yet queried)
  int passes_ = 0;  // SCF passes of this molecule (first pass, stability rungs)
  size_t nn_ = 0;
  long long wcap_ = 1;
  const double* final_pt_ = nullptr;
  const double* final_pa_ = nullptr;
  const double* final_pb_ = nullptr;
  std::vector<int> hblk_;

  double* work_matrix() { return B_.A.as<double>(); }
  double* slot(int head, int l, int depth, int mats) {
    return B_.hist.as<double>() + (size_t)((head + l) % depth) * mats * nn_;
  }
  int copy(const double* src, double* dst) {
    CUDA_TRY(c_, cudaMemcpyAsync(dst, src, 8 * nn_, cudaMemcpyDeviceToDevice, c_->stream));
    return PM3GPU_OK;
  }
  // C = alpha op(A) op(B) + beta C (column-major) on the context's stream, by the hand-written
  // DMMA GEMM (dgemm.cuh); launches are added to *count (the context's counter by default). The
  // split-K workspace grows only for shapes that split, none of which runs under graph capture
  // (the captured multi-launch reduction's rank-2b updates have K = 2b).
  int gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double* A, int lda, const double* B, int ldb,
           double beta, double* C, int ldc, int* count = nullptr) {
    const dg::Plan p = dg::plan(m, n, k, c_->sms);
    if (p.work_doubles > 0) CUDA_TRY(c_, B_.gwork.ensure(8 * p.work_doubles));
    const int r = dg::gemm(c_->stream, c_->sms, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                           B_.gwork.as<double>());
    if (r < 0) return fail(c_, PM3GPU_CUDA_ERROR, std::string("DGEMM launch: ") + cudaGetErrorString(cudaGetLastError()));
    *(count ? count : &c_->launches) += r;
    return PM3GPU_OK;
  }

  int finish(double* out) {
    large::finish_sum<<<1, large::kBlock, 0, c_->stream>>>(B_.part.as<double>(), large::kRedBlocks, B_.scal.as<double>());
    ++c_->launches;
    CUDA_TRY(c_, cudaMemcpyAsync(out, B_.scal.p, 8, cudaMemcpyDeviceToHost, c_->stream));
    CUDA_TRY(c_, cudaStreamSynchronize(c_->stream));
    return PM3GPU_OK;
  }
  int dot(const double* x, const double* y, const double* x2, const double* y2, double* out) {
    large::dot_kernel<<<large::kRedBlocks, large::kBlock, 0, c_->stream>>>(x, y, x2, y2, nn_, B_.part.as<double>());
    ++c_->launches;
    return finish(out);
  }
  int sqdiff(const double* x, const double* y, double* out) {
    large::sqdiff_kernel<<<large::kRedBlocks, large::kBlock, 0, c_->stream>>>(x, y, nn_, B_.part.as<double>());
    ++c_->launches;
    return finish(out);
  }

  // F = H + J(Pt) - K (fock.rs:285-332); RHF exchange from Pt/2, UHF from Pa / Pb.
  int fock(const double* Pt, const double* Pa, const double* Pb, double* F, double* G) {
    const int gN = grid_for((size_t)N_ * 16);
    large::pack_density_kernel<<<gN, large::kBlock, 0, c_->stream>>>(m_, Pt, B_.dpk.as<double>(), B_.jacc.as<double>());
    const long long np = (long long)N_ * (N_ - 1) / 2;
    const int gp = grid_for((size_t)std::max<long long>(np, 1));
    const int ga = (N_ + large::kBlock / 32 - 1) / (large::kBlock / 32);  // one warp per atom
    large::coulomb_atoms_kernel<<<ga, large::kBlock, 0, c_->stream>>>(m_, B_.W.as<double>(), B_.dpk.as<double>(),
                                                                      B_.jacc.as<double>());
    ++c_->launches;
    if (Pb)
      large::fock_pairs_kernel<true><<<gp, large::kBlock, 0, c_->stream>>>(
          m_, B_.W.as<double>(), B_.H.as<double>(), B_.dpk.as<double>(), B_.jacc.as<double>(), Pt, Pa, Pb, F, G);
    else
      large::fock_pairs_kernel<false><<<gp, large::kBlock, 0, c_->stream>>>(
          m_, B_.W.as<double>(), B_.H.as<double>(), B_.dpk.as<double>(), B_.jacc.as<double>(), Pt, Pa, Pb, F, G);
    large::fock_diag_kernel<<<gN, large::kBlock, 0, c_->stream>>>(m_, B_.H.as<double>(), B_.jacc.as<double>(), Pt, Pa,
                                                                  Pb, F, G);
    c_->launches += 3;
    CUDA_TRY(c_, cudaGetLastError());
    return PM3GPU_OK;
  }
  // E = F P - P F (scf.rs:1039-1054): row-major F P is the column-major product P F.
  // Mixed mode (lowp) takes the product from split-BF16 tensor-core GEMMs with FP32 accumulation.
  int commutator(const double* F, const double* P, double* E, bool lowp = false) {
    if (lowp) {  // C = F P^T = F P (P symmetric), both operands K-major rows
      int rc;
      const int ldp = (n_ + 7) & ~7;
      if ((rc = split(F, n_, n_, n_, ldp, 0)) || (rc = split(P, n_, n_, n_, ldp, 1)) ||
          (rc = gemm_split(n_, n_, n_, ldp, 0, 1)))
        return rc;
      return combine_transpose(E, 1.0, -1.0);
    }
    const double one = 1.0, zero = 0.0;
    GEMM_TRY(gemm(false, false, n_, n_, n_, one, P, n_, F, n_, zero, E, n_));
    large::antisym_kernel<<<grid_for(nn_), large::kBlock, 0, c_->stream>>>(E, n_);
    ++c_->launches;
    return PM3GPU_OK;
  }
  // P = w X X^T over the first k eigenvectors of the last eigensolve (X is n x ld, row-major).
  int density_from_x(int k, int ld, double w, double* P, bool lowp = false) {
    if (k == 0) {
      CUDA_TRY(c_, cudaMemsetAsync(P, 0, 8 * nn_, c_->stream));
      return PM3GPU_OK;
    }
    if (lowp) {  // C = X X^T over the first k columns: one split; the result is symmetrised
      const double* X = B_.X.as<double>();
      const int ldp = (k + 7) & ~7;
      int rc;
      if ((rc = split(X, n_, k, ld, ldp, 0)) || (rc = gemm_split(n_, n_, k, ldp, 0, 0))) return rc;
      return combine_transpose(P, 0.5 * w, 0.5 * w);
    }
    const double zero = 0.0;
    GEMM_TRY(gemm(true, false, n_, n_, k, w, B_.X.as<double>(), ld, B_.X.as<double>(), ld, zero, P, n_));
    return PM3GPU_OK;
  }

  // Split the rows x cols matrix x (leading dimension ldx) into the BF16 hi / lo pair of operand
  // slot s, stored with leading dimension ldo (a multiple of 8, zero beyond cols).
  int split(const double* x, int rows, int cols, int ldx, int ldo, int s) {
    const size_t cnt = (size_t)rows * ldo;
    CUDA_TRY(c_, B_.mh[s].ensure(2 * cnt));
    CUDA_TRY(c_, B_.ml[s].ensure(2 * cnt));
    large::split_pad_kernel<<<grid_for(cnt), large::kBlock, 0, c_->stream>>>(
        x, rows, cols, ldx, B_.mh[s].as<__nv_bfloat16>(), B_.ml[s].as<__nv_bfloat16>(), ldo);
    ++c_->launches;
    CUDA_TRY(c_, cudaGetLastError());
    return PM3GPU_OK;
  }
  // c32 (m x m row-major FP32) = A B^T with A the split operand of slot sa and B that of slot sb
  // (m x k each, leading dimension ld): hi hi + hi lo + lo hi accumulated in FP32 in tensor memory
  // by the hand-written tcgen05 kernel (tc_gemm.cuh), one launch.
  int gemm_split(int m, int m2, int k, int ld, int sa, int sb) {
    CUDA_TRY(c_, B_.c32.ensure(4 * (size_t)m * m2));
    CUDA_TRY(c_, B_.tcerr.ensure(sizeof(int)));
    if (!B_.tcerr_zeroed) {
      CUDA_TRY(c_, cudaMemsetAsync(B_.tcerr.p, 0, sizeof(int), c_->stream));
      B_.tcerr_zeroed = true;
    }
    if (!tc::launch_split_gemm(m, m2, k, B_.mh[sa].as<__nv_bfloat16>(), B_.ml[sa].as<__nv_bfloat16>(), ld,
                               B_.mh[sb].as<__nv_bfloat16>(), B_.ml[sb].as<__nv_bfloat16>(), ld, B_.c32.as<float>(), m2,
                               B_.tcerr.as<int>(), c_->stream))
      return fail(c_, PM3GPU_CUDA_ERROR, "split-BF16 GEMM: tensor map or kernel attribute could not be set");
    ++c_->launches;
    CUDA_TRY(c_, cudaGetLastError());
    int flag = 0;
    CUDA_TRY(c_, cudaMemcpyAsync(&flag, B_.tcerr.p, sizeof(int), cudaMemcpyDeviceToHost, c_->stream));
    CUDA_TRY(c_, cudaStreamSynchronize(c_->stream));
    if (flag) return fail(c_, PM3GPU_CUDA_ERROR, "split-BF16 GEMM: a pipeline wait in the kernel ran out");
    return PM3GPU_OK;
  }
  // out = a c32 + b c32^T in FP64 (row-major n x n).
  int combine_transpose(double* out, double a, double b) {
    const size_t tiles = (size_t)((n_ + 31) / 32) * ((n_ + 31) / 32);
    large::transpose_combine_kernel<<<grid_for(tiles, 1), large::kBlock, 0, c_->stream>>>(B_.c32.as<float>(), out, n_, a,
                                                                                         b);
    ++c_->launches;
    CUDA_TRY(c_, cudaGetLastError());
    return PM3GPU_OK;
  }

  // The whole reduction is one fixed sequence of kernels and DGEMMs for a given matrix size and
  // set of buffers, so it is captured once into a CUDA graph and replayed in later SCF
  // iterations (it is ~5 launches per column). Streams that cannot be captured run it directly.
  int run_tridiag(double* A) {
    if (coop_grid() > 0) {  // one cooperative launch per panel: few enough launches to issue directly
      int launches = 0;
      const int rc = enqueue_tridiag(A, launches);
      c_->launches += launches;
      return rc;
    }
    TriGraph& g = B_.tg;
    const void* key[TriGraph::kKeys] = {A,        B_.V.p,  B_.Wp.p,    B_.vcol.p, B_.y.p,   B_.wtmp.p,
                                        B_.ps.p,  B_.s64.p, B_.part.p, B_.part2.p, B_.d.p,   B_.e.p,
                                        B_.tau.p, B_.tp.p, B_.ctr.p, B_.refl.p, (const void*)c_->stream};
    bool hit = g.exec != nullptr && g.n == n_;
    for (int k = 0; hit && k < TriGraph::kKeys; ++k) hit = g.key[k] == key[k];
    if (!hit) {
      g.reset();
      if (cudaStreamBeginCapture(c_->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        (void)cudaGetLastError();
        int launches = 0;
        const int rc = enqueue_tridiag(A, launches);
        c_->launches += launches;
        return rc;
      }
      int launches = 0;
      const int rc = enqueue_tridiag(A, launches);
      cudaGraph_t graph = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(c_->stream, &graph);
      if (rc != PM3GPU_OK || ec != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return rc != PM3GPU_OK ? rc : fail(c_, PM3GPU_CUDA_ERROR, std::string("graph capture: ") + cudaGetErrorString(ec));
      }
      const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ei != cudaSuccess) {
        g.exec = nullptr;
        return fail(c_, PM3GPU_CUDA_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(ei));
      }
      g.n = n_;
      g.launches = launches;
      for (int k = 0; k < TriGraph::kKeys; ++k) g.key[k] = key[k];
    }
    CUDA_TRY(c_, cudaGraphLaunch(g.exec, c_->stream));
    c_->launches += g.launches;
    return PM3GPU_OK;
  }

  // Grid of the cooperative panel kernel for this matrix size, 0 when the multi-launch path runs
  // instead (no cooperative launch, PM3GPU_COOP_PANELS=0, or more 64-row stripes than blocks:
  // each block owns one stripe).
  int coop_grid() {
    if (!c_->coop_panels) return 0;
    if ((c_->force_coop >= 0 ? c_->force_coop : tune_lookup(c_->tune_large, n_, 1)) == 0) return 0;
    if (coop_g_ < 0) {
      int occ = 0, coop = 0;
      if (cudaFuncSetAttribute(large::panel_coop_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)large::kCoopSmem) != cudaSuccess ||
          cudaFuncSetAttribute(large::panel_coop_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)large::kCoopSmem) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, large::panel_coop_kernel<true>, large::kBlock,
                                                        large::kCoopSmem) != cudaSuccess ||
          cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c_->device) != cudaSuccess) {
        (void)cudaGetLastError();
        occ = coop = 0;
      }
      coop_g_ = (coop && occ > 0) ? std::min(occ, 2) * c_->sms : 0;
    }
    if ((long long)coop_g_ * large::kTile < n_) return 0;
    // A small matrix has a few stripes and GEMV tiles (n = 204: 4 and 10), so most blocks of the
    // full grid only wait at the two grid barriers of each column; 64 blocks (the fewest the kernel
    // takes: blocks 0-63 each finish one component of W^T v, V^T v) shorten both barriers and the
    // cross-block sums.
    if (n_ <= kCoopSmallN) return std::min(coop_g_, 64);
    return coop_g_;
  }
  static constexpr int kCoopSmallN = 512;  // at most 8 stripes of 64 rows

  // Enqueues the blocked reduction of A (no host synchronisation inside).
  int enqueue_tridiag(double* A, int& launches) {
    int n = n_;
    double* d = B_.d.as<double>();
    double* e = B_.e.as<double>();
    double* tau = B_.tau.as<double>();
    double* V = B_.V.as<double>();
    double* W = B_.Wp.as<double>();
    double* vcol = B_.vcol.as<double>();
    const double one = 1.0, mone = -1.0;
    const int G = coop_grid();
    large::GridSync* gs = nullptr;
    double *X = nullptr, *Y = nullptr;
    if (G > 0) {
      CUDA_TRY(c_, B_.gsync.ensure(sizeof(large::GridSync)));
      CUDA_TRY(c_, B_.vw.ensure(8 * (size_t)n * large::kCoopLd));
      CUDA_TRY(c_, B_.wv.ensure(8 * (size_t)n * large::kCoopLd));
      gs = B_.gsync.as<large::GridSync>();
      X = B_.vw.as<double>();
      Y = B_.wv.as<double>();
      CUDA_TRY(c_, cudaMemsetAsync(gs, 0, sizeof(large::GridSync), c_->stream));
    }
    for (int p = 0; p < n - 2; p += large::kPanel) {
      int b = std::min(large::kPanel, n - 2 - p);
      if (G > 0) {
        double *tp = B_.tp.as<double>(), *pn = B_.part.as<double>();
        double *ps = B_.ps.as<double>(), *st = B_.s64.as<double>(), *pq = B_.part2.as<double>();
        void* args[] = {&A, &n, &p, &b, &X, &Y, &d, &e, &tau, &tp, &pn, &ps, &st, &pq, &gs};
        const void* fn = (n & 1) ? (const void*)large::panel_coop_kernel<false> : (const void*)large::panel_coop_kernel<true>;
        CUDA_TRY(c_, cudaLaunchCooperativeKernel(fn, dim3(G), dim3(large::kBlock), args,
                                                 large::kCoopSmem, c_->stream));
        ++launches;
        const int q = p + b, m = n - q;
        if (m > 0) {  // A[q:, q:] -= X Y^T (row-major); column-major: C -= Yc^T Xc, inner dimension 2b
          double* C = A + (size_t)q * n + q;
          const double* Xq = X + (size_t)q * large::kCoopLd;
          const double* Yq = Y + (size_t)q * large::kCoopLd;
          if (b == large::kPanel) {
            GEMM_TRY(gemm(true, false, m, m, 2 * b, mone, Yq, large::kCoopLd, Xq, large::kCoopLd, one, C, n, &launches));
          } else {  // last, narrower panel: columns b.. of X and Y are not part of it
            GEMM_TRY(gemm(true, false, m, m, b, mone, Yq, large::kCoopLd, Xq, large::kCoopLd, one, C, n, &launches));
            GEMM_TRY(gemm(true, false, m, m, b, mone, Yq + large::kPanel, large::kCoopLd, Xq + large::kPanel, large::kCoopLd, one, C, n, &launches));
          }
        }
        continue;
      }
      for (int j = 0; j < b; ++j) {
        const int i = p + j;
        const int m = n - i - 1;
        const int gu = grid_for((size_t)(n - i), large::kBlock, large::kRedBlocks);
        double* refl = B_.refl.as<double>();
        unsigned int* ctr = B_.ctr.as<unsigned int>();
        large::panel_update_kernel<<<gu, large::kBlock, 0, c_->stream>>>(A, n, i, j, V, W, B_.part2.as<double>(), ctr,
                                                                         d, e, tau, refl);
        const int nt = (m + large::kTile - 1) / large::kTile;
        const long long ntiles = (long long)nt * (nt + 1) / 2;
        large::symv_tiles_kernel<<<(unsigned)ntiles, large::kBlock, 0, c_->stream>>>(A, n, i, refl, B_.tp.as<double>());
        const int gg = std::max(1, std::min((m + 31) / 32, large::kRedBlocks));
        large::symv_gather_kernel<<<gg, large::kBlock, 0, c_->stream>>>(A, n, i, j, V, W, refl, B_.tp.as<double>(),
                                                                        B_.y.as<double>(), B_.ps.as<double>(), ctr + 1,
                                                                        B_.s64.as<double>());
        const int gw = grid_for((size_t)m, large::kBlock, large::kRedBlocks);
        large::panel_wfix_kernel<<<gw, large::kBlock, 0, c_->stream>>>(A, n, i, j, V, W, vcol, B_.y.as<double>(),
                                                                        B_.s64.as<double>(), refl,
                                                                        B_.wtmp.as<double>(), B_.part.as<double>());
        large::panel_wfinal_kernel<<<grid_for((size_t)n, large::kBlock, large::kRedBlocks), large::kBlock, 0,
                                     c_->stream>>>(n, i, j, vcol, V, W, B_.wtmp.as<double>(), B_.part.as<double>(), gw,
                                                   tau + i);
        launches += 5;  // update, tiles, gather, wfix, wfinal
      }
      const int q = p + b, m = n - q;
      if (m > 0) {  // A[q:, q:] -= V W^T + W V^T (row-major); column-major: C -= Wc^T Vc + Vc^T Wc
        double* C = A + (size_t)q * n + q;
        const double* Vq = V + (size_t)q * large::kPanel;
        const double* Wq = W + (size_t)q * large::kPanel;
        GEMM_TRY(gemm(true, false, m, m, b, mone, Wq, large::kPanel, Vq, large::kPanel, one, C, n, &launches));
        GEMM_TRY(gemm(true, false, m, m, b, mone, Vq, large::kPanel, Wq, large::kPanel, one, C, n, &launches));
      }
    }
    large::tail_kernel<<<1, 1, 0, c_->stream>>>(A, n, d, e, tau);
    ++launches;
    CUDA_TRY(c_, cudaGetLastError());
    return PM3GPU_OK;
  }

  // Lowest kval eigenvalues of the tridiagonal in B_.d / B_.e (host bookkeeping of splits).
  int eigenvalues(int kval, std::vector<double>& lam, std::vector<double>& dl, bool warm) {
    const int n = n_;
    std::vector<double> d(n), e(n);
    CUDA_TRY(c_, cudaMemcpyAsync(d.data(), B_.d.p, 8 * (size_t)n, cudaMemcpyDeviceToHost, c_->stream));
    CUDA_TRY(c_, cudaMemcpyAsync(e.data(), B_.e.p, 8 * (size_t)n, cudaMemcpyDeviceToHost, c_->stream));
    CUDA_TRY(c_, cudaStreamSynchronize(c_->stream));
    return eigenvalues_host(d, e, kval, lam, dl, warm);
  }
  int eigenvalues_host(std::vector<double>& d, std::vector<double>& e, int kval, std::vector<double>& lam,
                       std::vector<double>& dl, bool warm) {
    const int n = n_;
    constexpr double eps = 2.220446049250313e-16;
    double gl = d[0], gu = d[0];
    for (int i = 0; i < n; ++i) {
      const double rad = (i + 1 < n ? std::fabs(e[i]) : 0.0) + (i > 0 ? std::fabs(e[i - 1]) : 0.0);
      gl = std::min(gl, d[i] - rad);
      gu = std::max(gu, d[i] + rad);
    }
    const double tnorm = std::max(std::fabs(gl), std::fabs(gu));
    const double cut = 1000.0 * eps * tnorm;
    std::vector<double> e2(n);
    hblk_.assign(1, 0);
    double emax = 0.0;
    for (int i = 0; i < n; ++i) {
      double ei = (i + 1 < n) ? e[i] : 0.0;
      if (i + 1 < n && std::fabs(ei) <= cut) {
        ei = 0.0;
        e[i] = 0.0;
        hblk_.push_back(i + 1);
      }
      e2[i] = ei * ei;
      emax = std::max(emax, ei * ei);
    }
    hblk_.push_back(n);
    pivmin_ = 2.2250738585072014e-308 * std::max(1.0, emax);
    tnorm_ = tnorm;
    const double glo = gl - 4.0 * eps * tnorm * n - 1.0e-300, ghi = gu + 4.0 * eps * tnorm * n + 1.0e-300;
    CUDA_TRY(c_, B_.e2.ensure(8 * (size_t)n));
    CUDA_TRY(c_, B_.blk.ensure(4 * hblk_.size()));
    CUDA_TRY(c_, B_.lam.ensure(8 * (size_t)n));
    CUDA_TRY(c_, B_.dlam.ensure(16 * (size_t)n));
    CUDA_TRY(c_, cudaMemcpyAsync(B_.e.p, e.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, c_->stream));
    CUDA_TRY(c_, cudaMemcpyAsync(B_.e2.p, e2.data(), 8 * (size_t)n, cudaMemcpyHostToDevice, c_->stream));
    CUDA_TRY(c_, cudaMemcpyAsync(B_.blk.p, hblk_.data(), 4 * hblk_.size(), cudaMemcpyHostToDevice, c_->stream));
    const bool seeded = warm && (int)lam.size() == kval && (int)dl.size() == kval;
    double* prev = B_.dlam.as<double>();
    double* dprev = prev + n;
    if (seeded) {
      CUDA_TRY(c_, cudaMemcpyAsync(prev, lam.data(), 8 * (size_t)kval, cudaMemcpyHostToDevice, c_->stream));
      CUDA_TRY(c_, cudaMemcpyAsync(dprev, dl.data(), 8 * (size_t)kval, cudaMemcpyHostToDevice, c_->stream));
    }
    int g = 32;
    while (g > 1 && (size_t)kval * g > 65536) g >>= 1;
    const int threads = kval * g;
    large::multisect_kernel<<<(threads + large::kBlock - 1) / large::kBlock, large::kBlock, 0, c_->stream>>>(
        B_.d.as<double>(), B_.e2.as<double>(), n, kval, g, glo, ghi, pivmin_, tnorm_, seeded ? prev : nullptr,
        seeded ? dprev : nullptr, B_.lam.as<double>());
    ++c_->launches;
    CUDA_TRY(c_, cudaGetLastError());
    std::vector<double> nl(kval);
    CUDA_TRY(c_, cudaMemcpyAsync(nl.data(), B_.lam.p, 8 * (size_t)kval, cudaMemcpyDeviceToHost, c_->stream));
    CUDA_TRY(c_, cudaStreamSynchronize(c_->stream));
    dl.assign(kval, 1.0e30);
    if (seeded)
      for (int j = 0; j < kval; ++j) dl[j] = nl[j] - lam[j];
    lam.swap(nl);
    return PM3GPU_OK;
  }

  // Eigen-decomposition of the symmetric matrix in A (destroyed): kval lowest eigenvalues into
  // lam, kvec eigenvectors into B_.X (n x kvec, row-major). `tri` receives the tridiagonal.
  int eigensolve(double* A, int kval, int kvec, std::vector<double>& lam, std::vector<double>& dl, bool warm,
                 std::vector<double>* tri) {
    const int n = n_;
    const size_t K = (size_t)std::max(kvec, 1);
    {
      const int rc = prepare_reduction();
      if (rc) return rc;
    }
    double* d = B_.d.as<double>();
    double* e = B_.e.as<double>();
    double* tau = B_.tau.as<double>();
    double* V = B_.V.as<double>();
    double* W = B_.Wp.as<double>();
    const double one = 1.0, mone = -1.0, zero = 0.0;
    // ---- 1. Householder tridiagonalisation (sytrd/latrd, lower), replayed from a CUDA graph
    {
      const int rc = run_tridiag(A);
      if (rc) return rc;
    }
    tick(kLgTridiag);
    // ---- 2. eigenvalues (host split bookkeeping, device multisection)
    {
      std::vector<double> hd(n), he(n);
      CUDA_TRY(c_, cudaMemcpyAsync(hd.data(), d, 8 * (size_t)n, cudaMemcpyDeviceToHost, c_->stream));
      CUDA_TRY(c_, cudaMemcpyAsync(he.data(), e, 8 * (size_t)n, cudaMemcpyDeviceToHost, c_->stream));
      large::GridSync gsh{};
      if (coop_grid() > 0)
        CUDA_TRY(c_, cudaMemcpyAsync(&gsh, B_.gsync.p, sizeof(gsh), cudaMemcpyDeviceToHost, c_->stream));
      CUDA_TRY(c_, cudaStreamSynchronize(c_->stream));
      if (gsh.err) return fail(c_, PM3GPU_CUDA_ERROR, "Householder panel: a grid barrier wait ran out");
      if (tri) {
        tri->assign(2 * (size_t)n, 0.0);
        std::copy(hd.begin(), hd.end(), tri->begin());
        std::copy(he.begin(), he.end(), tri->begin() + n);
      }
      int rc = eigenvalues_host(hd, he, kval, lam, dl, warm);
      if (rc) return rc;
    }
    tick(kLgEigval);
    if (kvec <= 0) return PM3GPU_OK;
    // ---- 3. eigenvectors of the tridiagonal
    CUDA_TRY(c_, B_.X.ensure(8 * (size_t)n * K));
    CUDA_TRY(c_, B_.Xt.ensure(8 * (size_t)n * K));
    for (DevBuf* bf : {&B_.Dp, &B_.Lp, &B_.Um}) CUDA_TRY(c_, bf->ensure(8 * (size_t)n * K));
    double* X = B_.X.as<double>();
    large::twisted_kernel<<<(kvec + large::kBlock - 1) / large::kBlock, large::kBlock, 0, c_->stream>>>(
        d, e, B_.e2.as<double>(), n, kvec, B_.lam.as<double>(), B_.blk.as<int>(), (int)hblk_.size() - 1, pivmin_, tnorm_,
        X, B_.Dp.as<double>(), B_.Lp.as<double>(), B_.Um.as<double>());
    ++c_->launches;
    CUDA_TRY(c_, cudaGetLastError());
    tick(kLgEigvec);
    // ---- 4. back-transformation X <- Q X, blocks of kWy reflectors from the last to the first
    CUDA_TRY(c_, B_.Gm.ensure(8 * (size_t)large::kWy * large::kWy));
    CUDA_TRY(c_, B_.Tm.ensure(8 * (size_t)large::kWy * large::kWy));
    CUDA_TRY(c_, B_.Z1.ensure(8 * K * large::kWy));
    CUDA_TRY(c_, B_.Z2.ensure(8 * K * large::kWy));
    CUDA_TRY(c_, B_.Vw.ensure(8 * (size_t)n * large::kWy));
    double* Vw = B_.Vw.as<double>();
    const int nbk = n - 2 > 0 ? (n - 2 + large::kWy - 1) / large::kWy : 0;
    for (int bi = nbk - 1; bi >= 0; --bi) {
      const int p = bi * large::kWy, b = std::min(large::kWy, n - 2 - p);
      large::block_v_kernel<<<grid_for((size_t)n * large::kWy), large::kBlock, 0, c_->stream>>>(A, n, p, b, Vw);
      ++c_->launches;
      const int r0 = p + 1, m = n - r0;
      const double* Vr = Vw + (size_t)r0 * large::kWy;
      double* Xr = X + (size_t)r0 * K;
      // G = V^T V (b x b); column-major: Vc Vc^T
      GEMM_TRY(gemm(false, true, b, b, m, one, Vr, large::kWy, Vr, large::kWy, zero, B_.Gm.as<double>(), b));
      large::wy_t_block_kernel<<<1, large::kWy, 0, c_->stream>>>(B_.Gm.as<double>(), tau, p, b, B_.Tm.as<double>());
      ++c_->launches;
      // Z = V^T X  -> column-major Zc = Xc Vc^T (K x b)
      GEMM_TRY(gemm(false, true, (int)K, b, m, one, Xr, (int)K, Vr, large::kWy, zero, B_.Z1.as<double>(), (int)K));
      // Z2 = T Z -> Z2c = Zc T^T, T row-major = column-major T^T
      GEMM_TRY(gemm(false, false, (int)K, b, b, one, B_.Z1.as<double>(), (int)K, B_.Tm.as<double>(), large::kWy, zero,
                    B_.Z2.as<double>(), (int)K));
      // X -= V Z2 -> Xc -= Z2c Vc
      GEMM_TRY(gemm(false, false, (int)K, m, b, mone, B_.Z2.as<double>(), (int)K, Vr, large::kWy, one, Xr, (int)K));
    }
    tick(kLgBack);
    // ---- 5. orthonormalise: X <- X (3I - X^T X) / 2 until max |X^T X - I| < 1e-13; at most
    // kNsSteps updates, the defect measured after each. A defect still at or above kOrthAccept
    // after the last update is a linear-algebra failure (PM3GPU_LINALG), not a silent result.
    CUDA_TRY(c_, B_.Mm.ensure(8 * K * K));
    CUDA_TRY(c_, B_.Gk.ensure(8 * K * K));
    double* Gk = B_.Gk.as<double>();
    last_ns_steps_ = 0;
    last_defect_ = INFINITY;
    for (int step = 0; step <= kNsSteps; ++step) {
      GEMM_TRY(gemm(false, true, (int)K, (int)K, n, one, X, (int)K, X, (int)K, zero, Gk, (int)K));
      large::orth_defect_kernel<<<large::kRedBlocks, large::kBlock, 0, c_->stream>>>(Gk, (int)K, B_.part.as<double>());
      ++c_->launches;
      std::vector<double> mx(large::kRedBlocks);
      CUDA_TRY(c_, cudaMemcpyAsync(mx.data(), B_.part.p, 8 * mx.size(), cudaMemcpyDeviceToHost, c_->stream));
      CUDA_TRY(c_, cudaStreamSynchronize(c_->stream));
      double defect = 0.0;
      for (double v : mx) defect = std::max(defect, v);
      last_defect_ = defect;
      if (!(defect < 0.5)) return fail(c_, PM3GPU_LINALG, "large eigensolver: eigenvectors far from orthonormal");
      if (defect < 1.0e-13) break;
      if (step == kNsSteps) {
        char msg[160];
        std::snprintf(msg, sizeof msg,
                      "large eigensolver: occupied vectors orthonormal only to %.3e after %d Newton-Schulz steps",
                      defect, kNsSteps);
        if (!(defect < kOrthAccept)) return fail(c_, PM3GPU_LINALG, msg);
        break;
      }
      ++last_ns_steps_;
      large::ns_matrix_kernel<<<grid_for(K * K), large::kBlock, 0, c_->stream>>>(Gk, B_.Mm.as<double>(), (int)K);
      ++c_->launches;
      // X M (row-major) -> column-major M Xc (M symmetric)
      GEMM_TRY(gemm(false, false, (int)K, n, (int)K, one, B_.Mm.as<double>(), (int)K, X, (int)K, zero, B_.Xt.as<double>(), (int)K));
      std::swap(B_.X, B_.Xt);
      X = B_.X.as<double>();
    }
    tick(kLgOrth);
    return PM3GPU_OK;
  }

  // Largest |F X - X diag(lam)| over the k occupied eigenpairs of the last eigensolve (X = B_.X,
  // lam = B_.lam), F symmetric row-major: one DGEMM and a max reduction.
  int eigen_residual(const double* F, int k, double* out) {
    const int n = n_;
    const double one = 1.0, zero = 0.0;
    CUDA_TRY(c_, B_.Xt.ensure(8 * (size_t)n * k));
    // row-major Y = F X  ->  column-major Yc = Xc F (F symmetric)
    GEMM_TRY(gemm(false, false, k, n, n, one, B_.X.as<double>(), k, F, n, zero, B_.Xt.as<double>(), k));
    large::eig_residual_kernel<<<large::kRedBlocks, large::kBlock, 0, c_->stream>>>(
        B_.Xt.as<double>(), B_.X.as<double>(), B_.lam.as<double>(), n, k, B_.part.as<double>());
    ++c_->launches;
    CUDA_TRY(c_, cudaGetLastError());
    std::vector<double> mx(large::kRedBlocks);
    CUDA_TRY(c_, cudaMemcpyAsync(mx.data(), B_.part.p, 8 * mx.size(), cudaMemcpyDeviceToHost, c_->stream));
    CUDA_TRY(c_, cudaStreamSynchronize(c_->stream));
    double r = 0.0;
    for (double v : mx) r = std::max(r, v);
    *out = r;
    return PM3GPU_OK;
  }

  // Work buffers of the Householder reduction for this matrix size.
  int prepare_reduction() {
    const int n = n_;
    for (DevBuf* b : {&B_.d, &B_.e, &B_.tau, &B_.y, &B_.wtmp, &B_.vcol}) CUDA_TRY(c_, b->ensure(8 * (size_t)n));
    CUDA_TRY(c_, B_.V.ensure(8 * (size_t)n * large::kPanel));
    CUDA_TRY(c_, B_.Wp.ensure(8 * (size_t)n * large::kPanel));
    CUDA_TRY(c_, B_.ps.ensure(8 * 64 * (size_t)large::kRedBlocks));
    CUDA_TRY(c_, B_.s64.ensure(8 * 64));
    const long long nt = (n + large::kTile - 1) / large::kTile;  // absolute stripes (covers the trailing ones)
    CUDA_TRY(c_, B_.tp.ensure(8 * (size_t)(2 * large::kTile) * (size_t)std::max<long long>(nt * (nt + 1) / 2, 1)));
    if (!B_.ctr.p) {
      CUDA_TRY(c_, B_.ctr.ensure(256));
      CUDA_TRY(c_, cudaMemsetAsync(B_.ctr.p, 0, 256, c_->stream));
    }
    CUDA_TRY(c_, B_.refl.ensure(256));
    return PM3GPU_OK;
  }

  // Mulliken charges and the dipole about the centre of mass (dipole.rs:64-144) from the atom
  // blocks of the total density.
  int properties(const double* Pt, LargeRun& R) {
    CUDA_TRY(c_, B_.blocks.ensure(8 * 16 * (size_t)N_));
    large::atom_blocks_kernel<<<grid_for((size_t)N_ * 16), large::kBlock, 0, c_->stream>>>(m_, Pt, B_.blocks.as<double>());
    ++c_->launches;
    std::vector<double> blk(16 * (size_t)N_), xyz(3 * (size_t)N_);
    CUDA_TRY(c_, cudaMemcpyAsync(blk.data(), B_.blocks.p, 8 * blk.size(), cudaMemcpyDeviceToHost, c_->stream));
    CUDA_TRY(c_, cudaMemcpyAsync(xyz.data(), m_.xyz, 8 * xyz.size(), cudaMemcpyDeviceToHost, c_->stream));
    CUDA_TRY(c_, cudaStreamSynchronize(c_->stream));
    R.charges.assign(N_, 0.0);
    double mt = 0.0, cm[3] = {0, 0, 0};
    for (int a = 0; a < N_; ++a) {
      const ElemDev& el = c_->h_elem[hz_[a]];
      double pop = 0.0;
      for (int k = 0; k < el.norb; ++k) pop += blk[16 * (size_t)a + 5 * k];
      R.charges[a] = el.core - pop;
      mt += el.mass;
      for (int k = 0; k < 3; ++k) cm[k] += el.mass * xyz[3 * (size_t)a + k];
    }
    for (int k = 0; k < 3; ++k) cm[k] = mt > 0.0 ? cm[k] / mt : 0.0;
    double mu[3] = {0, 0, 0};
    for (int a = 0; a < N_; ++a) {
      const ElemDev& el = c_->h_elem[hz_[a]];
      double pop = 0.0;
      for (int k = 0; k < el.norb; ++k) pop += blk[16 * (size_t)a + 5 * k];
      for (int ax = 0; ax < 3; ++ax) {
        const double disp = xyz[3 * (size_t)a + ax] - cm[ax];
        double elc = pop * disp;
        if (el.norb == 4) elc += 2.0 * blk[16 * (size_t)a + ax + 1] * el.dd;
        mu[ax] += disp * el.core - elc;
      }
    }
    for (int ax = 0; ax < 3; ++ax) R.o.dipole[ax] = mu[ax] * kAuDipoleToDebye;
    return PM3GPU_OK;
  }

  double pivmin_ = 0.0, tnorm_ = 0.0;
  // Newton-Schulz bookkeeping of the last eigensolve: defect max |X^T X - I| after the last
  // measured step, and the number of updates applied
  static constexpr int kNsSteps = 5;
  static constexpr double kOrthAccept = 1.0e-11;
  double last_defect_ = 0.0;
  int last_ns_steps_ = 0;
  std::chrono::steady_clock::time_point t0_ = std::chrono::steady_clock::now();

 public:
  // Phase clock (profiling only: each tick waits for the stream).
  void tick(int phase) {
    if (!c_->profile) return;
    cudaStreamSynchronize(c_->stream);
    const auto t = std::chrono::steady_clock::now();
    c_->large_ms[phase] += std::chrono::duration<double, std::milli>(t - t0_).count();
    t0_ = t;
  }
};
