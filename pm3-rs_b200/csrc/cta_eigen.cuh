// Symmetric eigensolver for one matrix per CTA (n <= kMaxN), replacing the reference's faer
// `self_adjoint_eigen` (pm3-rs src/linalg.rs:221-263) on the SCF path:
//   1. Householder reduction to tridiagonal form, the matrix held as a packed lower triangle
//      (row-major: element (r, c), r >= c, at r(r+1)/2 + c) in shared memory (or global memory
//      when it does not fit). Reflectors stay in the strictly-lower part of column i.
//   2. Eigenvalues of the tridiagonal T by Sturm-count bisection, one thread per eigenvalue.
//   3. Eigenvectors of T by twisted (N_r D_r N_r^T) factorisation, one thread per vector,
//      on the unreduced block holding the eigenvalue (T is split where |e_i| <= 1000 eps ||T||,
//      which separates exact degeneracies); members of a within-block cluster (gap below
//      1e-7 ||T||) after the first are redone by inverse iteration with re-orthogonalisation.
//   4. Back-transformation Z = Q Y, one warp per pair of vectors held in registers.
// Only the eigenpairs the SCF needs are formed (the occupied block, plus one more value for
// the frontier gap). Eigenvalues come out ascending, as the reference requires.
#pragma once
#include "cta_blas.cuh"

namespace pm3gpu {

constexpr int kMaxN = 256;          // largest basis handled by the per-CTA path
constexpr int kRowT = kMaxN / 32;   // rows per lane in warp-per-row loops

__device__ __forceinline__ int tri(int r) { return r * (r + 1) / 2; }
__device__ __forceinline__ double ap_get(const double* A, int r, int c) { return r >= c ? A[tri(r) + c] : A[tri(c) + r]; }

struct EigenScratch {
  double* d;     // [n] diagonal of T
  double* e;     // [n] off-diagonal of T (e[i] couples i, i+1); zeroed where T splits
  double* e2;    // [n] e^2
  double* tau;   // [n] reflector scales
  double* v;     // [n] current reflector
  double* p;     // [n] symv result
  double* lam;   // [n] eigenvalues (ascending)
  int* blk;      // [n+1] block starts (blk[0] = 0, ..., blk[nb] = n)
  int* nblk;     // [1]
  int* vinfo;    // [n] per eigenvector: its block index
  double* red;   // reduction scratch (>= 8 * kWarps)
  double* misc;  // [8] broadcast scalars
};

// ---------------------------------------------------------------- 1. tridiagonalisation
__device__ void tridiagonalize(int n, double* A, const EigenScratch& s) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = 0; i + 2 < n; ++i) {
    // x = A[i+1.., i]; annihilate A[i+2.., i]
    double part = 0.0;
    for (int r = i + 2 + tid; r < n; r += kThreads) {
      const double x = A[tri(r) + i];
      part += x * x;
    }
    const double xn2 = block_sum(part, s.red);
    const double alpha = A[tri(i + 1) + i];
    double beta = 0.0, tau = 0.0, scal = 0.0;
    if (xn2 > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
      tau = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    if (tid == 0) {
      s.tau[i] = tau;
      s.e[i] = xn2 > 0.0 ? beta : alpha;
      s.d[i] = A[tri(i) + i];
    }
    if (xn2 == 0.0) {  // already reduced: nothing to apply (uniform branch)
      __syncthreads();
      continue;
    }
    for (int r = i + 1 + tid; r < n; r += kThreads) {
      double vr = 1.0;
      if (r > i + 1) {
        vr = A[tri(r) + i] * scal;
        A[tri(r) + i] = vr;
      }
      s.v[r] = vr;
    }
    __syncthreads();
    // p = tau * A22 v (A22 = A[i+1.., i+1..]); warp per row, lanes across the row
    double dpart = 0.0;
    for (int r = i + 1 + warp; r < n; r += kWarps) {
      double acc = 0.0;
      for (int c = i + 1 + lane; c < n; c += 32) acc = fma(ap_get(A, r, c), s.v[c], acc);
      acc = warp_sum(acc) * tau;
      if (lane == 0) s.p[r] = acc;
      dpart = fma(acc, s.v[r], dpart);
    }
    const double dot = block_sum(lane == 0 ? dpart : 0.0, s.red);
    const double a2 = -0.5 * tau * dot;
    // A22 -= v w^T + w v^T with w = p + a2 v
    for (int r = i + 1 + warp; r < n; r += kWarps) {
      const double vr = s.v[r], wr = s.p[r] + a2 * vr;
      double* row = A + tri(r);
      for (int c = i + 1 + lane; c <= r; c += 32) {
        const double vc = s.v[c], wc = s.p[c] + a2 * vc;
        row[c] -= vr * wc + wr * vc;
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      s.d[n - 2] = A[tri(n - 2) + n - 2];
      s.e[n - 2] = A[tri(n - 1) + n - 2];
      s.tau[n - 2] = 0.0;
    }
    s.d[n - 1] = A[tri(n - 1) + n - 1];
    s.e[n - 1] = 0.0;
  }
  __syncthreads();
}

// ------------------------------------------------------------- 2. split + eigenvalues
// Sturm count: number of eigenvalues of T[lo..hi] below x.
__device__ __forceinline__ int sturm(const double* d, const double* e2, int lo, int hi, double x, double pivmin) {
  int cnt = 0;
  double q = d[lo] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += q < 0.0;
  for (int i = lo + 1; i <= hi; ++i) {
    q = (d[i] - x) - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
  }
  return cnt;
}

// Splits T where the coupling is negligible and computes the lowest `kval` eigenvalues.
// Leaves pivmin / tnorm in misc[0] / misc[1].
__device__ void tridiag_eigenvalues(int n, int kval, const EigenScratch& s) {
  const int tid = threadIdx.x;
  constexpr double eps = 2.220446049250313e-16;
  if (tid == 0) {
    // Gershgorin bounds of the unsplit T, then split where |e_i| <= 1000 eps ||T||: an
    // absolute criterion, so exactly degenerate eigenvalues (which Householder leaves joined
    // by couplings of a few eps ||T||) land in separate blocks.
    double gl = s.d[0], gu = s.d[0];
    for (int i = 0; i < n; ++i) {
      const double rad = (i + 1 < n ? fabs(s.e[i]) : 0.0) + (i > 0 ? fabs(s.e[i - 1]) : 0.0);
      gl = fmin(gl, s.d[i] - rad);
      gu = fmax(gu, s.d[i] + rad);
    }
    const double tnorm = fmax(fabs(gl), fabs(gu));
    const double cut = 1000.0 * eps * tnorm;
    int nb = 0;
    s.blk[0] = 0;
    double emax = 0.0;
    for (int i = 0; i < n; ++i) {
      double ei = (i + 1 < n) ? s.e[i] : 0.0;
      if (i + 1 < n && fabs(ei) <= cut) {
        ei = 0.0;
        s.e[i] = 0.0;
        s.blk[++nb] = i + 1;
      }
      s.e2[i] = ei * ei;
      emax = fmax(emax, ei * ei);
    }
    s.blk[++nb] = n;
    *s.nblk = nb;
    s.misc[0] = 2.2250738585072014e-308 * fmax(1.0, emax);  // pivmin
    s.misc[1] = tnorm;
    s.misc[2] = gl - 4.0 * eps * tnorm * n - 1.0e-300;
    s.misc[3] = gu + 4.0 * eps * tnorm * n + 1.0e-300;
  }
  __syncthreads();
  const double pivmin = s.misc[0], glo = s.misc[2], ghi = s.misc[3];
  for (int j = tid; j < kval; j += kThreads) {
    double lo = glo, hi = ghi;
    for (int it = 0; it < 128; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (mid <= lo || mid >= hi) break;
      if (hi - lo <= 2.0 * eps * fmax(fabs(lo), fabs(hi)) + 4.0 * pivmin) break;
      if (sturm(s.d, s.e2, 0, n - 1, mid, pivmin) > j) hi = mid;
      else lo = mid;
    }
    s.lam[j] = 0.5 * (lo + hi);
  }
  __syncthreads();
}

// ------------------------------------------------------------- 3. tridiagonal eigenvectors
// Eigenvector j (< kvec) of T into Y[j*n .. j*n+n) (zero outside its block). `tf` is per-CTA
// global scratch of kvec * 6n doubles.
__device__ void tridiag_vectors(int n, int kvec, double* Y, double* tf, const EigenScratch& s) {
  const int tid = threadIdx.x;
  const double pivmin = s.misc[0], tnorm = s.misc[1];
  const int nb = *s.nblk;
  const double win = 1.0e-11 * fmax(tnorm, 1.0);
  for (int j = tid; j < kvec; j += kThreads) {
    const double lam = s.lam[j];
    // which unreduced block holds this eigenvalue (degenerate copies go to successive blocks)
    int pos = j - sturm(s.d, s.e2, 0, n - 1, lam - win, pivmin);
    int b = -1, sub = 0;
    for (int q = 0; q < nb && b < 0; ++q) {
      const int lo = s.blk[q], hi = s.blk[q + 1] - 1;
      const int c = sturm(s.d, s.e2, lo, hi, lam + win, pivmin) - sturm(s.d, s.e2, lo, hi, lam - win, pivmin);
      if (pos < c) {
        b = q;
        sub = pos;
      } else {
        pos -= c;
      }
    }
    if (b < 0) b = 0;  // inconsistent counts (not expected): block 0
    (void)sub;
    s.vinfo[j] = b;
    const int lo = s.blk[b], hi = s.blk[b + 1] - 1, m = hi - lo + 1;
    double* y = Y + (size_t)j * n;
    for (int i = 0; i < n; ++i) y[i] = 0.0;
    if (m == 1) {
      y[lo] = 1.0;
      continue;
    }
    double* Dp = tf + (size_t)j * 6 * n;
    double* Lp = Dp + n;
    double* Um = Lp + n;
    // T - lam = L+ D+ L+^T (top-down)
    double dp = s.d[lo] - lam;
    for (int i = 0; i < m - 1; ++i) {
      if (fabs(dp) < pivmin) dp = dp < 0.0 ? -pivmin : pivmin;
      Dp[i] = dp;
      const double ei = s.e[lo + i];
      Lp[i] = ei / dp;
      dp = (s.d[lo + i + 1] - lam) - Lp[i] * ei;
    }
    if (fabs(dp) < pivmin) dp = dp < 0.0 ? -pivmin : pivmin;
    Dp[m - 1] = dp;
    // T - lam = U- D- U-^T (bottom-up), twist index r minimising |gamma|
    double dm = s.d[hi] - lam;
    if (fabs(dm) < pivmin) dm = dm < 0.0 ? -pivmin : pivmin;
    double best = fabs(Dp[m - 1] + dm - (s.d[hi] - lam));
    int r = m - 1;
    for (int i = m - 2; i >= 0; --i) {
      const double ei = s.e[lo + i];
      Um[i] = ei / dm;
      dm = (s.d[lo + i] - lam) - Um[i] * ei;
      if (fabs(dm) < pivmin) dm = dm < 0.0 ? -pivmin : pivmin;
      const double g = fabs(Dp[i] + dm - (s.d[lo + i] - lam));
      if (g < best) {
        best = g;
        r = i;
      }
    }
    // solve N_r D_r N_r^T y = gamma_r e_r
    y[lo + r] = 1.0;
    for (int i = r - 1; i >= 0; --i) {
      double z = -Lp[i] * y[lo + i + 1];
      if (y[lo + i + 1] == 0.0 && i + 2 < m) z = -(s.e[lo + i + 1] / s.e[lo + i]) * y[lo + i + 2];
      y[lo + i] = z;
    }
    for (int i = r; i < m - 1; ++i) {
      double z = -Um[i] * y[lo + i];
      if (y[lo + i] == 0.0 && i >= 1) z = -(s.e[lo + i - 1] / s.e[lo + i]) * y[lo + i - 1];
      y[lo + i + 1] = z;
    }
    double nrm = 0.0;
    for (int i = lo; i <= hi; ++i) nrm += y[i] * y[i];
    nrm = 1.0 / sqrt(nrm);
    for (int i = lo; i <= hi; ++i) y[i] *= nrm;
  }
  __syncthreads();
  // Eigenvalues of one block closer than 1e-7 ||T||: the twisted vectors are not reliable
  // there, so every cluster member after the first is recomputed by inverse iteration on a
  // row-pivoted LU of T_b - lam, re-orthogonalised against the earlier members of its
  // cluster (the dstein scheme). One thread per block; clusters are rare.
  const double ctol = 1.0e-7 * fmax(tnorm, 1.0), tiny = 2.220446049250313e-16 * fmax(tnorm, 1.0);
  for (int b = tid; b < nb; b += kThreads) {
    const int lo = s.blk[b], hi = s.blk[b + 1] - 1, m = hi - lo + 1;
    int head = -1, prev = -1;
    for (int j = 0; j < kvec; ++j) {
      if (s.vinfo[j] != b) continue;
      if (prev < 0 || s.lam[j] - s.lam[prev] >= ctol) {
        head = j;
        prev = j;
        continue;
      }
      prev = j;
      double* dd = tf + (size_t)j * 6 * n;
      double* dl = dd + n;
      double* du = dl + n;
      double* du2 = du + n;
      double* pv = du2 + n;
      const double sg = s.lam[j];
      for (int i = 0; i < m; ++i) {
        dd[i] = s.d[lo + i] - sg;
        if (i + 1 < m) dl[i] = du[i] = s.e[lo + i];
      }
      for (int i = 0; i + 1 < m; ++i) {
        if (fabs(dd[i]) >= fabs(dl[i])) {
          if (dd[i] == 0.0) dd[i] = tiny;
          const double f = dl[i] / dd[i];
          dl[i] = f;
          dd[i + 1] -= f * du[i];
          if (i + 2 < m) du2[i] = 0.0;
          pv[i] = 0.0;
        } else {
          const double f = dd[i] / dl[i];
          dd[i] = dl[i];
          dl[i] = f;
          const double t = du[i];
          du[i] = dd[i + 1];
          dd[i + 1] = t - f * dd[i + 1];
          if (i + 2 < m) {
            du2[i] = du[i + 1];
            du[i + 1] = -f * du[i + 1];
          }
          pv[i] = 1.0;
        }
      }
      for (int i = 0; i < m; ++i)
        if (fabs(dd[i]) < tiny) dd[i] = dd[i] < 0.0 ? -tiny : tiny;
      double* x = Y + (size_t)j * n + lo;
      for (int i = 0; i < m; ++i) x[i] = sin(1.0 + 0.7 * i + 1.3 * j);
      for (int it = 0; it < 3; ++it) {
        for (int i = 0; i + 1 < m; ++i) {
          if (pv[i] == 0.0) {
            x[i + 1] -= dl[i] * x[i];
          } else {
            const double t = x[i];
            x[i] = x[i + 1];
            x[i + 1] = t - dl[i] * x[i];
          }
        }
        x[m - 1] /= dd[m - 1];
        if (m > 1) x[m - 2] = (x[m - 2] - du[m - 2] * x[m - 1]) / dd[m - 2];
        for (int i = m - 3; i >= 0; --i) x[i] = (x[i] - du[i] * x[i + 1] - du2[i] * x[i + 2]) / dd[i];
        for (int pass = 0; pass < 2; ++pass)
          for (int q = head; q < j; ++q) {
            if (s.vinfo[q] != b) continue;
            const double* yq = Y + (size_t)q * n + lo;
            double dot = 0.0;
            for (int i = 0; i < m; ++i) dot += yq[i] * x[i];
            for (int i = 0; i < m; ++i) x[i] -= dot * yq[i];
          }
        double nrm = 0.0;
        for (int i = 0; i < m; ++i) nrm += x[i] * x[i];
        nrm = 1.0 / sqrt(nrm);
        for (int i = 0; i < m; ++i) x[i] *= nrm;
      }
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------------- 4. back-transform
// Y[j] <- H(0) H(1) ... H(n-3) Y[j] for j < kvec, two vectors per warp held in registers.
__device__ void back_transform(int n, int kvec, const double* A, double* Y, const EigenScratch& s) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j0 = 2 * warp; j0 < kvec; j0 += 2 * kWarps) {
    const bool two = j0 + 1 < kvec;
    double* y0 = Y + (size_t)j0 * n;
    double* y1 = Y + (size_t)(two ? j0 + 1 : j0) * n;
    double z0[kRowT], z1[kRowT];
#pragma unroll
    for (int t = 0; t < kRowT; ++t) {
      const int r = lane + 32 * t;
      z0[t] = r < n ? y0[r] : 0.0;
      z1[t] = r < n ? y1[r] : 0.0;
    }
    for (int i = n - 3; i >= 0; --i) {
      const double tau = s.tau[i];
      if (tau == 0.0) continue;
      double a0 = 0.0, a1 = 0.0;
#pragma unroll
      for (int t = 0; t < kRowT; ++t) {
        const int r = lane + 32 * t;
        if (r > i && r < n) {
          const double vr = r == i + 1 ? 1.0 : A[tri(r) + i];
          a0 = fma(vr, z0[t], a0);
          a1 = fma(vr, z1[t], a1);
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
      }
      a0 *= tau;
      a1 *= tau;
#pragma unroll
      for (int t = 0; t < kRowT; ++t) {
        const int r = lane + 32 * t;
        if (r > i && r < n) {
          const double vr = r == i + 1 ? 1.0 : A[tri(r) + i];
          z0[t] -= a0 * vr;
          z1[t] -= a1 * vr;
        }
      }
    }
#pragma unroll
    for (int t = 0; t < kRowT; ++t) {
      const int r = lane + 32 * t;
      if (r < n) {
        y0[r] = z0[t];
        if (two) y1[r] = z1[t];
      }
    }
  }
  __syncthreads();
}

// All eigenvalues of the saved tridiagonal (d, e) -- used once at the end for the MO energies.
__device__ void all_eigenvalues(int n, const double* d, const double* e, double* out, const EigenScratch& s) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < n; ++i) {
      s.d[i] = d[i];
      s.e[i] = e[i];
    }
  }
  __syncthreads();
  tridiag_eigenvalues(n, n, s);
  for (int j = threadIdx.x; j < n; j += kThreads) out[j] = s.lam[j];
  __syncthreads();
}

}  // namespace pm3gpu
