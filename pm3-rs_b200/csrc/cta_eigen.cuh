// Symmetric eigensolver for one matrix per CTA (n <= kMaxN), replacing the reference's faer
// `self_adjoint_eigen` (pm3-rs src/linalg.rs:221-263) on the SCF path:
//   1. Householder reduction to tridiagonal form, the matrix held as a packed lower triangle
//      (row-major: element (r, c), r >= c, at r(r+1)/2 + c) in shared memory (or global memory
//      when it does not fit), a power-of-two group of threads per remaining row. Reflectors stay
//      in the strictly-lower part of column i.
//   2. Eigenvalues of the tridiagonal T by Sturm-count multisection, a group of lanes per
//      eigenvalue, started from the previous SCF iteration's eigenvalues when given.
//   3. Eigenvectors of T by twisted (N_r D_r N_r^T) factorisation, one thread per vector,
//      on the unreduced block holding the eigenvalue (T is split where |e_i| <= 1000 eps ||T||,
//      which separates exact degeneracies); members of a within-block cluster (gap below
//      1e-7 ||T||) after the first are redone by inverse iteration with re-orthogonalisation.
//   4. Back-transformation Z = Q Y, one warp per 2, 4 or 8 vectors held in registers (fewer rows
//      per lane for smaller bases, more vectors).
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
// Sum over the CTA with one barrier: `red` holds two alternating kWarps buffers, so a call may
// overwrite the buffer two calls back without waiting (the previous call's barrier separates them).
__device__ __forceinline__ double block_sum_alt(double v, double* red, int& parity) {
  v = warp_sum(v);
  double* buf = red + parity * kWarps;
  parity ^= 1;
  if ((threadIdx.x & 31) == 0) buf[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int i = 0; i < kWarps; ++i) t += buf[i];
  return t;
}

// Householder reduction (n <= kThreads). For column i, the m = n - i - 1 trailing rows get T
// threads each (T the largest power of two with T m <= kThreads, at most a warp), so that late
// columns, with few rows left, still keep the CTA busy. The T threads of row r split the
// matrix-vector product (its row segment c <= r, then the column below it) and the rank-2
// update of its row segment by interleaved columns, and combine the product by shuffles; the
// first of them contributes its element of the next column to the next reflector's norm.
// Three barriers per column. This sweep reduces columns [0, i_stop) of the n x n matrix and, with
// `close`, writes the last diagonal and off-diagonal entries; d, e, tau are indexed from the
// matrix's first row.
__device__ __forceinline__ void householder_columns(int n, double* __restrict__ A, double* v, double* p, double* red, double* tau_out,
                                    double* e_out, double* d_out, int i_stop, bool close) {
  // scratch pointers in registers: the stores below go through generic pointers, which
  // would otherwise force them to be re-read after every store
  struct {
    double *v, *p, *red, *tau, *e, *d;
  } s = {v, p, red, tau_out, e_out, d_out};
  const int t = threadIdx.x;
  int parity = 0;
  double xn2 = block_sum_alt(t >= 2 && t < n ? A[tri(t)] * A[tri(t)] : 0.0, s.red, parity);
  for (int i = 0; i < i_stop; ++i) {
    const double alpha = A[tri(i + 1) + i];
    double beta = alpha, tau = 0.0, scal = 0.0;
    if (xn2 > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
      tau = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    if (t == 0) {
      s.tau[i] = tau;
      s.e[i] = beta;
      s.d[i] = A[tri(i) + i];
    }
    if (xn2 == 0.0) {  // column already reduced (uniform): only the next norm is needed
      xn2 = block_sum_alt(t >= i + 3 && t < n ? A[tri(t) + i + 1] * A[tri(t) + i + 1] : 0.0, s.red, parity);
      continue;
    }
    if (t > i && t < n) {  // reflector: one thread per row
      double vr = 1.0;
      if (t > i + 1) {
        vr = A[tri(t) + i] * scal;
        A[tri(t) + i] = vr;
      }
      s.v[t] = vr;
    }
    __syncthreads();
    const int m = n - i - 1;
    const int lg = min(5, 31 - __clz(kThreads / m));
    const int T = 1 << lg, k = t & (T - 1), r = i + 1 + (t >> lg);
    const bool mine = r < n;
    const int tr = mine ? tri(r) : 0;
    // y_r = sum_{c > i} A(r, c) v_c; four independent accumulators per thread
    double y = 0.0;
    if (mine) {
      double y0 = 0.0, y1 = 0.0, y2 = 0.0, y3 = 0.0;
      const double* row = A + tr;
      int c = i + 1 + k;
      for (; c + 3 * T <= r; c += 4 * T) {
        y0 = fma(row[c], s.v[c], y0);
        y1 = fma(row[c + T], s.v[c + T], y1);
        y2 = fma(row[c + 2 * T], s.v[c + 2 * T], y2);
        y3 = fma(row[c + 3 * T], s.v[c + 3 * T], y3);
      }
      for (; c <= r; c += T) y0 = fma(row[c], s.v[c], y0);
      for (; c + 3 * T < n; c += 4 * T) {
        y0 = fma(A[tri(c) + r], s.v[c], y0);
        y1 = fma(A[tri(c + T) + r], s.v[c + T], y1);
        y2 = fma(A[tri(c + 2 * T) + r], s.v[c + 2 * T], y2);
        y3 = fma(A[tri(c + 3 * T) + r], s.v[c + 3 * T], y3);
      }
      for (; c < n; c += T) y1 = fma(A[tri(c) + r], s.v[c], y1);
      y = (y0 + y1) + (y2 + y3);
    }
    for (int o = T >> 1; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
    y *= tau;
    const double vr = mine ? s.v[r] : 0.0;
    if (mine && k == 0) s.p[r] = y;
    const double a2 = -0.5 * tau * block_sum_alt(mine && k == 0 ? y * vr : 0.0, s.red, parity);
    // A22 -= v w^T + w v^T (w = p + a2 v) on the row segments, keeping the next column's norm part
    double part = 0.0;
    if (mine) {
      const double wr = y + a2 * vr;
      double* row = A + tr;
      int c = i + 1 + k;
      for (; c + 3 * T <= r; c += 4 * T) {
        const double v0 = s.v[c], v1 = s.v[c + T], v2 = s.v[c + 2 * T], v3 = s.v[c + 3 * T];
        const double w0 = s.p[c] + a2 * v0, w1 = s.p[c + T] + a2 * v1, w2 = s.p[c + 2 * T] + a2 * v2,
                     w3 = s.p[c + 3 * T] + a2 * v3;
        const double a0 = row[c], a1 = row[c + T], a2_ = row[c + 2 * T], a3 = row[c + 3 * T];
        row[c] = a0 - (vr * w0 + wr * v0);
        row[c + T] = a1 - (vr * w1 + wr * v1);
        row[c + 2 * T] = a2_ - (vr * w2 + wr * v2);
        row[c + 3 * T] = a3 - (vr * w3 + wr * v3);
      }
      for (; c <= r; c += T) {
        const double vc = s.v[c], wc = s.p[c] + a2 * vc;
        row[c] -= vr * wc + wr * vc;
      }
      if (k == 0 && r >= i + 3) {
        const double x = row[i + 1];
        part = x * x;
      }
    }
    xn2 = block_sum_alt(part, s.red, parity);
  }
  if (close && t == 0) {
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

// Householder reduction of the packed n x n matrix A (shared or global memory).
__device__ void tridiagonalize(int n, double* __restrict__ A, const EigenScratch& s) {
  householder_columns(n, A, s.v, s.p, s.red, s.tau, s.e, s.d, n - 2, true);
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

// Sturm counts at M shifts at once, without divisions (see the ratio form above for the
// reference recurrence): p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2}; sign changes between
// consecutive values count the eigenvalues below x. Pairs are rescaled by powers of two every
// 8 steps (each step grows |p| by far less than 2^32 for the matrices here), exact for ratios.
template <int M>
__device__ __forceinline__ void sturm_multi(const double* __restrict__ d, const double* __restrict__ e2, int n,
                                            const double (&x)[M], double pivmin, int (&cnt)[M]) {
  (void)pivmin;
  constexpr double kBig = 0x1p256, kSmall = 0x1p-256;
  double p[M], pm[M];
  unsigned sg[M];
#pragma unroll
  for (int t = 0; t < M; ++t) {
    pm[t] = 1.0;
    p[t] = d[0] - x[t];
    sg[t] = __double_as_longlong(p[t]) < 0 ? 1u : 0u;
    cnt[t] = (int)sg[t];
  }
  int i = 1;
  for (; i + 8 <= n; i += 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const double di = d[i + u], ei = e2[i + u - 1];
#pragma unroll
      for (int t = 0; t < M; ++t) {
        const double pn = fma(di - x[t], p[t], -ei * pm[t]);
        const unsigned s = __double_as_longlong(pn) < 0 ? 1u : 0u;
        cnt[t] += (int)(s ^ sg[t]);
        sg[t] = s;
        pm[t] = p[t];
        p[t] = pn;
      }
    }
#pragma unroll
    for (int t = 0; t < M; ++t) {
      const double m = fmax(fabs(p[t]), fabs(pm[t]));
      const double sc = m > kBig ? kSmall : (m < kSmall ? kBig : 1.0);
      p[t] *= sc;
      pm[t] *= sc;
    }
  }
  for (; i < n; ++i) {
    const double di = d[i], ei = e2[i - 1];
#pragma unroll
    for (int t = 0; t < M; ++t) {
      const double pn = fma(di - x[t], p[t], -ei * pm[t]);
      const unsigned s = __double_as_longlong(pn) < 0 ? 1u : 0u;
      cnt[t] += (int)(s ^ sg[t]);
      sg[t] = s;
      pm[t] = p[t];
      p[t] = pn;
    }
  }
}

// Splits T where the coupling is negligible and computes the lowest `kval` eigenvalues.
// Leaves pivmin / tnorm in misc[0] / misc[1]. With `prev` (the same eigenvalues of the
// previous SCF iteration) and `dprev` (their last change) the search starts from a bracket
// around prev[j] once Sturm counts confirm it.
__device__ void tridiag_eigenvalues(int n, int kval, const EigenScratch& s_, const double* prev = nullptr,
                                    const double* dprev = nullptr) {
  struct {
    double *d, *e, *e2, *misc, *lam;
    int *blk, *nblk;
  } s = {s_.d, s_.e, s_.e2, s_.misc, s_.lam, s_.blk, s_.nblk};
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
  const double pivmin = s.misc[0], tnorm = s.misc[1], glo = s.misc[2], ghi = s.misc[3];
  // Multisection: a group of g lanes (a power of two, g <= 32, kval * g <= kThreads) brackets
  // one eigenvalue; each step the group takes Sturm counts at P = g * kPts interior points (kPts
  // per lane, evaluated together), which cuts the bracket by P + 1 instead of 2.
  // Invariant: count(lo) <= j < count(hi).
  constexpr int kPts = 2;
  int g = 1;
  while (g < 32 && kval * (2 * g) <= kThreads) g *= 2;
  const int P = g * kPts;
  const int lane = tid & 31;
  const int gbase = lane & ~(g - 1), gl = lane & (g - 1);
  const unsigned gbits = g == 32 ? 0xffffffffu : ((1u << g) - 1u);
  for (int j0 = 0; j0 < kval; j0 += kThreads / g) {
    const int j = j0 + tid / g;
    const bool active = j < kval;
    double lo = glo, hi = ghi;
    if (prev) {
      // warm bracket around the previous SCF iteration's value, widened until two Sturm
      // counts confirm that it holds eigenvalue j (else the Gershgorin interval stays)
      const double c0 = active ? prev[j] : 0.0;
      const double w0 = active ? fmax(4.0 * fabs(dprev[j]), 1.0e-9 * fmax(tnorm, 1.0)) : 0.0;
      double x[4];
      int cn[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {  // brackets w0 and 64 w0: lower ends on even t, upper on odd
        const double w = w0 * (t >= 2 ? 64.0 : 1.0);
        x[t] = (t & 1) ? fmin(c0 + w, ghi) : fmax(c0 - w, glo);
      }
      if (active) sturm_multi<4>(s.d, s.e2, n, x, pivmin, cn);
      if (active) {
        if (x[0] < x[1] && cn[0] <= j && cn[1] >= j + 1) {
          lo = x[0];
          hi = x[1];
        } else if (x[2] < x[3] && cn[2] <= j && cn[3] >= j + 1) {
          lo = x[2];
          hi = x[3];
        }
      }
    }
    bool act = active;
    for (int it = 0; it < 128; ++it) {
      if (act) {
        const double mid = 0.5 * (lo + hi);
        if (hi - lo <= 2.0 * eps * fmax(fabs(lo), fabs(hi)) + 4.0 * pivmin || !(mid > lo && mid < hi)) act = false;
      }
      if (!__any_sync(0xffffffffu, act)) break;
      double x[kPts];
      int cn[kPts];
#pragma unroll
      for (int t = 0; t < kPts; ++t) x[t] = lo + (hi - lo) * (double)(gl * kPts + t + 1) / (double)(P + 1);
      if (act) sturm_multi<kPts>(s.d, s.e2, n, x, pivmin, cn);
      int tf = kPts;  // this lane's first point above eigenvalue j
#pragma unroll
      for (int t = kPts - 1; t >= 0; --t)
        if (act && cn[t] > j) tf = t;
      const unsigned bal = __ballot_sync(0xffffffffu, act && tf < kPts);
      const unsigned mine = (bal >> gbase) & gbits;
      const int src = mine ? gbase + __ffs(mine) - 1 : gbase;
      const int tsrc = __shfl_sync(0xffffffffu, tf, src);
      if (act) {
        double nlo, nhi;
        if (mine == 0u) {  // every point is at or below eigenvalue j
          nlo = lo + (hi - lo) * (double)P / (double)(P + 1);
          nhi = hi;
        } else {
          const int f = (src - gbase) * kPts + tsrc;  // first point above it
          nlo = f > 0 ? lo + (hi - lo) * (double)f / (double)(P + 1) : lo;
          nhi = lo + (hi - lo) * (double)(f + 1) / (double)(P + 1);
        }
        if (!(nhi - nlo < hi - lo)) act = false;
        else {
          lo = nlo;
          hi = nhi;
        }
      }
    }
    if (active && gl == 0) s.lam[j] = 0.5 * (lo + hi);
  }
  __syncthreads();
}

// ------------------------------------------------------------- 3. tridiagonal eigenvectors
// Eigenvector j (< kvec) of T into Y[j*n .. j*n+n) (zero outside its block). `tf` is per-CTA
// global scratch of kvec * 6n doubles.
__device__ void tridiag_vectors(int n, int kvec, double* Y, double* tf, const EigenScratch& s_) {
  struct {
    const double *d, *e, *e2, *lam, *misc;
    const int *blk, *nblk;
    int* vinfo;
  } s = {s_.d, s_.e, s_.e2, s_.lam, s_.misc, s_.blk, s_.nblk, s_.vinfo};
  const int tid = threadIdx.x;
  const double pivmin = s.misc[0], tnorm = s.misc[1];
  const int nb = *s.nblk;
  const double win = 1.0e-11 * fmax(tnorm, 1.0);
  // Two halves of the CTA work on the same vectors: warps 0-3 (half 0) form the top-down
  // factorisation L+ D+ L+^T of T - lam, warps 4-7 (half 1) the bottom-up U- D- U-^T; both are
  // chains of divisions, so running them side by side halves the latency per vector. Then half 0
  // picks the twist index, and the halves fill the vector above and below it. Per-vector scratch
  // in tf (6 n): D+, L+, U-, D- (the pivots after clamping), then [twist, block], [norm parts].
  constexpr int kHalf = kThreads / 2;
  const int half = tid / kHalf, hj = tid % kHalf;
  for (int j = hj; j < kvec; j += kHalf) {
    const double lam = s.lam[j];
    // which unreduced block holds this eigenvalue (degenerate copies go to successive blocks);
    // an unsplit T (the usual case) has one block, and the three Sturm counts are not needed
    int pos = nb == 1 ? 0 : j - sturm(s.d, s.e2, 0, n - 1, lam - win, pivmin);
    int b = nb == 1 ? 0 : -1;
    for (int q = 0; q < nb && b < 0; ++q) {
      const int lo = s.blk[q], hi = s.blk[q + 1] - 1;
      const int c = sturm(s.d, s.e2, lo, hi, lam + win, pivmin) - sturm(s.d, s.e2, lo, hi, lam - win, pivmin);
      if (pos < c) b = q;
      else pos -= c;
    }
    if (b < 0) b = 0;  // inconsistent counts (not expected): block 0
    if (half == 0) s.vinfo[j] = b;
    const int lo = s.blk[b], hi = s.blk[b + 1] - 1, m = hi - lo + 1;
    double* y = Y + (size_t)j * n;
    for (int i = half; i < n; i += 2) y[i] = 0.0;
    if (m == 1) continue;
    double* Dp = tf + (size_t)j * 6 * n;
    double* Lp = Dp + n;
    double* Um = Lp + n;
    double* Dm = Um + n;
    if (half == 0) {  // T - lam = L+ D+ L+^T (top-down)
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
    } else {  // T - lam = U- D- U-^T (bottom-up)
      double dm = s.d[hi] - lam;
      if (fabs(dm) < pivmin) dm = dm < 0.0 ? -pivmin : pivmin;
      Dm[m - 1] = dm;
      for (int i = m - 2; i >= 0; --i) {
        const double ei = s.e[lo + i];
        Um[i] = ei / dm;
        dm = (s.d[lo + i] - lam) - Um[i] * ei;
        if (fabs(dm) < pivmin) dm = dm < 0.0 ? -pivmin : pivmin;
        Dm[i] = dm;
      }
    }
  }
  __syncthreads();
  // twist index r minimising |gamma_i| = |D+_i + D-_i - (d_i - lam)| (the largest index among ties,
  // as a downward scan with a strict comparison finds it)
  if (half == 0)
    for (int j = hj; j < kvec; j += kHalf) {
      const double lam = s.lam[j];
      const int b = s.vinfo[j], lo = s.blk[b], hi = s.blk[b + 1] - 1, m = hi - lo + 1;
      if (m == 1) continue;
      double* Dp = tf + (size_t)j * 6 * n;
      const double* Dm = Dp + 3 * n;
      double best = fabs(Dp[m - 1] + Dm[m - 1] - (s.d[hi] - lam));
      int r = m - 1;
      for (int i = m - 2; i >= 0; --i) {
        const double g = fabs(Dp[i] + Dm[i] - (s.d[lo + i] - lam));
        if (g < best) {
          best = g;
          r = i;
        }
      }
      reinterpret_cast<int*>(Dp + 4 * n)[0] = r;
    }
  __syncthreads();
  // solve N_r D_r N_r^T y = gamma_r e_r: half 0 the rows above r, half 1 from r down; partial norms
  for (int j = hj; j < kvec; j += kHalf) {
    const int b = s.vinfo[j], lo = s.blk[b], hi = s.blk[b + 1] - 1, m = hi - lo + 1;
    double* y = Y + (size_t)j * n;
    double* Dp = tf + (size_t)j * 6 * n;
    if (m == 1) {
      if (half == 0) y[lo] = 1.0;
      continue;
    }
    const double* Lp = Dp + n;
    const double* Um = Lp + n;
    const int r = reinterpret_cast<const int*>(Dp + 4 * n)[0];
    double nrm = 0.0;
    if (half == 0) {
      double yn = 1.0, ynn = 0.0;  // y[lo + i + 1], y[lo + i + 2]
      for (int i = r - 1; i >= 0; --i) {
        double z = -Lp[i] * yn;
        if (yn == 0.0 && i + 2 < m) z = -(s.e[lo + i + 1] / s.e[lo + i]) * ynn;
        y[lo + i] = z;
        nrm = fma(z, z, nrm);
        ynn = yn;
        yn = z;
      }
    } else {
      y[lo + r] = 1.0;
      nrm = 1.0;
      double yc = 1.0, yp = 0.0;  // y[lo + i], y[lo + i - 1] (the latter read only after a zero)
      for (int i = r; i < m - 1; ++i) {
        double z = -Um[i] * yc;
        if (yc == 0.0 && i >= 1) z = -(s.e[lo + i - 1] / s.e[lo + i]) * yp;
        y[lo + i + 1] = z;
        nrm = fma(z, z, nrm);
        yp = yc;
        yc = z;
      }
    }
    Dp[5 * n + half] = nrm;
  }
  __syncthreads();
  for (int j = hj; j < kvec; j += kHalf) {
    const int b = s.vinfo[j], lo = s.blk[b], hi = s.blk[b + 1] - 1, m = hi - lo + 1;
    if (m == 1) continue;
    const double* Dp = tf + (size_t)j * 6 * n;
    const int r = reinterpret_cast<const int*>(Dp + 4 * n)[0];
    const double scale = 1.0 / sqrt(Dp[5 * n] + Dp[5 * n + 1]);
    double* y = Y + (size_t)j * n;
    if (half == 0)
      for (int i = lo; i < lo + r; ++i) y[i] *= scale;
    else
      for (int i = lo + r; i <= hi; ++i) y[i] *= scale;
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
// One warp applies the reflectors to NV vectors at a time, RT rows per lane held in registers
// (n <= 32 RT). Per reflector the NV partial dot products are reduced together (their shuffle
// chains overlap), so the latency of a reflector is paid once for NV vectors.
template <int RT, int NV>
__device__ __forceinline__ void back_transform_t(int n, int kvec, const double* __restrict__ A, double* Y,
                                                 const double* __restrict__ tau_) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j0 = NV * warp; j0 < kvec; j0 += NV * kWarps) {
    double z[NV][RT];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double* y = Y + (size_t)(j0 + v < kvec ? j0 + v : j0) * n;
#pragma unroll
      for (int t = 0; t < RT; ++t) {
        const int r = lane + 32 * t;
        z[v][t] = r < n ? y[r] : 0.0;
      }
    }
    for (int i = n - 3; i >= 0; --i) {
      const double tau = tau_[i];
      if (tau == 0.0) continue;
      double vr[RT];
#pragma unroll
      for (int t = 0; t < RT; ++t) {
        const int r = lane + 32 * t;
        vr[t] = (r > i && r < n) ? (r == i + 1 ? 1.0 : A[tri(r) + i]) : 0.0;
      }
      double a[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        double acc = 0.0;
#pragma unroll
        for (int t = 0; t < RT; ++t) acc = fma(vr[t], z[v][t], acc);
        a[v] = acc;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int v = 0; v < NV; ++v) a[v] += __shfl_xor_sync(0xffffffffu, a[v], o);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double s = a[v] * tau;
#pragma unroll
        for (int t = 0; t < RT; ++t) z[v][t] = fma(-s, vr[t], z[v][t]);
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      if (j0 + v >= kvec) break;
      double* y = Y + (size_t)(j0 + v) * n;
#pragma unroll
      for (int t = 0; t < RT; ++t) {
        const int r = lane + 32 * t;
        if (r < n) y[r] = z[v][t];
      }
    }
  }
  __syncthreads();
}

// The reflectors of column i (v_{i+1} = 1, v_r = A(r, i) below) applied from the last to the
// first. Up to n = 64 each lane holds 2 rows and a warp 4 vectors (the n/2 or so occupied vectors
// then keep all eight warps busy, which measured faster than 8 vectors on four warps).
__device__ void back_transform(int n, int kvec, const double* __restrict__ A, double* Y, const EigenScratch& s_) {
  if (n <= 64) back_transform_t<2, 4>(n, kvec, A, Y, s_.tau);
  else if (n <= 128) back_transform_t<4, 4>(n, kvec, A, Y, s_.tau);
  else back_transform_t<kRowT, 2>(n, kvec, A, Y, s_.tau);
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
