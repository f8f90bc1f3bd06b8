// One Householder panel of the blocked lower reduction (the LAPACK sytrd/latrd scheme, the role
// of faer's self_adjoint_eigen tridiagonalisation behind src/linalg.rs:221-263) in a single
// cooperative launch: the kPanel columns of the panel run back to back inside one persistent
// grid with three grid-wide barriers per column, instead of five dependent launches per column.
//
// Ownership. The matrix is cut into absolute 64-row stripes; block c owns stripe c (rows
// 64c .. 64c+63) for the whole panel, its warp w rows 64c + w + 8t (t < 8), and keeps their
// rows of V and W in registers (lane k holding component k). The panel's V and W live in two
// n x 64 row-major buffers X = [V | W] and Y = [W | V], so the trailing update
// A22 -= V W^T + W V^T is the single GEMM X Y^T with inner dimension 64.
//
// Per column i = p + j (trailing block starts at s = i + 1), two grid-wide barriers:
//   A  rows r >= i of the owned stripes: a_r = A[i][r] - sum_{k<j} (V[r][k] W[i][k] + W[r][k] V[i][k]),
//      written back into row i; block partials of |a|^2 (r >= i+2) and of sum_r W[r][k] a_r,
//      sum_r V[r][k] a_r.                                                            barrier 1
//   B  every block forms the reflector (beta, tau, 1/(alpha-beta)) from the norm partials; the
//      grid runs the lower-triangle GEMV y = A22 v over the absolute 64 x 64 tiles (I >= J)
//      that meet the trailing block, row sums and column sums into per-tile slots, and the
//      block partials of v^T A22 v; blocks 0..63 finish s1 = W^T v and s2 = V^T v.    barrier 2
//   C  w . v = tau (v^T A22 v - 2 s1 . s2) (the same scalar as sum_r w_r v_r, without a third
//      reduction); each stripe owner adds up its rows of y from the slots (coalesced, in shared
//      memory), then w_r = tau (y_r - V[r] s1 - W[r] s2) and W[r][j] = w_r - (tau/2)(w . v) v_r;
//      v and W[:, j] into X / Y, v into row i (the stored reflector). The next column's step A
//      needs W[s][j], which another block owns: every block recomputes it from row s of y.
// Data written by another block inside the launch is read with ld.global.cg (L2), never through
// L1. The trailing block A22 itself is not written during the panel (only rows < s are), so its
// GEMV tiles are plain copies. Every sum runs in a fixed order: results do not depend on timing.
#pragma once
#include "large_scf.cuh"

namespace pm3gpu {
namespace large {

constexpr int kCoopRows = 8;         // rows per warp: a block owns one 64-row stripe
constexpr int kCoopLd = 2 * kPanel;  // row length of the X = [V | W] and Y = [W | V] buffers

struct GridSync {
  unsigned int count;
  unsigned int gen;
  int err;  // set when a barrier wait ran out; every block then leaves at its next barrier
  int pad;
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier of a cooperative launch (all blocks are resident): thread 0 of each block
// arrives with a release add, the last one to arrive publishes the next generation with a
// release store, the others poll it with acquire loads. Bounded: after ~2^24 polls the wait
// raises gs->err instead of spinning on.
__device__ __forceinline__ bool grid_sync(GridSync* gs, unsigned int& gen) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int g = gen;
    unsigned int arrived;
    asm volatile("atom.add.release.gpu.u32 %0, [%1], 1;" : "=r"(arrived) : "l"(&gs->count) : "memory");
    if (arrived == gridDim.x - 1) {
      gs->count = 0u;
      asm volatile("st.release.gpu.u32 [%0], %1;" ::"l"(&gs->gen), "r"(g + 1u) : "memory");
    } else {
      for (unsigned int spin = 0;; ++spin) {
        if (ld_acquire_u32(&gs->gen) != g) break;
        if (*(volatile int*)&gs->err != 0) break;
        if (spin > (1u << 24)) {
          atomicExch(&gs->err, 1);
          break;
        }
        if (spin > 64) __nanosleep(20);
      }
    }
    s_ok = *(volatile int*)&gs->err == 0;
  }
  __syncthreads();
  ++gen;
  return s_ok != 0;
}

// Sums over the warp of eight per-lane values at once (transpose-reduce: 9 shuffles instead of
// 40). Lane L ends with the total of value L >> 2, added in a fixed order.
__device__ __forceinline__ double warp_sum8(const double (&x)[8], int lane) {
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  double r1[4], r2[2];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double send = b4 ? x[k] : x[k + 4];
    r1[k] = (b4 ? x[k + 4] : x[k]) + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const double send = b3 ? r1[k] : r1[k + 2];
    r2[k] = (b3 ? r1[k + 2] : r1[k]) + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  double r = (b2 ? r2[1] : r2[0]) + __shfl_xor_sync(0xffffffffu, b2 ? r2[0] : r2[1], 4);
  r += __shfl_xor_sync(0xffffffffu, r, 2);
  r += __shfl_xor_sync(0xffffffffu, r, 1);
  return r;
}

constexpr int kStages = 3;  // tiles of the GEMV pipeline per block (3 x 32 KB of shared memory)
constexpr size_t kCoopSmem = (size_t)kStages * kTile * kTile * sizeof(double);

// 16-byte asynchronous global -> shared copy through L2 only; ok = false writes zeros.
__device__ __forceinline__ void cp_async16(double* smem, const double* gmem, bool ok) {
  const unsigned int sa = (unsigned int)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(gmem), "r"(ok ? 16 : 0) : "memory");
}
// 8-byte asynchronous global -> shared copy; ok = false writes zeros (nothing is read).
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool ok) {
  const unsigned int sa = (unsigned int)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(sa), "l"(gmem), "r"(ok ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Fixed-order sum of x[0], x[stride], ... (cnt terms) by one warp; every lane gets lane 0's value.
// Loads go out in batches of 8 per lane before any add, so a grid's worth of block partials
// costs about one L2 round trip rather than one per term.
__device__ __forceinline__ double warp_sum_cg(const double* x, int cnt, int lane, int stride = 1) {
  double s = 0.0;
  for (int b0 = 0; b0 < cnt; b0 += 32 * 8) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int b = b0 + lane + 32 * u;
      v[u] = b < cnt ? __ldcg(x + (size_t)b * stride) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) s += v[u];
  }
  s = warp_sum(s);
  return __shfl_sync(0xffffffffu, s, 0);
}

// kEven: n is even, so every 16-byte pair of a row starts 16-byte aligned (row starts are)
template <bool kEven>
__global__ void __launch_bounds__(kBlock, 2)
    panel_coop_kernel(double* A, int n, int p, int b, double* X, double* Y, double* d, double* e, double* tau,
                      double* tp, double* part_n, double* part_s, double* s_tot, double* part_q, GridSync* gs) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int G = gridDim.x, c = blockIdx.x;
  const int nts = (n + kTile - 1) / kTile;  // absolute stripes
  const int row0 = c * kTile + warp;        // this warp's rows: row0 + 8t
  const bool owner = c < nts;
  __shared__ double sred[kBlock / 32][64];
  __shared__ double cs2[2][kBlock / 32][kTile];  // GEMV column partials, double-buffered
  double(*cs)[kTile] = cs2[0];                    // small block reductions outside the GEMV
  __shared__ double y_s[kTile];
  __shared__ double s_scal[4];  // 1/(alpha - beta), tau, -(tau/2)(w . v), W[s][j] of the column
  __shared__ double s_a[kBlock / 32][kCoopRows];  // a_r of the owned rows
  __shared__ unsigned int s_gen;
  extern __shared__ __align__(16) double tiles[];  // kStages x 64 x 64 GEMV tiles
  if (threadIdx.x == 0) {
    s_gen = ld_acquire_u32(&gs->gen);
    s_scal[3] = 0.0;
  }
  __syncthreads();
  unsigned int gen = s_gen;
  double vreg[kCoopRows], wreg[kCoopRows];
#pragma unroll
  for (int t = 0; t < kCoopRows; ++t) vreg[t] = wreg[t] = 0.0;
  double prev_tt = 0.0;  // tau of the previous column
  for (int j = 0; j < b; ++j) {
    const int i = p + j, s = i + 1;
    double* rowi = A + (size_t)i * n;
    // GEMV tiles of this column (step B): which tiles does not depend on the reflector, and A22 is
    // not written during the panel, so the first two copies go out before barrier 1.
    const int I0 = s / kTile;  // first stripe that meets the trailing block
    const int ntr = nts - I0;
    const long long ntiles = (long long)ntr * (ntr + 1) / 2;
    const long long t0 = ntiles * c / G, t1 = ntiles * (c + 1) / G;
    const int my = (int)(t1 - t0);
    int Ii = 0, Ji = 0;  // tile coordinates (relative to I0) of the next copy
    {
      int Ir = (int)((sqrt(8.0 * (double)t0 + 1.0) - 1.0) * 0.5);
      while ((long long)(Ir + 1) * (Ir + 2) / 2 <= t0) ++Ir;
      while ((long long)Ir * (Ir + 1) / 2 > t0) --Ir;
      Ii = Ir;
      Ji = (int)(t0 - (long long)Ir * (Ir + 1) / 2);
    }
    int Iv = Ii, Jv = Ji, Ic = Ii, Jc = Ji;  // next v fetch, next reduction
    auto step = [](int& I, int& J) {
      if (++J > I) {
        ++I;
        J = 0;
      }
    };
    auto issue = [&](int k) {
      if (k < my) {
        double* T = tiles + (size_t)(k % kStages) * kTile * kTile;
        const int rb = (I0 + Ii) * kTile, cb = (I0 + Ji) * kTile;
        if (kEven) {
#pragma unroll
          for (int q = 0; q < kTile * kTile / 2 / kBlock; ++q) {
            const int el = threadIdx.x + kBlock * q, r = rb + (el >> 5), col = cb + 2 * (el & 31);
            const bool ok = r < n && col < n;
            cp_async16(T + 2 * el, ok ? A + (size_t)r * n + col : A, ok);
          }
        } else {
#pragma unroll
          for (int q = 0; q < kTile * kTile / kBlock; ++q) {
            const int el = threadIdx.x + kBlock * q, r = rb + (el >> 6), col = cb + (el & 63);
            const bool ok = r < n && col < n;
            cp_async8(T + el, ok ? A + (size_t)r * n + col : A, ok);
          }
        }
        step(Ii, Ji);
      }
      cp_async_commit();  // one group per step, empty past the end: the wait counts stay fixed
    };
    // ---------------------------------------------------------------- A: update row i
    {
      // Row i of V and W: entries j-1 were written by their owner in the previous step C with no
      // barrier since, so they come from this block's own copies (V[i][j-1] = 1 with a reflection)
      double Vi = lane + 1 < j ? __ldcg(X + (size_t)i * kCoopLd + lane) : 0.0;
      double Wi = lane + 1 < j ? __ldcg(X + (size_t)i * kCoopLd + kPanel + lane) : 0.0;
      if (j > 0 && lane == j - 1) {
        Vi = prev_tt != 0.0 ? 1.0 : 0.0;
        Wi = s_scal[3];
      }
      double prod[kCoopRows];
#pragma unroll
      for (int t = 0; t < kCoopRows; ++t) prod[t] = vreg[t] * Wi + wreg[t] * Vi;
      const double sum = warp_sum8(prod, lane);  // lane 4t: row t
      double a = 0.0;
      {
        const int t = lane >> 2, r = row0 + 8 * t;
        if ((lane & 3) == 0 && owner && r >= i && r < n) {
          a = rowi[r] - sum;
          rowi[r] = a;
          s_a[warp][t] = a;
        }
      }
      double normp = 0.0, s1p = 0.0, s2p = 0.0;
#pragma unroll
      for (int t = 0; t < kCoopRows; ++t) {
        const double at = __shfl_sync(0xffffffffu, a, 4 * t);
        const int r = row0 + 8 * t;
        if (owner && r >= i + 2 && r < n) {
          normp = fma(at, at, normp);
          s1p = fma(wreg[t], at, s1p);
          s2p = fma(vreg[t], at, s2p);
        }
      }
      sred[warp][lane] = s1p;
      sred[warp][32 + lane] = s2p;
      if (lane == 0) cs[warp][0] = normp;
      __syncthreads();
      if (threadIdx.x < 64) {
        double u = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) u += sred[w][threadIdx.x];
        part_s[(size_t)c * 64 + threadIdx.x] = u;
      }
      if (threadIdx.x == 64) {
        double u = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) u += cs[w][0];
        part_n[c] = u;
      }
    }
    issue(0);
    issue(1);
    if (!grid_sync(gs, gen)) return;
    // ---------------------------------------------------------------- B: reflector, GEMV, s
    if (warp == 0) {
      const double alpha = lane == 0 ? __ldcg(rowi + s) : 0.0;
      const double xn2 = warp_sum_cg(part_n, G, lane);
      if (lane == 0) {
        double beta = alpha, tt = 0.0, sc = 0.0;
        if (xn2 > 0.0) {
          beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
          tt = (beta - alpha) / beta;
          sc = 1.0 / (alpha - beta);
        }
        s_scal[0] = sc;
        s_scal[1] = tt;
        if (c == 0) {
          d[i] = __ldcg(rowi + i);
          e[i] = beta;
          tau[i] = tt;
        }
      }
    }
    __syncthreads();
    const double sc = s_scal[0], tt = s_scal[1];
    double quadp = 0.0;  // this thread's share of v^T A22 v
    if (tt != 0.0) {
      // GEMV over a contiguous range of the trailing tiles (row-major order over I >= J >= I0):
      // a 3-stage cp.async pipeline keeps two 64 x 64 tiles in flight while a third is reduced.
      // Tiles are copied whole (only the matrix edge is zero-filled): entries outside the
      // trailing block meet v = 0 and add nothing to the rows and columns that are used.
      auto vval = [&](int col) {  // v over the whole row: 0 before the trailing block and past n
        return (col < s || col >= n) ? 0.0 : (col == s ? 1.0 : __ldcg(rowi + col) * sc);
      };
      double nvc0 = 0.0, nvc1 = 0.0, nvr[kTile / 8], vr[kTile / 8];
      int nvI = -1;
      auto fetch_v = [&]() {
        const int cb = (I0 + Jv) * kTile;
        nvc0 = vval(cb + lane);
        nvc1 = vval(cb + lane + 32);
        if (Iv != nvI) {  // row values change only with the stripe
          nvI = Iv;
#pragma unroll
          for (int q = 0; q < kTile / 8; ++q) nvr[q] = vval((I0 + Iv) * kTile + warp + 8 * q);
        }
        step(Iv, Jv);
      };
      // s1 = W^T v, s2 = V^T v over rows > i, components < j (v_s = 1, v_r = a_r sc beyond):
      // c < 32 is W-based (W at X[., 32 + k]), c >= 32 V-based (V at X[., k]). Done before the
      // GEMV so that these blocks do not arrive last at barrier 2.
      if (c < 64 && warp == 0) {
        const int k = c & 31;
        double tot = 0.0;
        if (k < j) {
          const double acc = warp_sum_cg(part_s + c, G, lane, 64);
          tot = __ldcg(X + (size_t)s * kCoopLd + (c < 32 ? kPanel : 0) + k) + sc * acc;
        }
        if (lane == 0) s_tot[c] = tot;
      }
      if (my > 0) fetch_v();
      for (int k = 0; k < my; ++k) {
        issue(k + 2);
        const double vc0 = nvc0, vc1 = nvc1;
#pragma unroll
        for (int q = 0; q < kTile / 8; ++q) vr[q] = nvr[q];
        if (k + 1 < my) fetch_v();
        const int I = I0 + Ic, J = I0 + Jc;
        step(Ic, Jc);
        cp_async_wait<kStages - 1>();
        __syncthreads();  // tile k visible to all threads; cs2[k & 1] free (read two tiles ago)
        const double* T = tiles + (size_t)(k % kStages) * kTile * kTile;
        double col0 = 0.0, col1 = 0.0, rs[kTile / 8];
#pragma unroll
        for (int q = 0; q < kTile / 8; ++q) {
          const double* tr = T + (warp + 8 * q) * kTile;
          const double a0 = tr[lane], a1 = tr[lane + 32];
          rs[q] = fma(a0, vc0, a1 * vc1);
          col0 = fma(a0, vr[q], col0);
          col1 = fma(a1, vr[q], col1);
        }
        double* slot = tp + ((size_t)I * (I + 1) / 2 + J) * (2 * kTile);
        {
          const double rsum = warp_sum8(rs, lane);
          if ((lane & 3) == 0) {
            double vq = vr[0];
#pragma unroll
            for (int q = 1; q < kTile / 8; ++q)
              if ((lane >> 2) == q) vq = vr[q];
            slot[warp + 8 * (lane >> 2)] = rsum;
            quadp = fma(I == J ? rsum : 2.0 * rsum, vq, quadp);  // off-diagonal tiles stand for two
          }
        }
        double(*csk)[kTile] = cs2[k & 1];
        csk[warp][lane] = col0;
        csk[warp][lane + 32] = col1;
        __syncthreads();  // column partials complete; every warp is done with this stage
        if (I != J && threadIdx.x < kTile) {  // diagonal tiles: only their row sums are used
          double u = 0.0;
          for (int w = 0; w < kBlock / 32; ++w) u += csk[w][threadIdx.x];
          slot[kTile + threadIdx.x] = u;
        }
      }
      cp_async_wait<0>();
    } else {
      cp_async_wait<0>();  // the early copies land before the stages are reused
    }
    {  // block partial of v^T A22 v (every block writes one, zero without a reflection)
      quadp = warp_sum(quadp);
      __syncthreads();  // cs2 reads of the last tile are done
      if (lane == 0) cs[warp][0] = quadp;
      __syncthreads();
      if (threadIdx.x == 0) {
        double u = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) u += cs[w][0];
        part_q[c] = u;
      }
    }
    if (!grid_sync(gs, gen)) return;
    // ---------------------------------------------------------------- C: y, w, v, W
    const bool active = owner && tt != 0.0 && c * kTile + kTile > s;  // block-uniform
    if (active) {  // y over this stripe: the 8 warps split the tile slots, fixed order
      double acc0 = 0.0, acc1 = 0.0;
      for (int J0 = I0 + warp; J0 < nts; J0 += 8 * (kBlock / 32)) {  // 8 slots in flight per warp
        double x0[8], x1[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int J = J0 + u * (kBlock / 32);
          x0[u] = x1[u] = 0.0;
          if (J < nts) {
            const size_t sl = J <= c ? ((size_t)c * (c + 1) / 2 + J) * (2 * kTile)
                                     : ((size_t)J * (J + 1) / 2 + c) * (2 * kTile) + kTile;
            x0[u] = __ldcg(tp + sl + lane);
            x1[u] = __ldcg(tp + sl + lane + 32);
          }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          acc0 += x0[u];
          acc1 += x1[u];
        }
      }
      sred[warp][lane] = acc0;
      sred[warp][lane + 32] = acc1;
    }
    const double s1k = tt != 0.0 ? __ldcg(s_tot + lane) : 0.0, s2k = tt != 0.0 ? __ldcg(s_tot + 32 + lane) : 0.0;
    if (warp == 0) {  // -(tau/2)(w . v), then W[s][j] for the next column (every block, same order)
      double a2 = 0.0, ws = 0.0;
      if (tt != 0.0) {
        const double quad = warp_sum_cg(part_q, G, lane);
        double s12 = warp_sum(s1k * s2k);
        s12 = __shfl_sync(0xffffffffu, s12, 0);
        a2 = -0.5 * tt * (tt * (quad - 2.0 * s12));
        // row s of y: stripe I0, offset o; then w_s and W[s][j] = w_s + a2 (v_s = 1)
        const int o = s - I0 * kTile;
        double ys = 0.0;
        for (int J0 = I0 + lane; J0 < nts; J0 += 32 * 4) {
          double x[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int J = J0 + 32 * u;
            x[u] = J < nts ? __ldcg(tp + (J == I0 ? ((size_t)I0 * (I0 + 1) / 2 + I0) * (2 * kTile) + o
                                                 : ((size_t)J * (J + 1) / 2 + I0) * (2 * kTile) + kTile + o))
                           : 0.0;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) ys += x[u];
        }
        ys = warp_sum(ys);
        const double vs = lane < j ? __ldcg(X + (size_t)s * kCoopLd + lane) : 0.0;
        const double wsk = lane < j ? __ldcg(X + (size_t)s * kCoopLd + kPanel + lane) : 0.0;
        double corr = warp_sum(vs * s1k + wsk * s2k);
        ys = __shfl_sync(0xffffffffu, ys, 0);
        corr = __shfl_sync(0xffffffffu, corr, 0);
        ws = tt * (ys - corr) + a2;
      }
      if (lane == 0) {
        s_scal[2] = a2;
        s_scal[3] = ws;
      }
    }
    __syncthreads();
    if (active && threadIdx.x < kTile) {
      double u = 0.0;
      for (int w = 0; w < kBlock / 32; ++w) u += sred[w][threadIdx.x];
      y_s[threadIdx.x] = u;
    }
    __syncthreads();
    {
      const double a2 = s_scal[2];
      double prod[kCoopRows];
#pragma unroll
      for (int t = 0; t < kCoopRows; ++t) prod[t] = vreg[t] * s1k + wreg[t] * s2k;
      const double corr = warp_sum8(prod, lane);  // lane 4t: row t
      double wn = 0.0, v = 0.0;
      {
        const int t = lane >> 2, r = row0 + 8 * t;
        if ((lane & 3) == 0 && owner && r < n) {
          if (r > i && tt != 0.0) {
            v = r == s ? 1.0 : s_a[warp][t] * sc;
            wn = tt * (y_s[warp + 8 * t] - corr) + a2 * v;
          }
          if (r > s) rowi[r] = v;
          X[(size_t)r * kCoopLd + j] = v;  // zero for r <= i
          X[(size_t)r * kCoopLd + kPanel + j] = wn;
          Y[(size_t)r * kCoopLd + j] = wn;
          Y[(size_t)r * kCoopLd + kPanel + j] = v;
        }
      }
#pragma unroll
      for (int t = 0; t < kCoopRows; ++t) {
        const double vt = __shfl_sync(0xffffffffu, v, 4 * t), wt = __shfl_sync(0xffffffffu, wn, 4 * t);
        if (lane == j) {
          vreg[t] = vt;
          wreg[t] = wt;
        }
      }
    }
    prev_tt = tt;
    __syncthreads();  // s_scal, s_a, sred and cs are rewritten by the next column
  }
}

}  // namespace large
}  // namespace pm3gpu
