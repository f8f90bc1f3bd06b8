// CTA-level building blocks: reductions and a shared-memory tiled FP64 GEMM used by the
// per-molecule SCF (commutator F.P and the density C_occ C_occ^T).
#pragma once
#include <cuda_runtime.h>

namespace pm3gpu {

constexpr int kThreads = 256;  // threads per SCF CTA
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum of `v` over the CTA; every thread gets the result. `red` needs kWarps doubles.
__device__ __forceinline__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int i = 0; i < kWarps; ++i) t += red[i];
  return t;
}
__device__ __forceinline__ double block_max(double v, double* red) {
  v = warp_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = red[0];
#pragma unroll
  for (int i = 1; i < kWarps; ++i) t = fmax(t, red[i]);
  return t;
}
// Several sums at once: v[0..K) per thread -> out[0..K) (in shared memory, visible to all
// threads after return). `red` needs K * kWarps doubles.
template <int K>
__device__ __forceinline__ void block_sums(double (&v)[K], double* red, double* out) {
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
  __syncthreads();
  if (l == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) red[k * kWarps + w] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double t = 0.0;
    for (int i = 0; i < kWarps; ++i) t += red[threadIdx.x * kWarps + i];
    out[threadIdx.x] = t;
  }
  __syncthreads();
}

// This thread's 4 + 4 elements of the 64 x 16 chunks of op(A) and op(B) at k0 (the layout of
// cta_gemm's shared tiles), zero outside the matrices.
template <bool TA, bool TB>
__device__ __forceinline__ void cta_gemm_fetch(double (&pa)[4], double (&pb)[4], int k0, int i0, int j0, int m, int n,
                                               int k, const double* __restrict__ A, int lda,
                                               const double* __restrict__ B, int ldb) {
  constexpr int BM = 64, BN = 64, BK = 16;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = threadIdx.x + q * kThreads;
    int ii, kk;
    if (TA) { ii = e % BM; kk = e / BM; } else { kk = e % BK; ii = e / BK; }
    const int gi = i0 + ii, gk = k0 + kk;
    pa[q] = (gi < m && gk < k) ? (TA ? A[(size_t)gk * lda + gi] : A[(size_t)gi * lda + gk]) : 0.0;
    int jj;
    if (TB) { kk = e % BK; jj = e / BK; } else { jj = e % BN; kk = e / BN; }
    const int gj = j0 + jj, gk2 = k0 + kk;
    pb[q] = (gj < n && gk2 < k) ? (TB ? B[(size_t)gj * ldb + gk2] : B[(size_t)gk2 * ldb + gj]) : 0.0;
  }
}

// C (m x n) = alpha * op(A) * op(B) with op(A) m x k, op(B) k x n; A, B row-major in global
// memory. TA: A stored as k x m (use its transpose). Each output element goes through
// `epi(i, j, value)`. Tiles of 64 x 64, k-chunks of 16 (the next chunk's loads in flight while the
// current one is multiplied), 4 x 4 outputs per thread; `tile` needs 2 * 64 * 17 doubles of shared
// memory. If `lower_only`, only tiles touching the lower
// triangle (i >= j) are computed (for symmetric results).
template <bool TA, bool TB, class Epi>
__device__ void cta_gemm(int m, int n, int k, double alpha, const double* __restrict__ A, int lda,
                         const double* __restrict__ B, int ldb, double* tile, bool lower_only, Epi epi) {
  constexpr int BM = 64, BN = 64, BK = 16;
  double* As = tile;              // [BK][BM+1]
  double* Bs = tile + BK * (BM + 1);  // [BK][BN+1]
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads
  const int tiles_m = (m + BM - 1) / BM, tiles_n = (n + BN - 1) / BN;
  for (int t = 0; t < tiles_m * tiles_n; ++t) {
    const int bi = t / tiles_n, bj = t % tiles_n;
    if (lower_only && bj > bi) continue;  // uniform across the CTA
    const int i0 = bi * BM, j0 = bj * BN;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;
    // the next k-chunk's elements are loaded into registers while the current one is multiplied
    // (each thread holds 4 of op(A) and 4 of op(B): 64 x 16 / 256 threads)
    double pa[4], pb[4];
    cta_gemm_fetch<TA, TB>(pa, pb, 0, i0, j0, m, n, k, A, lda, B, ldb);
    for (int k0 = 0; k0 < k; k0 += BK) {
      __syncthreads();  // the previous chunk's products have read As, Bs
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = threadIdx.x + q * kThreads;
        int ii, kk;
        if (TA) { ii = e % BM; kk = e / BM; } else { kk = e % BK; ii = e / BK; }
        As[kk * (BM + 1) + ii] = pa[q];
        int jj;
        if (TB) { kk = e % BK; jj = e / BK; } else { jj = e % BN; kk = e / BN; }
        Bs[kk * (BN + 1) + jj] = pb[q];
      }
      __syncthreads();
      if (k0 + BK < k) cta_gemm_fetch<TA, TB>(pa, pb, k0 + BK, i0, j0, m, n, k, A, lda, B, ldb);
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        double a[4], b[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          a[q] = As[kk * (BM + 1) + ty + 16 * q];
          b[q] = Bs[kk * (BN + 1) + tx + 16 * q];
        }
#pragma unroll
        for (int p = 0; p < 4; ++p)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[p][q] = fma(a[p], b[q], acc[p][q]);
      }
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int gi = i0 + ty + 16 * p, gj = j0 + tx + 16 * q;
        if (gi < m && gj < n) epi(gi, gj, alpha * acc[p][q]);
      }
  }
  __syncthreads();
}

}  // namespace pm3gpu
