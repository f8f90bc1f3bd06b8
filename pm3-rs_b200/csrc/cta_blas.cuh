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

// C (m x n) = alpha * op(A) * op(B) with op(A) m x k, op(B) k x n; A, B row-major in global
// memory. TA: A stored as k x m (use its transpose). Each output element goes through
// `epi(i, j, value)`. Tiles of 64 x 64, k-chunks of 16, 4 x 4 outputs per thread; `tile`
// needs 2 * 64 * 17 doubles of shared memory. If `lower_only`, only tiles touching the lower
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
    for (int k0 = 0; k0 < k; k0 += BK) {
      __syncthreads();
      // load op(A)[i0..i0+64, k0..k0+16] into As[kk][ii]
      for (int e = threadIdx.x; e < BM * BK; e += kThreads) {
        int ii, kk;
        if (TA) { ii = e % BM; kk = e / BM; } else { kk = e % BK; ii = e / BK; }
        const int gi = i0 + ii, gk = k0 + kk;
        double v = 0.0;
        if (gi < m && gk < k) v = TA ? A[(size_t)gk * lda + gi] : A[(size_t)gi * lda + gk];
        As[kk * (BM + 1) + ii] = v;
      }
      for (int e = threadIdx.x; e < BK * BN; e += kThreads) {
        int jj, kk;
        if (TB) { kk = e % BK; jj = e / BK; } else { jj = e % BN; kk = e / BN; }
        const int gj = j0 + jj, gk = k0 + kk;
        double v = 0.0;
        if (gj < n && gk < k) v = TB ? B[(size_t)gj * ldb + gk] : B[(size_t)gk * ldb + gj];
        Bs[kk * (BN + 1) + jj] = v;
      }
      __syncthreads();
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
