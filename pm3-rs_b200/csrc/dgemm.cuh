// FP64 GEMM on the FP64 tensor pipe (DMMA), for the whole-GPU path's dense products: the
// commutator F P and the density X^T X of the SCF loop (pm3-rs src/scf.rs:1039-1054, 982-992),
// and the eigensolver's Householder trailing updates, compact-WY back-transformation and
// Newton-Schulz orthonormalisation that replace faer's self_adjoint_eigen (src/linalg.rs:221-263).
//
// C = alpha op(A) op(B) + beta C, column-major, op = N or T (the BLAS dgemm contract). Blackwell has
// no tcgen05 kind for FP64, so the products are `mma.sync.m16n8k8.f64`. One CTA of 8 warps per
// BM x BN tile of C; each warp owns a (16 MT) x (8 NT) block as MT x NT MMA tiles; K advances in
// steps of 16 through a 3- or 4-stage cp.async pipeline of 16-byte copies (`Tile` below: the
// shared layout follows the operand's contiguous direction). The tile shape follows the problem:
// 128 x 128 (64 accumulators per thread, one CTA per SM) for large outputs with a long K, 128 x 64
// (two CTAs per SM, more bytes in flight) for the low-K trailing updates, and 128 x 32 / 32 x 128
// (two CTAs per SM) for outputs one panel wide. C goes out through shared memory, 64 (or all)
// columns at a time, so every global access is a coalesced column run with 16 loads of the old C
// in flight per thread. Outputs with fewer tiles than resident CTA slots and a long K split K over
// the grid's z dimension (as many slices as fill the slots in one wave); the partial products go
// to a workspace and one kernel sums them in a fixed order, so results repeat bit for bit.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

namespace pm3gpu {
namespace dg {

constexpr int kBK = 16, kThreads = 256;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// 8-byte asynchronous copy; src_bytes = 0 writes a zero (the source is not read)
__device__ __forceinline__ void cp8(double* dst, const double* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes));
}
// 16-byte asynchronous copy (both addresses 16-byte aligned); the bytes past src_bytes are zero
__device__ __forceinline__ void cp16(double* dst, const double* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Shared-memory tile of one operand, R rows (of op(A), or columns of op(B)) by kBK k's. When the
// global matrix is contiguous in r the tile is k-major, S[kk][r] with rows of R + 4 doubles;
// when it is contiguous in k the tile is r-major, S[r][kk] with rows of 20 doubles. Either way
// 16-byte copies move pairs of consecutive doubles and each half-warp's fragment loads hit 16
// distinct banks (row strides of 4 mod 16 doubles).
template <bool KContig, int R>
struct Tile {
  static constexpr int LD = KContig ? kBK + 4 : R + 4;
  static constexpr int SIZE = KContig ? R * LD : kBK * LD;
  __device__ static __forceinline__ int at(int r, int kk) { return KContig ? r * LD + kk : kk * LD + r; }
};

// Tile shapes: BM x BN outputs per CTA, warps (BM / 16 MT) x (BN / 8 NT) = 8; MinBlocks = the CTAs
// per SM that the shared memory and registers allow.
template <int BM_, int BN_, int MT_, int NT_, int MinBlocks_, int Stages_>
struct Shape {
  static constexpr int BM = BM_, BN = BN_, MT = MT_, NT = NT_, MinBlocks = MinBlocks_, STAGES = Stages_;
  static constexpr int WM = 16 * MT, WN = 8 * NT;
  static constexpr int WARPS_M = BM / WM;
  static_assert((BM / WM) * (BN / WN) == 8, "eight warps per CTA");
  // the larger of the two layouts, so one size serves every operand orientation
  static constexpr int TILE_A =
      Tile<false, BM>::SIZE > Tile<true, BM>::SIZE ? Tile<false, BM>::SIZE : Tile<true, BM>::SIZE;
  static constexpr int TILE_B =
      Tile<false, BN>::SIZE > Tile<true, BN>::SIZE ? Tile<false, BN>::SIZE : Tile<true, BN>::SIZE;
  static constexpr int LC = BM + 4;  // epilogue staging: CW columns of BM rows
  static constexpr int PIPE = STAGES * (TILE_A + TILE_B);
  static constexpr int CW = (PIPE / LC) >= BN ? BN : ((PIPE / LC) >= 64 && BN % 64 == 0 ? 64 : 32);
  static_assert(BN % CW == 0 && (BM * CW) % kThreads == 0, "epilogue chunks");
  static constexpr int SMEM = 8 * (PIPE > CW * LC ? PIPE : CW * LC);
};
using ShapeL = Shape<128, 128, 4, 4, 1, 4>;  // large outputs, long K
using ShapeM = Shape<128, 64, 2, 4, 2, 3>;   // low K: two CTAs per SM
using ShapeN = Shape<128, 32, 2, 2, 2, 3>;   // one panel wide (n <= 32)
using ShapeW = Shape<32, 128, 2, 2, 2, 3>;   // one panel tall (m <= 32)

// Stage one K-step of op(X) into the tile S. KContig: the element (r, kk) sits at X[kk + r ld];
// otherwise at X[r + kk ld]. Out-of-range elements are zero. With `vec` (ld even, X 16-byte
// aligned) pairs of consecutive doubles move as 16-byte copies.
template <bool KContig, int R>
__device__ __forceinline__ void load_tile(double* S, const double* X, int ld, int r0, int rows, int k0, int kdim,
                                          bool vec) {
  using T = Tile<KContig, R>;
  const int t = threadIdx.x;
  if (vec) {
#pragma unroll
    for (int q = 0; q < (kBK * R) / (2 * kThreads); ++q) {
      const int idx = t + q * kThreads;
      int kk, r, avail;
      const double* src;
      if (!KContig) {  // pairs (r, r + 1): runs of R / 2 pairs per k-row
        kk = idx / (R / 2);
        r = 2 * (idx % (R / 2));
        const int gr = r0 + r, gk = k0 + kk;
        avail = gk < kdim ? min(max(rows - gr, 0), 2) : 0;
        src = avail ? X + (size_t)gk * ld + gr : X;
      } else {  // pairs (kk, kk + 1): 8 pairs per r
        kk = 2 * (idx & 7);
        r = idx >> 3;
        const int gr = r0 + r, gk = k0 + kk;
        avail = gr < rows ? min(max(kdim - gk, 0), 2) : 0;
        src = avail ? X + (size_t)gr * ld + gk : X;
      }
      cp16(S + T::at(r, kk), src, 8 * avail);
    }
  } else {
#pragma unroll
    for (int q = 0; q < (kBK * R) / kThreads; ++q) {
      const int idx = t + q * kThreads;
      int kk, r;
      if (!KContig) {
        kk = idx / R;
        r = idx % R;
      } else {
        kk = idx & 15;
        r = idx >> 4;
      }
      const int gr = r0 + r, gk = k0 + kk;
      const bool ok = gr < rows && gk < kdim;
      const double* src = ok ? (KContig ? X + (size_t)gr * ld + gk : X + (size_t)gk * ld + gr) : X;
      cp8(S + T::at(r, kk), src, ok ? 8 : 0);
    }
  }
}

// One CTA: the BM x BN tile (blockIdx.x, blockIdx.y) of C over the K range of blockIdx.z. With
// `part` set, the raw products go to part (tile-major, BM-row columns, splits stacked) instead of C.
template <class S, bool TA, bool TB>
__global__ void __launch_bounds__(kThreads, S::MinBlocks)
    dgemm_kernel(int m, int n, int k, double alpha, const double* __restrict__ A, int lda,
                 const double* __restrict__ B, int ldb, double beta, double* __restrict__ C, int ldc, int kchunk,
                 double* __restrict__ part, int vec_a, int vec_b) {
  constexpr int kStages = S::STAGES;
  using TA_ = Tile<TA, S::BM>;
  using TB_ = Tile<!TB, S::BN>;
  extern __shared__ __align__(16) double dg_smem[];
  double* As = dg_smem;
  double* Bs = dg_smem + kStages * S::TILE_A;
  const int m0 = blockIdx.x * S::BM, n0 = blockIdx.y * S::BN;
  const int kb = blockIdx.z * kchunk, ke = min(k, kb + kchunk);
  const int nk = ke > kb ? (ke - kb + kBK - 1) / kBK : 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp % S::WARPS_M) * S::WM, wn = (warp / S::WARPS_M) * S::WN;
  const int g = lane >> 2, tg = lane & 3;
  double acc[S::MT][S::NT][4];
#pragma unroll
  for (int a = 0; a < S::MT; ++a)
#pragma unroll
    for (int b = 0; b < S::NT; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;

  // op(A) element (i, kk): A[i + kk lda] (N) or A[kk + i lda] (T); op(B) element (kk, j):
  // B[kk + j ldb] (N: contiguous in kk) or B[j + kk ldb] (T)
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) {
      load_tile<TA, S::BM>(As + s * S::TILE_A, A, lda, m0, m, kb + s * kBK, ke, vec_a);
      load_tile<!TB, S::BN>(Bs + s * S::TILE_B, B, ldb, n0, n, kb + s * kBK, ke, vec_b);
    }
    cp_commit();
  }
  for (int it = 0; it < nk; ++it) {
    cp_wait<kStages - 2>();
    __syncthreads();
    {  // refill the stage consumed at the previous step
      const int nx = it + kStages - 1;
      if (nx < nk) {
        const int st = nx % kStages;
        load_tile<TA, S::BM>(As + st * S::TILE_A, A, lda, m0, m, kb + nx * kBK, ke, vec_a);
        load_tile<!TB, S::BN>(Bs + st * S::TILE_B, B, ldb, n0, n, kb + nx * kBK, ke, vec_b);
      }
      cp_commit();
    }
    const double* as = As + (it % kStages) * S::TILE_A;
    const double* bs = Bs + (it % kStages) * S::TILE_B;
#pragma unroll
    for (int k8 = 0; k8 < kBK; k8 += 8) {
      double af[S::MT][4], bf[S::NT][2];
#pragma unroll
      for (int a = 0; a < S::MT; ++a) {
        const int r = wm + 16 * a + g;
        af[a][0] = as[TA_::at(r, k8 + tg)];
        af[a][1] = as[TA_::at(r + 8, k8 + tg)];
        af[a][2] = as[TA_::at(r, k8 + tg + 4)];
        af[a][3] = as[TA_::at(r + 8, k8 + tg + 4)];
      }
#pragma unroll
      for (int b = 0; b < S::NT; ++b) {
        const int r = wn + 8 * b + g;
        bf[b][0] = bs[TB_::at(r, k8 + tg)];
        bf[b][1] = bs[TB_::at(r, k8 + tg + 4)];
      }
#pragma unroll
      for (int a = 0; a < S::MT; ++a)
#pragma unroll
        for (int b = 0; b < S::NT; ++b)
          asm volatile(
              "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
              "{%0,%1,%2,%3};\n"
              : "+d"(acc[a][b][0]), "+d"(acc[a][b][1]), "+d"(acc[a][b][2]), "+d"(acc[a][b][3])
              : "d"(af[a][0]), "d"(af[a][1]), "d"(af[a][2]), "d"(af[a][3]), "d"(bf[b][0]), "d"(bf[b][1]));
    }
  }
  cp_wait<0>();
  __syncthreads();  // the pipeline buffers become the epilogue's staging area

  // Epilogue, CW columns of the tile at a time: the warps owning them write their accumulators
  // (rows wm + 16a + g (+8), columns wn + 8b + 2tg (+1)) to Cs[col][row]; then each thread moves
  // its elements of the chunk (element q: row (t + 256 q) % BM, column (t + 256 q) / BM), loading
  // 16 old values of C at a time before combining and storing them.
  double* Cs = dg_smem;
  double* P = part ? part + ((size_t)blockIdx.z * gridDim.x * gridDim.y + (size_t)blockIdx.y * gridDim.x + blockIdx.x) *
                                (size_t)(S::BM * S::BN)
                   : nullptr;
  constexpr int CW = S::CW, kPer = (S::BM * CW) / kThreads;
  for (int c0 = 0; c0 < S::BN; c0 += CW) {
    if (wn + S::WN > c0 && wn < c0 + CW) {
#pragma unroll
      for (int a = 0; a < S::MT; ++a)
#pragma unroll
        for (int b = 0; b < S::NT; ++b)
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const int i = wm + 16 * a + g + 8 * (c >> 1), j = wn + 8 * b + 2 * tg + (c & 1) - c0;
            if (j >= 0 && j < CW) Cs[j * S::LC + i] = acc[a][b][c];
          }
    }
    __syncthreads();
    if (P) {
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const int e = threadIdx.x + q * kThreads, ii = e % S::BM, jj = e / S::BM;
        P[(size_t)(c0 + jj) * S::BM + ii] = Cs[jj * S::LC + ii];
      }
    } else if (beta == 0.0) {
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const int e = threadIdx.x + q * kThreads, ii = e % S::BM, jj = e / S::BM;
        const int i = m0 + ii, j = n0 + c0 + jj;
        if (i < m && j < n) C[(size_t)j * ldc + i] = alpha * Cs[jj * S::LC + ii];
      }
    } else {
      constexpr int kGroup = kPer < 16 ? kPer : 16;  // loads of the old C in flight per thread
#pragma unroll
      for (int q0 = 0; q0 < kPer; q0 += kGroup) {
        double old[kGroup];
#pragma unroll
        for (int q = 0; q < kGroup; ++q) {
          const int e = threadIdx.x + (q0 + q) * kThreads, ii = e % S::BM, jj = e / S::BM;
          const int i = m0 + ii, j = n0 + c0 + jj;
          old[q] = (i < m && j < n) ? C[(size_t)j * ldc + i] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kGroup; ++q) {
          const int e = threadIdx.x + (q0 + q) * kThreads, ii = e % S::BM, jj = e / S::BM;
          const int i = m0 + ii, j = n0 + c0 + jj;
          if (i < m && j < n) C[(size_t)j * ldc + i] = fma(alpha, Cs[jj * S::LC + ii], beta * old[q]);
        }
      }
    }
    __syncthreads();
  }
}

// C = alpha sum_z part[z] + beta C, the splits summed in order (tiles of bm x bn).
__global__ void dgemm_reduce_kernel(int m, int n, int bm, int bn, int splits, int tiles_m, int tiles_n, double alpha,
                                    const double* __restrict__ part, double beta, double* __restrict__ C, int ldc) {
  const size_t total = (size_t)m * n;
  const size_t tile = (size_t)bm * bn, stride = (size_t)tiles_m * tiles_n * tile;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % m), j = (int)(e / m);
    const size_t off = ((size_t)(j / bn) * tiles_m + i / bm) * tile + (size_t)(j % bn) * bm + i % bm;
    double s = 0.0;
    for (int z = 0; z < splits; ++z) s += part[off + z * stride];
    double* cp = C + (size_t)j * ldc + i;
    *cp = beta == 0.0 ? alpha * s : fma(alpha, s, beta * *cp);
  }
}

enum Kind { kL = 0, kM = 1, kN = 2, kW = 3 };

struct Plan {
  int kind, bm, bn, tiles_m, tiles_n, splits, kchunk;
  size_t work_doubles;  // split-K workspace
};
inline Plan plan(int m, int n, int k, int sms) {
  Plan p{};
  if (n <= 32) p.kind = kN;
  else if (m <= 32) p.kind = kW;
  else if (k <= 128) p.kind = kM;
  else p.kind = kL;
  static const int bms[4] = {ShapeL::BM, ShapeM::BM, ShapeN::BM, ShapeW::BM};
  static const int bns[4] = {ShapeL::BN, ShapeM::BN, ShapeN::BN, ShapeW::BN};
  static const int per_sm[4] = {ShapeL::MinBlocks, ShapeM::MinBlocks, ShapeN::MinBlocks, ShapeW::MinBlocks};
  p.bm = bms[p.kind];
  p.bn = bns[p.kind];
  p.tiles_m = (m + p.bm - 1) / p.bm;
  p.tiles_n = (n + p.bn - 1) / p.bn;
  const int tiles = p.tiles_m * p.tiles_n, slots = sms * per_sm[p.kind];
  int splits = 1;  // as many K slices as fill the resident slots in one wave
  if (tiles * 2 <= slots && k >= 1024) splits = std::max(1, std::min(slots / tiles, k / 256));
  int kchunk = (k + splits - 1) / splits;
  kchunk = std::max(kBK, (kchunk + kBK - 1) / kBK * kBK);
  p.splits = std::max(1, (k + kchunk - 1) / kchunk);
  p.kchunk = kchunk;
  p.work_doubles = p.splits > 1 ? (size_t)p.splits * tiles * p.bm * p.bn : 0;
  return p;
}

template <class S>
inline cudaError_t set_attributes_for() {
  cudaError_t e = cudaSuccess;
  auto one = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM);
  };
  one((const void*)dgemm_kernel<S, false, false>);
  one((const void*)dgemm_kernel<S, false, true>);
  one((const void*)dgemm_kernel<S, true, false>);
  one((const void*)dgemm_kernel<S, true, true>);
  return e;
}
// The shared-memory attribute of every variant, on the current device.
inline cudaError_t set_attributes() {
  cudaError_t e = set_attributes_for<ShapeL>();
  if (e == cudaSuccess) e = set_attributes_for<ShapeM>();
  if (e == cudaSuccess) e = set_attributes_for<ShapeN>();
  if (e == cudaSuccess) e = set_attributes_for<ShapeW>();
  return e;
}

template <class S>
inline void launch(const dim3& grid, cudaStream_t stream, bool ta, bool tb, int m, int n, int k, double alpha,
                   const double* A, int lda, const double* B, int ldb, double beta, double* C, int ldc, int kchunk,
                   double* part) {
  const int va = (lda % 2 == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0);
  const int vb = (ldb % 2 == 0) && ((reinterpret_cast<uintptr_t>(B) & 15) == 0);
  if (!ta && !tb)
    dgemm_kernel<S, false, false><<<grid, kThreads, S::SMEM, stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                       kchunk, part, va, vb);
  else if (!ta && tb)
    dgemm_kernel<S, false, true><<<grid, kThreads, S::SMEM, stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                      kchunk, part, va, vb);
  else if (ta && !tb)
    dgemm_kernel<S, true, false><<<grid, kThreads, S::SMEM, stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                      kchunk, part, va, vb);
  else
    dgemm_kernel<S, true, true><<<grid, kThreads, S::SMEM, stream>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                     kchunk, part, va, vb);
}

// Launch C = alpha op(A) op(B) + beta C on `stream` (set_attributes must have run on this device).
// `work` must hold plan(..).work_doubles. Returns the number of kernels launched, or -1 on a launch
// error (cudaGetLastError has it).
inline int gemm(cudaStream_t stream, int sms, bool ta, bool tb, int m, int n, int k, double alpha, const double* A,
                int lda, const double* B, int ldb, double beta, double* C, int ldc, double* work) {
  if (m <= 0 || n <= 0) return 0;
  const Plan p = plan(m, n, k, sms);
  if (p.splits > 1 && work == nullptr) return -1;
  const dim3 grid(p.tiles_m, p.tiles_n, p.splits);
  double* part = p.splits > 1 ? work : nullptr;
  switch (p.kind) {
    case kL: launch<ShapeL>(grid, stream, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, p.kchunk, part); break;
    case kM: launch<ShapeM>(grid, stream, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, p.kchunk, part); break;
    case kN: launch<ShapeN>(grid, stream, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, p.kchunk, part); break;
    default: launch<ShapeW>(grid, stream, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, p.kchunk, part); break;
  }
  if (cudaPeekAtLastError() != cudaSuccess) return -1;
  if (p.splits == 1) return 1;
  const size_t total = (size_t)m * n;
  const int blocks = (int)std::min<size_t>((total + 255) / 256, (size_t)sms * 8);
  dgemm_reduce_kernel<<<blocks, 256, 0, stream>>>(m, n, p.bm, p.bn, p.splits, p.tiles_m, p.tiles_n, alpha, part, beta,
                                                  C, ldc);
  return cudaPeekAtLastError() != cudaSuccess ? -1 : 2;
}

}  // namespace dg
}  // namespace pm3gpu
