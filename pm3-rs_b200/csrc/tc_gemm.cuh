// Split-BF16 GEMM on the fifth-generation tensor cores (tcgen05, sm_100a) for the mixed-precision
// dense products of the whole-GPU path: the commutator F P (pm3-rs src/scf.rs:1039-1054) and the
// density X X^T (src/scf.rs:982-992, src/linalg.rs:128-147).
//
// An FP64 operand x is carried as two BF16 numbers, hi = bf16(x) and lo = bf16(x - hi), and
//   C = A B^T ~ A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T
// (the lo lo term is below FP32 accumulation noise). One launch accumulates all three products into
// a single FP32 accumulator in tensor memory, so the three GEMMs are one pass over K.
//
// Layout: A is M x K and B is N x K, both row-major with K contiguous ("K-major"), BF16, leading
// dimension a multiple of 8 elements (16-byte rows for TMA). C is M x N row-major FP32.
//
// One CTA of 128 threads per 128 x 256 output tile:
//   warp 0 lane 0   TMA producer: per K block of 64, the four 128-byte-swizzled tiles A_hi, A_lo
//                   (128 x 64) and B_hi, B_lo (256 x 64) into one of two shared-memory stages
//                   (96 KB each), completion counted on the stage's "full" mbarrier;
//   warp 1 lane 0   MMA issuer: 3 products x 4 K-slices of tcgen05.mma.cta_group::1.kind::f16
//                   (M 128, N 256, K 16) per stage into a 256-column TMEM accumulator, then
//                   tcgen05.commit to the stage's "empty" mbarrier (frees it for the producer)
//                   and, after the last stage, to the "accumulator" mbarrier;
//   all 4 warps     epilogue: tcgen05.ld of the accumulator rows (warp w owns TMEM lanes
//                   32w..32w+31) and the FP32 stores.
// Out-of-range rows and K columns of a tile are zero-filled by TMA; stores are masked.
//
// Every mbarrier wait is bounded: a wait that runs out sets the launch's error flag, the roles
// stop, and the CTA still waits (bounded) for the copies and products it issued and frees its
// tensor memory before it returns. The host turns the flag into an error.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

namespace pm3gpu {
namespace tc {

constexpr int kBM = 128, kBN = 256, kBK = 64;  // output tile; K block = one 128-byte row of BF16
constexpr int kStages = 2;
constexpr int kThreads = 128;
constexpr uint32_t kTileA = kBM * kBK * 2;               // 16 KB
constexpr uint32_t kTileB = kBN * kBK * 2;               // 32 KB
constexpr uint32_t kStageBytes = 2 * kTileA + 2 * kTileB;  // A_hi, A_lo, B_hi, B_lo: 96 KB
constexpr uint32_t kSmemBytes = kStages * kStageBytes + 1024 + 128;  // + alignment slack + barriers
constexpr uint32_t kTmemCols = 256;                      // FP32 accumulator, 128 lanes x 256 columns
constexpr int kWaitLimit = 1 << 20;                      // polls of one mbarrier wait before giving up
// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), A and B BF16 (bits 7-9,
// 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor of a K-major tile in the 128-byte swizzle layout that TMA writes
// for a box 64 BF16 wide: rows of 128 bytes, 8-row groups 1024 bytes apart (stride byte offset),
// leading byte offset unused for this layout (16), descriptor version 1 (bits 46-47), swizzle mode
// 128B (2 at bits 61-63). The tile must start on a 1024-byte boundary (base offset 0); moving to
// the next 16-element K slice inside the swizzle row adds 32 bytes to the start address.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)(16 >> 4) << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase with the given parity; false when it ran out or another role failed.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* fail) {
  for (int i = 0; i < kWaitLimit; ++i) {
    if (mbar_test(bar, parity)) return true;
    if ((i & 255) == 255 && *fail) return false;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(kThreads, 1)
    split_gemm_kernel(const __grid_constant__ CUtensorMap mAhi, const __grid_constant__ CUtensorMap mAlo,
                      const __grid_constant__ CUtensorMap mBhi, const __grid_constant__ CUtensorMap mBlo, int M, int N,
                      int K, float* __restrict__ C, int ldc, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;  // stage tiles on 1024-byte boundaries
  const uint32_t bar0 = base + kStages * kStageBytes;
  // barriers: full[0..1] at bar0, empty[0..1] at bar0 + 16, accumulator at bar0 + 32
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 16u + 8u * s; };
  const uint32_t accum_bar = bar0 + 32u;
  unsigned char* gen = smem_raw + (base - raw);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gen + kStages * kStageBytes + 40);
  volatile int* fail = reinterpret_cast<volatile int*>(gen + kStages * kStageBytes + 44);
  int* issued_p = reinterpret_cast<int*>(gen + kStages * kStageBytes + 48);

  // a CTA of a launch that has already failed does nothing (before any allocation), so that a
  // systematic failure costs one wave of bounded waits, not every tile's; one thread reads the flag
  // so that the whole CTA takes the same branch
  __shared__ int skip;
  if (threadIdx.x == 0) skip = *reinterpret_cast<volatile int*>(err);
  __syncthreads();
  if (skip) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int nkb = (K + kBK - 1) / kBK;

  if (warp == 0) {  // the whole warp allocates the accumulator columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    mbar_init(accum_bar, 1);
    *fail = 0;
    *issued_p = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {  // ---- TMA producer
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mAhi)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mBhi)) : "memory");
    int issued = 0;
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb & 1;
      if (kb >= kStages && !mbar_wait(empty_bar(s), ((kb >> 1) - 1) & 1, fail)) {
        *fail = 1;
        break;
      }
      const uint32_t st = base + s * kStageBytes;
      mbar_expect_tx(full_bar(s), kStageBytes);
      tma_load_2d(st, &mAhi, kb * kBK, m0, full_bar(s));
      tma_load_2d(st + kTileA, &mAlo, kb * kBK, m0, full_bar(s));
      tma_load_2d(st + 2 * kTileA, &mBhi, kb * kBK, n0, full_bar(s));
      tma_load_2d(st + 2 * kTileA + kTileB, &mBlo, kb * kBK, n0, full_bar(s));
      issued = kb + 1;
    }
    *issued_p = issued;
  } else if (warp == 1 && lane == 0) {  // ---- MMA issuer
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb & 1;
      if (!mbar_wait(full_bar(s), (kb >> 1) & 1, fail)) {
        *fail = 1;
        break;
      }
      tc_fence_after();
      const uint32_t st = base + s * kStageBytes;
      const uint32_t a_hi = st, a_lo = st + kTileA, b_hi = st + 2 * kTileA, b_lo = st + 2 * kTileA + kTileB;
#pragma unroll
      for (int k = 0; k < kBK / 16; ++k) {
        const uint32_t off = 32u * k;  // 16 BF16 = 32 bytes along the swizzled row
        umma_f16(tmem, sw128_desc(a_hi + off), sw128_desc(b_hi + off), (kb | k) != 0);
        umma_f16(tmem, sw128_desc(a_hi + off), sw128_desc(b_lo + off), 1u);
        umma_f16(tmem, sw128_desc(a_lo + off), sw128_desc(b_hi + off), 1u);
      }
      umma_commit(empty_bar(s));  // arrives once these products have read the stage
    }
    umma_commit(accum_bar);  // every product issued so far, also on the error path
  }
  __syncwarp();

  // ---- epilogue: accumulator rows -> FP32 C. The accumulator barrier is waited for on every
  // path (products still in flight must finish before the tensor memory is freed).
  int never = 0;
  const bool done = mbar_wait(accum_bar, 0, &never);
  if (!done && threadIdx.x == 0) *fail = 1;
  __syncthreads();
  const bool ok = !*fail;
  tc_fence_after();
  if (ok && nkb > 0) {
    const int row = warp * 32 + lane;
    const int gm = m0 + row;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c0 = 0; c0 < kBN; c0 += 32) {
      uint32_t r[32];
      tmem_ld32(lane_base + (uint32_t)c0, r);
      if (gm < M) {
        float* dst = C + (size_t)gm * ldc + n0 + c0;
        const int left = N - (n0 + c0);
        if (left >= 32 && (ldc & 3) == 0) {
#pragma unroll
          for (int j = 0; j < 32; j += 4)
            *reinterpret_cast<float4*>(dst + j) = make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]),
                                                              __uint_as_float(r[j + 2]), __uint_as_float(r[j + 3]));
        } else {
          for (int j = 0; j < 32 && j < left; ++j) dst[j] = __uint_as_float(r[j]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    if (*fail) {
      // bounded wait for the stage copies that were issued but never consumed, so that no TMA
      // write lands in shared memory after the CTA has gone
      const int issued = *issued_p;
      for (int kb = (issued > kStages ? issued - kStages : 0); kb < issued; ++kb)
        (void)mbar_wait(full_bar(kb & 1), (kb >> 1) & 1, &never);
      atomicExch(err, 1);
    }
  }
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ------------------------------------------------------------------ MLP layers
// One hidden layer of the learned-guess network on the same machinery (no counterpart in the
// reference): H = silu(A W^T + b) with A (M x K, K = 64 or 256) and W^T (256 x K) K-major BF16, one
// product per K slice, FP32 accumulator in tensor memory, bias + SiLU + BF16 rounding in the
// epilogue (the rounding points of the mma.sync path: FP32 pre-activation, BF16 activation). With
// HEAD the epilogue also applies the 256 x 8 output layer to the BF16 activations of its row
// (Y = H W4 + b4, FP32), so the last hidden activations never leave the SM. Stage = A tile
// (128 x 64) + W tile (256 x 64), 48 KB; two stages, two CTAs per SM.
constexpr uint32_t kMlpStage = kTileA + kTileB;
constexpr uint32_t kMlpSmem = kStages * kMlpStage + 1024 + 128;

template <bool HEAD>
__global__ void __launch_bounds__(kThreads, 2)
    mlp_layer_kernel(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mW, int M, int K,
                     const float* __restrict__ bias, __nv_bfloat16* __restrict__ H, const __nv_bfloat16* __restrict__ W4,
                     const float* __restrict__ b4, float* __restrict__ Y, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  const uint32_t bar0 = base + kStages * kMlpStage;
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 16u + 8u * s; };
  const uint32_t accum_bar = bar0 + 32u;
  unsigned char* gen = smem_raw + (base - raw);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gen + kStages * kMlpStage + 40);
  volatile int* fail = reinterpret_cast<volatile int*>(gen + kStages * kMlpStage + 44);
  int* issued_p = reinterpret_cast<int*>(gen + kStages * kMlpStage + 48);

  __shared__ int skip;
  if (threadIdx.x == 0) skip = *reinterpret_cast<volatile int*>(err);
  __syncthreads();
  if (skip) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * kBM;
  const int nkb = (K + kBK - 1) / kBK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    mbar_init(accum_bar, 1);
    *fail = 0;
    *issued_p = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {  // ---- TMA producer
    int issued = 0;
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb & 1;
      if (kb >= kStages && !mbar_wait(empty_bar(s), ((kb >> 1) - 1) & 1, fail)) {
        *fail = 1;
        break;
      }
      const uint32_t st = base + s * kMlpStage;
      mbar_expect_tx(full_bar(s), kMlpStage);
      tma_load_2d(st, &mA, kb * kBK, m0, full_bar(s));
      tma_load_2d(st + kTileA, &mW, kb * kBK, 0, full_bar(s));
      issued = kb + 1;
    }
    *issued_p = issued;
  } else if (warp == 1 && lane == 0) {  // ---- MMA issuer
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb & 1;
      if (!mbar_wait(full_bar(s), (kb >> 1) & 1, fail)) {
        *fail = 1;
        break;
      }
      tc_fence_after();
      const uint32_t st = base + s * kMlpStage;
#pragma unroll
      for (int k = 0; k < kBK / 16; ++k)
        umma_f16(tmem, sw128_desc(st + 32u * k), sw128_desc(st + kTileA + 32u * k), (kb | k) != 0);
      umma_commit(empty_bar(s));
    }
    umma_commit(accum_bar);
  }
  __syncwarp();

  int never = 0;
  const bool done = mbar_wait(accum_bar, 0, &never);
  if (!done && threadIdx.x == 0) *fail = 1;
  __syncthreads();
  const bool ok = !*fail;
  tc_fence_after();
  if (ok && nkb > 0) {
    const int row = warp * 32 + lane;
    const int gm = m0 + row;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    float y[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
    for (int c0 = 0; c0 < kBN; c0 += 32) {
      uint32_t r[32];
      tmem_ld32(lane_base + (uint32_t)c0, r);
      float h[32];  // BF16-rounded activations of columns c0 .. c0 + 31
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const float z = __uint_as_float(r[j]) + __ldg(bias + c0 + j);
        h[j] = __bfloat162float(__float2bfloat16(z / (1.0f + __expf(-z))));
      }
      if (!HEAD) {
        if (gm < M) {  // 64 bytes of the row: four 16-byte stores of packed pairs
          uint4* dst = reinterpret_cast<uint4*>(H + (size_t)gm * kBN + c0);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            uint32_t w[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const __nv_bfloat162 b2 = __floats2bfloat162_rn(h[8 * q + 2 * e], h[8 * q + 2 * e + 1]);
              w[e] = (uint32_t)__bfloat16_as_ushort(b2.x) | ((uint32_t)__bfloat16_as_ushort(b2.y) << 16);
            }
            dst[q] = make_uint4(w[0], w[1], w[2], w[3]);
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const __nv_bfloat16* w = W4 + (size_t)(c0 + j) * 8;
#pragma unroll
          for (int o = 0; o < 8; ++o) y[o] = fmaf(h[j], __bfloat162float(w[o]), y[o]);
        }
      }
    }
    if (HEAD && gm < M) {
      float4* dst = reinterpret_cast<float4*>(Y + (size_t)gm * 8);
      dst[0] = make_float4(y[0] + b4[0], y[1] + b4[1], y[2] + b4[2], y[3] + b4[3]);
      dst[1] = make_float4(y[4] + b4[4], y[5] + b4[5], y[6] + b4[6], y[7] + b4[7]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    if (*fail) {
      const int issued = *issued_p;
      for (int kb = (issued > kStages ? issued - kStages : 0); kb < issued; ++kb)
        (void)mbar_wait(full_bar(kb & 1), (kb >> 1) & 1, &never);
      atomicExch(err, 1);
    }
  }
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ------------------------------------------------------------------ host side
// cuTensorMapEncodeTiled from the driver (through the runtime's entry-point query: no link
// dependency on libcuda), resolved once per process.
inline PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Tensor map of a K-major BF16 matrix (rows x k used, leading dimension ld elements, ld a multiple
// of 8 so rows start on 16 bytes) read in boxes of 64 (K) x box_rows with the 128-byte swizzle.
inline bool map_kmajor(CUtensorMap* m, const void* base, int rows, int k, int ld, int box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
  if (!enc || (ld & 7) != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0 || rows < 1 || k < 1) return false;
  cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// A kernel's dynamic shared-memory limit, raised once per device and kernel (`tag` < 32): the
// attribute is per device, and setting it again on every launch is not free (with other streams
// busy the call can wait for their work, which would hold back this stream's next launches).
inline bool smem_attr_once(const void* kernel, int bytes, int tag) {
  static std::mutex mu;
  static std::vector<uint32_t> done;  // per device: bit `tag` set once the attribute is in place
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return false;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)done.size() <= dev) done.resize(dev + 1, 0u);
  if (done[dev] & (1u << tag)) return true;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess) return false;
  done[dev] |= 1u << tag;
  return true;
}

// C (M x N, row-major FP32, ldc) = A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T with A (M x K, lda) and
// B (N x K, ldb) K-major BF16 on `stream`; err (device int) is set if a wait in the kernel ran
// out. Returns false when a tensor map cannot be made (bad alignment or no driver entry point).
inline bool launch_split_gemm(int M, int N, int K, const __nv_bfloat16* Ahi, const __nv_bfloat16* Alo, int lda,
                              const __nv_bfloat16* Bhi, const __nv_bfloat16* Blo, int ldb, float* C, int ldc, int* err,
                              cudaStream_t stream) {
  CUtensorMap a_hi, a_lo, b_hi, b_lo;
  if (!map_kmajor(&a_hi, Ahi, M, K, lda, kBM) || !map_kmajor(&a_lo, Alo, M, K, lda, kBM) ||
      !map_kmajor(&b_hi, Bhi, N, K, ldb, kBN) || !map_kmajor(&b_lo, Blo, N, K, ldb, kBN))
    return false;
  if (!smem_attr_once((const void*)split_gemm_kernel, (int)kSmemBytes, 0)) return false;
  const dim3 grid((unsigned)((N + kBN - 1) / kBN), (unsigned)((M + kBM - 1) / kBM));
  split_gemm_kernel<<<grid, kThreads, kSmemBytes, stream>>>(a_hi, a_lo, b_hi, b_lo, M, N, K, C, ldc, err);
  return true;
}

// One learned-guess layer: A (M x K, ld K) and Wt (256 x K, ld K) K-major BF16, bias (256 FP32).
// Without W4: H (M x 256 BF16, row-major) = silu(A Wt^T + bias). With W4 (256 x 8 BF16, in x out)
// and b4 (8 FP32): Y (M x 8 FP32) = bf16(silu(A Wt^T + bias)) W4 + b4. Returns false when a
// tensor map or the kernel attribute cannot be set.
inline bool launch_mlp_layer(int M, int K, const __nv_bfloat16* A, const __nv_bfloat16* Wt, const float* bias,
                             __nv_bfloat16* H, const __nv_bfloat16* W4, const float* b4, float* Y, int* err,
                             cudaStream_t stream) {
  if (M < 1 || (K != 64 && K != 256)) return false;
  CUtensorMap ma, mw;
  if (!map_kmajor(&ma, A, M, K, K, kBM) || !map_kmajor(&mw, Wt, kBN, K, K, kBN)) return false;
  const dim3 grid((unsigned)((M + kBM - 1) / kBM));
  if (W4) {
    if (!smem_attr_once((const void*)mlp_layer_kernel<true>, (int)kMlpSmem, 2)) return false;
    mlp_layer_kernel<true><<<grid, kThreads, kMlpSmem, stream>>>(ma, mw, M, K, bias, nullptr, W4, b4, Y, err);
  } else {
    if (!smem_attr_once((const void*)mlp_layer_kernel<false>, (int)kMlpSmem, 1)) return false;
    mlp_layer_kernel<false><<<grid, kThreads, kMlpSmem, stream>>>(ma, mw, M, K, bias, H, nullptr, nullptr, nullptr,
                                                                  err);
  }
  return true;
}

}  // namespace tc
}  // namespace pm3gpu
