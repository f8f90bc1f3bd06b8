// Learned initial density (no counterpart in the reference, whose guesses are SAD, core
// Hamiltonian and symmetry-broken SAD, src/scf.rs:855-916). A 3 x 256 MLP in BF16 with FP32
// accumulation predicts, for every atom and every atom pair of a molecule, the rotation-invariant
// elements of its density block from element one-hots, 32 Gaussian distance functions (6 A
// cutoff) and coordination counts. Pair blocks are described in the bond frame (x along a -> b):
// P[s_a][s_b] = ss, P[s_a][p_b] = s_sigma u, P[p_a][s_b] = sigma_s u,
// P[p_a][p_b] = sigma_sigma u u^T + pi_pi (I - u u^T); atom blocks by P_ss and the mean p
// population. The assembled matrix, scaled to the electron count, gives the first Fock matrix;
// its aufbau density is where the SCF iteration starts.
//
// Everything runs on the device: features, training targets from converged densities, the GEMMs
// (mma.sync m16n8k16 BF16 -> FP32, hand-written), activations, loss, backward pass, Adam, and the
// assembly of the guess.
#pragma once
#include <cuda_bf16.h>

#include "pm3_elements.h"

namespace pm3gpu {
namespace guess {

constexpr int kIn = 64;     // input features (padded)
constexpr int kHid = 256;   // hidden width
constexpr int kOut = 8;     // outputs (5 used, padded)
constexpr int kRbf = 32;
constexpr double kCutoffA = 6.0;          // Angstrom
constexpr double kBohrA = 0.529177210903;  // Angstrom per Bohr
constexpr int kElems = 8;   // one-hot slots: H C N O F S Cl other
// parameter layout (FP32 master copy): W1 b1 W2 b2 W3 b3 W4 b4, weights row-major (in x out)
constexpr int kW1 = 0, kB1 = kW1 + kIn * kHid, kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid, kW3 = kB2 + kHid,
              kB3 = kW3 + kHid * kHid, kW4 = kB3 + kHid, kB4 = kW4 + kHid * kOut, kParams = kB4 + kOut;

struct Mol {
  int atom0, natom, nao;
  int pad;
  long long row0;      // first feature row (self rows, then pairs a < b)
  long long dens_off;  // density block of this molecule (nao^2), target or guess
};

__device__ __forceinline__ int elem_slot(int z) {
  switch (z) {
    case 1: return 0;
    case 6: return 1;
    case 7: return 2;
    case 8: return 3;
    case 9: return 4;
    case 16: return 5;
    case 17: return 6;
    default: return 7;
  }
}

// row -> (molecule, atoms a, b); self rows have a == b. Pairs are ordered with the atom of more
// orbitals first (then by index), the same ordering in training and inference.
__device__ __forceinline__ void decode_row(const Mol* mols, int nmol, long long row, const ElemDev* elem,
                                           const int* z, int& mi, int& a, int& b) {
  int lo = 0, hi = nmol - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (mols[mid].row0 <= row) lo = mid;
    else hi = mid - 1;
  }
  mi = lo;
  const Mol& M = mols[lo];
  const long long loc = row - M.row0;
  if (loc < M.natom) {
    a = b = (int)loc;
    return;
  }
  const int t = (int)(loc - M.natom), N = M.natom;
  const double bb = 2.0 * N - 1.0;
  int uu = (int)floor((bb - sqrt(bb * bb - 8.0 * t)) * 0.5);
  if (uu < 0) uu = 0;
  while (uu > 0 && uu * (2 * N - uu - 1) / 2 > t) --uu;
  while ((uu + 1) * (2 * N - uu - 2) / 2 <= t) ++uu;
  const int u = uu, v = t - uu * (2 * N - uu - 1) / 2 + uu + 1;
  const bool hu = elem[z[M.atom0 + u]].norb == 4, hv = elem[z[M.atom0 + v]].norb == 4;
  a = (hu || !hv) ? u : v;
  b = a == u ? v : u;
}

// coordination count of each atom: sum over the molecule of 1 / (1 + exp(10 (d - 1.8 A)))
__global__ void coord_kernel(const Mol* mols, int nmol, const int* atom_mol, const double* xyz, int total_atoms,
                             float* coord) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total_atoms) return;
  const Mol& M = mols[atom_mol[g]];
  double c = 0.0;
  for (int k = 0; k < M.natom; ++k) {
    const int h = M.atom0 + k;
    if (h == g) continue;
    const double dx = xyz[3 * h] - xyz[3 * g], dy = xyz[3 * h + 1] - xyz[3 * g + 1], dz = xyz[3 * h + 2] - xyz[3 * g + 2];
    const double d = sqrt(dx * dx + dy * dy + dz * dz) * kBohrA;
    c += 1.0 / (1.0 + exp(10.0 * (d - 1.8)));
  }
  coord[g] = (float)c;
}

// feature rows (BF16, kIn per row)
__global__ void features_kernel(const Mol* mols, int nmol, const ElemDev* elem, const int* z, const double* xyz,
                                const float* coord, long long rows, __nv_bfloat16* X) {
  for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < rows;
       row += (long long)gridDim.x * blockDim.x) {
    int mi, a, b;
    decode_row(mols, nmol, row, elem, z, mi, a, b);
    const Mol& M = mols[mi];
    const int ga = M.atom0 + a, gb = M.atom0 + b;
    float f[kIn];
#pragma unroll
    for (int k = 0; k < kIn; ++k) f[k] = 0.0f;
    f[elem_slot(z[ga])] = 1.0f;
    f[kElems + elem_slot(z[gb])] = 1.0f;
    double d = 0.0;
    if (a != b) {
      const double dx = xyz[3 * gb] - xyz[3 * ga], dy = xyz[3 * gb + 1] - xyz[3 * ga + 1],
                   dz = xyz[3 * gb + 2] - xyz[3 * ga + 2];
      d = sqrt(dx * dx + dy * dy + dz * dz) * kBohrA;
    }
    const double fc = d < kCutoffA ? 0.5 * (cos(3.141592653589793 * d / kCutoffA) + 1.0) : 0.0;
    const double w = kCutoffA / (kRbf - 1), gam = 1.0 / (2.0 * w * w);
#pragma unroll
    for (int k = 0; k < kRbf; ++k) {
      const double mu = k * w;
      f[2 * kElems + k] = (float)(fc * exp(-gam * (d - mu) * (d - mu)));
    }
    f[2 * kElems + kRbf] = 0.25f * coord[ga];
    f[2 * kElems + kRbf + 1] = 0.25f * coord[gb];
    f[2 * kElems + kRbf + 2] = a == b ? 1.0f : 0.0f;
    __nv_bfloat16* xr = X + row * kIn;
#pragma unroll
    for (int k = 0; k < kIn; ++k) xr[k] = __float2bfloat16(f[k]);
  }
}

// bond unit vector a -> b
__device__ __forceinline__ void bond_dir(const double* xyz, int ga, int gb, double u[3]) {
  const double dx = xyz[3 * gb] - xyz[3 * ga], dy = xyz[3 * gb + 1] - xyz[3 * ga + 1], dz = xyz[3 * gb + 2] - xyz[3 * ga + 2];
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  u[0] = dx / r;
  u[1] = dy / r;
  u[2] = dz / r;
}

// training targets and masks from converged densities
__global__ void targets_kernel(const Mol* mols, int nmol, const ElemDev* elem, const int* z, const double* xyz,
                               const int* ao, const double* dens, long long rows, float* T, float* Mk) {
  for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < rows;
       row += (long long)gridDim.x * blockDim.x) {
    int mi, a, b;
    decode_row(mols, nmol, row, elem, z, mi, a, b);
    const Mol& M = mols[mi];
    const int ga = M.atom0 + a, gb = M.atom0 + b;
    const int na = elem[z[ga]].norb, nb = elem[z[gb]].norb;
    const int oa = ao[ga], ob = ao[gb], n = M.nao;
    const double* P = dens + M.dens_off;
    auto p = [&](int i, int j) { return P[(size_t)(oa + i) * n + ob + j]; };
    float t[kOut] = {0, 0, 0, 0, 0, 0, 0, 0}, m[kOut] = {0, 0, 0, 0, 0, 0, 0, 0};
    t[0] = (float)p(0, 0);
    m[0] = 1.0f;
    if (a == b) {
      if (na == 4) {
        const float pp = (float)((p(1, 1) + p(2, 2) + p(3, 3)) / 3.0);
        t[3] = pp;
        t[4] = pp;
        m[3] = m[4] = 1.0f;
      }
    } else {
      double u[3];
      bond_dir(xyz, ga, gb, u);
      if (nb == 4) {
        t[1] = (float)(p(0, 1) * u[0] + p(0, 2) * u[1] + p(0, 3) * u[2]);
        m[1] = 1.0f;
      }
      if (na == 4) {
        t[2] = (float)(p(1, 0) * u[0] + p(2, 0) * u[1] + p(3, 0) * u[2]);
        m[2] = 1.0f;
      }
      if (na == 4 && nb == 4) {
        double ss = 0.0, tr = 0.0;
        for (int k = 0; k < 3; ++k) {
          tr += p(1 + k, 1 + k);
          for (int l = 0; l < 3; ++l) ss += u[k] * p(1 + k, 1 + l) * u[l];
        }
        t[3] = (float)ss;
        t[4] = (float)(0.5 * (tr - ss));
        m[3] = m[4] = 1.0f;
      }
    }
#pragma unroll
    for (int k = 0; k < kOut; ++k) {
      T[row * kOut + k] = t[k];
      Mk[row * kOut + k] = m[k];
    }
  }
}

// initial densities from the predictions (FP32 outputs Y, kOut per row), into a zeroed buffer
__global__ void assemble_kernel(const Mol* mols, int nmol, const ElemDev* elem, const int* z, const double* xyz,
                                const int* ao, const float* Y, long long rows, double* dens) {
  for (long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x; row < rows;
       row += (long long)gridDim.x * blockDim.x) {
    int mi, a, b;
    decode_row(mols, nmol, row, elem, z, mi, a, b);
    const Mol& M = mols[mi];
    const int ga = M.atom0 + a, gb = M.atom0 + b;
    const int na = elem[z[ga]].norb, nb = elem[z[gb]].norb;
    const int oa = ao[ga], ob = ao[gb], n = M.nao;
    double* P = dens + M.dens_off;
    const float* y = Y + row * kOut;
    if (a == b) {
      P[(size_t)oa * n + oa] = y[0];
      if (na == 4)
        for (int k = 1; k < 4; ++k) P[(size_t)(oa + k) * n + oa + k] = 0.5 * (y[3] + y[4]);
      continue;
    }
    double u[3];
    bond_dir(xyz, ga, gb, u);
    auto put = [&](int i, int j, double v) {
      P[(size_t)(oa + i) * n + ob + j] = v;
      P[(size_t)(ob + j) * n + oa + i] = v;
    };
    put(0, 0, y[0]);
    if (nb == 4)
      for (int k = 0; k < 3; ++k) put(0, 1 + k, y[1] * u[k]);
    if (na == 4)
      for (int k = 0; k < 3; ++k) put(1 + k, 0, y[2] * u[k]);
    if (na == 4 && nb == 4)
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l) put(1 + k, 1 + l, y[3] * u[k] * u[l] + y[4] * ((k == l ? 1.0 : 0.0) - u[k] * u[l]));
  }
}

// ---------------------------------------------------------------- BF16 tensor-core GEMM
// C (M x N, FP32, row-major ldc) = op(A) (M x K) * op(B) (K x N) with BF16 operands:
// op(A)(m, k) = TA ? A[k * lda + m] : A[m * lda + k]; op(B)(k, n) = TB ? B[n * ldb + k] : B[k * ldb + n].
// 64 x 64 block tiles, K in steps of 32 staged in shared memory (k-contiguous, padded), four warps
// of 32 x 32, each a 2 x 4 grid of mma.sync.m16n8k16 (row.col, FP32 accumulate). Ragged edges
// are zero-filled on load and masked on store.
constexpr int kGT = 64, kGK = 32, kGPad = 8;
__device__ __forceinline__ unsigned pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
}
template <bool TA, bool TB>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                        int lda, const __nv_bfloat16* __restrict__ B, int ldb,
                                                        float* __restrict__ C, int ldc, int accumulate) {
  __shared__ __nv_bfloat16 As[kGT][kGK + kGPad];
  __shared__ __nv_bfloat16 Bs[kGT][kGK + kGPad];
  const int m0 = blockIdx.y * kGT, n0 = blockIdx.x * kGT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0f;
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
  for (int k0 = 0; k0 < K; k0 += kGK) {
    for (int e = threadIdx.x; e < kGT * kGK; e += 128) {
      const int r = e / kGK, kk = e % kGK;
      const int gm = m0 + r, gk = k0 + kk;
      As[r][kk] = (gm < M && gk < K) ? (TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk]) : zero;
      const int gn = n0 + r;
      Bs[r][kk] = (gn < N && gk < K) ? (TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn]) : zero;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < kGK; ks += 16) {
      unsigned af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + g;
        af[i][0] = pack2(As[r][ks + 2 * t], As[r][ks + 2 * t + 1]);
        af[i][1] = pack2(As[r + 8][ks + 2 * t], As[r + 8][ks + 2 * t + 1]);
        af[i][2] = pack2(As[r][ks + 2 * t + 8], As[r][ks + 2 * t + 9]);
        af[i][3] = pack2(As[r + 8][ks + 2 * t + 8], As[r + 8][ks + 2 * t + 9]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + j * 8 + g;
        bfr[j][0] = pack2(Bs[c][ks + 2 * t], Bs[c][ks + 2 * t + 1]);
        bfr[j][1] = pack2(Bs[c][ks + 2 * t + 8], Bs[c][ks + 2 * t + 9]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          asm volatile(
              "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
              "{%0,%1,%2,%3};\n"
              : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
              : "r"(af[i][0]), "r"(af[i][1]), "r"(af[i][2]), "r"(af[i][3]), "r"(bfr[j][0]), "r"(bfr[j][1]));
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = m0 + wm + i * 16 + g + (q >= 2 ? 8 : 0);
        const int c = n0 + wn + j * 8 + 2 * t + (q & 1);
        if (r < M && c < N) {
          float* dst = C + (size_t)r * ldc + c;
          *dst = accumulate ? *dst + acc[i][j][q] : acc[i][j][q];
        }
      }
}

// ---------------------------------------------------------------- MLP pieces
__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}
// Z += b; H = silu(Z) (BF16) -- hidden layers; for the output layer (act = 0) only Z += b
__global__ void bias_act_kernel(float* Z, const float* b, int cols, long long rows, __nv_bfloat16* H, int act) {
  const long long total = rows * cols;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const float z = Z[k] + b[k % cols];
    Z[k] = z;
    if (act) H[k] = __float2bfloat16(silu(z));
  }
}
// masked squared error: dY = 2 m (Y - T) / count (BF16); the block sums of m (Y - T)^2 are added
// into *accum (reporting only)
__global__ void loss_kernel(const float* Y, const float* T, const float* Mk, long long n, float inv_count,
                            __nv_bfloat16* dY, float* accum) {
  float s = 0.0f;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const float d = (Y[k] - T[k]) * Mk[k];
    s += d * d;
    dY[k] = __float2bfloat16(2.0f * d * inv_count);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ float red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float u = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) u += red[w];
    atomicAdd(accum, u);
  }
}
// dZ = dH * silu'(Z) (BF16); dH given in FP32
__global__ void dact_kernel(const float* dH, const float* Z, long long n, __nv_bfloat16* dZ) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    dZ[k] = __float2bfloat16(dH[k] * dsilu(Z[k]));
}
// db[c] = sum over rows of dZ[r][c]
__global__ void colsum_kernel(const __nv_bfloat16* dZ, int cols, long long rows, float* db) {
  const int c = blockIdx.x;
  float s = 0.0f;
  for (long long r = threadIdx.x; r < rows; r += blockDim.x) s += __bfloat162float(dZ[r * cols + c]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ float red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float u = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) u += red[w];
    db[c] = u;
  }
}
// Adam step on the FP32 master parameters; refreshes the BF16 copies
__global__ void adam_kernel(float* p, const float* gr, float* m, float* v, int n, float lr, float b1, float b2,
                            float c1, float c2, __nv_bfloat16* pb) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float gk = gr[k];
    const float mk = b1 * m[k] + (1.0f - b1) * gk, vk = b2 * v[k] + (1.0f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    const float q = p[k] - lr * (mk / c1) / (sqrtf(vk / c2) + 1.0e-8f);
    p[k] = q;
    pb[k] = __float2bfloat16(q);
  }
}
// Wt (out x in) = W^T for a row-major (in x out) weight: the K-major B operand of the tcgen05 layers.
__global__ void transpose_w_kernel(const __nv_bfloat16* __restrict__ W, int kin, int kout, __nv_bfloat16* __restrict__ Wt) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kin * kout; e += gridDim.x * blockDim.x) {
    const int n = e / kin, k = e % kin;
    Wt[e] = W[(size_t)k * kout + n];
  }
}

__global__ void to_bf16_kernel(const float* p, int n, __nv_bfloat16* pb) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) pb[k] = __float2bfloat16(p[k]);
}
// gather rows idx[0..B) of X (kIn) / T, Mk (kOut) into contiguous minibatch buffers
__global__ void gather_rows_kernel(const long long* idx, int B, const __nv_bfloat16* X, const float* T, const float* Mk,
                                   __nv_bfloat16* Xb, float* Tb, float* Mb) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < B * kIn; e += gridDim.x * blockDim.x) {
    const int r = e / kIn, c = e % kIn;
    Xb[e] = X[idx[r] * kIn + c];
    if (c < kOut) {
      Tb[r * kOut + c] = T[idx[r] * kOut + c];
      Mb[r * kOut + c] = Mk[idx[r] * kOut + c];
    }
  }
}

}  // namespace guess
}  // namespace pm3gpu
