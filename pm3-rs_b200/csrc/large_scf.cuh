// Whole-GPU kernels for one large molecule (basis beyond one CTA): the same run_pm3 SCF as the
// per-CTA path, with every step spread over the device. Pair integrals, H_core and the Fock
// build run one thread per atom pair (src/hamiltonian.rs:191-344, src/fock.rs:93-332), the sums
// into each atom's diagonal block one warp per atom in a fixed order (no atomics: repeated solves
// agree bit for bit); the dense products (commutator, density, the eigensolver's trailing updates
// and back-transformation) are DMMA DGEMMs (dgemm.cuh) issued by the host driver; the multi-launch
// Householder panel (the cooperative one is panel_coop.cuh), the Sturm multisection, the
// twisted-factorisation eigenvectors, the compact-WY factors and all reductions are here.
#pragma once
#include <cuda_bf16.h>

#include "scf_kernel.cuh"

namespace pm3gpu {
namespace large {

constexpr int kBlock = 256;   // threads per block of the grid kernels (matches the CTA helpers)
constexpr int kPanel = 32;    // Householder panel width
constexpr int kRedBlocks = 1184;  // partial-sum slots of the grid reductions (8 per SM)

// Device view of one molecule.
struct Mol {
  const ElemDev* elem;
  const PairDev* pairs;
  const int* z;             // [N]
  const double* xyz;        // [3N] Bohr
  const int* ao;            // [N] first AO of each atom
  const int* sprow;         // [N+1] prefix sums of packed orbital-pair sizes (10 sp, 1 s)
  const long long* sroff;   // [N] pair-table row offsets
  int N, n;
};

__device__ __forceinline__ long long pair_count(int N) { return (long long)N * (N - 1) / 2; }
__device__ __forceinline__ const double* pair_block(const Mol& m, const double* W, int u, int v) {
  const int su = m.sprow[u + 1] - m.sprow[u];
  return W + m.sroff[u] + (long long)su * (m.sprow[v] - m.sprow[u + 1]);
}

// ---------------------------------------------------------------- reductions (deterministic)
// Each block writes one partial; finish_sum adds the partials in a fixed order.
__device__ __forceinline__ void block_partial(double v, double* partial) {
  __shared__ double red[kBlock / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < kBlock / 32; ++i) t += red[i];
    partial[blockIdx.x] = t;
  }
}
__global__ void __launch_bounds__(kBlock) finish_sum(const double* partial, int np, double* out) {
  double v = 0.0;
  for (int i = threadIdx.x; i < np; i += kBlock) v += partial[i];
  __shared__ double red[kBlock / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < kBlock / 32; ++i) t += red[i];
    *out = t;
  }
}
// sum_k x_k y_k (+ sum_k x2_k y2_k when x2 is given)
__global__ void __launch_bounds__(kBlock) dot_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                                     const double* __restrict__ x2, const double* __restrict__ y2,
                                                     size_t cnt, double* partial) {
  double s = 0.0;
  for (size_t k = blockIdx.x * (size_t)kBlock + threadIdx.x; k < cnt; k += (size_t)gridDim.x * kBlock) {
    s = fma(x[k], y[k], s);
    if (x2) s = fma(x2[k], y2[k], s);
  }
  block_partial(s, partial);
}
// sum_k (x_k - y_k)^2
__global__ void __launch_bounds__(kBlock) sqdiff_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                                        size_t cnt, double* partial) {
  double s = 0.0;
  for (size_t k = blockIdx.x * (size_t)kBlock + threadIdx.x; k < cnt; k += (size_t)gridDim.x * kBlock) {
    const double d = x[k] - y[k];
    s = fma(d, d, s);
  }
  block_partial(s, partial);
}
// max_k |x_k - y_k| (one partial per block)
__global__ void __launch_bounds__(kBlock) absdiff_max_kernel(const double* __restrict__ x,
                                                             const double* __restrict__ y, size_t cnt,
                                                             double* partial) {
  double s = 0.0;
  for (size_t k = blockIdx.x * (size_t)kBlock + threadIdx.x; k < cnt; k += (size_t)gridDim.x * kBlock)
    s = fmax(s, fabs(x[k] - y[k]));
  s = warp_max(s);
  __shared__ double red[kBlock / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < kBlock / 32; ++i) t = fmax(t, red[i]);
    partial[blockIdx.x] = t;
  }
}

// ---------------------------------------------------------------- H_core and the pair table
// Pair table W, the resonance blocks of H and the core-core energy, one thread per pair; the
// electron-core blocks are summed per atom by core_atoms_kernel.
__global__ void __launch_bounds__(kBlock) core_pairs_kernel(Mol m, double* H, double* W, double* partial) {
  const long long np = pair_count(m.N);
  double ecc = 0.0;
  for (long long t = blockIdx.x * (long long)kBlock + threadIdx.x; t < np; t += (long long)gridDim.x * kBlock) {
    int u, v;
    pair_uv(m.N, (int)t, u, v);
    const ElemDev& eu = m.elem[m.z[u]];
    const ElemDev& ev = m.elem[m.z[v]];
    const bool hu = eu.norb == 4, hv = ev.norb == 4;
    const int a = (hu || !hv) ? u : v, b = a == u ? v : u;
    double* w = const_cast<double*>(pair_block(m, W, u, v));
    ecc += core_pair(m.elem[m.z[a]], m.elem[m.z[b]], eu, ev, *m.pairs, m.xyz + 3 * (size_t)a, m.xyz + 3 * (size_t)b,
                     m.ao[a], m.ao[b], (size_t)m.n, nullptr, nullptr, w, H);
  }
  block_partial(ecc, partial);
}
// Electron-core attraction blocks summed per atom (hamiltonian.rs:191-344): one warp per atom x,
// lanes over the partners y in a fixed order, so H_core does not depend on timing.
__global__ void __launch_bounds__(kBlock) core_atoms_kernel(Mol m, double* hacc) {
  const int lane = threadIdx.x & 31, x = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
  if (x >= m.N) return;  // whole warps
  const ElemDev& ex = m.elem[m.z[x]];
  const double* px = m.xyz + 3 * (size_t)x;
  double acc[10] = {};
  for (int y = lane; y < m.N; y += 32) {
    if (y == x) continue;
    const double* py = m.xyz + 3 * (size_t)y;
    const double d[3] = {py[0] - px[0], py[1] - px[1], py[2] - px[2]};
    const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const double dv[3] = {d[0] / r * r, d[1] / r * r, d[2] / r * r};  // as core_pair forms it
    double blk[10];
    core_attraction(ex, m.elem[m.z[y]], dv, blk);
#pragma unroll
    for (int k = 0; k < 10; ++k)
      if (k < (ex.norb == 4 ? 10 : 1)) acc[k] += blk[k];
  }
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    const double t = warp_sum(acc[k]);
    if (lane == 0) hacc[10 * (size_t)x + k] = t;
  }
}
// atom-diagonal blocks of H: U + the summed electron-core attractions
__global__ void __launch_bounds__(kBlock) core_diag_kernel(Mol m, const double* hacc, double* H) {
  for (int k = blockIdx.x * kBlock + threadIdx.x; k < m.N * 16; k += gridDim.x * kBlock) {
    const int a = k >> 4, mu = (k >> 2) & 3, nu = k & 3;
    const ElemDev& e = m.elem[m.z[a]];
    if (mu >= e.norb || nu >= e.norb) continue;
    double h = hacc[a * 10 + pk(mu, nu)];
    if (mu == nu) h += mu == 0 ? e.uss : e.upp;
    H[(size_t)(m.ao[a] + mu) * m.n + m.ao[a] + nu] = h;
  }
}
// SAD guess (scf.rs:855-881) into a zeroed P; `tilt` = atom of the symmetry-broken tilt or -1
__global__ void __launch_bounds__(kBlock) sad_kernel(Mol m, double* P, double scale, int tilt) {
  for (int a = blockIdx.x * kBlock + threadIdx.x; a < m.N; a += gridDim.x * kBlock) {
    const ElemDev& e = m.elem[m.z[a]];
    const int o = m.ao[a];
    P[(size_t)o * m.n + o] = e.occ_s * scale;
    if (e.norb == 4) {
      double pz = e.occ_p / 3.0;
      for (int k = 1; k < 4; ++k) P[(size_t)(o + k) * m.n + o + k] = pz * scale;
      if (a == tilt) {  // scf.rs:894-916: 0.2 e from pz to px on the most p-rich atom
        const double t = fmin(0.2, pz);
        P[(size_t)(o + 3) * m.n + o + 3] = (pz - t) * scale;
        P[(size_t)(o + 1) * m.n + o + 1] = (pz + t) * scale;
      }
    }
  }
}

// ---------------------------------------------------------------- Fock build
// packed atomic densities (fock.rs:93-100) and zeroed Coulomb accumulators
__global__ void __launch_bounds__(kBlock) pack_density_kernel(Mol m, const double* Pt, double* dpk, double* jacc) {
  for (int k = blockIdx.x * kBlock + threadIdx.x; k < m.N * 10; k += gridDim.x * kBlock) {
    const int a = k / 10, p = k % 10;
    const int no = m.elem[m.z[a]].norb;
    jacc[k] = 0.0;
    double v = 0.0;
    if (no == 4 || p == 0) {
      int hi, lo;
      unpk(p, hi, lo);
      const int oa = m.ao[a];
      v = Pt[(size_t)(oa + hi) * m.n + oa + lo];
      if (hi != lo) v *= 2.0;
    }
    dpk[k] = v;
  }
}
// Two-centre Coulomb sums of the Fock build, J_x[p] = sum_{y != x} sum_q (x p | y q) Pbar_y[q]
// (fock.rs:106-159), one warp per atom x, lanes over the partners in a fixed order (the pair
// kernel leaves them out), so the Fock matrix does not depend on timing. Pair blocks are stored
// in (a, b) orientation, a the atom with more orbitals (the first one on a tie).
__global__ void __launch_bounds__(kBlock) coulomb_atoms_kernel(Mol m, const double* W, const double* dpk, double* jacc) {
  const int lane = threadIdx.x & 31, x = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
  if (x >= m.N) return;  // whole warps
  const int sx = m.sprow[x + 1] - m.sprow[x];
  double acc[10] = {};
  for (int y = lane; y < m.N; y += 32) {
    if (y == x) continue;
    const int sy = m.sprow[y + 1] - m.sprow[y];
    const int u = min(x, y), v = max(x, y);
    const int su = u == x ? sx : sy, sv = u == x ? sy : sx;
    const bool x_rows = ((su == 10 || sv != 10) ? u : v) == x;  // x is the block's row atom
    const double* w = pair_block(m, W, u, v);
    const double* dy = dpk + 10 * (size_t)y;
#pragma unroll
    for (int p = 0; p < 10; ++p) {
      if (p >= sx) break;
      double t = 0.0;
#pragma unroll
      for (int q = 0; q < 10; ++q) {
        if (q >= sy) break;
        t = fma(dy[q], x_rows ? w[p * sy + q] : w[q * sx + p], t);
      }
      acc[p] += t;
    }
  }
#pragma unroll
  for (int p = 0; p < 10; ++p) {
    const double t = warp_sum(acc[p]);
    if (lane == 0 && p < sx) jacc[10 * (size_t)x + p] = t;
  }
}
template <bool UHF>
__global__ void __launch_bounds__(kBlock) fock_pairs_kernel(Mol m, const double* W, const double* H, const double* dpk,
                                                            double* jacc, const double* Pt, const double* Pa,
                                                            const double* Pb, double* F, double* G) {
  const long long np = pair_count(m.N);
  for (long long t = blockIdx.x * (long long)kBlock + threadIdx.x; t < np; t += (long long)gridDim.x * kBlock) {
    int u, v;
    pair_uv(m.N, (int)t, u, v);
    const int su = m.sprow[u + 1] - m.sprow[u], sv = m.sprow[v + 1] - m.sprow[v];
    const bool hu = su == 10, hv = sv == 10;
    const int a = (hu || !hv) ? u : v, b = a == u ? v : u;
    const double* w = pair_block(m, W, u, v);
    const int oa = m.ao[a], ob = m.ao[b];
    if (hu && hv) fock_pair<4, 4, UHF, false>(m.n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
    else if (hu || hv) fock_pair<4, 1, UHF, false>(m.n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
    else fock_pair<1, 1, UHF, false>(m.n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
  }
}
// atom-diagonal blocks: H + one-centre J - K + two-centre J
__global__ void __launch_bounds__(kBlock) fock_diag_kernel(Mol m, const double* H, const double* jacc, const double* Pt,
                                                           const double* Pa, const double* Pb, double* F, double* G) {
  const bool uhf = Pb != nullptr;
  for (int k = blockIdx.x * kBlock + threadIdx.x; k < m.N * 16; k += gridDim.x * kBlock) {
    const int a = k >> 4, mu = (k >> 2) & 3, nu = k & 3;
    const ElemDev& e = m.elem[m.z[a]];
    const int no = e.norb;
    if (mu >= no || nu >= no) continue;
    const int oa = m.ao[a];
    double ja = 0.0, ka = 0.0, kb = 0.0;
    for (int la = 0; la < no; ++la)
      for (int si = 0; si < no; ++si) {
        const double coul = oc_integral(e, mu, nu, la, si), exch = oc_integral(e, mu, la, nu, si);
        const size_t ix = (size_t)(oa + la) * m.n + oa + si;
        ja = fma(Pt[ix], coul, ja);
        if (uhf) {
          ka = fma(Pa[ix], exch, ka);
          kb = fma(Pb[ix], exch, kb);
        } else {
          ka = fma(0.5 * Pt[ix], exch, ka);
        }
      }
    const size_t ix = (size_t)(oa + mu) * m.n + oa + nu;
    const double base = H[ix] + jacc[a * 10 + pk(mu, nu)] + ja;
    F[ix] = base - ka;
    if (uhf) G[ix] = base - kb;
  }
}

// ---------------------------------------------------------------- elementwise helpers
// E <- E - E^T, zero diagonal (the commutator FP - PF from the product FP)
__global__ void __launch_bounds__(kBlock) antisym_kernel(double* E, int n) {
  const size_t nn = (size_t)n * n;
  for (size_t k = blockIdx.x * (size_t)kBlock + threadIdx.x; k < nn; k += (size_t)gridDim.x * kBlock) {
    const int i = (int)(k / n), j = (int)(k % n);
    if (j < i) {
      const double lo = E[k], up = E[(size_t)j * n + i];
      E[k] = lo - up;
      E[(size_t)j * n + i] = up - lo;
    } else if (j == i) {
      E[k] = 0.0;
    }
  }
}
// ---------------------------------------------------------------- split-BF16 products (mixed mode)
// x = hi + lo with hi = bf16(x) and lo = bf16(x - hi), both rounded to nearest even: 16
// significant bits, relative representation error <= 2^-17. A product a b is then taken as
// hi_a hi_b + hi_a lo_b + lo_a hi_b (each term exact in FP32, accumulated in FP32 on the tensor
// cores); the dropped lo_a lo_b term is 2^-16 of the product.
__global__ void __launch_bounds__(kBlock) split_bf16_kernel(const double* __restrict__ x, __nv_bfloat16* __restrict__ hi,
                                                            __nv_bfloat16* __restrict__ lo, size_t cnt) {
  for (size_t k = blockIdx.x * (size_t)kBlock + threadIdx.x; k < cnt; k += (size_t)gridDim.x * kBlock) {
    const double v = x[k];
    const __nv_bfloat16 h = __double2bfloat16(v);
    hi[k] = h;
    lo[k] = __double2bfloat16(v - (double)__bfloat162float(h));
  }
}
// The same split of a row-major rows x cols matrix (leading dimension ldx) into hi / lo copies with
// leading dimension ldo >= cols, the columns beyond cols zero (TMA wants 16-byte rows).
__global__ void __launch_bounds__(kBlock) split_pad_kernel(const double* __restrict__ x, int rows, int cols, int ldx,
                                                           __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo,
                                                           int ldo) {
  const size_t cnt = (size_t)rows * ldo;
  for (size_t k = blockIdx.x * (size_t)kBlock + threadIdx.x; k < cnt; k += (size_t)gridDim.x * kBlock) {
    const size_t r = k / ldo;
    const int c = (int)(k - r * ldo);
    const double v = c < cols ? x[r * ldx + c] : 0.0;
    const __nv_bfloat16 h = __double2bfloat16(v);
    hi[k] = h;
    lo[k] = __double2bfloat16(v - (double)__bfloat162float(h));
  }
}
// out[i][j] = a C[i][j] + b C[j][i] (row-major n x n, C in FP32, out in FP64): the commutator's
// antisymmetrisation (a = 1, b = -1) and the density's symmetrisation (a = b = w / 2). One block
// per 32 x 32 output tile; the mirrored tile is read through shared memory so both reads and the
// write are coalesced.
__global__ void __launch_bounds__(kBlock) transpose_combine_kernel(const float* __restrict__ C, double* __restrict__ out,
                                                                   int n, double a, double b) {
  __shared__ float t[32][33];
  const int tiles = (n + 31) / 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  for (int tile = blockIdx.x; tile < tiles * tiles; tile += gridDim.x) {
    const int i0 = (tile / tiles) * 32, j0 = (tile % tiles) * 32;
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {  // mirrored tile rows j0 + r, columns i0 + tx
      const int row = j0 + r, col = i0 + tx;
      t[r][tx] = (row < n && col < n) ? C[(size_t)row * n + col] : 0.0f;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
      const int row = i0 + r, col = j0 + tx;
      if (row < n && col < n)
        out[(size_t)row * n + col] = a * (double)C[(size_t)row * n + col] + b * (double)t[tx][r];
    }
  }
}

struct Comb {
  const double* m[8];
  double c[8];
  int len;
};
// out = sum_l c_l M_l (+ shift (I - Pproj) when shift != 0)
__global__ void __launch_bounds__(kBlock) combine_kernel(Comb cb, const double* Pproj, double shift, int n, double* out) {
  const size_t nn = (size_t)n * n;
  for (size_t k = blockIdx.x * (size_t)kBlock + threadIdx.x; k < nn; k += (size_t)gridDim.x * kBlock) {
    double v = 0.0;
    for (int l = 0; l < cb.len; ++l) v = fma(cb.c[l], cb.m[l][k], v);
    if (shift != 0.0) v += shift * (((k / n) == (k % n) ? 1.0 : 0.0) - Pproj[k]);
    out[k] = v;
  }
}
// P <- (1 - lam) Pn + lam P (damping, scf.rs:1440-1448); Pn kept
__global__ void __launch_bounds__(kBlock) damp_kernel(const double* Pn, double* P, double lam, size_t cnt) {
  for (size_t k = blockIdx.x * (size_t)kBlock + threadIdx.x; k < cnt; k += (size_t)gridDim.x * kBlock)
    P[k] = (1.0 - lam) * Pn[k] + lam * P[k];
}
__global__ void __launch_bounds__(kBlock) add_kernel(const double* a, const double* b, double* out, size_t cnt) {
  for (size_t k = blockIdx.x * (size_t)kBlock + threadIdx.x; k < cnt; k += (size_t)gridDim.x * kBlock)
    out[k] = a[k] + b[k];
}
// M = 1.5 I - 0.5 G (one Newton-Schulz step towards the orthogonal polar factor)
__global__ void __launch_bounds__(kBlock) ns_matrix_kernel(const double* G, double* M, int k) {
  const size_t kk = (size_t)k * k;
  for (size_t q = blockIdx.x * (size_t)kBlock + threadIdx.x; q < kk; q += (size_t)gridDim.x * kBlock)
    M[q] = ((q / k) == (q % k) ? 1.5 : 0.0) - 0.5 * G[q];
}
// max |G - I|
__global__ void __launch_bounds__(kBlock) orth_defect_kernel(const double* G, int k, double* partial) {
  const size_t kk = (size_t)k * k;
  double s = 0.0;
  for (size_t q = blockIdx.x * (size_t)kBlock + threadIdx.x; q < kk; q += (size_t)gridDim.x * kBlock) {
    const double v = fabs(G[q] - ((q / k) == (q % k) ? 1.0 : 0.0));
    s = v == v ? fmax(s, v) : INFINITY;  // fmax would drop a NaN
  }
  s = warp_max(s);
  __shared__ double red[kBlock / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < kBlock / 32; ++i) t = fmax(t, red[i]);
    partial[blockIdx.x] = t;
  }
}

// Eigen residual of k computed eigenpairs: per-block partial maxima of |Y - X diag(lam)| with
// Y = F X (row-major n x k each); NaN counts as infinite.
__global__ void __launch_bounds__(kBlock) eig_residual_kernel(const double* Y, const double* X, const double* lam,
                                                               int n, int k, double* partial) {
  const size_t nk = (size_t)n * k;
  double s = 0.0;
  for (size_t q = blockIdx.x * (size_t)kBlock + threadIdx.x; q < nk; q += (size_t)gridDim.x * kBlock) {
    const double v = fabs(Y[q] - X[q] * lam[q % k]);
    s = v == v ? fmax(s, v) : INFINITY;
  }
  s = warp_max(s);
  __shared__ double red[kBlock / 32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < kBlock / 32; ++i) t = fmax(t, red[i]);
    partial[blockIdx.x] = t;
  }
}

// ---------------------------------------------------------------- Householder tridiagonalisation
// Blocked lower reduction (the LAPACK sytrd/latrd scheme) of a full symmetric row-major A. For
// the panel starting at p, V and W (n x kPanel, row-major) hold the panel's reflectors and the
// vectors w_j such that the trailing matrix becomes A - V W^T - W V^T after the panel.
//
// Column i = p + j, step 1 (grid): bring row i (= column i below the diagonal: the trailing
// matrix is kept symmetric) up to date with the panel's earlier columns,
// a_r = A[i][r] - sum_{k<j} (V[r][k] W[i][k] + W[r][k] V[i][k]) for r >= i, in place, and the
// block partials of the reflector norm sum_{r >= i+2} a_r^2.
__global__ void __launch_bounds__(kBlock) panel_update_kernel(double* A, int n, int i, int j, const double* V,
                                                              const double* W, double* partial, unsigned int* counter,
                                                              double* d, double* e, double* tau, double* refl) {
  double* rowi = A + (size_t)i * n;
  const double* wi = W + (size_t)i * kPanel;
  const double* vi = V + (size_t)i * kPanel;
  double part = 0.0;
  for (int r = i + blockIdx.x * kBlock + threadIdx.x; r < n; r += gridDim.x * kBlock) {
    const double* vr = V + (size_t)r * kPanel;
    const double* wr = W + (size_t)r * kPanel;
    double a0 = rowi[r], a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int k = 0;
    for (; k + 3 < j; k += 4) {
      a0 -= vr[k] * wi[k] + wr[k] * vi[k];
      a1 -= vr[k + 1] * wi[k + 1] + wr[k + 1] * vi[k + 1];
      a2 -= vr[k + 2] * wi[k + 2] + wr[k + 2] * vi[k + 2];
      a3 -= vr[k + 3] * wi[k + 3] + wr[k + 3] * vi[k + 3];
    }
    for (; k < j; ++k) a0 -= vr[k] * wi[k] + wr[k] * vi[k];
    const double a = (a0 + a1) + (a2 + a3);
    rowi[r] = a;
    if (r >= i + 2) part = fma(a, a, part);
  }
  block_partial(part, partial);
  // the last block to finish forms the reflector scalars (no block waits for another)
  __threadfence();
  __shared__ bool last;
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  __shared__ double red[kBlock / 32];
  double x = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += kBlock) x += ((volatile double*)partial)[b];
  x = warp_sum(x);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    double xn2 = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) xn2 += red[w];
    const double alpha = ((volatile double*)rowi)[i + 1];
    double beta = alpha, tt = 0.0, sc = 0.0;
    if (xn2 > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
      tt = (beta - alpha) / beta;
      sc = 1.0 / (alpha - beta);
    }
    d[i] = ((volatile double*)rowi)[i];
    e[i] = beta;
    tau[i] = tt;
    refl[0] = sc;
    refl[1] = tt;
    *counter = 0u;
  }
}
// Symmetric GEMV over the lower triangle only (half the HBM traffic of a full GEMV): y = A22 v in
// 64 x 64 tiles (I >= J) of A22 = A[i+1.., i+1..]. A tile contributes the row sums A_IJ v_J to
// y_I and, off the diagonal, the column sums A_IJ^T v_I to y_J; both go to per-tile slots
// (64 + 64 values) that symv_gather adds up in a fixed order.
constexpr int kTile = 64;
__global__ void __launch_bounds__(kBlock) symv_tiles_kernel(const double* __restrict__ A, int n, int i,
                                                            const double* __restrict__ refl, double* tp) {
  const double* rowi = A + (size_t)i * n;
  const double scal = refl[0], t = refl[1];
  const int m = n - i - 1;
  const long long tidx = blockIdx.x;
  int I = (int)((sqrt(8.0 * (double)tidx + 1.0) - 1.0) * 0.5);
  while ((long long)(I + 1) * (I + 2) / 2 <= tidx) ++I;
  while ((long long)I * (I + 1) / 2 > tidx) --I;
  const int J = (int)(tidx - (long long)I * (I + 1) / 2);
  const double* aa = rowi + i + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c0 = J * kTile + lane, c1 = c0 + 32;
  auto vval = [&](int c) { return c == 0 ? 1.0 : aa[c] * scal; };
  const double vc0 = (t != 0.0 && c0 < m) ? vval(c0) : 0.0, vc1 = (t != 0.0 && c1 < m) ? vval(c1) : 0.0;
  double rs[kTile / 8];
  double col0 = 0.0, col1 = 0.0;
#pragma unroll
  for (int q = 0; q < kTile / 8; ++q) {
    const int rl = warp + 8 * q, r = I * kTile + rl;
    rs[q] = 0.0;
    if (r < m && t != 0.0) {
      const double* row = A + (size_t)(i + 1 + r) * n + i + 1;
      const double a0 = c0 < m ? row[c0] : 0.0, a1 = c1 < m ? row[c1] : 0.0;
      rs[q] = fma(a0, vc0, a1 * vc1);
      if (I != J) {
        const double vr = vval(r);
        col0 = fma(a0, vr, col0);
        col1 = fma(a1, vr, col1);
      }
    }
  }
  double* slot = tp + (size_t)tidx * (2 * kTile);
#pragma unroll
  for (int q = 0; q < kTile / 8; ++q) {
    const double v = warp_sum(rs[q]);
    if (lane == 0) slot[warp + 8 * q] = v;
  }
  __shared__ double cs[8][kTile];
  cs[warp][lane] = col0;
  cs[warp][lane + 32] = col1;
  __syncthreads();
  if (threadIdx.x < kTile) {
    double u = 0.0;
    for (int w = 0; w < 8; ++w) u += cs[w][threadIdx.x];
    slot[kTile + threadIdx.x] = u;
  }
}
// y_r = (row sums of stripe I over J <= I) + (column sums of the tiles below in column stripe I),
// one thread per r; then s1 = W[:, :j]^T v and s2 = V[:, :j]^T v (one warp per row, lane k
// accumulating component k) into block partials, which the last block to finish adds into s.
__global__ void __launch_bounds__(kBlock) symv_gather_kernel(const double* __restrict__ A, int n, int i, int j,
                                                             const double* __restrict__ V,
                                                             const double* __restrict__ W,
                                                             const double* __restrict__ refl, const double* tp,
                                                             double* y, double* partial_s, unsigned int* counter,
                                                             double* s) {
  const double* rowi = A + (size_t)i * n;
  const double scal = refl[0];
  const double xn2 = refl[1] != 0.0 ? 1.0 : 0.0;  // a reflection exists
  const int m = n - i - 1;
  const int nt = (m + kTile - 1) / kTile;
  const double* aa = rowi + i + 1;
  {  // y over one 64-row stripe per block iteration: the 8 warps split its nt tile slots
    __shared__ double ys[8][kTile];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int I = blockIdx.x; I < nt; I += gridDim.x) {
      const long long base = (long long)I * (I + 1) / 2;
      double y0 = 0.0, y1 = 0.0;
      for (int J = warp; J < nt; J += 8) {
        const size_t sl = J <= I ? (size_t)(base + J) * (2 * kTile) : (size_t)((long long)J * (J + 1) / 2 + I) * (2 * kTile) + kTile;
        y0 += tp[sl + lane];
        y1 += tp[sl + lane + 32];
      }
      ys[warp][lane] = y0;
      ys[warp][lane + 32] = y1;
      __syncthreads();
      if (threadIdx.x < kTile) {
        double u = 0.0;
        for (int w = 0; w < 8; ++w) u += ys[w][threadIdx.x];
        const int r = I * kTile + threadIdx.x;
        if (r < m) y[r] = u;
      }
      __syncthreads();
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double s1 = 0.0, s2 = 0.0;
  if (xn2 > 0.0 && lane < j)
    for (int rr = blockIdx.x * (kBlock / 32) + warp; rr < m; rr += gridDim.x * (kBlock / 32)) {
      const double vr = rr == 0 ? 1.0 : aa[rr] * scal;
      const size_t ix = (size_t)(i + 1 + rr) * kPanel + lane;
      s1 = fma(W[ix], vr, s1);
      s2 = fma(V[ix], vr, s2);
    }
  __shared__ double rs2[2][kBlock / 32][32];
  rs2[0][warp][lane] = s1;
  rs2[1][warp][lane] = s2;
  __syncthreads();
  if (threadIdx.x < 64) {
    const int which = threadIdx.x >> 5, k = threadIdx.x & 31;
    double u = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) u += rs2[which][w][k];
    partial_s[(size_t)blockIdx.x * 64 + threadIdx.x] = u;
  }
  // the last block to finish adds the block partials (no block waits for another)
  __threadfence();
  __shared__ bool last;
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last) {
    __threadfence();
    if (threadIdx.x < 64) {
      double u = 0.0;
      for (unsigned b = 0; b < gridDim.x; ++b) u += ((volatile double*)partial_s)[(size_t)b * 64 + threadIdx.x];
      s[threadIdx.x] = u;
    }
    if (threadIdx.x == 0) *counter = 0u;
  }
}
// Step 4 (grid): v into V[:, j], vcol and row i (the stored reflector, A[i][r] for r >= i+2);
// w = tau (y - V s1 - W s2) over rows > i; block partials of w . v.
__global__ void __launch_bounds__(kBlock) panel_wfix_kernel(double* A, int n, int i, int j, double* V, const double* W,
                                                            double* vcol, const double* y, const double* s,
                                                            const double* __restrict__ refl, double* wtmp,
                                                            double* partial) {
  double* rowi = A + (size_t)i * n;
  const double sc = refl[0], tt = refl[1];
  const int m = n - i - 1;
  double dp = 0.0;
  for (int rr = blockIdx.x * kBlock + threadIdx.x; rr < m; rr += gridDim.x * kBlock) {
    const size_t r = (size_t)(i + 1 + rr);
    const double v = tt == 0.0 ? 0.0 : (rr == 0 ? 1.0 : rowi[r] * sc);
    double w = 0.0;
    if (tt != 0.0) {
      const double* vr = V + r * kPanel;
      const double* wr = W + r * kPanel;
      double w0 = y[rr], w1 = 0.0, w2 = 0.0, w3 = 0.0;
      int k = 0;
      for (; k + 3 < j; k += 4) {
        w0 -= vr[k] * s[k] + wr[k] * s[32 + k];
        w1 -= vr[k + 1] * s[k + 1] + wr[k + 1] * s[33 + k];
        w2 -= vr[k + 2] * s[k + 2] + wr[k + 2] * s[34 + k];
        w3 -= vr[k + 3] * s[k + 3] + wr[k + 3] * s[35 + k];
      }
      for (; k < j; ++k) w0 -= vr[k] * s[k] + wr[k] * s[32 + k];
      w = tt * ((w0 + w1) + (w2 + w3));
    }
    wtmp[rr] = w;
    dp = fma(w, v, dp);
    V[r * kPanel + j] = v;
    vcol[r] = v;
    if (rr > 0) rowi[r] = v;
  }
  block_partial(dp, partial);
}
// Step 5 (grid): W[:, j] = w - (tau/2)(w . v) v over rows > i (zero above, as V[:, j])
__global__ void __launch_bounds__(kBlock) panel_wfinal_kernel(int n, int i, int j, const double* vcol, double* V,
                                                              double* W, const double* wtmp, const double* partial,
                                                              int np, const double* tau_i) {
  __shared__ double red[kBlock / 32];
  double t = 0.0;
  for (int b = threadIdx.x; b < np; b += kBlock) t += partial[b];
  t = warp_sum(t);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  double dotwv = 0.0;
  for (int w = 0; w < kBlock / 32; ++w) dotwv += red[w];
  const double a2 = -0.5 * (*tau_i) * dotwv;
  for (int r = blockIdx.x * kBlock + threadIdx.x; r < n; r += gridDim.x * kBlock) {
    double w = 0.0;
    if (r > i) w = wtmp[r - i - 1] + a2 * vcol[r];
    else V[(size_t)r * kPanel + j] = 0.0;
    W[(size_t)r * kPanel + j] = w;
  }
}
// The last 2 x 2 of the tridiagonal after the final trailing update.
__global__ void tail_kernel(const double* A, int n, double* d, double* e, double* tau) {
  if (n >= 2) {
    d[n - 2] = A[(size_t)(n - 2) * n + n - 2];
    e[n - 2] = A[(size_t)(n - 1) * n + n - 2];
    tau[n - 2] = 0.0;
  }
  d[n - 1] = A[(size_t)(n - 1) * n + n - 1];
  e[n - 1] = 0.0;
}
// Back-transformation blocks: kWy reflectors (four panels) per compact-WY block, so that its
// products are GEMMs 128 wide instead of 32.
constexpr int kWy = 4 * kPanel;
// V (n x kWy, row-major) of the reflectors [p, p + b): column k is reflector p + k (zero above row
// p + k + 1, one there, A's stored entries below); columns b .. kWy - 1 zero.
__global__ void __launch_bounds__(kBlock) block_v_kernel(const double* A, int n, int p, int b, double* V) {
  for (size_t q = blockIdx.x * (size_t)kBlock + threadIdx.x; q < (size_t)n * kWy; q += (size_t)gridDim.x * kBlock) {
    const int r = (int)(q / kWy), k = (int)(q % kWy);
    const int i = p + k;
    double v = 0.0;
    if (k < b) v = r <= i ? 0.0 : (r == i + 1 ? 1.0 : A[(size_t)i * n + r]);
    V[q] = v;
  }
}
// T (kWy x kWy, row-major, upper triangular) of H(p) ... H(p+b-1) = I - V T V^T from the Gram
// G = V^T V (b x b) and tau: T[k][k] = tau_k, T[m][k] = -tau_k sum_{m <= l < k} T[m][l] G[l][k].
// Row m depends only on its own earlier entries, so thread m forms row m alone (no barriers).
__global__ void __launch_bounds__(kWy) wy_t_block_kernel(const double* __restrict__ G, const double* __restrict__ tau,
                                                         int p, int b, double* __restrict__ T) {
  const int m = threadIdx.x;
  double* row = T + (size_t)m * kWy;
  for (int k = 0; k < kWy; ++k) row[k] = 0.0;
  if (m >= b) return;
  row[m] = tau[p + m];
  for (int k = m + 1; k < b; ++k) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int l = m;
    for (; l + 3 < k; l += 4) {
      a0 = fma(row[l], G[(size_t)l * b + k], a0);
      a1 = fma(row[l + 1], G[(size_t)(l + 1) * b + k], a1);
      a2 = fma(row[l + 2], G[(size_t)(l + 2) * b + k], a2);
      a3 = fma(row[l + 3], G[(size_t)(l + 3) * b + k], a3);
    }
    for (; l < k; ++l) a0 = fma(row[l], G[(size_t)l * b + k], a0);
    row[k] = -tau[p + k] * ((a0 + a1) + (a2 + a3));
  }
}

// ---------------------------------------------------------------- tridiagonal eigenproblem
// Lowest kval eigenvalues of T (d, e2 with splits already zeroed) by division-free multisection,
// a group of g lanes per eigenvalue (the per-CTA scheme of cta_eigen.cuh over a whole grid).
__global__ void __launch_bounds__(kBlock) multisect_kernel(const double* d, const double* e2, int n, int kval,
                                                           int g, double glo, double ghi, double pivmin, double tnorm,
                                                           const double* prev, const double* dprev, double* lam) {
  constexpr double eps = 2.220446049250313e-16;
  constexpr int kPts = 2;
  const int gt = blockIdx.x * kBlock + threadIdx.x;
  const int j = gt / g, gl = gt % g;
  const int lane = threadIdx.x & 31;
  const int gbase = lane & ~(g - 1);
  const unsigned gbits = g == 32 ? 0xffffffffu : ((1u << g) - 1u);
  const int P = g * kPts;
  const bool active = j < kval;
  double lo = glo, hi = ghi;
  if (prev) {
    const double c0 = active ? prev[j] : 0.0;
    const double w0 = active ? fmax(4.0 * fabs(dprev[j]), 1.0e-9 * fmax(tnorm, 1.0)) : 0.0;
    double x[4];
    int cn[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const double w = w0 * (t >= 2 ? 64.0 : 1.0);
      x[t] = (t & 1) ? fmin(c0 + w, ghi) : fmax(c0 - w, glo);
    }
    if (active) {
      sturm_multi<4>(d, e2, n, x, pivmin, cn);
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
  for (int it = 0; it < 160; ++it) {
    if (act) {
      const double mid = 0.5 * (lo + hi);
      if (hi - lo <= 2.0 * eps * fmax(fabs(lo), fabs(hi)) + 4.0 * pivmin || !(mid > lo && mid < hi)) act = false;
    }
    if (!__any_sync(0xffffffffu, act)) break;
    double x[kPts];
    int cn[kPts];
#pragma unroll
    for (int t = 0; t < kPts; ++t) x[t] = lo + (hi - lo) * (double)(gl * kPts + t + 1) / (double)(P + 1);
    if (act) sturm_multi<kPts>(d, e2, n, x, pivmin, cn);
    int tf = kPts;
#pragma unroll
    for (int t = kPts - 1; t >= 0; --t)
      if (act && cn[t] > j) tf = t;
    const unsigned bal = __ballot_sync(0xffffffffu, act && tf < kPts);
    const unsigned mine = (bal >> gbase) & gbits;
    const int src = mine ? gbase + __ffs(mine) - 1 : gbase;
    const int tsrc = __shfl_sync(0xffffffffu, tf, src);
    if (act) {
      double nlo, nhi;
      if (mine == 0u) {
        nlo = lo + (hi - lo) * (double)P / (double)(P + 1);
        nhi = hi;
      } else {
        const int f = (src - gbase) * kPts + tsrc;
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
  if (active && gl == 0) lam[j] = 0.5 * (lo + hi);
}
// Eigenvector j < kvec of T by twisted factorisation (thread per vector), written as column j of
// Y (n x kvec, row-major); zero outside the unreduced block that holds eigenvalue j. Scratch
// arrays are interleaved by vector (element i of vector j at i * kvec + j) so a warp's accesses
// coalesce. `blk` lists the nb + 1 block starts.
__global__ void __launch_bounds__(kBlock) twisted_kernel(const double* d, const double* e, const double* e2, int n,
                                                         int kvec, const double* lam, const int* blk, int nb,
                                                         double pivmin, double tnorm, double* Y, double* Dp, double* Lp,
                                                         double* Um) {
  const int j = blockIdx.x * kBlock + threadIdx.x;
  if (j >= kvec) return;
  const double lj = lam[j];
  const double win = 1.0e-11 * fmax(tnorm, 1.0);
  const size_t K = (size_t)kvec;
  // which unreduced block holds this eigenvalue (equal eigenvalues go to successive blocks)
  int pos = j - sturm(d, e2, 0, n - 1, lj - win, pivmin);
  int b = -1;
  for (int q = 0; q < nb && b < 0; ++q) {
    const int lo = blk[q], hi = blk[q + 1] - 1;
    const int cnt = sturm(d, e2, lo, hi, lj + win, pivmin) - sturm(d, e2, lo, hi, lj - win, pivmin);
    if (pos < cnt) b = q;
    else pos -= cnt;
  }
  if (b < 0) b = 0;
  const int lo = blk[b], hi = blk[b + 1] - 1, m = hi - lo + 1;
  for (int i = 0; i < n; ++i) Y[i * K + j] = 0.0;
  if (m == 1) {
    Y[(size_t)lo * K + j] = 1.0;
    return;
  }
  double dp = d[lo] - lj;
  for (int i = 0; i < m - 1; ++i) {
    if (fabs(dp) < pivmin) dp = dp < 0.0 ? -pivmin : pivmin;
    Dp[(lo + i) * K + j] = dp;
    const double ei = e[lo + i];
    const double l = ei / dp;
    Lp[(lo + i) * K + j] = l;
    dp = (d[lo + i + 1] - lj) - l * ei;
  }
  if (fabs(dp) < pivmin) dp = dp < 0.0 ? -pivmin : pivmin;
  Dp[(size_t)hi * K + j] = dp;
  double dm = d[hi] - lj;
  if (fabs(dm) < pivmin) dm = dm < 0.0 ? -pivmin : pivmin;
  double best = fabs(Dp[(size_t)hi * K + j] + dm - (d[hi] - lj));
  int r = m - 1;
  for (int i = m - 2; i >= 0; --i) {
    const double ei = e[lo + i];
    const double u = ei / dm;
    Um[(lo + i) * K + j] = u;
    dm = (d[lo + i] - lj) - u * ei;
    if (fabs(dm) < pivmin) dm = dm < 0.0 ? -pivmin : pivmin;
    const double gm = fabs(Dp[(lo + i) * K + j] + dm - (d[lo + i] - lj));
    if (gm < best) {
      best = gm;
      r = i;
    }
  }
  // N_r D_r N_r^T y = gamma_r e_r
  double ynext = 1.0, ynext2 = 0.0;  // y[i+1], y[i+2] going up
  double yrm1 = 0.0;                 // y[r-1], seeds the downward sweep
  Y[(size_t)(lo + r) * K + j] = 1.0;
  double nrm = 1.0;
  for (int i = r - 1; i >= 0; --i) {
    double zv = -Lp[(lo + i) * K + j] * ynext;
    if (ynext == 0.0 && i + 2 < m) zv = -(e[lo + i + 1] / e[lo + i]) * ynext2;
    Y[(size_t)(lo + i) * K + j] = zv;
    nrm = fma(zv, zv, nrm);
    if (i == r - 1) yrm1 = zv;
    ynext2 = ynext;
    ynext = zv;
  }
  double yprev = 1.0, yprev2 = yrm1;  // y[i], y[i-1] going down
  for (int i = r; i < m - 1; ++i) {
    double zv = -Um[(lo + i) * K + j] * yprev;
    if (yprev == 0.0 && i >= 1) zv = -(e[lo + i - 1] / e[lo + i]) * yprev2;
    Y[(size_t)(lo + i + 1) * K + j] = zv;
    nrm = fma(zv, zv, nrm);
    yprev2 = yprev;
    yprev = zv;
  }
  const double sc = 1.0 / sqrt(nrm);
  for (int i = lo; i <= hi; ++i) Y[(size_t)i * K + j] *= sc;
}

// ---------------------------------------------------------------- properties
// per-atom diagonal density blocks (16 per atom, row-major 4 x 4) for charges and dipole
__global__ void __launch_bounds__(kBlock) atom_blocks_kernel(Mol m, const double* P, double* out) {
  for (int k = blockIdx.x * kBlock + threadIdx.x; k < m.N * 16; k += gridDim.x * kBlock) {
    const int a = k >> 4, mu = (k >> 2) & 3, nu = k & 3;
    const int no = m.elem[m.z[a]].norb;
    out[k] = (mu < no && nu < no) ? P[(size_t)(m.ao[a] + mu) * m.n + m.ao[a] + nu] : 0.0;
  }
}

}  // namespace large
}  // namespace pm3gpu
