// Grimme D3 dispersion (zero damping, coordination-number-interpolated C6) for a batch of molecules:
// the post-SCF classical correction of PM3-D3 (pm3-rs src/corrections/d3.rs:360-458 energy,
// src/corrections/mod.rs:129-160 variant selection, src/scf.rs:740-743 where it joins the total
// energy, src/gradient.rs:324-357 where its gradient joins the SCF gradient). Included by pm3gpu.cu
// inside its private namespace, before run_batch.
//
// Layout: one thread per atom of the batch, looping over the other atoms of its molecule (found by
// a binary search over the molecule offsets), in three passes that only gather:
//   1. coordination numbers  cn_i = sum_j 1 / (1 + exp(-16 (rco_ij / r_ij - 1)))       (k1 = 16)
//   2. the ordered pair sum E = -1/2 Eh sum_i sum_{j != i} C6_ij (s6 f6 / r^6 + s8 q_ij f8 / r^8),
//      its derivative with respect to cn_i and the direct (fixed-cn) gradient on atom i
//   3. the chain through the coordination numbers, (dE/dcn_i + dE/dcn_j) dcn/dr_ij per pair
// and a per-molecule sum of the row energies. C6_ij is the Gaussian-weighted average of the
// element pair's reference C6 values (k3 = -4) over (cn of the higher-Z atom, cn of the lower-Z
// atom), in the order the reference's table lists them; for two atoms of one element the ordered
// pairs (i, j) and (j, i) can differ, so both are evaluated, as the reference's ordered loop does.
// Derivatives are analytic: f = 1 / (1 + u), u = 6 (rs R0 / r)^alpha gives
// d(f / r^n)/dr = f / r^(n+1) (alpha u f - n), and dC6/dcn follows from the quotient rule on the
// weights. Every sum is in FP64 and runs in a fixed order, so the result is deterministic. The pair
// loops touch each molecule's coordinates from L1; per atom the work is O(n) and the whole
// correction is a few microseconds for the batches the SCF solves in milliseconds. The host side
// (buffers, launches, the variant's sum) is corrections.cuh.
#pragma once
#include "pm3_d3_table.h"

namespace d3k {

constexpr double kA0 = 0.529177210903;   // BOHR_TO_ANGSTROM
constexpr double kEh = 27.211386245988;  // HARTREE_TO_EV

struct Tables {
  double r2r4[PM3_D3_NELEM], rcov[PM3_D3_NELEM], r0ab[PM3_D3_NELEM][PM3_D3_NELEM];
  double ref[PM3_D3_NREF][3];
  int off[PM3_D3_NPAIR + 1];
  signed char idx[128];
};
__device__ Tables g_tab;

// D3Params::pm3_d3 (set 1) and D3Params::pm3_d3h4 (set 2), d3.rs:36-60
struct Params {
  double s6, s8, rs6, rs8, alp6, alp8;
};
__host__ __device__ inline Params params_of(int set) {
  if (set == 1) return {1.0, 0.612, 1.345, 1.0, 14.0, 16.0};
  return {1.0, 0.0, 0.90, 1.0e-10, 22.0, 24.0};
}

// The reference's load-time transforms (d3.rs:84-158).
inline void host_tables(Tables& t) {
  for (signed char& v : t.idx) v = -1;
  for (int e = 0; e < PM3_D3_NELEM; ++e) {
    const int z = pm3_d3_z[e];
    t.idx[z] = (signed char)e;
    t.r2r4[e] = std::sqrt(0.5 * pm3_d3_r2r4_raw[e] * std::sqrt((double)z));
    t.rcov[e] = 4.0 / 3.0 * pm3_d3_rcov_raw[e] / kA0;
    for (int f = 0; f < PM3_D3_NELEM; ++f) t.r0ab[e][f] = pm3_d3_r0ab_ang[e][f] / kA0;
  }
  for (int k = 0; k < PM3_D3_NREF; ++k)
    for (int c = 0; c < 3; ++c) t.ref[k][c] = pm3_d3_ref[k][c];
  for (int p = 0; p <= PM3_D3_NPAIR; ++p) t.off[p] = pm3_d3_pair_off[p];
}

__device__ __forceinline__ int mol_of(const int32_t* offs, int n_mol, int t) {
  int lo = 0, hi = n_mol;  // offs[lo] <= t < offs[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (offs[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int elem_of(int z) { return (z > 0 && z < 128) ? g_tab.idx[z] : -1; }

// getc6 (d3.rs:212-236) for the ordered pair (i, j), with its derivatives by cn_i and cn_j.
__device__ inline void c6_of(int ei, int ej, double cni, double cnj, double& c6, double& dci, double& dcj) {
  const bool sw = ei < ej;
  const int a = sw ? ej : ei, b = sw ? ei : ej;
  const int p = a * (a + 1) / 2 + b;
  const double ca = sw ? cnj : cni, cb = sw ? cni : cnj;
  double num = 0.0, den = 0.0, na = 0.0, nb = 0.0, da_ = 0.0, db_ = 0.0;
  for (int k = g_tab.off[p]; k < g_tab.off[p + 1]; ++k) {
    const double c = g_tab.ref[k][0];
    const double da = ca - g_tab.ref[k][1];
    const double db = cb - g_tab.ref[k][2];
    const double t = exp((da * da + db * db) * -4.0);
    num = num + t * c;
    den = den + t;
    const double ta = -8.0 * da * t, tb = -8.0 * db * t;
    na += ta * c;
    nb += tb * c;
    da_ += ta;
    db_ += tb;
  }
  if (den > 0.0) {
    c6 = num / den;
    const double dA = (na - c6 * da_) / den, dB = (nb - c6 * db_) / den;
    dci = sw ? dB : dA;
    dcj = sw ? dA : dB;
  } else {
    c6 = dci = dcj = 0.0;
  }
}

__global__ void __launch_bounds__(128) cn_kernel(int total, int n_mol, const int32_t* __restrict__ offs,
                                                 const int32_t* __restrict__ set, const int32_t* __restrict__ z,
                                                 const double* __restrict__ xyz, double* __restrict__ cn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int m = mol_of(offs, n_mol, i);
  if (!set[m]) return;
  const int ei = elem_of(z[i]);
  double acc = 0.0;
  if (ei >= 0) {
    const double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
    for (int j = offs[m]; j < offs[m + 1]; ++j) {
      const int ej = elem_of(z[j]);
      if (j == i || ej < 0) continue;
      const double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      const double rco = g_tab.rcov[ei] + g_tab.rcov[ej];
      acc = acc + 1.0 / (exp((1.0 / r * rco - 1.0) * -16.0) + 1.0);
    }
  }
  cn[i] = acc;
}

__global__ void __launch_bounds__(128) pair_kernel(int total, int n_mol, const int32_t* __restrict__ offs,
                                                   const int32_t* __restrict__ set, const int32_t* __restrict__ z,
                                                   const double* __restrict__ xyz, const double* __restrict__ cn,
                                                   double* __restrict__ e6row, double* __restrict__ e8row,
                                                   double* __restrict__ dedcn, double* __restrict__ gdir, int want_grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int m = mol_of(offs, n_mol, i);
  if (!set[m]) return;
  const Params P = params_of(set[m]);
  const int ei = elem_of(z[i]);
  double e6 = 0.0, e8 = 0.0, de = 0.0, g[3] = {0.0, 0.0, 0.0};
  if (ei >= 0) {
    const double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
    const double cni = cn[i];
    for (int j = offs[m]; j < offs[m + 1]; ++j) {
      const int ej = elem_of(z[j]);
      if (j == i || ej < 0) continue;
      const double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      const double r2 = r * r;
      const double r6 = r2 * r2 * r2;
      const double r8 = r6 * r2;
      const double cnj = cn[j];
      double cij, aij, bij;
      c6_of(ei, ej, cni, cnj, cij, aij, bij);
      const double q = 3.0 * g_tab.r2r4[ei] * g_tab.r2r4[ej];
      const double rr = 1.0 / r * g_tab.r0ab[ei][ej];
      const double u6 = pow(rr * P.rs6, P.alp6) * 6.0, u8 = pow(rr * P.rs8, P.alp8) * 6.0;
      const double f6 = 1.0 / (u6 + 1.0), f8 = 1.0 / (u8 + 1.0);
      e6 = e6 + cij * f6 / r6;
      e8 = e8 + cij * q * f8 / r8;
      if (want_grad) {
        double cji = cij, bji = aij;  // (j, i): same key and oriented cn unless one element
        if (ei == ej) {
          double aji;
          c6_of(ej, ei, cnj, cni, cji, aji, bji);
        }
        const double w = P.s6 * f6 / r6 + P.s8 * q * f8 / r8;
        de += w * (aij + bji);
        const double d6 = f6 / (r6 * r) * (P.alp6 * u6 * f6 - 6.0);
        const double d8 = f8 / (r8 * r) * (P.alp8 * u8 * f8 - 8.0);
        const double dh = (cij + cji) * (P.s6 * d6 + P.s8 * q * d8) / r;
        g[0] -= dh * dx;
        g[1] -= dh * dy;
        g[2] -= dh * dz;
      }
    }
  }
  e6row[i] = e6;
  e8row[i] = e8;
  if (want_grad) {
    const double k = -0.5 * kEh;
    dedcn[i] = k * de;
    for (int c = 0; c < 3; ++c) gdir[3 * i + c] = k * g[c];
  }
}

__global__ void __launch_bounds__(128) chain_kernel(int total, int n_mol, const int32_t* __restrict__ offs,
                                                    const int32_t* __restrict__ set, const int32_t* __restrict__ z,
                                                    const double* __restrict__ xyz, const double* __restrict__ dedcn,
                                                    const double* __restrict__ gdir, double* __restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int m = mol_of(offs, n_mol, i);
  if (!set[m]) return;
  const int ei = elem_of(z[i]);
  double g[3] = {gdir[3 * i], gdir[3 * i + 1], gdir[3 * i + 2]};
  if (ei >= 0) {
    const double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
    const double di = dedcn[i];
    for (int j = offs[m]; j < offs[m + 1]; ++j) {
      const int ej = elem_of(z[j]);
      if (j == i || ej < 0) continue;
      const double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      const double rco = g_tab.rcov[ei] + g_tab.rcov[ej];
      const double e = exp((1.0 / r * rco - 1.0) * -16.0);
      const double s = 1.0 / (e + 1.0);
      const double ds = -16.0 * rco * e * s * s / (r * r);  // d s / d r
      const double f = (di + dedcn[j]) * ds / r;
      g[0] -= f * dx;
      g[1] -= f * dy;
      g[2] -= f * dz;
    }
  }
  for (int c = 0; c < 3; ++c) grad[3 * i + c] = g[c];
}

__global__ void energy_kernel(int n_mol, const int32_t* __restrict__ offs, const int32_t* __restrict__ set,
                              const double* __restrict__ e6row, const double* __restrict__ e8row,
                              double* __restrict__ energy) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n_mol || !set[m]) return;
  const Params P = params_of(set[m]);
  double e6 = 0.0, e8 = 0.0;
  for (int i = offs[m]; i < offs[m + 1]; ++i) {
    e6 += e6row[i];
    e8 += e8row[i];
  }
  energy[m] = -(e6 * P.s6 + e8 * P.s8) * (0.5 * kEh);
}

}  // namespace d3k

// The D3 tables in each device's memory, uploaded once per device. The device must be current.
cudaError_t d3_ready(int device) {
  static std::mutex mu;
  static std::vector<char> done;
  std::lock_guard<std::mutex> lk(mu);
  if (device < 0) return cudaErrorInvalidDevice;
  if ((int)done.size() <= device) done.resize(device + 1, 0);
  if (done[device]) return cudaSuccess;
  static d3k::Tables host;
  d3k::host_tables(host);
  const cudaError_t e = cudaMemcpyToSymbol(d3k::g_tab, &host, sizeof(host));
  if (e == cudaSuccess) done[device] = 1;
  return e;
}
