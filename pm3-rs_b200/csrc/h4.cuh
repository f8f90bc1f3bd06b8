// The H4 hydrogen-bond correction, the H-H repulsion and the halogen-bond (X) correction of the
// PM3-D3H4 family for a batch of molecules (pm3-rs src/corrections/h4.rs:243-387 and
// src/corrections/hx.rs:64-88; combined per variant as src/corrections/mod.rs:129-160). Included by
// pm3gpu.cu inside its private namespace, after d3.cuh.
//
// One CTA per molecule, three phases separated by barriers:
//   A. per atom a: its covalent valence V_a = sum_k cval(a, k) (the C^2 seventh-order switch between
//      the covalent-radius sum r0 and 1.6 r0), for N and O its hydrogen and non-hydrogen parts, and
//      from them the scale factors a triple uses with their derivatives by those sums: the water
//      factor of an O donor, the NR4+ factor of an N donor, the carboxylate factor of an O acceptor
//      (its nearest bonded carbon and that carbon's other oxygen found as the reference finds them);
//   B. every N/O pair closer than 5.5 Angstrom against the hydrogens within the 1.15 Angstrom donor
//      bond of either (the only ones a triple can count): the triple value
//      e_radial(R_DA) e_angular(pi - angle DHA) s_water s_NR4 s_COO e_para, its direct gradient on
//      D, A and H, and the adjoints of the valence sums it read (FP64 atomics);
//   C. per atom: the chain through the valence switches (gathered, each pair once per side), the
//      H-H repulsion rows and the Cl-to-N/O halogen-bond rows with their gradients.
// Units follow the reference: distances in Angstrom inside the terms, energies in kcal/mol until
// the final KCAL_TO_EV. The derivative rules at the branch points are those of the reference's
// dual numbers (src/dual.rs): |x| takes +1 at 0, acos has zero derivative where 1 - c^2 <= 1e-14,
// a clamped cosine and a branch on a value carry no derivative.
#pragma once

namespace h4k {

constexpr double kA0 = 0.529177210903;
constexpr double kKcal = 1.0 / 23.06054783061903;  // KCAL_TO_EV
constexpr double kPi = 3.14159265358979323846;
constexpr int kThreads = 256;

// covalent radii (Angstrom) of elements 1..17 (h4.rs:81-89, MOPAC radii_C)
__constant__ double c_cov[17] = {0.37, 0.32, 1.34, 0.90, 0.82, 0.77, 0.75, 0.73, 0.71,
                                 0.69, 1.54, 1.30, 1.18, 1.11, 1.06, 1.02, 0.99};
__device__ __forceinline__ double cov(int z) { return (z >= 1 && z <= 17) ? c_cov[z - 1] : 0.0; }

// Per-atom scratch, indexed by the atom's position in the batch.
struct Scratch {
  double *V, *Hs, *Os;                        // valence sums
  double *sw, *swH, *swO;                     // water factor of an O donor and its derivatives
  double *chd, *chdV;                         // NR4+ factor of an N donor
  double *cha, *chaO1, *chaCC, *chaO2;        // carboxylate factor of an O acceptor
  int *cc, *o2;                               // its carbon and second oxygen (-1: none)
  double *adjH, *adjO, *adjV;                 // dE/d(valence sums), kcal/mol
  double* gB;                                 // phase-B gradient, kcal/mol/Bohr
};

// 1 - (35 x^4 - 84 x^5 + 70 x^6 - 20 x^7) and its derivative
__device__ __forceinline__ void switch7(double x, double& v, double& dv) {
  const double x2 = x * x, x3 = x2 * x, x4 = x2 * x2, x5 = x4 * x, x6 = x4 * x2, x7 = x6 * x;
  v = -(x7 * -20.0 + x6 * 70.0 + x5 * -84.0 + x4 * 35.0) + 1.0;
  dv = -(x6 * -140.0 + x5 * 420.0 + x4 * -420.0 + x3 * 140.0);
}

// cvalence_contribution_g (h4.rs:128-143) at distance r (Angstrom), with d/dr
__device__ __forceinline__ void cval(int za, int zb, double r, double& v, double& dv) {
  const double r0 = cov(za) + cov(zb);
  const double r1 = r0 * 1.6;
  if (r == 0.0 || r >= r1) {
    v = dv = 0.0;
  } else if (r <= r0) {
    v = 1.0;
    dv = 0.0;
  } else {
    double s, ds;
    switch7((r - r0) / (r1 - r0), s, ds);
    v = s;
    dv = ds / (r1 - r0);
  }
}

__device__ __forceinline__ double dist_b(const double* xyz, int a, int b) {
  const double dx = xyz[3 * a] - xyz[3 * b], dy = xyz[3 * a + 1] - xyz[3 * b + 1], dz = xyz[3 * a + 2] - xyz[3 * b + 2];
  return sqrt(dx * dx + dy * dy + dz * dz);
}

// f_dev (h4.rs:43-50): 1 - |cv - t| inside 1, else 0; derivative by cv
__device__ __forceinline__ void f_dev(double cv, double t, double& f, double& df) {
  const double u = cv - t;
  const double dev = u >= 0.0 ? u : -u;
  if (dev < 1.0) {
    f = 1.0 - dev;
    df = u >= 0.0 ? -1.0 : 1.0;
  } else {
    f = df = 0.0;
  }
}

__device__ __forceinline__ double e_para(int d, int a) {
  if (d == 8 && a == 8) return 2.71;
  if (d == 8 && a == 7) return 4.37;
  if (d == 7 && a == 8) return 2.29;
  if (d == 7 && a == 7) return 3.86;
  return 0.0;
}

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < kThreads / 32; ++k) s += red[k];
  return s;  // valid on thread 0
}

// grid: one CTA per entry of mols; variant[m] >= 2 (H4 + H-H), 3 adds X. energy[3 m + {0,1,2}]
// receives (H4, H-H, X) in eV, grad[3 atom] the gradient of their sum in eV/Bohr (overwritten).
__global__ void __launch_bounds__(kThreads) h4_kernel(const int32_t* __restrict__ mols, const int32_t* __restrict__ offs,
                                                      const int32_t* __restrict__ variant,
                                                      const int32_t* __restrict__ z,
                                                      const double* __restrict__ xyz, Scratch S,
                                                      double* __restrict__ energy, double* __restrict__ grad) {
  __shared__ double red[kThreads / 32];
  const int m = mols[blockIdx.x];
  const int a0 = offs[m], a1 = offs[m + 1];
  const int var = variant[m];
  const double cut_dh2 = (1.15 / kA0) * (1.15 / kA0);

  // ---------------------------------------------------------------- A. valence sums, scale factors
  for (int a = a0 + threadIdx.x; a < a1; a += kThreads) {
    const int za = z[a];
    double V = 0.0, Hs = 0.0, Os = 0.0, cdist = INFINITY;
    int cc = -1;
    for (int k = a0; k < a1; ++k) {
      double v, dv;
      const double r = dist_b(xyz, a, k) * kA0;
      cval(za, z[k], r, v, dv);
      V = V + v;
      if (z[k] == 1) Hs = Hs + v;
      else Os = Os + v;
      if (za == 8 && v > 0.0 && z[k] == 6 && r < cdist) {
        cdist = r;
        cc = k;
      }
    }
    S.V[a] = V;
    S.Hs[a] = Hs;
    S.Os[a] = Os;
    // water factor (h4.rs:146-180), O donors
    double sw = 1.0, swH = 0.0, swO = 0.0;
    if (za == 8 && Hs >= 1.0) {
      const double slope = 0.91 - 1.0;
      double fv = 0.0, dfv = 0.0;
      if (Hs > 1.0 && Hs <= 2.0) {
        fv = Hs - 1.0;
        dfv = 1.0;
      } else if (Hs > 2.0 && Hs < 3.0) {
        fv = -Hs + 3.0;
        dfv = -1.0;
      }
      const bool on = (1.0 - Os) > 0.0;
      const double fv2 = on ? -Os + 1.0 : 0.0, dfv2 = on ? -1.0 : 0.0;
      sw = fv * fv2 * slope + 1.0;
      swH = dfv * fv2 * slope;
      swO = fv * dfv2 * slope;
    }
    S.sw[a] = sw;
    S.swH[a] = swH;
    S.swO[a] = swO;
    // NR4+ factor (h4.rs:183-193), N donors
    const bool nr4 = za == 7 && V > 3.0;
    S.chd[a] = nr4 ? (V - 3.0) * (2.5390633931627 - 1.0) + 1.0 : 1.0;
    S.chdV[a] = nr4 ? 2.5390633931627 - 1.0 : 0.0;
    // carboxylate factor (h4.rs:196-240), O acceptors
    double cha = 1.0, dO1 = 0.0, dCC = 0.0, dO2 = 0.0;
    int o2 = -1;
    if (za == 8 && cc >= 0) {
      double cvcc = 0.0, odist = INFINITY;
      for (int k = a0; k < a1; ++k) {
        double v, dv;
        const double r = dist_b(xyz, cc, k) * kA0;
        cval(z[cc], z[k], r, v, dv);
        cvcc = cvcc + v;
        if (v > 0.0 && k != a && z[k] == 8 && r < odist) {
          odist = r;
          o2 = k;
        }
      }
      if (o2 >= 0) {
        double cvo2 = 0.0;
        for (int k = a0; k < a1; ++k) {
          double v, dv;
          cval(z[o2], z[k], dist_b(xyz, o2, k) * kA0, v, dv);
          cvo2 = cvo2 + v;
        }
        double f1, d1, f2, d2, f3, d3;
        f_dev(V, 1.0, f1, d1);
        f_dev(cvo2, 1.0, f2, d2);
        f_dev(cvcc, 3.0, f3, d3);
        const double mc = 0.88610264413703 - 1.0;
        cha = f1 * f2 * f3 * mc + 1.0;
        dO1 = d1 * f2 * f3 * mc;
        dO2 = f1 * d2 * f3 * mc;
        dCC = f1 * f2 * d3 * mc;
      }
    }
    S.cha[a] = cha;
    S.chaO1[a] = dO1;
    S.chaCC[a] = dCC;
    S.chaO2[a] = dO2;
    S.cc[a] = (o2 >= 0) ? cc : -1;
    S.o2[a] = o2;
    S.adjH[a] = S.adjO[a] = S.adjV[a] = 0.0;
    S.gB[3 * a] = S.gB[3 * a + 1] = S.gB[3 * a + 2] = 0.0;
  }
  __syncthreads();

  // ---------------------------------------------------------------- B. donor-hydrogen-acceptor triples
  double eh4 = 0.0;
  for (int i = a0 + threadIdx.x; i < a1; i += kThreads) {
    const int zi = z[i];
    if (zi != 7 && zi != 8) continue;
    for (int j = i + 1; j < a1; ++j) {
      const int zj = z[j];
      if (zj != 7 && zj != 8) continue;
      const double dxa = xyz[3 * j] - xyz[3 * i], dya = xyz[3 * j + 1] - xyz[3 * i + 1], dza = xyz[3 * j + 2] - xyz[3 * i + 2];
      const double rij = sqrt(dxa * dxa + dya * dya + dza * dza);
      const double rda = rij * kA0;
      if (rda >= 5.5) continue;
      for (int h = a0; h < a1; ++h) {
        if (z[h] != 1) continue;
        double u[3], w[3];
        for (int c = 0; c < 3; ++c) {
          u[c] = xyz[3 * i + c] - xyz[3 * h + c];
          w[c] = xyz[3 * j + c] - xyz[3 * h + c];
        }
        const double ru2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        const double rw2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
        if (ru2 >= cut_dh2 && rw2 >= cut_dh2) continue;  // no donor bond: the triple cannot count
        const double rih = sqrt(ru2), rjh = sqrt(rw2);
        const double cs = (u[0] * w[0] + u[1] * w[1] + u[2] * w[2]) / (rih * rjh);
        const bool clamped = cs >= 1.0 || cs <= -1.0;
        const double cl = cs >= 1.0 ? 1.0 : (cs <= -1.0 ? -1.0 : cs);
        const double angle = -acos(cl) + kPi;
        if (angle >= kPi / 2.0) continue;
        const bool idon = rih < rjh;
        const int d = idon ? i : j, ac = idon ? j : i;
        const double rdh = (idon ? rih : rjh) * kA0;
        if (rdh >= 1.15) continue;
        const double ep = e_para(z[d], z[ac]);
        if (ep == 0.0) continue;
        // radial polynomial and its derivative (h4.rs:97-106)
        const double r1 = rda, r2 = r1 * r1, r3 = r2 * r1, r4 = r2 * r2, r5 = r4 * r1, r6 = r4 * r2, r7 = r6 * r1;
        const double rad = r7 * -0.003034074074073135 + r6 * 0.07357629629627092 + r5 * -0.700871111110828 +
                           r4 * 3.2530962962946175 + r3 * -7.206874074068388 + r2 * 5.317546666655722 +
                           r1 * 3.407360000011028 - 4.685120000004504;
        const double drad = r6 * (7 * -0.003034074074073135) + r5 * (6 * 0.07357629629627092) +
                            r4 * (5 * -0.700871111110828) + r3 * (4 * 3.2530962962946175) +
                            r2 * (3 * -7.206874074068388) + r1 * (2 * 5.317546666655722) + 3.407360000011028;
        // angular term (h4.rs:109-113)
        const double aa = angle * (1.0 / (kPi / 2.0));
        const double a2 = aa * aa, a3 = a2 * aa, a4 = a2 * a2, a5 = a4 * aa, a6 = a4 * a2, a7 = a6 * aa;
        const double X = a7 * -20.0 + a6 * 70.0 + a5 * -84.0 + a4 * 35.0;
        const double dX = a6 * -140.0 + a5 * 420.0 + a4 * -420.0 + a3 * 140.0;
        const double ang = -(X * X) + 1.0;
        const double dang = -2.0 * X * dX * (1.0 / (kPi / 2.0));  // d ang / d angle
        const double one_m = 1.0 - cl * cl;
        const double dangle = (!clamped && one_m > 1.0e-14) ? 1.0 / sqrt(one_m) : 0.0;  // d angle / d cos
        const bool wat = z[d] == 8 && z[ac] == 8;
        const double sw = wat ? S.sw[d] : 1.0;
        const double chd = S.chd[d], cha = S.cha[ac];
        const double T = rad * ang * 1.0 * sw * chd * cha * ep;
        eh4 += T;
        // direct gradient: R_DA on i, j; the cosine on i, j, h
        const double f = sw * chd * cha * ep;
        const double gr = drad * ang * f * kA0 / rij;  // times (x_i - x_j) on i
        const double gc = rad * dang * dangle * f;
        const double inv = 1.0 / (rih * rjh);
        double gi[3], gj[3];
        for (int c = 0; c < 3; ++c) {
          const double du = w[c] * inv - cs * u[c] / ru2;  // d cos / d u
          const double dw = u[c] * inv - cs * w[c] / rw2;  // d cos / d w
          const double dr = (c == 0 ? dxa : c == 1 ? dya : dza);
          gi[c] = gc * du - gr * dr;
          gj[c] = gc * dw + gr * dr;
          atomicAdd(&S.gB[3 * h + c], -gc * (du + dw));
        }
        for (int c = 0; c < 3; ++c) {
          atomicAdd(&S.gB[3 * i + c], gi[c]);
          atomicAdd(&S.gB[3 * j + c], gj[c]);
        }
        // adjoints of the valence sums behind the scale factors
        const double P = rad * ang * ep;
        if (wat) {
          atomicAdd(&S.adjH[d], P * chd * cha * S.swH[d]);
          atomicAdd(&S.adjO[d], P * chd * cha * S.swO[d]);
        }
        if (S.chdV[d] != 0.0) atomicAdd(&S.adjV[d], P * sw * cha * S.chdV[d]);
        const int cc = S.cc[ac];
        if (cc >= 0) {
          const double q = P * sw * chd;
          atomicAdd(&S.adjV[ac], q * S.chaO1[ac]);
          atomicAdd(&S.adjV[cc], q * S.chaCC[ac]);
          atomicAdd(&S.adjV[S.o2[ac]], q * S.chaO2[ac]);
        }
      }
    }
  }
  const double Eh4 = block_sum(eh4, red);
  __syncthreads();  // every phase-B atomic is in place

  // ---------------------------------------------------------------- C. valence chain, H-H, X
  double ehh = 0.0, ex = 0.0;
  for (int x = a0 + threadIdx.x; x < a1; x += kThreads) {
    const int zx = z[x];
    double g[3] = {S.gB[3 * x], S.gB[3 * x + 1], S.gB[3 * x + 2]};
    const double aVx = S.adjV[x], aHx = S.adjH[x], aOx = S.adjO[x];
    for (int a = a0; a < a1; ++a) {
      if (a == x) continue;
      const int za = z[a];
      const double dx = xyz[3 * x] - xyz[3 * a], dy = xyz[3 * x + 1] - xyz[3 * a + 1], dz = xyz[3 * x + 2] - xyz[3 * a + 2];
      const double rb = sqrt(dx * dx + dy * dy + dz * dz);
      const double r = rb * kA0;
      double v, dv;
      cval(za, zx, r, v, dv);
      double s = 0.0;  // d E / d r (kcal/mol/Angstrom)
      if (dv != 0.0) {
        const double wgt = S.adjV[a] + aVx + (zx == 1 ? S.adjH[a] : S.adjO[a]) + (za == 1 ? aHx : aOx);
        s += wgt * dv;
      }
      if (zx == 1 && za == 1) {  // H-H repulsion (h4.rs:342-348, 369-387)
        const double e = exp((r / 2.23 - 1.0) * -6.86);
        const double q = 1.0 / (e + 1.0);
        ehh = ehh + (1.0 - q) * 1.55;
        s += -1.55 * (6.86 / 2.23) * e * q * q;
      }
      if (var == 3 && r <= 8.0) {  // halogen bonds (hx.rs:64-88): Cl to N and O
        const bool xh = zx == 17 && (za == 7 || za == 8), ah = za == 17 && (zx == 7 || zx == 8);
        if (xh || ah) {
          const int acc = xh ? za : zx;
          const double A = acc == 7 ? 1.0489e12 : 4.6783e8, B = acc == 7 ? -9.946 : -6.867;
          const double t = exp(r * B) * A;
          if (xh) ex = ex + t;
          s += t * B;
        }
      }
      if (s != 0.0) {
        const double f = s * kA0 / rb;
        g[0] += f * dx;
        g[1] += f * dy;
        g[2] += f * dz;
      }
    }
    for (int c = 0; c < 3; ++c) grad[3 * x + c] = g[c] * kKcal;
  }
  const double Ehh = block_sum(ehh, red);
  __syncthreads();
  const double Ex = block_sum(ex, red);
  if (threadIdx.x == 0) {
    energy[3 * m] = Eh4 * kKcal;
    energy[3 * m + 1] = Ehh * (0.5 * kKcal);
    energy[3 * m + 2] = (var == 3) ? Ex * kKcal : 0.0;
  }
}

}  // namespace h4k

// MOPAC's MMOK amide term (pm3-rs src/corrections/mmok.rs:97-143): for every (O, C, N, H) with
// C-N < 1.65, C=O < 1.35 and N-H < 1.30 Angstrom, AMIDE_K sin^2 of the O-C-N-H torsion, in the
// reference's polynomial form ((n1 x n2) . b2)^2 / (|n1|^2 |n2|^2 |b2|^2), zero where that
// denominator is at most 1e-30. The gradient comes from forward-mode dual numbers carrying the 12
// coordinates of the quadruple, one evaluation per term.
namespace mmk {

constexpr double kAmideK = 7.185300 / 23.06054783061903;  // eV

struct D12 {
  double v, d[12];
};
__device__ __forceinline__ D12 dsub(const D12& a, const D12& b) {
  D12 r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < 12; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
__device__ __forceinline__ D12 dadd(const D12& a, const D12& b) {
  D12 r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < 12; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
__device__ __forceinline__ D12 dmul(const D12& a, const D12& b) {
  D12 r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < 12; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}

__device__ inline void sin2_torsion(const double* xyz, const int* at, double& s, double* g) {
  D12 p[4][3];
  for (int a = 0; a < 4; ++a)
    for (int c = 0; c < 3; ++c) {
      p[a][c].v = xyz[3 * at[a] + c];
#pragma unroll
      for (int k = 0; k < 12; ++k) p[a][c].d[k] = (k == 3 * a + c) ? 1.0 : 0.0;
    }
  D12 b1[3], b2[3], b3[3], n1[3], n2[3], m[3];
  for (int c = 0; c < 3; ++c) {
    b1[c] = dsub(p[1][c], p[0][c]);
    b2[c] = dsub(p[2][c], p[1][c]);
    b3[c] = dsub(p[3][c], p[2][c]);
  }
  auto cross = [](const D12* a, const D12* b, D12* o) {
    o[0] = dsub(dmul(a[1], b[2]), dmul(a[2], b[1]));
    o[1] = dsub(dmul(a[2], b[0]), dmul(a[0], b[2]));
    o[2] = dsub(dmul(a[0], b[1]), dmul(a[1], b[0]));
  };
  auto dot = [](const D12* a, const D12* b) { return dadd(dadd(dmul(a[0], b[0]), dmul(a[1], b[1])), dmul(a[2], b[2])); };
  cross(b1, b2, n1);
  cross(b2, b3, n2);
  cross(n1, n2, m);
  const D12 t = dot(m, b2);
  const D12 num = dmul(t, t);
  const D12 den = dmul(dmul(dot(n1, n1), dot(n2, n2)), dot(b2, b2));
  if (den.v <= 1.0e-30) {
    s = 0.0;
    for (int k = 0; k < 12; ++k) g[k] = 0.0;
    return;
  }
  s = num.v / den.v;
  for (int k = 0; k < 12; ++k) g[k] = (num.d[k] * den.v - num.v * den.d[k]) / (den.v * den.v);
}

__device__ __forceinline__ bool bonded(const double* xyz, int i, int j, double mx) {
  double d2 = 0.0;
  for (int k = 0; k < 3; ++k) d2 += (xyz[3 * i + k] - xyz[3 * j + k]) * (xyz[3 * i + k] - xyz[3 * j + k]);
  return d2 < mx * mx;
}

// grid: one CTA per entry of mols; energy[m] (eV) written, grad[3 atom] accumulated (zeroed first)
__global__ void __launch_bounds__(128) mmok_kernel(const int32_t* __restrict__ mols, const int32_t* __restrict__ offs,
                                                   const int32_t* __restrict__ z, const double* __restrict__ xyz,
                                                   double* __restrict__ energy, double* __restrict__ grad) {
  __shared__ double red[4];
  const int m = mols[blockIdx.x];
  const int a0 = offs[m], a1 = offs[m + 1];
  const double co = 1.35 / h4k::kA0, cn = 1.65 / h4k::kA0, nh = 1.30 / h4k::kA0;
  double e = 0.0;
  for (int ni = a0 + threadIdx.x; ni < a1; ni += blockDim.x) {
    if (z[ni] != 7) continue;
    for (int ci = a0; ci < a1; ++ci) {
      if (z[ci] != 6 || !bonded(xyz, ni, ci, cn)) continue;
      for (int oi = a0; oi < a1; ++oi) {
        if (z[oi] != 8 || !bonded(xyz, ci, oi, co)) continue;
        for (int hi = a0; hi < a1; ++hi) {
          if (z[hi] != 1 || !bonded(xyz, ni, hi, nh)) continue;
          const int at[4] = {oi, ci, ni, hi};
          double s, g[12];
          sin2_torsion(xyz, at, s, g);
          e = e + s * kAmideK;
          for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 3; ++c) atomicAdd(&grad[3 * at[a] + c], g[3 * a + c] * kAmideK);
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) energy[m] = red[0] + red[1] + red[2] + red[3];
}

}  // namespace mmk
