// CPU oracle for the Grimme D3 dispersion correction of pm3-rs (TEST INFRASTRUCTURE ONLY): a C++
// restatement of src/corrections/d3.rs (zero damping, CN-interpolated C6) for molecules, generic
// over the scalar as the reference is, so that the gradient comes from forward-mode dual numbers
// seeded one atom at a time exactly as src/gradient.rs:324-357 (add_correction_gradient) does.
// It is the checker of the GPU library's D3 kernels, which use hand-derived analytic derivatives
// instead; the two share only the data header.
#include <cmath>
#include <cstring>
#include <vector>

#include "../pm3-rs_b200/csrc/pm3_d3_table.h"
#include "pm3_oracle.h"

namespace {

constexpr double kA0 = 0.529177210903;        // BOHR_TO_ANGSTROM (constants.rs:24,36)
constexpr double kEh = 27.211386245988;       // HARTREE_TO_EV (constants.rs:21,33)

// value + gradient with respect to the three coordinates of one seeded atom
struct Dual {
  double v = 0.0, d[3] = {0.0, 0.0, 0.0};
  Dual() = default;
  Dual(double x) : v(x) {}  // NOLINT: constants promote
};
inline Dual operator+(Dual a, const Dual& b) {
  a.v += b.v;
  for (int k = 0; k < 3; ++k) a.d[k] += b.d[k];
  return a;
}
inline Dual operator-(Dual a, const Dual& b) {
  a.v -= b.v;
  for (int k = 0; k < 3; ++k) a.d[k] -= b.d[k];
  return a;
}
inline Dual operator-(Dual a) {
  a.v = -a.v;
  for (int k = 0; k < 3; ++k) a.d[k] = -a.d[k];
  return a;
}
inline Dual operator*(const Dual& a, const Dual& b) {
  Dual r(a.v * b.v);
  for (int k = 0; k < 3; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
inline Dual operator/(const Dual& a, const Dual& b) {
  Dual r(a.v / b.v);
  for (int k = 0; k < 3; ++k) r.d[k] = (a.d[k] * b.v - a.v * b.d[k]) / (b.v * b.v);
  return r;
}
inline Dual chain(const Dual& a, double f, double df) {
  Dual r(f);
  for (int k = 0; k < 3; ++k) r.d[k] = df * a.d[k];
  return r;
}
inline double val(double x) { return x; }
inline double val(const Dual& x) { return x.v; }
inline double s_sqrt(double x) { return std::sqrt(x); }
inline Dual s_sqrt(const Dual& x) {
  const double s = std::sqrt(x.v);
  return chain(x, s, 0.5 / s);
}
inline double s_exp(double x) { return std::exp(x); }
inline Dual s_exp(const Dual& x) {
  const double e = std::exp(x.v);
  return chain(x, e, e);
}
inline double s_recip(double x) { return 1.0 / x; }
inline Dual s_recip(const Dual& x) { return chain(x, 1.0 / x.v, -1.0 / (x.v * x.v)); }
inline double s_powf(double x, double a) { return std::pow(x, a); }
inline Dual s_powf(const Dual& x, double a) { return chain(x, std::pow(x.v, a), a * std::pow(x.v, a - 1.0)); }

struct Tables {
  int idx[128];
  double r2r4[PM3_D3_NELEM], rcov[PM3_D3_NELEM], r0ab[PM3_D3_NELEM][PM3_D3_NELEM];
  Tables() {
    for (int& v : idx) v = -1;
    for (int e = 0; e < PM3_D3_NELEM; ++e) {
      const int z = pm3_d3_z[e];
      idx[z] = e;
      r2r4[e] = std::sqrt(0.5 * pm3_d3_r2r4_raw[e] * std::sqrt((double)z));  // d3.rs:140-141
      rcov[e] = 4.0 / 3.0 * pm3_d3_rcov_raw[e] / kA0;
      for (int f = 0; f < PM3_D3_NELEM; ++f) r0ab[e][f] = pm3_d3_r0ab_ang[e][f] / kA0;  // d3.rs:114-121
    }
  }
};
const Tables& tables() {
  static const Tables t;
  return t;
}

template <class S>
S dist(const S* a, const S* b) {
  const S dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return s_sqrt(dx * dx + dy * dy + dz * dz);
}

// getc6 (d3.rs:212-236): Gaussian weights exp(k3 ((cn_a - ref_a)^2 + (cn_b - ref_b)^2)), k3 = -4
template <class S>
S getc6(int ei, int ej, const S& cni, const S& cnj) {
  const int a = ei >= ej ? ei : ej, b = ei >= ej ? ej : ei;
  const int p = a * (a + 1) / 2 + b;
  const S& ca = ei >= ej ? cni : cnj;
  const S& cb = ei >= ej ? cnj : cni;
  S num(0.0), den(0.0);
  for (int k = pm3_d3_pair_off[p]; k < pm3_d3_pair_off[p + 1]; ++k) {
    const S da = ca - S(pm3_d3_ref[k][1]);
    const S db = cb - S(pm3_d3_ref[k][2]);
    const S t = s_exp((da * da + db * db) * S(-4.0));
    num = num + t * S(pm3_d3_ref[k][0]);
    den = den + t;
  }
  if (val(den) > 0.0) return num / den;
  return S(0.0);
}

// coordination_numbers_g (d3.rs:173-209), k1 = 16
template <class S>
void coordination(int n, const int* e, const S* pos, std::vector<S>& cn) {
  const Tables& T = tables();
  cn.assign(n, S(0.0));
  for (int i = 0; i < n; ++i) {
    if (e[i] < 0) continue;
    for (int j = 0; j < n; ++j) {
      if (i == j || e[j] < 0) continue;
      const S r = dist(pos + 3 * j, pos + 3 * i);
      const double rco = T.rcov[e[i]] + T.rcov[e[j]];
      cn[i] = cn[i] + s_recip(s_exp((s_recip(r) * S(rco) - S(1.0)) * S(-16.0)) + S(1.0));
    }
  }
}

struct Params {
  double s6, s8, rs6, rs8, alp6, alp8;
};
// D3Params::pm3_d3 / pm3_d3h4 (d3.rs:36-60)
Params params_of(int variant) {
  if (variant == 1) return {1.0, 0.612, 1.345, 1.0, 14.0, 16.0};
  return {1.0, 0.0, 0.90, 1.0e-10, 22.0, 24.0};
}

// d3_energy_cluster_g (d3.rs:398-458) for a molecule: the ordered pair sum with weight 1/2
template <class S>
S energy(int n, const int* e, const S* pos, const Params& p) {
  const Tables& T = tables();
  std::vector<S> cn;
  coordination(n, e, pos, cn);
  S e6(0.0), e8(0.0);
  for (int i = 0; i < n; ++i) {
    if (e[i] < 0) continue;
    for (int j = 0; j < n; ++j) {
      if (j == i || e[j] < 0) continue;
      const S r = dist(pos + 3 * j, pos + 3 * i);
      const S r2 = r * r;
      const S r6 = r2 * r2 * r2;
      const S r8 = r6 * r2;
      const S c6 = getc6(e[i], e[j], cn[i], cn[j]);
      const S c8 = c6 * S(3.0 * T.r2r4[e[i]] * T.r2r4[e[j]]);
      const S rr = s_recip(r) * S(T.r0ab[e[i]][e[j]]);
      const S damp6 = s_recip(s_powf(rr * S(p.rs6), p.alp6) * S(6.0) + S(1.0));
      const S damp8 = s_recip(s_powf(rr * S(p.rs8), p.alp8) * S(6.0) + S(1.0));
      e6 = e6 + c6 * damp6 / r6;
      e8 = e8 + c8 * damp8 / r8;
    }
  }
  return -(e6 * S(p.s6) + e8 * S(p.s8)) * S(0.5 * kEh);
}

void elements(int n, const int* z, std::vector<int>& e) {
  const Tables& T = tables();
  e.resize(n);
  for (int i = 0; i < n; ++i) e[i] = (z[i] > 0 && z[i] < 128) ? T.idx[z[i]] : -1;
}

}  // namespace

extern "C" {

int oracle_d3(int n_atoms, const int* z, const double* xyz_bohr, int variant, double* energy_ev, double* gradient,
              double* cn_out) {
  if (n_atoms < 0 || (n_atoms > 0 && (!z || !xyz_bohr)) || !energy_ev || variant < 1 || variant > 2) return 1;
  std::vector<int> e;
  elements(n_atoms, z, e);
  const Params p = params_of(variant);
  *energy_ev = energy<double>(n_atoms, e.data(), xyz_bohr, p);
  if (cn_out) {
    std::vector<double> cn;
    coordination<double>(n_atoms, e.data(), xyz_bohr, cn);
    std::memcpy(cn_out, cn.data(), sizeof(double) * n_atoms);
  }
  if (gradient) {
    std::vector<Dual> pos(3 * (size_t)n_atoms);
    for (int a = 0; a < n_atoms; ++a) {
      for (int k = 0; k < 3 * n_atoms; ++k) pos[k] = Dual(xyz_bohr[k]);
      for (int k = 0; k < 3; ++k) pos[3 * a + k].d[k] = 1.0;
      const Dual ed = energy<Dual>(n_atoms, e.data(), pos.data(), p);
      for (int k = 0; k < 3; ++k) gradient[3 * a + k] = ed.d[k];
    }
  }
  return 0;
}

double oracle_d3_c6(int zi, int zj, double cni, double cnj) {
  std::vector<int> e;
  const int z[2] = {zi, zj};
  elements(2, z, e);
  if (e[0] < 0 || e[1] < 0) return 0.0;
  return getc6<double>(e[0], e[1], cni, cnj);
}

}  // extern "C"
