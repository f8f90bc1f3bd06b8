// CPU oracle for the post-SCF corrections of pm3-rs (TEST INFRASTRUCTURE ONLY): a C++ restatement of
// src/corrections/d3.rs (Grimme D3, zero damping, CN-interpolated C6), src/corrections/h4.rs (the
// H4 hydrogen-bond term and the H-H repulsion) and src/corrections/hx.rs (the halogen-bond term)
// for molecules, combined per variant as src/corrections/mod.rs:129-160 does. Generic over the
// scalar as the reference is, so that the gradient comes from forward-mode dual numbers seeded one
// atom at a time exactly as src/gradient.rs:324-357 (add_correction_gradient) does. It is the
// checker of the GPU library's correction kernels, which use hand-derived derivatives instead; the
// two share only the D3 data header.
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
inline Dual s_powf(const Dual& x, double a) {
  return chain(x, std::pow(x.v, a), x.v > 0.0 ? a * std::pow(x.v, a - 1.0) : 0.0);
}
inline double s_powi(double x, int n) { return std::pow(x, n); }
inline Dual s_powi(const Dual& x, int n) {
  return chain(x, std::pow(x.v, n), x.v != 0.0 ? n * std::pow(x.v, n - 1) : 0.0);
}
inline double s_abs(double x) { return std::fabs(x); }
inline Dual s_abs(const Dual& x) { return x.v >= 0.0 ? x : -x; }
// acos with the reference's derivative rule (dual.rs: zero where 1 - v^2 <= 1e-14)
inline double s_acos(double x) { return std::acos(x); }
inline Dual s_acos(const Dual& x) {
  const double one_m = 1.0 - x.v * x.v;
  return chain(x, std::acos(x.v), one_m > 1.0e-14 ? -1.0 / std::sqrt(one_m) : 0.0);
}

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

// ---------------------------------------------------------------- H4 and H-H (h4.rs)
constexpr double kKcalToEv = 1.0 / 23.06054783061903;  // KCAL_TO_EV (constants.rs:27,37)
constexpr double kPi = 3.14159265358979323846;
// covalent radii (Angstrom) of elements 1..17, the head of h4.rs:81-89 (radii_C of MOPAC)
const double kCovRad[17] = {0.37, 0.32, 1.34, 0.90, 0.82, 0.77, 0.75, 0.73, 0.71,
                            0.69, 1.54, 1.30, 1.18, 1.11, 1.06, 1.02, 0.99};
double cov_radius(int z) { return (z >= 1 && z <= 17) ? kCovRad[z - 1] : 0.0; }

template <class S>
S dist_ang(const S* pos, int a, int b) {
  return dist(pos + 3 * a, pos + 3 * b) * S(kA0);
}

template <class S>
S poly7_switch(const S& x) {  // 1 - (35 x^4 - 84 x^5 + 70 x^6 - 20 x^7)
  return -(s_powi(x, 7) * S(-20.0) + s_powi(x, 6) * S(70.0) + s_powi(x, 5) * S(-84.0) + s_powi(x, 4) * S(35.0)) +
         S(1.0);
}

// cvalence_contribution_g (h4.rs:128-143)
template <class S>
S cvalence(const int* z, const S* pos, int a, int b) {
  const double r0 = cov_radius(z[a]) + cov_radius(z[b]);
  const double r1 = r0 * 1.6;
  const S r = dist_ang(pos, a, b);
  const double rv = val(r);
  if (rv == 0.0 || rv >= r1) return S(0.0);
  if (rv <= r0) return S(1.0);
  const S x = (r - S(r0)) / S(r1 - r0);
  return poly7_switch(x);
}

template <class S>
S e_radial(const S& rda) {  // h4.rs:97-106
  return s_powi(rda, 7) * S(-0.003034074074073135) + s_powi(rda, 6) * S(0.07357629629627092) +
         s_powi(rda, 5) * S(-0.700871111110828) + s_powi(rda, 4) * S(3.2530962962946175) +
         s_powi(rda, 3) * S(-7.206874074068388) + s_powi(rda, 2) * S(5.317546666655722) +
         rda * S(3.407360000011028) - S(4.685120000004504);
}

template <class S>
S e_angular(const S& angle) {  // h4.rs:109-113
  const S a = angle * S(1.0 / (kPi / 2.0));
  const S x = s_powi(a, 7) * S(-20.0) + s_powi(a, 6) * S(70.0) + s_powi(a, 5) * S(-84.0) + s_powi(a, 4) * S(35.0);
  return -(x * x) + S(1.0);
}

double e_para(int d, int a) {  // h4.rs:116-124
  if (d == 8 && a == 8) return 2.71;
  if (d == 8 && a == 7) return 4.37;
  if (d == 7 && a == 8) return 2.29;
  if (d == 7 && a == 7) return 3.86;
  return 0.0;
}

template <class S>
S f_dev(const S& cv, double target) {  // h4.rs:43-50
  const S dev = s_abs(cv - S(target));
  if (val(dev) < 1.0) return S(1.0) - dev;
  return S(0.0);
}

template <class S>
S scale_water(int n, const int* z, const S* pos, int donor, int acceptor) {  // h4.rs:146-180
  if (z[donor] != 8 || z[acceptor] != 8) return S(1.0);
  S hyd(0.0), oth(0.0);
  for (int k = 0; k < n; ++k) {
    const S c = cvalence(z, pos, donor, k);
    if (z[k] == 1) hyd = hyd + c;
    else oth = oth + c;
  }
  if (val(hyd) < 1.0) return S(1.0);
  const double slope = 0.91 - 1.0;
  const double vv = val(hyd);
  S fv(0.0);
  if (vv > 1.0 && vv <= 2.0) fv = hyd - S(1.0);
  else if (vv > 2.0 && vv < 3.0) fv = -hyd + S(3.0);
  const S fv2 = (1.0 - val(oth)) > 0.0 ? -oth + S(1.0) : S(0.0);
  return fv * fv2 * S(slope) + S(1.0);
}

template <class S>
S scale_charged_donor(int n, const int* z, const S* pos, int donor) {  // h4.rs:183-193
  if (z[donor] != 7) return S(1.0);
  S v(0.0);
  for (int k = 0; k < n; ++k) v = v + cvalence(z, pos, donor, k);
  const S vv = val(v) > 3.0 ? v - S(3.0) : S(0.0);
  return vv * S(2.5390633931627 - 1.0) + S(1.0);
}

template <class S>
S scale_charged_acceptor(int n, const int* z, const S* pos, int acceptor) {  // h4.rs:196-240
  if (z[acceptor] != 8) return S(1.0);
  const int o1 = acceptor;
  double cdist = INFINITY;
  int cc = -1;
  S cv_o1(0.0);
  for (int k = 0; k < n; ++k) {
    const S v = cvalence(z, pos, o1, k);
    cv_o1 = cv_o1 + v;
    const double d = val(dist_ang(pos, o1, k));
    if (val(v) > 0.0 && z[k] == 6 && d < cdist) {
      cdist = d;
      cc = k;
    }
  }
  if (cc < 0) return S(1.0);
  double odist = INFINITY;
  int o2 = -1;
  S cv_cc(0.0);
  for (int k = 0; k < n; ++k) {
    const S v = cvalence(z, pos, cc, k);
    cv_cc = cv_cc + v;
    const double d = val(dist_ang(pos, cc, k));
    if (val(v) > 0.0 && k != o1 && z[k] == 8 && d < odist) {
      odist = d;
      o2 = k;
    }
  }
  if (o2 < 0) return S(1.0);
  S cv_o2(0.0);
  for (int k = 0; k < n; ++k) cv_o2 = cv_o2 + cvalence(z, pos, o2, k);
  return f_dev(cv_o1, 1.0) * f_dev(cv_o2, 1.0) * f_dev(cv_cc, 3.0) * S(0.88610264413703 - 1.0) + S(1.0);
}

// h4_energy_cluster_g (h4.rs:265-339) for a molecule
template <class S>
S h4_energy(int n, const int* z, const S* pos) {
  auto don_acc = [](int q) { return q == 7 || q == 8; };
  S sum(0.0);
  for (int i = 0; i < n; ++i) {
    if (!don_acc(z[i])) continue;
    for (int j = i + 1; j < n; ++j) {
      if (!don_acc(z[j])) continue;
      const S rda = dist(pos + 3 * j, pos + 3 * i) * S(kA0);
      if (val(rda) >= 5.5) continue;
      for (int h = 0; h < n; ++h) {
        if (z[h] != 1) continue;
        S vih[3], vjh[3];
        for (int c = 0; c < 3; ++c) {
          vih[c] = pos[3 * i + c] - pos[3 * h + c];
          vjh[c] = pos[3 * j + c] - pos[3 * h + c];
        }
        const S rih = s_sqrt(vih[0] * vih[0] + vih[1] * vih[1] + vih[2] * vih[2]);
        const S rjh = s_sqrt(vjh[0] * vjh[0] + vjh[1] * vjh[1] + vjh[2] * vjh[2]);
        const S cs = (vih[0] * vjh[0] + vih[1] * vjh[1] + vih[2] * vjh[2]) / (rih * rjh);
        const S cl = val(cs) >= 1.0 ? S(1.0) : val(cs) <= -1.0 ? S(-1.0) : cs;  // clamp_unit
        const S dha = s_acos(cl);
        const S angle = -dha + S(kPi);
        if (val(angle) >= kPi / 2.0) continue;
        const bool i_don = val(rih) < val(rjh);
        const int donor = i_don ? i : j, acceptor = i_don ? j : i;
        const S rdh = (i_don ? rih : rjh) * S(kA0);
        const S rah = (i_don ? rjh : rih) * S(kA0);
        if (val(rdh) >= 1.15) continue;
        const double ep = e_para(z[donor], z[acceptor]);
        if (ep == 0.0) continue;
        S bsw(1.0);
        if (val(rdh) > 1.15) {  // h4.rs:314-321 (unreachable after the 1.15 cut; kept as written)
          const S x = (rdh - S(1.15)) / (rdh * S(0.5) + rah * S(0.5) - S(1.15));
          bsw = poly7_switch(x);
        }
        const S sw = scale_water(n, z, pos, donor, acceptor);
        const S chd = scale_charged_donor(n, z, pos, donor);
        const S cha = scale_charged_acceptor(n, z, pos, acceptor);
        sum = sum + e_radial(rda) * e_angular(angle) * bsw * sw * chd * cha * S(ep);
      }
    }
  }
  return sum * S(kKcalToEv);
}

// hh_rep_energy_cluster_g (h4.rs:369-387) with poly_hh_g (h4.rs:342-348)
template <class S>
S hh_energy(int n, const int* z, const S* pos) {
  S sum(0.0);
  for (int i = 0; i < n; ++i) {
    if (z[i] != 1) continue;
    for (int j = 0; j < n; ++j) {
      if (j == i || z[j] != 1) continue;
      const S r = dist(pos + 3 * i, pos + 3 * j) * S(kA0);
      sum = sum + (S(1.0) - s_recip(s_exp((r / S(2.23) - S(1.0)) * S(-6.86)) + S(1.0))) * S(1.55);
    }
  }
  return sum * S(0.5 * kKcalToEv);
}

// hx_energy_cluster_g (hx.rs:64-88): Cl (the one halogen of the s/p set) to N and O
template <class S>
S hx_energy(int n, const int* z, const S* pos) {
  S sum(0.0);
  for (int i = 0; i < n; ++i) {
    if (z[i] != 17) continue;
    for (int j = 0; j < n; ++j) {
      if (i == j) continue;
      double a, b;
      if (z[j] == 7) {
        a = 1.0489e12;
        b = -9.946;
      } else if (z[j] == 8) {
        a = 4.6783e8;
        b = -6.867;
      } else {
        continue;
      }
      const S rab = dist(pos + 3 * j, pos + 3 * i) * S(kA0);
      if (val(rab) > 8.0) continue;
      sum = sum + s_exp(rab * S(b)) * S(a);
    }
  }
  return sum * S(kKcalToEv);
}

// ---------------------------------------------------------------- MMOK amide term (mmok.rs)
constexpr double kAmideKEv = 7.185300 / 23.06054783061903;  // AMIDE_K_KCAL / EV_TO_KCAL (mmok.rs:39-42)

// sin^2 of the p0-p1-p2-p3 torsion, polynomial form (mmok.rs:64-89)
template <class S>
S sin2_torsion(const S* p0, const S* p1, const S* p2, const S* p3) {
  S b1[3], b2[3], b3[3], n1[3], n2[3], m[3];
  for (int k = 0; k < 3; ++k) {
    b1[k] = p1[k] - p0[k];
    b2[k] = p2[k] - p1[k];
    b3[k] = p3[k] - p2[k];
  }
  auto cross = [](const S* a, const S* b, S* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  auto dot = [](const S* a, const S* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  cross(b1, b2, n1);
  cross(b2, b3, n2);
  cross(n1, n2, m);
  const S num = s_powi(dot(m, b2), 2);
  const S den = dot(n1, n1) * dot(n2, n2) * dot(b2, b2);
  if (val(den) <= 1.0e-30) return S(0.0);
  return num / den;
}

// amide_torsions (mmok.rs:97-125): (O, C, N, H) with C-N < 1.65, C=O < 1.35, N-H < 1.30 Angstrom
void amide_torsions(int n, const int* z, const double* pos, std::vector<int>& out) {
  auto bonded = [&](int i, int j, double mx) {
    double d2 = 0.0;
    for (int k = 0; k < 3; ++k) d2 += (pos[3 * i + k] - pos[3 * j + k]) * (pos[3 * i + k] - pos[3 * j + k]);
    return d2 < mx * mx;
  };
  const double co = 1.35 / kA0, cn = 1.65 / kA0, nh = 1.30 / kA0;
  out.clear();
  for (int ni = 0; ni < n; ++ni) {
    if (z[ni] != 7) continue;
    for (int ci = 0; ci < n; ++ci) {
      if (z[ci] != 6 || !bonded(ni, ci, cn)) continue;
      for (int oi = 0; oi < n; ++oi) {
        if (z[oi] != 8 || !bonded(ci, oi, co)) continue;
        for (int hi = 0; hi < n; ++hi)
          if (z[hi] == 1 && bonded(ni, hi, nh)) {
            out.push_back(oi);
            out.push_back(ci);
            out.push_back(ni);
            out.push_back(hi);
          }
      }
    }
  }
}

// amide_correction_g (mmok.rs:132-143): topology from the coordinate values
template <class S>
S mmok_energy(int n, const int* z, const S* pos) {
  std::vector<double> v(3 * (size_t)n);
  for (size_t k = 0; k < v.size(); ++k) v[k] = val(pos[k]);
  std::vector<int> q;
  amide_torsions(n, z, v.data(), q);
  S e(0.0);
  for (size_t t = 0; t < q.size(); t += 4)
    e = e + sin2_torsion(pos + 3 * q[t], pos + 3 * q[t + 1], pos + 3 * q[t + 2], pos + 3 * q[t + 3]) * S(kAmideKEv);
  return e;
}

// correction_energy_cluster_g (mod.rs:129-160) for a molecule: variant 1 = PM3-D3, 2 = PM3-D3H4,
// 3 = PM3-D3H4X; parts[4] = (d3, h4, hh, hx)
// correction_energy_with_mmok_g (mod.rs:78-91): variant 0 has no variant term; parts[5] =
// (d3, h4, hh, hx, mmok)
template <class S>
S correction(int n, const int* z, const int* e, const S* pos, int variant, int mmok, S* parts) {
  for (int k = 0; k < 5; ++k) parts[k] = S(0.0);
  if (variant >= 1) parts[0] = energy(n, e, pos, params_of(variant == 1 ? 1 : 2));
  if (variant >= 2) {
    parts[1] = h4_energy(n, z, pos);
    parts[2] = hh_energy(n, z, pos);
  }
  if (variant == 3) parts[3] = hx_energy(n, z, pos);
  const S base = parts[0] + parts[1] + parts[2] + parts[3];
  if (!mmok) return base;
  parts[4] = mmok_energy(n, z, pos);
  return base + parts[4];
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

int oracle_corrections(int n_atoms, const int* z, const double* xyz_bohr, int variant, int mmok, double* parts_ev,
                       double* gradient) {
  if (n_atoms < 0 || (n_atoms > 0 && (!z || !xyz_bohr)) || !parts_ev || variant < 0 || variant > 3) return 1;
  std::vector<int> e;
  elements(n_atoms, z, e);
  double parts[5];
  correction<double>(n_atoms, z, e.data(), xyz_bohr, variant, mmok, parts);
  for (int k = 0; k < 5; ++k) parts_ev[k] = parts[k];
  if (gradient) {
    std::vector<Dual> pos(3 * (size_t)n_atoms);
    Dual dp[5];
    for (int a = 0; a < n_atoms; ++a) {
      for (int k = 0; k < 3 * n_atoms; ++k) pos[k] = Dual(xyz_bohr[k]);
      for (int k = 0; k < 3; ++k) pos[3 * a + k].d[k] = 1.0;
      const Dual ed = correction<Dual>(n_atoms, z, e.data(), pos.data(), variant, mmok, dp);
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
