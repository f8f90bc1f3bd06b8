// CPU oracle for the molecular PM3 single point of pm3-rs -- TEST INFRASTRUCTURE ONLY.
//
// A C++ restatement of the reference's CPU algorithm, used by tests/, by smoke() and by the
// CPU-baseline leg of bench.py to check (and time beside) the GPU library. Every function
// cites the reference file:line it follows (paths relative to the pm3-rs project root).
// The product library never links or loads this file.
#include "pm3_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../pm3-rs_b200/csrc/pm3_param_table.h"

namespace {

// ---------------------------------------------------------------- constants (constants.rs:21-64)
constexpr double EV = 27.211386245988;
constexpr double A0 = 0.529177210903;
constexpr double EV_TO_KCAL = 23.06054783061903;
constexpr double AU_DIPOLE_TO_DEBYE = 2.541746473;

// ---------------------------------------------------------------- dual numbers (dual.rs:13-260)
struct Dual {
  double v;
  double d[3];
};
inline double val(double x) { return x; }
inline double val(const Dual& x) { return x.v; }
template <class S> inline S cst(double x);
template <> inline double cst<double>(double x) { return x; }
template <> inline Dual cst<Dual>(double x) { return Dual{x, {0, 0, 0}}; }
inline Dual dvar(double x, int k) {
  Dual r{x, {0, 0, 0}};
  r.d[k] = 1.0;
  return r;
}
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]}}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]}}; }
inline Dual operator-(Dual a) { return {-a.v, {-a.d[0], -a.d[1], -a.d[2]}}; }
inline Dual operator*(Dual a, Dual b) {
  return {a.v * b.v, {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2]}};
}
inline Dual operator/(Dual a, Dual b) {
  double inv = 1.0 / b.v, q = a.v * inv;
  return {q, {(a.d[0] - q * b.d[0]) * inv, (a.d[1] - q * b.d[1]) * inv, (a.d[2] - q * b.d[2]) * inv}};
}
inline Dual operator+(Dual a, double b) { return {a.v + b, {a.d[0], a.d[1], a.d[2]}}; }
inline Dual operator+(double b, Dual a) { return a + b; }
inline Dual operator-(Dual a, double b) { return {a.v - b, {a.d[0], a.d[1], a.d[2]}}; }
inline Dual operator-(double b, Dual a) { return {b - a.v, {-a.d[0], -a.d[1], -a.d[2]}}; }
inline Dual operator*(Dual a, double b) { return {a.v * b, {a.d[0] * b, a.d[1] * b, a.d[2] * b}}; }
inline Dual operator*(double b, Dual a) { return a * b; }
inline Dual operator/(Dual a, double b) { return a * (1.0 / b); }
inline Dual chain(Dual a, double f, double df) { return {f, {a.d[0] * df, a.d[1] * df, a.d[2] * df}}; }
inline double dsqrt(double x) { return std::sqrt(x); }
inline Dual dsqrt(Dual a) { double s = std::sqrt(a.v); return chain(a, s, 0.5 / s); }
inline double drecip(double x) { return 1.0 / x; }
inline Dual drecip(Dual a) { double r = 1.0 / a.v; return chain(a, r, -r * r); }
inline double dexp(double x) { return std::exp(x); }
inline Dual dexp(Dual a) { double e = std::exp(a.v); return chain(a, e, e); }
inline double dpowf(double x, double p) { return std::pow(x, p); }
inline Dual dpowf(Dual a, double p) { double f = std::pow(a.v, p); return chain(a, f, p * std::pow(a.v, p - 1.0)); }
template <class S> inline S dpowi(S x, int n) {
  S r = cst<S>(1.0);
  for (int i = 0; i < n; ++i) r = r * x;
  return r;
}
inline double dabs(double x) { return std::fabs(x); }
inline Dual dabs(Dual a) { return a.v < 0 ? -a : a; }

// ---------------------------------------------------------------- parameters (params.rs:155-343)
struct Elem {
  int z = 0, norb = 0, n = 0;
  double uss, upp, zs, zp, bs, bp, gss, gsp, gpp, gp2, hsp, alpha;
  std::vector<std::array<double, 3>> gauss;
  double core, occ_s, occ_p, eheat_ev, e_isol, mass;
  double dd, qq, rho0, rho1, rho2;
  double po[10];
  double ddp[7];
  bool has_p() const { return norb >= 4; }
};

// params.rs:570-580
double multipole_pqn(int z) {
  if (z <= 2) return 1.0;
  if (z <= 10) return 2.0;
  if (z <= 18) return 3.0;
  return 0.0;
}
// params.rs:584-594
double dd_charge_sep(double qn, double zs, double zp) {
  return (2.0 * qn + 1.0) * std::pow(4.0 * zs * zp, qn + 0.5) / std::pow(zs + zp, 2.0 * qn + 2.0) /
         std::sqrt(3.0);
}
double qq_charge_sep(double qn, double zp) { return std::sqrt((4.0 * qn * qn + 6.0 * qn + 2.0) / 20.0) / zp; }
// params.rs:605-622: exactly five secant steps
double additive_rho1(double hsp_ev, double dd) {
  double hsp = std::max(hsp_ev, 1.0e-7) / EV;
  auto g = [&](double d) { return 0.5 * d - 0.5 / std::sqrt(4.0 * dd * dd + 1.0 / (d * d)); };
  double gdd1 = std::pow(hsp / (dd * dd), 1.0 / 3.0);
  double d1 = gdd1, d2 = gdd1 + 0.04;
  for (int it = 0; it < 5; ++it) {
    double df = d2 - d1, h1 = g(d1), h2 = g(d2);
    if (std::fabs(h2 - h1) < 1.0e-25) break;
    double d3 = d1 + df * (hsp - h1) / (h2 - h1);
    d1 = d2;
    d2 = d3;
  }
  return 0.5 / d2;
}
// params.rs:629-649
double additive_rho2(double hpp_ev, double qq) {
  double hpp = hpp_ev / EV;
  auto g = [&](double q) {
    return 0.25 * q - 0.5 / std::sqrt(4.0 * qq * qq + 1.0 / (q * q)) + 0.25 / std::sqrt(8.0 * qq * qq + 1.0 / (q * q));
  };
  double qq4 = qq * qq * qq * qq;
  double gqq = std::pow(16.0 * hpp / (48.0 * qq4), 0.2);
  double q1 = gqq, q2 = gqq + 0.04;
  for (int it = 0; it < 5; ++it) {
    double qf = q2 - q1, h1 = g(q1), h2 = g(q2);
    if (std::fabs(h2 - h1) < 1.0e-25) break;
    double q3 = q1 + qf * (hpp - h1) / (h2 - h1);
    q1 = q2;
    q2 = q3;
  }
  return 0.5 / q2;
}
// params.rs:542-560
double gssc(double ios) { return std::max(ios - 1.0, 0.0); }
double gspc(double ios, double iop) { return ios * iop; }
double hspc(double ios, double iop) { return -iop * ios * 0.5; }
double gp2c(double iop) {
  long k = (long)iop, l = std::min(k, 6 - k);
  return (double)((k * (k - 1)) / 2) + (double)(l * (l - 1)) / 4.0;
}
double gppc(double iop) {
  long k = (long)iop, l = std::min(k, 6 - k);
  return -((double)(l * (l - 1))) / 4.0;
}

struct Params {
  Elem el[19];
  bool have[19] = {false};
  double pair_alpha[19][19], pair_x[19][19];
  bool have_pair[19][19];
  Params() {
    for (int i = 0; i < 19; ++i)
      for (int j = 0; j < 19; ++j) have_pair[i][j] = false;
    for (int k = 0; k < PM3_N_RAW_ELEMENTS; ++k) {
      const Pm3RawElement& r = PM3_RAW_ELEMENTS[k];
      Elem e;
      e.z = r.z;
      e.norb = r.zp > 0.0 ? 4 : 1;  // params.rs:195-203
      e.n = r.npq_s;
      e.uss = r.uss; e.upp = r.upp; e.zs = r.zs; e.zp = r.zp; e.bs = r.betas; e.bp = r.betap;
      e.gss = r.gss; e.gsp = r.gsp; e.gpp = r.gpp; e.gp2 = r.gp2;
      e.hsp = std::max(r.hsp, 1.0e-7);  // params.rs:217
      e.alpha = r.alp;
      for (int g = 0; g < 4; ++g)
        if (r.gauss[g][0] != 0.0 || r.gauss[g][1] != 0.0)
          e.gauss.push_back({r.gauss[g][0], r.gauss[g][1], r.gauss[g][2]});
      e.core = r.tore;
      e.occ_s = r.ios; e.occ_p = r.iop;
      e.eheat_ev = r.eheat_kcal / EV_TO_KCAL;
      e.mass = r.mass;
      if (e.norb >= 4 && e.zp > 0.0) {  // params.rs:245-255
        double zp = std::max(e.zp, 0.3), qn = multipole_pqn(e.z);
        e.dd = dd_charge_sep(qn, e.zs, zp);
        e.qq = qq_charge_sep(qn, zp);
        double hpp = std::max(0.5 * (e.gpp - e.gp2), 0.1);
        e.rho1 = additive_rho1(e.hsp, e.dd);
        e.rho2 = additive_rho2(hpp, e.qq);
      } else {
        e.dd = e.qq = e.rho1 = e.rho2 = 0.0;
      }
      e.rho0 = e.gss > 0.0 ? 0.5 * EV / e.gss : 0.0;  // params.rs:259-266
      if (e.z == 1) {  // params.rs:273-289
        e.e_isol = e.uss;
      } else {
        e.e_isol = e.uss * r.ios + e.upp * r.iop + e.gss * gssc(r.ios) + e.gpp * gppc(r.iop) +
                   e.gsp * gspc(r.ios, r.iop) + e.gp2 * gp2c(r.iop) + e.hsp * hspc(r.ios, r.iop);
      }
      for (double& v : e.po) v = 0.0;
      for (double& v : e.ddp) v = 0.0;
      if (e.norb >= 4) {  // params.rs:694-703
        e.po[1] = e.rho0; e.po[2] = e.rho1; e.po[3] = e.rho2; e.po[7] = e.rho0; e.po[9] = e.rho0;
        e.ddp[2] = e.dd;
        e.ddp[3] = e.qq * std::sqrt(2.0);
      } else {
        e.po[1] = e.rho0; e.po[7] = e.rho0; e.po[9] = e.rho0;
      }
      el[e.z] = e;
      have[e.z] = true;
    }
    for (int k = 0; k < PM3_N_RAW_PAIRS; ++k) {
      const Pm3RawPair& p = PM3_RAW_PAIRS[k];
      int a = std::max(p.zi, p.zj), b = std::min(p.zi, p.zj);
      pair_alpha[a][b] = pair_alpha[b][a] = p.alpb;
      pair_x[a][b] = pair_x[b][a] = p.xfac;
      have_pair[a][b] = have_pair[b][a] = true;
    }
  }
  const Elem* get(int z) const { return (z > 0 && z < 19 && have[z]) ? &el[z] : nullptr; }
};
// The parameter set in use: the standard one (Pm3Parameters::standard, params.rs:133-137) unless
// oracle_set_parameters replaced it (the &Pm3Parameters argument of run_pm3, scf.rs:450-452).
Params& params_mut() {
  static Params p;
  return p;
}
const Params& params() { return params_mut(); }

// ---------------------------------------------------------------- integrals (integrals.rs)
inline int pack(int a, int b) {
  int h = a >= b ? a : b, l = a >= b ? b : a;
  return h * (h + 1) / 2 + l;
}

// integrals.rs:25-59
template <class S> void rotation_to_x(S vx, S vy, S vz, S r[3][3]) {
  if (val(vx) < 0.0) {
    S one = cst<S>(1.0);
    S ux = vx - one, uy = vy, uz = vz;
    S factor = drecip(ux * ux + uy * uy + uz * uz) * (-2.0);
    r[0][0] = one + factor * ux * ux; r[0][1] = factor * ux * uy; r[0][2] = factor * ux * uz;
    r[1][0] = factor * uy * ux; r[1][1] = one + factor * uy * uy; r[1][2] = factor * uy * uz;
    r[2][0] = factor * uz * ux; r[2][1] = factor * uz * uy; r[2][2] = one + factor * uz * uz;
  } else {
    S qy = vz, qz = cst<S>(0.0) - vy, qw = vx + 1.0;
    S inv = drecip(dsqrt(qy * qy + qz * qz + qw * qw));
    qy = qy * inv; qz = qz * inv; qw = qw * inv;
    r[0][0] = (qy * qy + qz * qz) * (-2.0) + 1.0; r[0][1] = qz * qw * (-2.0); r[0][2] = qy * qw * 2.0;
    r[1][0] = qz * qw * 2.0; r[1][1] = qz * qz * (-2.0) + 1.0; r[1][2] = qy * qz * 2.0;
    r[2][0] = qy * qw * (-2.0); r[2][1] = qy * qz * 2.0; r[2][2] = qy * qy * (-2.0) + 1.0;
  }
}

// Multipole view of an element used by the local integral kernels.
struct Mp {
  double dd, qq, rho0, rho1, rho2;
};
inline Mp mp_of(const Elem& e) { return {e.dd, e.qq, e.rho0, e.rho1, e.rho2}; }

// integrals.rs:289-309
template <class S> void local_xh(const Mp& ei, const Mp& ej, S r, S ri[4]) {
  const double ev1 = EV / 2.0, ev2 = EV / 4.0;
  double da = ei.dd, qa = ei.qq * 2.0;
  double aee = (ei.rho0 + ej.rho0) * (ei.rho0 + ej.rho0);
  double ade = (ei.rho1 + ej.rho0) * (ei.rho1 + ej.rho0);
  double aqe = (ei.rho2 + ej.rho0) * (ei.rho2 + ej.rho0);
  S ee = drecip(dsqrt(r * r + aee)) * EV;
  S ev1dsqr6 = drecip(dsqrt(r * r + aqe)) * ev1;
  ri[0] = ee;
  ri[1] = drecip(dsqrt((r + da) * (r + da) + ade)) * ev1 - drecip(dsqrt((r - da) * (r - da) + ade)) * ev1;
  ri[2] = ee + drecip(dsqrt((r + qa) * (r + qa) + aqe)) * ev2 + drecip(dsqrt((r - qa) * (r - qa) + aqe)) * ev2 - ev1dsqr6;
  ri[3] = ee + drecip(dsqrt(r * r + qa * qa + aqe)) * ev1 - ev1dsqr6;
}

// integrals.rs:311-464
template <class S> void local_xx(const Mp& ei, const Mp& ej, S r, S ri[22]) {
  const double ev1 = EV / 2.0, ev2 = EV / 4.0, ev3 = EV / 8.0, ev4 = EV / 16.0;
  double da = ei.dd, db = ej.dd, qa = ei.qq * 2.0, qb = ej.qq * 2.0, qa1 = ei.qq, qb1 = ej.qq;
  auto sq = [](double x) { return x * x; };
  double aee = sq(ei.rho0 + ej.rho0), ade = sq(ei.rho1 + ej.rho0), aqe = sq(ei.rho2 + ej.rho0);
  double aed = sq(ei.rho0 + ej.rho1), aeq = sq(ei.rho0 + ej.rho2), axx = sq(ei.rho1 + ej.rho1);
  double adq = sq(ei.rho1 + ej.rho2), aqd = sq(ei.rho2 + ej.rho1), aqq = sq(ei.rho2 + ej.rho2);
  auto g = [](S x, double c) { return drecip(dsqrt(x + c)); };
  auto sq2 = [](S a, double c) { return drecip(dsqrt(a * a + c)); };
  S ee = drecip(dsqrt(r * r + aee)) * EV;
  S dze = sq2(r - da, ade) * ev1 - sq2(r + da, ade) * ev1;
  S ev1dsqr6 = drecip(dsqrt(r * r + aqe)) * ev1;
  S qzze = sq2(r - qa, aqe) * ev2 + sq2(r + qa, aqe) * ev2 - ev1dsqr6;
  S qxxe = g(r * r + qa * qa, aqe) * ev1 - ev1dsqr6;
  S edz = sq2(r + db, aed) * ev1 - sq2(r - db, aed) * ev1;
  S ev1dsqr12 = drecip(dsqrt(r * r + aeq)) * ev1;
  S eqzz = sq2(r - qb, aeq) * ev2 + sq2(r + qb, aeq) * ev2 - ev1dsqr12;
  S eqxx = g(r * r + qb * qb, aeq) * ev1 - ev1dsqr12;
  S ev2dsqr20 = sq2(r + da, adq) * ev2;
  S ev2dsqr22 = sq2(r - da, adq) * ev2;
  S ev2dsqr24 = sq2(r - db, aqd) * ev2;
  S ev2dsqr26 = sq2(r + db, aqd) * ev2;
  S ev2dsqr36 = drecip(dsqrt(r * r + aqq)) * ev2;
  S ev2dsqr39 = g(r * r + qa * qa, aqq) * ev2;
  S ev2dsqr40 = g(r * r + qb * qb, aqq) * ev2;
  S ev3dsqr42 = sq2(r - qb, aqq) * ev3;
  S ev3dsqr44 = sq2(r + qb, aqq) * ev3;
  S ev3dsqr46 = sq2(r + qa, aqq) * ev3;
  S ev3dsqr48 = sq2(r - qa, aqq) * ev3;
  ri[0] = ee;
  ri[1] = cst<S>(0.0) - dze;
  ri[2] = ee + qzze;
  ri[3] = ee + qxxe;
  ri[4] = cst<S>(0.0) - edz;
  ri[5] = sq2(r + da - db, axx) * ev2 + sq2(r - da + db, axx) * ev2 - sq2(r - da - db, axx) * ev2 - sq2(r + da + db, axx) * ev2;
  ri[6] = g(r * r + (da - db) * (da - db), axx) * ev1 - g(r * r + (da + db) * (da + db), axx) * ev1;
  ri[7] = cst<S>(0.0) - edz + sq2(r + qa - db, aqd) * ev3 - sq2(r + qa + db, aqd) * ev3 + sq2(r - qa - db, aqd) * ev3 -
          sq2(r - qa + db, aqd) * ev3 - ev2dsqr24 + ev2dsqr26;
  ri[8] = cst<S>(0.0) - edz - ev2dsqr24 + g((r - db) * (r - db) + qa * qa, aqd) * ev2 + ev2dsqr26 -
          g((r + db) * (r + db) + qa * qa, aqd) * ev2;
  ri[9] = g((r + qa1) * (r + qa1) + (qa1 - db) * (qa1 - db), aqd) * ev2 -
          g((r - qa1) * (r - qa1) + (qa1 - db) * (qa1 - db), aqd) * ev2 -
          g((r + qa1) * (r + qa1) + (qa1 + db) * (qa1 + db), aqd) * ev2 +
          g((r - qa1) * (r - qa1) + (qa1 + db) * (qa1 + db), aqd) * ev2;
  ri[10] = ee + eqzz;
  ri[11] = ee + eqxx;
  ri[12] = cst<S>(0.0) - dze + sq2(r + da - qb, adq) * ev3 - sq2(r - da - qb, adq) * ev3 + sq2(r + da + qb, adq) * ev3 -
           sq2(r - da + qb, adq) * ev3 + ev2dsqr22 - ev2dsqr20;
  ri[13] = cst<S>(0.0) - dze - ev2dsqr20 + g((r + da) * (r + da) + qb * qb, adq) * ev2 + ev2dsqr22 -
           g((r - da) * (r - da) + qb * qb, adq) * ev2;
  ri[14] = g((r - qb1) * (r - qb1) + (da - qb1) * (da - qb1), adq) * ev2 -
           g((r + qb1) * (r + qb1) + (da - qb1) * (da - qb1), adq) * ev2 -
           g((r - qb1) * (r - qb1) + (da + qb1) * (da + qb1), adq) * ev2 +
           g((r + qb1) * (r + qb1) + (da + qb1) * (da + qb1), adq) * ev2;
  ri[15] = ee + eqzz + qzze + sq2(r + qa - qb, aqq) * ev4 + sq2(r + qa + qb, aqq) * ev4 + sq2(r - qa - qb, aqq) * ev4 +
           sq2(r - qa + qb, aqq) * ev4 - ev3dsqr48 - ev3dsqr46 - ev3dsqr42 - ev3dsqr44 + ev2dsqr36;
  ri[16] = ee + eqzz + qxxe + g((r - qb) * (r - qb) + qa * qa, aqq) * ev3 + g((r + qb) * (r + qb) + qa * qa, aqq) * ev3 -
           ev3dsqr42 - ev3dsqr44 - ev2dsqr39 + ev2dsqr36;
  ri[17] = ee + eqxx + qzze + g((r + qa) * (r + qa) + qb * qb, aqq) * ev3 + g((r - qa) * (r - qa) + qb * qb, aqq) * ev3 -
           ev3dsqr46 - ev3dsqr48 - ev2dsqr40 + ev2dsqr36;
  S qxxqxx = g(r * r + (qa - qb) * (qa - qb), aqq) * ev3 + g(r * r + (qa + qb) * (qa + qb), aqq) * ev3 - ev2dsqr39 -
             ev2dsqr40 + ev2dsqr36;
  ri[18] = ee + eqxx + qxxe + qxxqxx;
  double dm = (qa1 - qb1) * (qa1 - qb1), dp = (qa1 + qb1) * (qa1 + qb1);
  S t1 = r + qa1 - qb1, t2 = r + qa1 + qb1, t3 = r - qa1 - qb1, t4 = r - qa1 + qb1;
  ri[19] = g(t1 * t1 + dm, aqq) * ev3 - g(t2 * t2 + dm, aqq) * ev3 - g(t3 * t3 + dm, aqq) * ev3 + g(t4 * t4 + dm, aqq) * ev3 -
           g(t1 * t1 + dp, aqq) * ev3 + g(t2 * t2 + dp, aqq) * ev3 + g(t3 * t3 + dp, aqq) * ev3 - g(t4 * t4 + dp, aqq) * ev3;
  S qxxqyy = g(r * r + qa * qa + qb * qb, aqq) * ev2 - ev2dsqr39 - ev2dsqr40 + ev2dsqr36;
  ri[20] = ee + eqxx + qxxe + qxxqyy;
  ri[21] = (qxxqxx - qxxqyy) * 0.5;
}

// integrals.rs:466-478
template <class S> void build_wxh(const S ri[4], const S r0[3], const S r1[3], const S r2[3], S wxh[10]) {
  wxh[pack(0, 0)] = ri[0];
  for (int k = 0; k < 3; ++k) wxh[pack(k + 1, 0)] = ri[1] * r0[k];
  for (int k = 0; k < 3; ++k)
    for (int l = 0; l <= k; ++l) {
      S t0 = r0[k] * r0[l];
      S t1 = r1[k] * r1[l] + r2[k] * r2[l];
      wxh[pack(k + 1, l + 1)] = ri[2] * t0 + ri[3] * t1;
    }
}

// integrals.rs:480-552
template <class S> void rotate_xx(const S ri[22], const S r0[3], const S r1[3], const S r2[3], S w[100]) {
  int idx = 0;
  for (int kk = 0; kk < 4; ++kk)
    for (int ll = 0; ll <= kk; ++ll)
      for (int mm = 0; mm < 4; ++mm)
        for (int nn = 0; nn <= mm; ++nn) {
          int k = kk - 1, l = ll - 1, m = mm - 1, n = nn - 1;
          S v;
          if (kk == 0) {
            if (mm == 0) v = ri[0];
            else if (nn == 0) v = ri[4] * r0[m];
            else v = ri[10] * (r0[m] * r0[n]) + ri[11] * (r1[m] * r1[n] + r2[m] * r2[n]);
          } else if (ll == 0) {
            if (mm == 0) v = ri[1] * r0[k];
            else if (nn == 0) v = ri[5] * (r0[k] * r0[m]) + ri[6] * (r1[k] * r1[m] + r2[k] * r2[m]);
            else {
              S t0 = r0[k] * r0[m] * r0[n];
              S t1 = (r1[m] * r1[n] + r2[m] * r2[n]) * r0[k];
              S mix = r1[k] * (r1[n] * r0[m] + r1[m] * r0[n]) + r2[k] * (r2[m] * r0[n] + r2[n] * r0[m]);
              v = ri[12] * t0 + ri[13] * t1 + ri[14] * mix;
            }
          } else if (mm == 0) {
            S t0 = r0[k] * r0[l];
            S t1 = r1[k] * r1[l] + r2[k] * r2[l];
            v = ri[2] * t0 + ri[3] * t1;
          } else if (nn == 0) {
            S t0 = r0[k] * r0[l] * r0[m];
            S t1 = (r1[k] * r1[l] + r2[k] * r2[l]) * r0[m];
            S t2 = r1[l] * r1[m] + r2[l] * r2[m];
            v = ri[7] * t0 + ri[8] * t1 + ri[9] * (r0[k] * t2 + r0[l] * (r1[k] * r1[m] + r2[k] * r2[m]));
          } else {
            S t0 = r0[k] * r0[l] * r0[m] * r0[n];
            v = ri[15] * t0;
            v = v + ri[16] * ((r1[k] * r1[l] + r2[k] * r2[l]) * r0[m] * r0[n]);
            v = v + ri[17] * ((r1[m] * r1[n] + r2[m] * r2[n]) * (r0[k] * r0[l]));
            v = v + ri[18] * (r1[k] * r1[l] * r1[m] * r1[n] + r2[k] * r2[l] * r2[m] * r2[n]);
            S mix1 = r0[m] * (r1[l] * r1[n] + r2[l] * r2[n]);
            S mix2 = r0[n] * (r1[l] * r1[m] + r2[l] * r2[m]);
            S val5 = r0[k] * (mix1 + mix2) + r0[l] * (r0[m] * (r1[k] * r1[n] + r2[k] * r2[n]) + r0[n] * (r1[k] * r1[m] + r2[k] * r2[m]));
            v = v + ri[19] * val5;
            v = v + ri[20] * (r1[k] * r1[l] * r2[m] * r2[n] + r2[k] * r2[l] * r1[m] * r1[n]);
            S cross = (r1[k] * r2[l] + r2[k] * r1[l]) * (r1[m] * r2[n] + r2[m] * r1[n]);
            v = v + ri[21] * cross;
          }
          w[idx++] = v;
        }
}

// integrals.rs:234-271 (MOPAC spcore); block is 4x4 row-major
template <class S> void core_attraction(const Elem& orb, const Elem& core, const S dvec[3], S block[16]) {
  for (int i = 0; i < 16; ++i) block[i] = cst<S>(0.0);
  S r = dsqrt(dvec[0] * dvec[0] + dvec[1] * dvec[1] + dvec[2] * dvec[2]);
  double core_rho = core.po[9];
  block[0] = drecip(dsqrt(r * r + (orb.po[1] + core_rho) * (orb.po[1] + core_rho))) * (-core.core * EV);
  if (orb.z < 3 || !orb.has_p()) return;
  S inv = drecip(r);
  S x[3] = {dvec[0] * inv, dvec[1] * inv, dvec[2] * inv};
  S rot[3][3];
  rotation_to_x(cst<S>(0.0) - x[0], cst<S>(0.0) - x[1], cst<S>(0.0) - x[2], rot);
  Mp oc{orb.ddp[2], orb.ddp[3] / std::sqrt(2.0), orb.po[1], orb.po[2], orb.po[3]};
  Mp pc{0.0, 0.0, core_rho, 0.0, 0.0};
  S loc[4], packed[10];
  local_xh(oc, pc, r, loc);
  build_wxh(loc, rot[0], rot[1], rot[2], packed);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) block[a * 4 + b] = packed[pack(a, b)] * (-core.core);
}

// integrals.rs:167-230. w has pa*pb entries (row-major, pa rows).
template <class S> void pair_two_electron(const Elem& ei, const Elem& ej, const S dvec[3], S* w, S e1b[16], S e2a[16]) {
  S r = dsqrt(dvec[0] * dvec[0] + dvec[1] * dvec[1] + dvec[2] * dvec[2]);
  S inv = drecip(r);
  S x[3] = {dvec[0] * inv, dvec[1] * inv, dvec[2] * inv};
  core_attraction(ei, ej, dvec, e1b);
  S md[3] = {cst<S>(0.0) - dvec[0], cst<S>(0.0) - dvec[1], cst<S>(0.0) - dvec[2]};
  core_attraction(ej, ei, md, e2a);
  S rot[3][3];
  rotation_to_x(cst<S>(0.0) - x[0], cst<S>(0.0) - x[1], cst<S>(0.0) - x[2], rot);
  bool hi = ei.has_p(), hj = ej.has_p();
  if (!hi && !hj) {
    double aee = (ei.rho0 + ej.rho0) * (ei.rho0 + ej.rho0);
    w[0] = drecip(dsqrt(r * r + aee)) * EV;
    return;
  }
  if (hi && !hj) {
    S ri[4];
    local_xh(mp_of(ei), mp_of(ej), r, ri);
    build_wxh(ri, rot[0], rot[1], rot[2], w);
    return;
  }
  S ri[22];
  local_xx(mp_of(ei), mp_of(ej), r, ri);
  rotate_xx(ri, rot[0], rot[1], rot[2], w);
}

// ---------------------------------------------------------------- overlap (overlap.rs)
// overlap.rs:763-774
template <class S> void aintgs(S x, S a[13]) {
  for (int i = 0; i < 13; ++i) a[i] = cst<S>(0.0);
  if (std::fabs(val(x)) < 1.0e-12) return;
  S inv = drecip(x);
  a[0] = dexp(cst<S>(0.0) - x) * inv;
  for (int i = 1; i < 13; ++i) a[i] = a[0] + a[i - 1] * inv * (double)i;
}
// overlap.rs:814-850
template <class S> void bintgs(S x, S b[13]) {
  for (int i = 0; i < 13; ++i) b[i] = cst<S>(0.0);
  double absx = std::fabs(val(x));
  if (absx > 3.0) {
    S inv = drecip(x);
    S tx = dexp(x) * inv;
    S tmx = dexp(cst<S>(0.0) - x) * inv * (-1.0);
    b[0] = tx + tmx;
    for (int i = 1; i < 13; ++i) {
      double sign = (i % 2 == 0) ? 1.0 : -1.0;
      b[i] = tx * sign + tmx + b[i - 1] * inv * (double)i;
    }
  } else {
    S term = cst<S>(1.0);
    for (int m = 0; m < 40; ++m) {
      for (int k = 0; k < 13; ++k)
        if ((k + m) % 2 == 0) b[k] = b[k] + term * (2.0 / (double)(k + m + 1));
      term = term * (cst<S>(0.0) - x) * (1.0 / (double)(m + 1));
    }
  }
}

// overlap.rs:266-475 (n <= 3 analytic branches). ea has the larger principal quantum number.
template <class S> bool overlap_locals(const Elem& ea, const Elem& eb, S r, S out[5]) {
  int jcall = 0;
  int na = ea.n, nb = eb.n;
  if (na == 1 && nb == 1) jcall = 2;
  else if (na == 2 && nb == 1) jcall = 3;
  else if (na == 2 && nb == 2) jcall = 4;
  else if (na == 3 && nb == 1) jcall = 431;
  else if (na == 3 && nb == 2) jcall = 5;
  else if (na == 3 && nb == 3) jcall = 6;
  if (jcall == 0) return false;
  double za[2] = {ea.zs, ea.zp}, zb[2] = {eb.zs, eb.zp};
  double sums[4] = {za[0] + zb[0], za[1] + zb[0], za[0] + zb[1], za[1] + zb[1]};
  double smallest = std::numeric_limits<double>::infinity();
  for (double s : sums)
    if (s > 0.0) smallest = std::min(smallest, s);
  smallest *= 0.5;
  if (std::isfinite(smallest) && val(r) * smallest > 300.0) {
    for (int i = 0; i < 5; ++i) out[i] = cst<S>(0.0);
    return true;
  }
  S a111[13], b111[13], a211[13], b211[13], a121[13], b121[13], a22[13], b22[13];
  aintgs(r * (0.5 * (za[0] + zb[0])), a111); bintgs(r * (0.5 * (za[0] - zb[0])), b111);
  aintgs(r * (0.5 * (za[1] + zb[0])), a211); bintgs(r * (0.5 * (za[1] - zb[0])), b211);
  aintgs(r * (0.5 * (za[0] + zb[1])), a121); bintgs(r * (0.5 * (za[0] - zb[1])), b121);
  aintgs(r * (0.5 * (za[1] + zb[1])), a22); bintgs(r * (0.5 * (za[1] - zb[1])), b22);
  S s111 = cst<S>(0.0), s211 = cst<S>(0.0), s121 = cst<S>(0.0), s221 = cst<S>(0.0), s222 = cst<S>(0.0);
  const double sq3 = std::sqrt(3.0);
  switch (jcall) {
    case 2:
      s111 = dpowf(r * r * (za[0] * zb[0]), 1.5) * (a111[2] * b111[0] - b111[2] * a111[0]) / 4.0;
      break;
    case 3:
      s111 = dpowi(r, 4) * (std::pow(zb[0], 1.5) * std::pow(za[0], 2.5)) *
             (a111[3] * b111[0] - b111[3] * a111[0] + a111[2] * b111[1] - b111[2] * a111[1]) / (sq3 * 8.0);
      s211 = dpowi(r, 4) * (std::pow(zb[0], 1.5) * std::pow(za[1], 2.5)) *
             (a211[2] * b211[0] - b211[2] * a211[0] + a211[3] * b211[1] - b211[3] * a211[1]) / 8.0;
      break;
    case 4: {
      s111 = dpowi(r, 5) * std::pow(zb[0] * za[0], 2.5) * (a111[4] * b111[0] + b111[4] * a111[0] - a111[2] * b111[2] * 2.0) / 48.0;
      s211 = dpowi(r, 5) * std::pow(zb[0] * za[1], 2.5) *
             (a211[3] * (b211[0] - b211[2]) - a211[1] * (b211[2] - b211[4]) + b211[3] * (a211[0] - a211[2]) -
              b211[1] * (a211[2] - a211[4])) / (16.0 * sq3);
      s121 = dpowi(r, 5) * std::pow(zb[1] * za[0], 2.5) *
             (a121[3] * (b121[0] - b121[2]) - a121[1] * (b121[2] - b121[4]) - b121[3] * (a121[0] - a121[2]) +
              b121[1] * (a121[2] - a121[4])) / (16.0 * sq3);
      S w = dpowi(r, 5) * std::pow(zb[1] * za[1], 2.5) / 16.0;
      s221 = cst<S>(0.0) - (w * (b22[2] * (a22[4] + a22[0]) - a22[2] * (b22[4] + b22[0])));
      s222 = w * (a22[4] * (b22[0] - b22[2]) - b22[4] * (a22[0] - a22[2]) - a22[2] * b22[0] + b22[2] * a22[0]) * 0.5;
      break;
    }
    case 431:
      s111 = dpowi(r, 5) * (std::pow(zb[0], 1.5) * std::pow(za[0], 3.5)) *
             (a111[4] * b111[0] + b111[1] * a111[3] * 2.0 - a111[1] * b111[3] * 2.0 - b111[4] * a111[0]) /
             (std::sqrt(10.0) * 24.0);
      s211 = dpowi(r, 5) * (std::pow(zb[0], 1.5) * std::pow(za[1], 3.5)) *
             (a211[3] * (b211[0] + b211[2]) - a211[1] * (b211[4] + b211[2]) + b211[1] * (a211[2] + a211[4]) -
              b211[3] * (a211[2] + a211[0])) / (8.0 * std::sqrt(30.0));
      break;
    case 5:
      s111 = dpowi(r, 6) * (std::pow(zb[0], 2.5) * std::pow(za[0], 3.5)) *
             (a111[5] * b111[0] + b111[1] * a111[4] - b111[2] * a111[3] * 2.0 - a111[2] * b111[3] * 2.0 +
              b111[4] * a111[1] + b111[5] * a111[0]) / (std::sqrt(30.0) * 48.0);
      s211 = dpowi(r, 6) * (std::pow(zb[0], 2.5) * std::pow(za[1], 3.5)) *
             (a211[4] * b211[0] + b211[1] * a211[5] - b211[3] * a211[3] * 2.0 - a211[2] * b211[2] * 2.0 +
              a211[1] * b211[5] + a211[0] * b211[4]) / (48.0 * std::sqrt(10.0));
      s121 = dpowi(r, 6) * (std::pow(zb[1], 2.5) * std::pow(za[0], 3.5)) *
             ((a121[4] * b121[0] - a121[5] * b121[1]) + (a121[3] * b121[1] - a121[4] * b121[2]) * 2.0 -
              (a121[1] * b121[3] - a121[2] * b121[4]) * 2.0 - (a121[0] * b121[4] - a121[1] * b121[5])) /
             (48.0 * std::sqrt(10.0));
      s221 = dpowi(r, 6) * (std::pow(zb[1], 2.5) * std::pow(za[1], 3.5)) *
             ((a22[3] * b22[0] - a22[5] * b22[2]) + (a22[2] * b22[1] - a22[4] * b22[3]) - (a22[1] * b22[2] - a22[3] * b22[4]) -
              (a22[0] * b22[3] - a22[2] * b22[5])) / (16.0 * std::sqrt(30.0));
      s222 = dpowi(r, 6) * (std::pow(zb[1], 2.5) * std::pow(za[1], 3.5)) *
             ((a22[5] - a22[3]) * (b22[0] - b22[2]) + (a22[4] - a22[2]) * (b22[1] - b22[3]) -
              (a22[3] - a22[1]) * (b22[2] - b22[4]) - (a22[2] - a22[0]) * (b22[3] - b22[5])) / (32.0 * std::sqrt(30.0));
      break;
    case 6:
      s111 = dpowi(r, 7) * std::pow(zb[0] * za[0], 3.5) *
             (a111[6] * b111[0] - b111[2] * a111[4] * 3.0 + a111[2] * b111[4] * 3.0 - a111[0] * b111[6]) / 1440.0;
      s211 = dpowi(r, 7) * std::pow(zb[0] * za[1], 3.5) *
             ((a211[5] * b211[0] + a211[6] * b211[1]) + (cst<S>(0.0) - a211[4] * b211[1] - a211[5] * b211[2]) -
              (a211[3] * b211[2] + a211[4] * b211[3]) * 2.0 - (cst<S>(0.0) - a211[2] * b211[3] - a211[3] * b211[4]) * 2.0 +
              (a211[1] * b211[4] + a211[2] * b211[5]) + (cst<S>(0.0) - a211[0] * b211[5] - a211[1] * b211[6])) /
             (480.0 * sq3);
      s121 = dpowi(r, 7) * std::pow(zb[1] * za[0], 3.5) *
             ((a121[5] * b121[0] - a121[6] * b121[1]) + (a121[4] * b121[1] - a121[5] * b121[2]) -
              (a121[3] * b121[2] - a121[4] * b121[3]) * 2.0 - (a121[2] * b121[3] - a121[3] * b121[4]) * 2.0 +
              (a121[1] * b121[4] - a121[2] * b121[5]) + (a121[0] * b121[5] - a121[1] * b121[6])) /
             (480.0 * sq3);
      s221 = dpowi(r, 7) * (std::pow(zb[1], 3.5) * std::pow(za[1], 3.5)) *
             ((a22[4] * b22[0] - a22[6] * b22[2]) - (a22[2] * b22[2] - a22[4] * b22[4]) * 2.0 +
              (a22[0] * b22[4] - a22[2] * b22[6])) / 480.0;
      s222 = dpowi(r, 7) * (std::pow(zb[1], 3.5) * std::pow(za[1], 3.5)) *
             ((a22[6] - a22[4]) * (b22[0] - b22[2]) - (a22[4] - a22[2]) * (b22[2] - b22[4]) * 2.0 +
              (a22[2] - a22[0]) * (b22[4] - b22[6])) / 960.0;
      break;
  }
  out[0] = s111; out[1] = s211; out[2] = s121; out[3] = s221; out[4] = s222;
  return true;
}

// overlap.rs:480-507
template <class S> void build_di(const S s[5], const S dir[3], S di[16]) {
  S rr[3][3];
  rotation_to_x(dir[0], dir[1], dir[2], rr);
  S ro[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) ro[a][b] = rr[b][a];
  di[0] = s[0];
  for (int a = 0; a < 3; ++a) {
    di[(1 + a) * 4 + 0] = s[1] * ro[a][0];
    di[0 * 4 + 1 + a] = cst<S>(0.0) - s[2] * ro[a][0];
  }
  S mm[3] = {cst<S>(0.0) - s[3], s[4], s[4]};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      S v = cst<S>(0.0);
      for (int k = 0; k < 3; ++k) v = v + ro[a][k] * mm[k] * ro[b][k];
      di[(1 + a) * 4 + 1 + b] = v;
    }
}

// overlap.rs:103-127 (f64) and 133-159 (Dual). dvec = R_j - R_i. Returns false when no
// analytic branch exists for the pair.
template <class S> bool diatom_overlap(const Elem& ei, const Elem& ej, const S dvec[3], S out[16]) {
  S r = dsqrt(dvec[0] * dvec[0] + dvec[1] * dvec[1] + dvec[2] * dvec[2]);
  if (val(r) < 1.0e-8) {
    for (int i = 0; i < 16; ++i) out[i] = cst<S>(i % 5 == 0 ? 1.0 : 0.0);
    return true;
  }
  bool swap = ei.n < ej.n;
  const Elem& ea = swap ? ej : ei;
  const Elem& eb = swap ? ei : ej;
  S inv = drecip(r);
  double sg = swap ? -1.0 : 1.0;
  S dir[3] = {dvec[0] * inv * sg, dvec[1] * inv * sg, dvec[2] * inv * sg};
  S loc[5];
  if (!overlap_locals(ea, eb, r, loc)) return false;
  S di[16];
  build_di(loc, dir, di);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) out[a * 4 + b] = swap ? di[b * 4 + a] : di[a * 4 + b];
  return true;
}

// ---------------------------------------------------------------- core-core (repulsion.rs:57-120)
template <class S> S pair_core_energy(const Elem& ei, const Elem& ej, S dist) {
  const Params& P = params();
  S ra = dist * A0;
  double rho = ei.po[9] + ej.po[9];
  S gab = drecip(dsqrt(dist * dist + rho * rho)) * EV;
  double cp = ei.core * ej.core;
  S bare = gab * cp;
  bool has_pair = false;
  double alpha = 0, x = 0;
  if (ei.norb != 0 && ej.norb != 0 && P.have_pair[ei.z][ej.z] && std::fabs(P.pair_x[ei.z][ej.z]) > 1.0e-5) {
    has_pair = true;
    alpha = P.pair_alpha[ei.z][ej.z];
    x = P.pair_x[ei.z][ej.z];
  }
  S e;
  if (has_pair) {
    double a = alpha < 1.0e-6 ? 1.2 : alpha;
    S scale = cst<S>(1.0) + dexp(ra * (-a)) * (2.0 * x);
    e = bare * scale;
  } else {
    S exi = dexp(ra * (-ei.alpha)), exj = dexp(ra * (-ej.alpha));
    S scale = exi + exj;
    int zs = ei.z + ej.z;
    if (zs == 8 || zs == 9) {
      if (ei.z == 7 || ei.z == 8) scale = scale + (ra - 1.0) * exi;
      if (ej.z == 7 || ej.z == 8) scale = scale + (ra - 1.0) * exj;
    }
    e = dabs(scale * bare) + bare;
  }
  if (!has_pair) {
    for (int pass = 0; pass < 2; ++pass) {
      const Elem& g = pass == 0 ? ei : ej;
      for (auto& t : g.gauss) {
        S delta = ra - t[2];
        S ax = delta * delta * t[1];
        if (val(ax) <= 25.0) e = e + dexp(cst<S>(0.0) - ax) * (cp * t[0]) / ra;
      }
    }
  }
  return e;
}

// ---------------------------------------------------------------- dense linear algebra
typedef void (*dsyevd_t)(const char*, const char*, const int*, double*, const int*, double*, double*,
                         const int*, int*, const int*, int*);
typedef void (*dgemm_t)(const char*, const char*, const int*, const int*, const int*, const double*,
                        const double*, const int*, const double*, const int*, const double*, double*,
                        const int*);
dsyevd_t g_dsyevd = nullptr;
dgemm_t g_dgemm = nullptr;

using Mat = std::vector<double>;  // row-major n x n

// Cyclic Jacobi (textbook); used when no LAPACK entry point was supplied.
bool jacobi_eigh(int n, Mat a, std::vector<double>& w, Mat& v) {
  v.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double x = a[(size_t)i * n + j] * a[(size_t)i * n + j];
        tot += x;
        if (i != j) off += x;
      }
    if (off <= 1e-30 * std::max(tot, 1e-300)) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = a[(size_t)p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
          a[(size_t)k * n + p] = c * akp - s * akq;
          a[(size_t)k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
          a[(size_t)p * n + k] = c * apk - s * aqk;
          a[(size_t)q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
          v[(size_t)k * n + p] = c * vkp - s * vkq;
          v[(size_t)k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return a[(size_t)x * n + x] < a[(size_t)y * n + y]; });
  w.resize(n);
  Mat vs((size_t)n * n);
  for (int c = 0; c < n; ++c) {
    w[c] = a[(size_t)order[c] * n + order[c]];
    for (int i = 0; i < n; ++i) vs[(size_t)i * n + c] = v[(size_t)i * n + order[c]];
  }
  v.swap(vs);
  return true;
}

// linalg.rs:221-263: eigenvalues ascending, eigenvectors as columns of a row-major matrix.
bool eigh(int n, const Mat& a, std::vector<double>& w, Mat& v) {
  if (n == 0) { w.clear(); v.clear(); return true; }
  if (!g_dsyevd) return jacobi_eigh(n, a, w, v);
  Mat z = a;  // symmetric: row-major == column-major
  w.assign(n, 0.0);
  int lwork = -1, liwork = -1, info = 0;
  double wq;
  int iwq;
  g_dsyevd("V", "L", &n, z.data(), &n, w.data(), &wq, &lwork, &iwq, &liwork, &info);
  lwork = (int)wq;
  liwork = iwq;
  std::vector<double> work(std::max(lwork, 1));
  std::vector<int> iwork(std::max(liwork, 1));
  g_dsyevd("V", "L", &n, z.data(), &n, w.data(), work.data(), &lwork, iwork.data(), &liwork, &info);
  if (info != 0) return false;
  v.assign((size_t)n * n, 0.0);  // z is column-major: z[i + j*n] = component i of vector j
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) v[(size_t)i * n + j] = z[(size_t)j * n + i];
  return true;
}

// C = A * B for row-major n x n (general)
void matmul(int n, const Mat& a, const Mat& b, Mat& c) {
  c.assign((size_t)n * n, 0.0);
  if (g_dgemm && n >= 32) {
    // row-major C = A B  <=>  column-major C^T = B^T A^T
    double one = 1.0, zero = 0.0;
    g_dgemm("N", "N", &n, &n, &n, &one, b.data(), &n, a.data(), &n, &zero, c.data(), &n);
    return;
  }
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) {
      double aik = a[(size_t)i * n + k];
      if (aik == 0.0) continue;
      const double* br = &b[(size_t)k * n];
      double* cr = &c[(size_t)i * n];
      for (int j = 0; j < n; ++j) cr[j] += aik * br[j];
    }
}

// linalg.rs:128-147: P = w * C[:, :k] C[:, :k]^T
Mat leading_columns_gram(int n, const Mat& c, int k, double wgt) {
  Mat p((size_t)n * n, 0.0);
  if (n == 0 || k == 0) return p;
  if (g_dgemm && n >= 32) {
    // row-major c (n x n). As column-major it is C^T (n x n); P^T = P = C_k C_k^T.
    // column-major: P = (C^T)[:k, :]^T (C^T)[:k, :]
    double zero = 0.0;
    g_dgemm("T", "N", &n, &n, &k, &wgt, c.data(), &n, c.data(), &n, &zero, p.data(), &n);
    return p;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = 0.0;
      for (int o = 0; o < k; ++o) s += c[(size_t)i * n + o] * c[(size_t)j * n + o];
      p[(size_t)i * n + j] = p[(size_t)j * n + i] = wgt * s;
    }
  return p;
}

double fdot(const Mat& a, const Mat& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}
double rms_diff(const Mat& a, const Mat& b) {
  double s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s += (a[i] - b[i]) * (a[i] - b[i]);
  return std::sqrt(s / (double)std::max<size_t>(a.size(), 1));
}

// ---------------------------------------------------------------- molecule / basis
struct Molecule {
  int natom = 0, nao = 0;
  std::vector<int> z;
  std::vector<double> xyz;  // Bohr
  std::vector<const Elem*> el;
  std::vector<int> off, norb;  // basis.rs:39-63
};

struct Error {
  int code;
  std::string msg;
};

bool build_molecule(int n, const int* z, const double* xyz, Molecule& m, Error& err) {
  m.natom = n;
  m.z.assign(z, z + n);
  m.xyz.assign(xyz, xyz + 3 * n);
  m.el.resize(n);
  m.off.resize(n);
  m.norb.resize(n);
  int nao = 0;
  for (int i = 0; i < n; ++i) {
    const Elem* e = params().get(z[i]);
    if (!e) {
      err = {2, "missing PM3 parameter block for Z=" + std::to_string(z[i])};
      return false;
    }
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(xyz[3 * i + k])) {
        err = {1, "non-finite coordinate"};
        return false;
      }
    m.el[i] = e;
    m.off[i] = nao;
    m.norb[i] = e->norb;
    nao += e->norb;
  }
  m.nao = nao;
  return true;
}

// ---------------------------------------------------------------- H_core (hamiltonian.rs:191-344)
struct PairInt {
  int a, b, na, nb;
  std::vector<double> w;  // pa x pb
};
struct Core {
  Mat h;
  std::vector<PairInt> pairs;
};

inline double beta_of(const Elem& e, int orb) { return orb == 0 ? e.bs : e.bp; }

bool build_core(const Molecule& m, Core& core, Error& err) {
  int n = m.nao;
  core.h.assign((size_t)n * n, 0.0);
  for (int i = 0; i < m.natom; ++i)
    for (int k = 0; k < m.norb[i]; ++k) core.h[(size_t)(m.off[i] + k) * n + m.off[i] + k] = k == 0 ? m.el[i]->uss : m.el[i]->upp;
  std::vector<std::pair<int, int>> idx;
  for (int u = 0; u < m.natom; ++u)
    for (int v = u + 1; v < m.natom; ++v) idx.push_back({u, v});
  size_t np = idx.size();
  core.pairs.resize(np);
  std::vector<double> blocks(np * 48);  // e1b, e2a, s per pair
  std::vector<int> bad(np, 0);
#pragma omp parallel for schedule(dynamic, 64) if (np > 4096)
  for (long t = 0; t < (long)np; ++t) {
    int u = idx[t].first, v = idx[t].second;
    const Elem &eu = *m.el[u], &ev = *m.el[v];
    int a = (eu.has_p() || !ev.has_p()) ? u : v;  // hamiltonian.rs:277-281
    int b = a == u ? v : u;
    const Elem &ea = *m.el[a], &eb = *m.el[b];
    double d[3] = {m.xyz[3 * b] - m.xyz[3 * a], m.xyz[3 * b + 1] - m.xyz[3 * a + 1], m.xyz[3 * b + 2] - m.xyz[3 * a + 2]};
    double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double dv[3] = {d[0] / r * r, d[1] / r * r, d[2] / r * r};  // integrals.rs:161-163
    PairInt& pi = core.pairs[t];
    pi.a = a; pi.b = b; pi.na = ea.norb; pi.nb = eb.norb;
    int pa = ea.norb * (ea.norb + 1) / 2, pb = eb.norb * (eb.norb + 1) / 2;
    pi.w.assign((size_t)pa * pb, 0.0);
    double* blk = &blocks[t * 48];
    pair_two_electron<double>(ea, eb, dv, pi.w.data(), blk, blk + 16);
    if (!diatom_overlap<double>(ea, eb, d, blk + 32)) bad[t] = 1;
  }
  for (size_t t = 0; t < np; ++t) {
    if (bad[t]) {
      err = {1, "no analytic overlap branch for this element pair"};
      return false;
    }
    const PairInt& pi = core.pairs[t];
    const double* blk = &blocks[t * 48];
    int oa = m.off[pi.a], ob = m.off[pi.b];
    for (int i = 0; i < pi.na; ++i)
      for (int j = 0; j < pi.na; ++j) core.h[(size_t)(oa + i) * n + oa + j] += blk[i * 4 + j];
    for (int i = 0; i < pi.nb; ++i)
      for (int j = 0; j < pi.nb; ++j) core.h[(size_t)(ob + i) * n + ob + j] += blk[16 + i * 4 + j];
    const Elem &ea = *m.el[pi.a], &eb = *m.el[pi.b];
    for (int i = 0; i < pi.na; ++i) {
      double bi = beta_of(ea, i);
      for (int j = 0; j < pi.nb; ++j) {
        double bj = beta_of(eb, j);
        double value = 0.5 * (bi + bj) * blk[32 + i * 4 + j];
        core.h[(size_t)(oa + i) * n + ob + j] = value;
        core.h[(size_t)(ob + j) * n + oa + i] = value;
      }
    }
  }
  return true;
}

// ---------------------------------------------------------------- Fock (fock.rs)
// fock.rs:244-282
double oc_two_electron(int a, int b, int c, int d, const Elem& e) {
  if (a == b && c == d) {
    if (a == 0 && c == 0) return e.gss;
    if (a == 0 || c == 0) return e.gsp;
    return a == c ? e.gpp : e.gp2;
  }
  int ba = std::min(a, b), bb = std::max(a, b), kc = std::min(c, d), kd = std::max(c, d);
  if (ba == 0 && bb != 0 && kc == 0 && kd != 0 && bb == kd) return e.hsp;
  if (ba != 0 && bb != 0 && ba != bb && ba == kc && bb == kd) return 0.5 * (e.gpp - e.gp2);
  return 0.0;
}

// fock.rs:285-332 (build_fock_spin): F = H + J(p_tot) - K(p_spin)
Mat build_fock_spin(const Molecule& m, const Core& core, const Mat& pt, const Mat& ps) {
  int n = m.nao;
  Mat f = core.h;
  for (int ia = 0; ia < m.natom; ++ia) {
    int off = m.off[ia], no = m.norb[ia];
    const Elem& e = *m.el[ia];
    for (int mu = 0; mu < no; ++mu)
      for (int nu = 0; nu < no; ++nu) {
        double acc = 0.0;
        for (int la = 0; la < no; ++la)
          for (int si = 0; si < no; ++si) {
            acc += pt[(size_t)(off + la) * n + off + si] * oc_two_electron(mu, nu, la, si, e);
            acc -= ps[(size_t)(off + la) * n + off + si] * oc_two_electron(mu, la, nu, si, e);
          }
        f[(size_t)(off + mu) * n + off + nu] += acc;
      }
  }
  // fock.rs:106-193: per-pair packed Coulomb mat-vecs + exchange into slots, then scatter.
  size_t np = core.pairs.size();
  const int STRIDE = 10 + 10 + 16;
  std::vector<double> slots(np * STRIDE);
#pragma omp parallel for schedule(static, 256) if (np > 8192)
  for (long t = 0; t < (long)np; ++t) {
    const PairInt& pi = core.pairs[t];
    double* s = &slots[t * STRIDE];
    for (int k = 0; k < STRIDE; ++k) s[k] = 0.0;
    int oa = m.off[pi.a], ob = m.off[pi.b], na = pi.na, nb = pi.nb;
    int pa = na * (na + 1) / 2, pb = nb * (nb + 1) / 2;
    double da[10], db[10];
    for (int mu = 0; mu < na; ++mu) {  // fock.rs:93-100
      da[pack(mu, mu)] = pt[(size_t)(oa + mu) * n + oa + mu];
      for (int nu = 0; nu < mu; ++nu) da[pack(mu, nu)] = 2.0 * pt[(size_t)(oa + mu) * n + oa + nu];
    }
    for (int mu = 0; mu < nb; ++mu) {
      db[pack(mu, mu)] = pt[(size_t)(ob + mu) * n + ob + mu];
      for (int nu = 0; nu < mu; ++nu) db[pack(mu, nu)] = 2.0 * pt[(size_t)(ob + mu) * n + ob + nu];
    }
    const double* w = pi.w.data();
    for (int p = 0; p < pa; ++p) {
      double acc = 0.0;
      for (int q = 0; q < pb; ++q) acc += db[q] * w[p * pb + q];
      s[p] = acc;
      for (int q = 0; q < pb; ++q) s[10 + q] += da[p] * w[p * pb + q];
    }
    for (int mu = 0; mu < na; ++mu)
      for (int nu = 0; nu < na; ++nu) {
        const double* row = w + pack(mu, nu) * pb;
        for (int la = 0; la < nb; ++la) {
          double acc = 0.0;
          for (int si = 0; si < nb; ++si) acc += ps[(size_t)(oa + nu) * n + ob + si] * row[pack(la, si)];
          s[20 + mu * 4 + la] -= acc;
        }
      }
  }
  for (size_t t = 0; t < np; ++t) {
    const PairInt& pi = core.pairs[t];
    const double* s = &slots[t * STRIDE];
    int oa = m.off[pi.a], ob = m.off[pi.b];
    for (int mu = 0; mu < pi.na; ++mu)
      for (int nu = 0; nu < pi.na; ++nu) f[(size_t)(oa + mu) * n + oa + nu] += s[pack(mu, nu)];
    for (int la = 0; la < pi.nb; ++la)
      for (int si = 0; si < pi.nb; ++si) f[(size_t)(ob + la) * n + ob + si] += s[10 + pack(la, si)];
    for (int mu = 0; mu < pi.na; ++mu)
      for (int la = 0; la < pi.nb; ++la) {
        double value = f[(size_t)(oa + mu) * n + ob + la] + s[20 + mu * 4 + la];
        f[(size_t)(oa + mu) * n + ob + la] = value;
        f[(size_t)(ob + la) * n + oa + mu] = value;
      }
  }
  return f;
}

// fock.rs:488-500
Mat build_fock(const Molecule& m, const Core& core, const Mat& p) {
  Mat half = p;
  for (double& v : half) v *= 0.5;
  return build_fock_spin(m, core, p, half);
}

// ---------------------------------------------------------------- SCF (scf.rs)
enum Accel { ACC_NONE = 0, ACC_CDIIS = 1, ACC_ADIIS = 2 };
enum Guess { G_AUTO = 0, G_SAD = 1, G_CORE = 2, G_SYM = 3 };

const int MAX_DIIS_DEPTH = 8;  // scf.rs:300
// scf.rs:309-331
size_t slot_bytes(int nao, int mps) { return (size_t)mps * nao * nao * 8; }
int diis_depth(int nao, int mps, int budget_mb) {
  if (budget_mb == 0) return MAX_DIIS_DEPTH;
  size_t per = slot_bytes(nao, mps);
  if (per == 0) return MAX_DIIS_DEPTH;
  size_t budget = (size_t)budget_mb * 1024 * 1024;
  return (int)std::min<size_t>(std::max<size_t>(budget / per, 2), MAX_DIIS_DEPTH);
}
bool diis_depth_fits(int nao, int mps, int budget_mb) {
  return budget_mb == 0 || 2 * slot_bytes(nao, mps) <= (size_t)budget_mb * 1024 * 1024;
}

// scf.rs:1039-1054
Mat commutator(int n, const Mat& f, const Mat& p) {
  Mat e;
  matmul(n, f, p, e);
  for (int i = 0; i < n; ++i) {
    e[(size_t)i * n + i] = 0.0;
    for (int j = 0; j < i; ++j) {
      double up = e[(size_t)j * n + i], lo = e[(size_t)i * n + j];
      e[(size_t)i * n + j] = lo - up;
      e[(size_t)j * n + i] = up - lo;
    }
  }
  return e;
}

// scf.rs:1501-1530
Mat combine(const std::vector<Mat>& fs, const std::vector<double>& c) {
  Mat out(fs[0].size(), 0.0);
  for (size_t i = 0; i < fs.size(); ++i) {
    double ci = c[i];
    for (size_t k = 0; k < out.size(); ++k) out[k] += ci * fs[i][k];
  }
  return out;
}

// scf.rs:1584-1630
bool solve_bordered_small(std::vector<std::vector<double>> m, std::vector<double> rhs, std::vector<double>& x) {
  int n = (int)m.size();
  for (int col = 0; col < n; ++col) {
    int pivot = col;
    double best = std::fabs(m[col][col]);
    for (int row = col + 1; row < n; ++row) {
      double v = std::fabs(m[row][col]);
      if (v > best) { best = v; pivot = row; }
    }
    if (best < 1.0e-12) return false;
    if (pivot != col) {
      std::swap(m[col], m[pivot]);
      std::swap(rhs[col], rhs[pivot]);
    }
    for (int row = col + 1; row < n; ++row) {
      double factor = m[row][col] / m[col][col];
      if (factor == 0.0) continue;
      for (int j = col; j < n; ++j) m[row][j] -= factor * m[col][j];
      rhs[row] -= factor * rhs[col];
    }
  }
  x.assign(n, 0.0);
  for (int col = n - 1; col >= 0; --col) {
    double sum = rhs[col];
    for (int j = col + 1; j < n; ++j) sum -= m[col][j] * x[j];
    x[col] = sum / m[col][col];
  }
  return true;
}

// scf.rs:1544-1580
bool diis_coeffs_from_gram(const std::vector<std::vector<double>>& gram, std::vector<double>& c) {
  int n = (int)gram.size();
  if (n < 2) return false;
  double scale = 0.0;
  for (auto& row : gram)
    for (double v : row) scale = std::max(scale, std::fabs(v));
  if (!std::isfinite(scale) || scale <= 0.0) return false;
  int dim = n + 1;
  std::vector<std::vector<double>> b(dim, std::vector<double>(dim, 0.0));
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) b[i][j] = gram[i][j] / scale;
    b[i][n] = -1.0;
    b[n][i] = -1.0;
  }
  std::vector<double> rhs(dim, 0.0);
  rhs[n] = -1.0;
  return solve_bordered_small(b, rhs, c);
}

// scf.rs:1677-1693
std::vector<double> simplex_project(const std::vector<double>& v) {
  std::vector<double> u = v;
  std::stable_sort(u.begin(), u.end(), [](double a, double b) { return a > b; });
  double css = 0.0, theta = 0.0;
  for (size_t j = 0; j < u.size(); ++j) {
    css += u[j];
    double t = (css - 1.0) / ((double)j + 1.0);
    if (u[j] - t > 0.0) theta = t;
  }
  std::vector<double> out(v.size());
  for (size_t i = 0; i < v.size(); ++i) out[i] = std::max(v[i] - theta, 0.0);
  return out;
}

// scf.rs:1637-1674
std::vector<double> solve_adiis_simplex(const std::vector<double>& d, const std::vector<std::vector<double>>& s) {
  int n = (int)d.size();
  double l = 1.0e-12;
  for (int i = 0; i < n; ++i) {
    double row = 0.0;
    for (int j = 0; j < n; ++j) row += std::fabs(s[i][j] + s[j][i]);
    l = std::max(l, row);
  }
  double lr = 1.0 / l;
  std::vector<double> c(n, 0.0);
  c[n - 1] = 1.0;
  for (int it = 0; it < 400; ++it) {
    std::vector<double> g(n), trial(n);
    for (int k = 0; k < n; ++k) {
      double acc = 2.0 * d[k];
      for (int j = 0; j < n; ++j) acc += (s[k][j] + s[j][k]) * c[j];
      g[k] = acc;
    }
    for (int i = 0; i < n; ++i) trial[i] = c[i] - lr * g[i];
    std::vector<double> proj = simplex_project(trial);
    double delta = 0.0;
    for (int i = 0; i < n; ++i) delta += std::fabs(proj[i] - c[i]);
    c = proj;
    if (delta < 1.0e-12) break;
  }
  return c;
}

// scf.rs:1065-1173
struct AccelHistory {
  int depth;
  bool keep;
  std::vector<Mat> focks, errors, dens;
  std::vector<std::vector<double>> b, mm;
  double push(Mat fock, Mat error, const Mat* density) {
    std::vector<double> brow;
    for (auto& e : errors) brow.push_back(fdot(e, error));
    double nsq = fdot(error, error);
    brow.push_back(nsq);
    for (size_t i = 0; i < b.size(); ++i) b[i].push_back(brow[i]);
    b.push_back(brow);
    if (keep && density) {
      std::vector<double> mrow;
      for (auto& f : focks) mrow.push_back(fdot(*density, f));
      mrow.push_back(fdot(*density, fock));
      for (size_t i = 0; i < mm.size(); ++i) mm[i].push_back(fdot(dens[i], fock));
      mm.push_back(mrow);
      dens.push_back(*density);
    }
    focks.push_back(std::move(fock));
    errors.push_back(std::move(error));
    while ((int)focks.size() > depth) {
      focks.erase(focks.begin());
      errors.erase(errors.begin());
      b.erase(b.begin());
      for (auto& row : b) row.erase(row.begin());
      if (keep) {
        dens.erase(dens.begin());
        mm.erase(mm.begin());
        for (auto& row : mm) row.erase(row.begin());
      }
    }
    return nsq;
  }
  bool cdiis(Mat& out) {
    std::vector<double> c;
    if (!diis_coeffs_from_gram(b, c)) return false;
    out = combine(focks, c);
    return true;
  }
  bool adiis(Mat& out) {
    int n = (int)focks.size();
    if (n < 2 || !keep) return false;
    int last = n - 1;
    double mnn = mm[last][last];
    std::vector<double> d(n);
    std::vector<std::vector<double>> s(n, std::vector<double>(n));
    for (int i = 0; i < n; ++i) d[i] = mm[i][last] - mnn;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) s[i][j] = mm[i][j] - mm[i][last] - mm[last][j] + mnn;
    out = combine(focks, solve_adiis_simplex(d, s));
    return true;
  }
};

struct State {
  Mat density, spin;
  bool has_spin = false;
  std::vector<double> eps, eps_b;
  bool has_beta = false;
  Mat coeff;
  int n_occ = 0, n_beta = 0;
  double electronic = 0.0, last_change = INFINITY;
  bool converged = false, unrestricted = false;
  int iterations = 0;
};

struct Opts {
  int max_scf;
  double e_tol, p_tol, adiis_switch, shift, damping;
  bool use_diis;
  int accel, guess, memory_mb;
};

// scf.rs:855-881
Mat sad_density(const Molecule& m) {
  int n = m.nao;
  Mat p((size_t)n * n, 0.0);
  for (int i = 0; i < m.natom; ++i) {
    int off = m.off[i];
    p[(size_t)off * n + off] = m.el[i]->occ_s;
    if (m.norb[i] >= 4)
      for (int k = 1; k < 4; ++k) p[(size_t)(off + k) * n + off + k] = m.el[i]->occ_p / 3.0;
  }
  return p;
}
// scf.rs:894-916
Mat symmetry_broken_density(const Molecule& m) {
  int n = m.nao;
  Mat p = sad_density(m);
  int target = -1;
  double best = 0.0;
  for (int i = 0; i < m.natom; ++i)
    if (m.norb[i] >= 4 && m.el[i]->occ_p > best) {
      best = m.el[i]->occ_p;
      target = i;
    }
  if (target >= 0) {
    int off = m.off[target];
    double tilt = std::min(0.2, p[(size_t)(off + 3) * n + off + 3]);
    p[(size_t)(off + 3) * n + off + 3] -= tilt;
    p[(size_t)(off + 1) * n + off + 1] += tilt;
  }
  return p;
}

// scf.rs:1179-1316
bool rhf_loop(const Molecule& m, const Core& core, int n_occ, const Opts& o, State& st, Error& err) {
  int n = m.nao;
  Mat density;
  if (o.guess == G_CORE) {  // scf.rs:919-935
    std::vector<double> w;
    Mat c;
    if (!eigh(n, core.h, w, c)) { err = {5, "eigensolver failed"}; return false; }
    density = leading_columns_gram(n, c, n_occ, 2.0);
  } else if (o.guess == G_SYM) {
    density = symmetry_broken_density(m);
  } else {
    density = sad_density(m);
  }
  double e_old = 0.0;
  std::vector<double> eps(n, 0.0);
  Mat coeff((size_t)n * n, 0.0);
  bool converged = false;
  double last_change = INFINITY;
  int iterations = 0;
  int accel = o.use_diis ? o.accel : ACC_NONE;
  bool keep = accel == ACC_ADIIS;
  if (keep && !diis_depth_fits(n, 3, o.memory_mb)) keep = false;
  if (accel == ACC_ADIIS && !keep) accel = ACC_CDIIS;
  AccelHistory hist{diis_depth(n, keep ? 3 : 2, o.memory_mb), keep, {}, {}, {}, {}, {}};
  for (int iter = 0; iter < o.max_scf; ++iter) {
    iterations = iter + 1;
    Mat f = build_fock(m, core, density);
    double e_elec = 0.5 * (fdot(density, core.h) + fdot(density, f));
    Mat f_use;
    if (accel == ACC_NONE) {
      f_use = std::move(f);
    } else {
      Mat e = commutator(n, f, density);
      double err_norm = std::sqrt(hist.push(std::move(f), std::move(e), keep ? &density : nullptr));
      bool ok = (accel == ACC_ADIIS && err_norm > o.adiis_switch) ? hist.adiis(f_use) : hist.cdiis(f_use);
      if (!ok) f_use = hist.focks.back();
    }
    std::vector<double> w;
    Mat c;
    if (!eigh(n, f_use, w, c)) { err = {5, "eigensolver failed"}; return false; }
    Mat p_new = leading_columns_gram(n, c, n_occ, 2.0);
    double dp = rms_diff(p_new, density);
    last_change = dp;
    double de = std::fabs(e_elec - e_old);
    eps = std::move(w);
    coeff = std::move(c);
    density = std::move(p_new);
    e_old = e_elec;
    if (iter > 0 && de < o.e_tol && dp < o.p_tol) {
      converged = true;
      break;
    }
  }
  Mat ff = build_fock(m, core, density);
  st = State();
  st.electronic = 0.5 * (fdot(density, core.h) + fdot(density, ff));
  st.density = std::move(density);
  st.eps = std::move(eps);
  st.coeff = std::move(coeff);
  st.n_occ = n_occ;
  st.n_beta = n_occ;
  st.converged = converged;
  st.last_change = last_change;
  st.iterations = iterations;
  st.unrestricted = false;
  return true;
}

// scf.rs:333-350
Mat level_shift(int n, const Mat& f, const Mat& p, double shift) {
  if (shift == 0.0) return f;
  Mat out = f;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) out[(size_t)i * n + j] += shift * ((i == j ? 1.0 : 0.0) - p[(size_t)i * n + j]);
  return out;
}

// scf.rs:1319-1496
bool uhf_loop(const Molecule& m, const Core& core, int na, int nb, const Opts& o, State& st, Error& err) {
  int n = m.nao;
  Mat pa, pb;
  if (o.guess == G_CORE) {  // scf.rs:938-979
    std::vector<double> w;
    Mat c;
    if (!eigh(n, core.h, w, c)) { err = {5, "eigensolver failed"}; return false; }
    pa = leading_columns_gram(n, c, na, 1.0);
    pb = leading_columns_gram(n, c, nb, 1.0);
  } else {
    Mat p = o.guess == G_SYM ? symmetry_broken_density(m) : sad_density(m);
    double ne = (double)(na + nb), fa = 0.5, fb = 0.5;
    if (ne > 0.0) { fa = na / ne; fb = nb / ne; }
    pa = p; pb = p;
    for (double& v : pa) v *= fa;
    for (double& v : pb) v *= fb;
  }
  double e_old = 0.0;
  std::vector<double> eps_a(n, 0.0), eps_b(n, 0.0);
  Mat ca((size_t)n * n, 0.0);
  bool converged = false;
  double last_change = INFINITY;
  int iterations = 0;
  std::vector<Mat> hfa, hfb, herr;
  int max_diis = diis_depth(n, 4, o.memory_mb);
  bool use_cdiis = o.use_diis && o.accel == ACC_CDIIS;
  for (int iter = 0; iter < o.max_scf; ++iter) {
    iterations = iter + 1;
    Mat pt = pa;
    for (size_t k = 0; k < pt.size(); ++k) pt[k] += pb[k];
    Mat fa = build_fock_spin(m, core, pt, pa);
    Mat fb = build_fock_spin(m, core, pt, pb);
    double e_elec = 0.5 * (fdot(pt, core.h) + fdot(pa, fa) + fdot(pb, fb));
    Mat fa_use, fb_use;
    if (use_cdiis) {
      Mat ea = commutator(n, fa, pa), eb = commutator(n, fb, pb);
      Mat er(2 * (size_t)n * n);
      std::copy(ea.begin(), ea.end(), er.begin());
      std::copy(eb.begin(), eb.end(), er.begin() + (size_t)n * n);
      hfa.push_back(fa);
      hfb.push_back(fb);
      herr.push_back(std::move(er));
      if ((int)hfa.size() > max_diis) {
        hfa.erase(hfa.begin());
        hfb.erase(hfb.begin());
        herr.erase(herr.begin());
      }
      std::vector<std::vector<double>> gram(herr.size(), std::vector<double>(herr.size()));
      for (size_t i = 0; i < herr.size(); ++i)
        for (size_t j = 0; j < herr.size(); ++j) gram[i][j] = fdot(herr[i], herr[j]);
      std::vector<double> c;
      if (diis_coeffs_from_gram(gram, c)) {
        fa_use = combine(hfa, c);
        fb_use = combine(hfb, c);
      } else {
        fa_use = fa;
        fb_use = fb;
      }
    } else {
      fa_use = fa;
      fb_use = fb;
    }
    Mat fad = level_shift(n, fa_use, pa, o.shift), fbd = level_shift(n, fb_use, pb, o.shift);
    std::vector<double> wa, wb;
    Mat cA, cB;
    if (!eigh(n, fad, wa, cA) || !eigh(n, fbd, wb, cB)) { err = {5, "eigensolver failed"}; return false; }
    Mat pa_new = leading_columns_gram(n, cA, na, 1.0);
    Mat pb_new = leading_columns_gram(n, cB, nb, 1.0);
    double dp = rms_diff(pa_new, pa) + rms_diff(pb_new, pb);
    last_change = dp;
    double lam = o.damping;
    if (lam > 0.0) {
      for (size_t k = 0; k < pa_new.size(); ++k) pa_new[k] = (1.0 - lam) * pa_new[k] + lam * pa[k];
      for (size_t k = 0; k < pb_new.size(); ++k) pb_new[k] = (1.0 - lam) * pb_new[k] + lam * pb[k];
    }
    double de = std::fabs(e_elec - e_old);
    eps_a = std::move(wa);
    eps_b = std::move(wb);
    ca = std::move(cA);
    pa = std::move(pa_new);
    pb = std::move(pb_new);
    e_old = e_elec;
    if (iter > 0 && de < o.e_tol && dp < o.p_tol) {
      converged = true;
      break;
    }
  }
  Mat density = pa, spin = pa;
  for (size_t k = 0; k < density.size(); ++k) {
    density[k] += pb[k];
    spin[k] -= pb[k];
  }
  Mat fa = build_fock_spin(m, core, density, pa), fb = build_fock_spin(m, core, density, pb);
  st = State();
  st.electronic = 0.5 * (fdot(density, core.h) + fdot(pa, fa) + fdot(pb, fb));
  st.density = std::move(density);
  st.spin = std::move(spin);
  st.has_spin = true;
  st.eps = std::move(eps_a);
  st.eps_b = std::move(eps_b);
  st.has_beta = true;
  st.coeff = std::move(ca);
  st.n_occ = na;
  st.n_beta = nb;
  st.converged = converged;
  st.last_change = last_change;
  st.iterations = iterations;
  st.unrestricted = true;
  return true;
}

// scf.rs:106-124
double frontier_gap(const State& s) {
  bool hh = s.n_occ > 0, hl = s.n_occ < (int)s.eps.size();
  double h = hh ? s.eps[s.n_occ - 1] : 0.0, l = hl ? s.eps[s.n_occ] : 0.0;
  if (s.has_beta) {
    if (s.n_beta > 0) { double bh = s.eps_b[s.n_beta - 1]; h = hh ? std::max(h, bh) : bh; hh = true; }
    if (s.n_beta < (int)s.eps_b.size()) { double bl = s.eps_b[s.n_beta]; l = hl ? std::min(l, bl) : bl; hl = true; }
  }
  if (hh && hl) return l - h;
  return INFINITY;
}

// ---------------------------------------------------------------- gradient (gradient.rs:306-599)
template <class S> void pair_dual_eval(const Elem& ea, const Elem& eb, const double d[3], S* w, S e1b[16], S e2a[16], S s[16]) {
  S dv[3] = {dvar(d[0], 0), dvar(d[1], 1), dvar(d[2], 2)};
  pair_two_electron<S>(ea, eb, dv, w, e1b, e2a);
  diatom_overlap<S>(ea, eb, dv, s);
}

void electronic_gradient(const Molecule& m, const Mat& pt, const Mat& pa, const Mat& pb, bool uhf, std::vector<double>& g) {
  int n = m.nao;
  std::vector<std::pair<int, int>> idx;
  for (int u = 0; u < m.natom; ++u)
    for (int v = u + 1; v < m.natom; ++v) idx.push_back({u, v});
  std::vector<double> fpair(idx.size() * 3);
  std::vector<int> ia(idx.size()), ib(idx.size());
#pragma omp parallel for schedule(dynamic, 64) if (idx.size() > 2048)
  for (long t = 0; t < (long)idx.size(); ++t) {
    int u = idx[t].first, v = idx[t].second;
    const Elem &eu = *m.el[u], &ev = *m.el[v];
    int a = (eu.has_p() || !ev.has_p()) ? u : v, b = a == u ? v : u;
    const Elem &ea = *m.el[a], &eb = *m.el[b];
    double d[3] = {m.xyz[3 * b] - m.xyz[3 * a], m.xyz[3 * b + 1] - m.xyz[3 * a + 1], m.xyz[3 * b + 2] - m.xyz[3 * a + 2]};
    Dual w[100], e1b[16], e2a[16], s[16];
    pair_dual_eval<Dual>(ea, eb, d, w, e1b, e2a, s);
    int oa = m.off[a], ob = m.off[b], na = ea.norb, nb = eb.norb, pb_ = nb * (nb + 1) / 2;
    double f[3] = {0, 0, 0};
    for (int i = 0; i < na; ++i) {
      double bi = beta_of(ea, i);
      for (int j = 0; j < nb; ++j) {
        double coef = pt[(size_t)(oa + i) * n + ob + j] * (bi + beta_of(eb, j));
        for (int ax = 0; ax < 3; ++ax) f[ax] += coef * s[i * 4 + j].d[ax];
      }
    }
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < na; ++j) {
        double coef = pt[(size_t)(oa + i) * n + oa + j];
        for (int ax = 0; ax < 3; ++ax) f[ax] += coef * e1b[i * 4 + j].d[ax];
      }
    for (int k = 0; k < nb; ++k)
      for (int l = 0; l < nb; ++l) {
        double coef = pt[(size_t)(ob + k) * n + ob + l];
        for (int ax = 0; ax < 3; ++ax) f[ax] += coef * e2a[k * 4 + l].d[ax];
      }
    for (int mu = 0; mu < na; ++mu)
      for (int nu = 0; nu < na; ++nu)
        for (int la = 0; la < nb; ++la)
          for (int si = 0; si < nb; ++si) {
            const Dual& dw = w[pack(mu, nu) * pb_ + pack(la, si)];
            double coul = pt[(size_t)(oa + mu) * n + oa + nu] * pt[(size_t)(ob + la) * n + ob + si];
            double exch;
            if (uhf)
              exch = -(pa[(size_t)(oa + mu) * n + ob + la] * pa[(size_t)(oa + nu) * n + ob + si] +
                       pb[(size_t)(oa + mu) * n + ob + la] * pb[(size_t)(oa + nu) * n + ob + si]);
            else
              exch = -0.5 * pt[(size_t)(oa + mu) * n + ob + la] * pt[(size_t)(oa + nu) * n + ob + si];
            double coef = coul + exch;
            for (int ax = 0; ax < 3; ++ax) f[ax] += coef * dw.d[ax];
          }
    for (int ax = 0; ax < 3; ++ax) fpair[t * 3 + ax] = f[ax];
    ia[t] = a;
    ib[t] = b;
  }
  for (size_t t = 0; t < idx.size(); ++t)
    for (int ax = 0; ax < 3; ++ax) {
      g[3 * ib[t] + ax] += fpair[t * 3 + ax];
      g[3 * ia[t] + ax] -= fpair[t * 3 + ax];
    }
}

// repulsion.rs:30-49
void core_core_gradient(const Molecule& m, std::vector<double>& g) {
  for (int i = 0; i < m.natom; ++i)
    for (int j = i + 1; j < m.natom; ++j) {
      double d[3] = {m.xyz[3 * j] - m.xyz[3 * i], m.xyz[3 * j + 1] - m.xyz[3 * i + 1], m.xyz[3 * j + 2] - m.xyz[3 * i + 2]};
      double dist = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      Dual e = pair_core_energy<Dual>(*m.el[i], *m.el[j], dvar(dist, 0));
      for (int ax = 0; ax < 3; ++ax) {
        double c = d[ax] / dist * (-e.d[0]);
        g[3 * i + ax] += c;
        g[3 * j + ax] -= c;
      }
    }
}

double core_core_energy(const Molecule& m) {  // repulsion.rs:13-27
  double e = 0.0;
  for (int i = 0; i < m.natom; ++i)
    for (int j = i + 1; j < m.natom; ++j) {
      double d[3] = {m.xyz[3 * j] - m.xyz[3 * i], m.xyz[3 * j + 1] - m.xyz[3 * i + 1], m.xyz[3 * j + 2] - m.xyz[3 * i + 2]};
      e += pair_core_energy<double>(*m.el[i], *m.el[j], std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
    }
  return e;
}

void set_err(char* buf, int len, const std::string& s) {
  if (buf && len > 0) {
    std::snprintf(buf, (size_t)len, "%s", s.c_str());
  }
}

}  // namespace

// ================================================================ C API
extern "C" {

void oracle_default_options(oracle_options* o) {  // scf.rs:259-287
  o->charge = 0.0;
  o->multiplicity = 1;
  o->max_scf = 200;
  o->e_tol = 1.0e-8;
  o->p_tol = 1.0e-7;
  o->use_diis = 1;
  o->accelerator = ACC_ADIIS;
  o->adiis_switch = 0.1;
  o->reference = 0;
  o->guess = 0;
  o->stability = 1;
  o->level_shift_ev = 0.0;
  o->damping = 0.0;
  o->scf_memory_mb = 512;
  o->variant = 0;
  o->mmok = 0;
}

void oracle_set_lapack(void* dsyevd, void* dgemm) {
  g_dsyevd = (dsyevd_t)dsyevd;
  g_dgemm = (dgemm_t)dgemm;
}

int oracle_nao(int n_atoms, const int* z) {
  int nao = 0;
  for (int i = 0; i < n_atoms; ++i) {
    const Elem* e = params().get(z[i]);
    if (!e) return -1;
    nao += e->norb;
  }
  return nao;
}

// Replace the parameter set by the caller's Pm3Element / PairParams values, used as given (the
// reference reads the derived multipole fields of Pm3Element directly and does not re-derive them).
int oracle_set_parameters(const oracle_element_params* elems, int n_elems, const oracle_pair_params* pairs,
                          int n_pairs) {
  Params P;
  for (int z = 0; z < 19; ++z) P.have[z] = false;
  for (int i = 0; i < 19; ++i)
    for (int j = 0; j < 19; ++j) P.have_pair[i][j] = false;
  for (int k = 0; k < n_elems; ++k) {
    const oracle_element_params& r = elems[k];
    if (r.z <= 0 || r.z >= 19 || (r.n_orb != 1 && r.n_orb != 4) || r.n_gauss < 0 || r.n_gauss > 4) return 1;
    Elem e;
    e.z = r.z;
    e.norb = r.n_orb;
    e.n = r.npq;
    e.uss = r.u_ss; e.upp = r.u_pp; e.zs = r.zeta_s; e.zp = r.zeta_p; e.bs = r.beta_s; e.bp = r.beta_p;
    e.gss = r.g_ss; e.gsp = r.g_sp; e.gpp = r.g_pp; e.gp2 = r.g_p2; e.hsp = r.h_sp;
    e.alpha = r.alpha;
    for (int g = 0; g < r.n_gauss; ++g) e.gauss.push_back({r.gauss[g][0], r.gauss[g][1], r.gauss[g][2]});
    e.core = r.core_charge; e.occ_s = r.occ_s; e.occ_p = r.occ_p;
    e.eheat_ev = r.eheat_ev; e.e_isol = r.e_isol; e.mass = r.mass;
    e.dd = r.dd; e.qq = r.qq; e.rho0 = r.rho0; e.rho1 = r.rho1; e.rho2 = r.rho2;
    for (int i = 0; i < 10; ++i) e.po[i] = r.po[i];
    for (int i = 0; i < 7; ++i) e.ddp[i] = r.ddp[i];
    P.el[e.z] = e;
    P.have[e.z] = true;
  }
  for (int k = 0; k < n_pairs; ++k) {
    const oracle_pair_params& q = pairs[k];
    if (q.zi <= 0 || q.zi >= 19 || q.zj <= 0 || q.zj >= 19) return 1;
    int a = std::max(q.zi, q.zj), b = std::min(q.zi, q.zj);
    P.pair_alpha[a][b] = P.pair_alpha[b][a] = q.alpha;
    P.pair_x[a][b] = P.pair_x[b][a] = q.x;
    P.have_pair[a][b] = P.have_pair[b][a] = true;
  }
  params_mut() = P;
  return 0;
}

void oracle_reset_parameters(void) { params_mut() = Params(); }

int oracle_element(int z, double* out) {
  const Elem* e = params().get(z);
  if (!e) return 2;
  double v[22] = {(double)e->norb, e->uss, e->upp, e->zs, e->zp, e->bs, e->bp, e->gss, e->gsp, e->gpp, e->gp2,
                  e->hsp, e->alpha, e->core, e->dd, e->qq, e->rho0, e->rho1, e->rho2, e->e_isol, e->eheat_ev, e->mass};
  std::memcpy(out, v, sizeof(v));
  return 0;
}

int oracle_pair(int za, int zb, const double* dvec, double* w, double* e1b, double* e2a, double* s, int* na, int* nb) {
  const Elem *ea = params().get(za), *eb = params().get(zb);
  if (!ea || !eb) return 2;
  double r = std::sqrt(dvec[0] * dvec[0] + dvec[1] * dvec[1] + dvec[2] * dvec[2]);
  double dv[3] = {dvec[0] / r * r, dvec[1] / r * r, dvec[2] / r * r};
  pair_two_electron<double>(*ea, *eb, dv, w, e1b, e2a);
  if (!diatom_overlap<double>(*ea, *eb, dvec, s)) return 1;
  *na = ea->norb;
  *nb = eb->norb;
  return 0;
}

int oracle_core_hamiltonian(int n_atoms, const int* z, const double* xyz, double* h) {
  Molecule m;
  Error err{0, ""};
  if (!build_molecule(n_atoms, z, xyz, m, err)) return err.code;
  Core core;
  if (!build_core(m, core, err)) return err.code;
  std::memcpy(h, core.h.data(), core.h.size() * sizeof(double));
  return 0;
}

int oracle_fock(int n_atoms, const int* z, const double* xyz, const double* p_tot, const double* p_spin, double* f) {
  Molecule m;
  Error err{0, ""};
  if (!build_molecule(n_atoms, z, xyz, m, err)) return err.code;
  Core core;
  if (!build_core(m, core, err)) return err.code;
  size_t nn = (size_t)m.nao * m.nao;
  Mat pt(p_tot, p_tot + nn), ps(p_spin, p_spin + nn);
  Mat ff = build_fock_spin(m, core, pt, ps);
  std::memcpy(f, ff.data(), nn * sizeof(double));
  return 0;
}

double oracle_core_core(int n_atoms, const int* z, const double* xyz) {
  Molecule m;
  Error err{0, ""};
  if (!build_molecule(n_atoms, z, xyz, m, err)) return NAN;
  return core_core_energy(m);
}

int oracle_fixed_density_gradient(int n_atoms, const int* z, const double* xyz, const double* p_tot, const double* pa,
                                  const double* pb, int uhf, double* grad) {
  Molecule m;
  Error err{0, ""};
  if (!build_molecule(n_atoms, z, xyz, m, err)) return err.code;
  size_t nn = (size_t)m.nao * m.nao;
  Mat pt(p_tot, p_tot + nn), A, B;
  if (uhf) {
    A.assign(pa, pa + nn);
    B.assign(pb, pb + nn);
  }
  std::vector<double> g(3 * (size_t)n_atoms, 0.0);
  core_core_gradient(m, g);
  electronic_gradient(m, pt, A, B, uhf != 0, g);
  std::memcpy(grad, g.data(), g.size() * sizeof(double));
  return 0;
}

int oracle_eigh(int n, const double* a, double* w, double* v) {
  Mat am(a, a + (size_t)n * n), vm;
  std::vector<double> wv;
  if (!eigh(n, am, wv, vm)) return 5;
  std::memcpy(w, wv.data(), (size_t)n * sizeof(double));
  std::memcpy(v, vm.data(), (size_t)n * n * sizeof(double));
  return 0;
}

// scf.rs:450-848 (run_pm3), plus gradient.rs:235-276 when a gradient buffer is given.
int oracle_single_point(int n_atoms, const int* z, const double* xyz_bohr, const oracle_options* opt, oracle_result* res,
                        double* charges, double* density, double* mo_energies, double* gradient, char* errbuf, int errlen) {
  oracle_options dflt;
  oracle_default_options(&dflt);
  const oracle_options& O = opt ? *opt : dflt;
  std::memset(res, 0, sizeof(*res));
  Molecule m;
  Error err{0, ""};
  if (n_atoms < 1) {
    set_err(errbuf, errlen, "no atoms");
    return 1;
  }
  if (O.multiplicity < 1) {
    set_err(errbuf, errlen, "multiplicity must be >= 1");
    return 1;
  }
  if (O.variant < 0 || O.variant > 3) {
    set_err(errbuf, errlen, "variant outside PM3 / PM3-D3 / PM3-D3H4 / PM3-D3H4X");
    return 1;
  }
  if (!build_molecule(n_atoms, z, xyz_bohr, m, err)) {
    set_err(errbuf, errlen, err.msg);
    return err.code;
  }
  Core core;
  if (!build_core(m, core, err)) {
    set_err(errbuf, errlen, err.msg);
    return err.code;
  }
  double n_elec = 0.0;
  for (int i = 0; i < m.natom; ++i) n_elec += m.el[i]->core;
  n_elec -= O.charge;
  long ne = std::lround(n_elec);
  if (std::fabs(n_elec - (double)ne) > 1.0e-6 || ne < 0) {
    set_err(errbuf, errlen, "invalid electron count");
    return 1;
  }
  long nu = O.multiplicity - 1;
  if (ne - nu < 0 || (ne - nu) % 2 != 0) {
    set_err(errbuf, errlen, "electron count is incompatible with multiplicity (need same parity)");
    return 1;
  }
  int n_alpha = (int)((ne + nu) / 2), n_beta = (int)((ne - nu) / 2);
  if (n_alpha > m.nao) {
    set_err(errbuf, errlen, "more electrons than orbitals");
    return 1;
  }
  bool use_uhf;
  if (O.reference == 0) use_uhf = n_alpha != n_beta;
  else if (O.reference == 2) use_uhf = true;
  else {
    if (n_alpha != n_beta) {
      set_err(errbuf, errlen, "RHF requested for an open-shell system; use UHF or Auto");
      return 1;
    }
    use_uhf = false;
  }
  auto run_scf = [&](double shift, double damping, int guess, int accel, bool force_uhf, State& st) -> bool {
    Opts o;
    o.max_scf = O.max_scf;
    o.e_tol = O.e_tol;
    o.p_tol = O.p_tol;
    o.adiis_switch = O.adiis_switch;
    o.shift = shift;
    o.damping = damping;
    o.use_diis = O.use_diis && accel != ACC_NONE;
    o.accel = accel;
    o.guess = guess;
    o.memory_mb = O.scf_memory_mb;
    Error e2{0, ""};
    bool ok = (use_uhf || force_uhf) ? uhf_loop(m, core, n_alpha, n_beta, o, st, e2) : rhf_loop(m, core, n_alpha, o, st, e2);
    if (!ok) err = e2;
    return ok;
  };
  bool steered = O.level_shift_ev != 0.0 || O.damping != 0.0;
  State state;
  bool ok = steered ? run_scf(O.level_shift_ev, O.damping, O.guess, O.accelerator, false, state)
                    : run_scf(0.0, 0.0, O.guess, O.accelerator, false, state);
  if (!ok) {
    set_err(errbuf, errlen, err.msg);
    return err.code;
  }
  int paths = 1;
  bool search = O.stability == 0 ? false : (O.stability == 2 ? !steered : (!steered && frontier_gap(state) < 6.0));
  double first_ev = state.electronic;
  if (search) {  // scf.rs:610-715
    int primary = O.guess == G_CORE ? G_CORE : G_SAD;
    int other = primary == G_CORE ? G_SAD : G_CORE;
    bool closed = !use_uhf;
    struct Rung { int guess, accel; double shift, damp; bool unrestricted; };
    Rung rungs[7] = {{primary, ACC_NONE, 0.0, 0.0, false},   {other, O.accelerator, 0.0, 0.0, false},
                     {other, ACC_NONE, 0.0, 0.0, false},     {G_SYM, O.accelerator, 0.0, 0.0, false},
                     {G_SYM, ACC_NONE, 0.0, 0.0, false},     {G_SYM, ACC_NONE, -2.0, 0.0, closed},
                     {primary, ACC_CDIIS, 0.0, 0.85, closed}};
    for (const Rung& r : rungs) {
      if (r.unrestricted != closed) continue;
      ++paths;
      State cand;
      if (!run_scf(r.shift, r.damp, r.guess, r.accel, r.unrestricted, cand)) continue;
      if (!cand.converged) continue;
      if (r.unrestricted) {
        double mx = 0.0;
        for (double v : cand.spin) mx = std::max(mx, std::fabs(v));
        if (!(mx < 1.0e-8)) continue;
        cand.has_spin = false;  // collapse_to_restricted (scf.rs:89-95)
        cand.has_beta = false;
        cand.n_beta = cand.n_occ;
        cand.unrestricted = false;
      }
      if (!state.converged || cand.electronic < state.electronic - 1.0e-6) state = std::move(cand);
    }
  }
  double improvement = std::max(first_ev - state.electronic, 0.0);
  double core_ev = core_core_energy(m);
  double electronic = state.electronic;
  // post-SCF classical correction of the method variant (scf.rs:740-743)
  double correction_ev = 0.0;
  if (O.variant != 0 || O.mmok) {
    double parts[5];
    oracle_corrections(n_atoms, z, xyz_bohr, O.variant, O.mmok, parts, nullptr);
    correction_ev = parts[0] + parts[1] + parts[2] + parts[3];
    if (O.mmok) correction_ev += parts[4];
  }
  double total = electronic + core_ev + correction_ev;
  double e_isol = 0.0, eheat = 0.0;
  for (int i = 0; i < m.natom; ++i) {
    e_isol += m.el[i]->e_isol;
    eheat += m.el[i]->eheat_ev;
  }
  res->nao = m.nao;
  res->electronic_ev = electronic;
  res->core_ev = core_ev;
  res->total_ev = total;
  res->heat_of_formation_kcal = (total - e_isol + eheat) * EV_TO_KCAL;
  res->iterations = state.iterations;
  res->converged = state.converged ? 1 : 0;
  res->unrestricted = state.unrestricted ? 1 : 0;
  res->scf_paths_tried = paths;
  res->scf_improvement_ev = improvement;
  res->n_occ = state.n_occ;
  res->n_beta = state.n_beta;
  res->last_change = state.last_change;
  if (!state.converged) {
    // the density of the last iteration still goes out, so that a run cut after k iterations can
    // be compared with another implementation's first k iterations
    if (density) std::memcpy(density, state.density.data(), sizeof(double) * (size_t)m.nao * m.nao);
    char msg[160];
    std::snprintf(msg, sizeof msg, "PM3 SCF did not converge after %d iterations (error=%.3e)", state.iterations, state.last_change);
    set_err(errbuf, errlen, msg);
    return 4;
  }
  int n = m.nao;
  for (int i = 0; i < m.natom; ++i) {  // scf.rs:762-772
    double pop = 0.0;
    for (int k = 0; k < m.norb[i]; ++k) pop += state.density[(size_t)(m.off[i] + k) * n + m.off[i] + k];
    charges[i] = m.el[i]->core - pop;
  }
  double mtot = 0.0, com[3] = {0, 0, 0};  // dipole.rs:64-77
  for (int i = 0; i < m.natom; ++i) {
    mtot += m.el[i]->mass;
    for (int k = 0; k < 3; ++k) com[k] += m.xyz[3 * i + k] * m.el[i]->mass;
  }
  for (int k = 0; k < 3; ++k) com[k] = mtot > 0 ? com[k] / mtot : 0.0;
  for (int ax = 0; ax < 3; ++ax) {  // dipole.rs:82-144
    double nuc = 0.0, elec = 0.0;
    for (int i = 0; i < m.natom; ++i) {
      double disp = m.xyz[3 * i + ax] - com[ax];
      nuc += disp * m.el[i]->core;
      int off = m.off[i];
      for (int k = 0; k < m.norb[i]; ++k) elec += state.density[(size_t)(off + k) * n + off + k] * disp;
      if (m.norb[i] >= 4) {
        int p = off + ax + 1;
        elec += state.density[(size_t)off * n + p] * m.el[i]->dd + state.density[(size_t)p * n + off] * m.el[i]->dd;
      }
    }
    res->dipole_debye[ax] = (nuc - elec) * AU_DIPOLE_TO_DEBYE;
  }
  // scf.rs:804-822
  bool ha = state.n_occ >= 1, la = state.n_occ < n;
  double homo = ha ? state.eps[state.n_occ - 1] : 0.0, lumo = la ? state.eps[state.n_occ] : 0.0;
  if (state.has_beta) {
    if (state.n_beta >= 1) { double h = state.eps_b[state.n_beta - 1]; homo = ha ? std::max(homo, h) : h; ha = true; }
    if (state.n_beta < n) { double l = state.eps_b[state.n_beta]; lumo = la ? std::min(lumo, l) : l; la = true; }
  }
  res->has_homo = ha;
  res->has_lumo = la;
  res->homo_ev = homo;
  res->lumo_ev = lumo;
  if (density) std::memcpy(density, state.density.data(), (size_t)n * n * sizeof(double));
  if (mo_energies) std::memcpy(mo_energies, state.eps.data(), (size_t)n * sizeof(double));
  if (gradient) {  // gradient.rs:240-276 (no field, no corrections)
    std::vector<double> g(3 * (size_t)m.natom, 0.0);
    core_core_gradient(m, g);
    if (state.unrestricted) {  // gradient.rs:494-521
      Mat pa(state.density.size()), pb(state.density.size());
      for (size_t k = 0; k < pa.size(); ++k) {
        pa[k] = 0.5 * (state.density[k] + state.spin[k]);
        pb[k] = 0.5 * (state.density[k] - state.spin[k]);
      }
      electronic_gradient(m, state.density, pa, pb, true, g);
    } else {
      Mat none;
      electronic_gradient(m, state.density, none, none, false, g);
    }
    if (O.variant != 0 || O.mmok) {  // add_correction_gradient (gradient.rs:324-357)
      std::vector<double> gd(g.size(), 0.0);
      double parts[5];
      oracle_corrections(n_atoms, z, xyz_bohr, O.variant, O.mmok, parts, gd.data());
      for (size_t k = 0; k < g.size(); ++k) g[k] += gd[k];
    }
    std::memcpy(gradient, g.data(), g.size() * sizeof(double));
  }
  return 0;
}

}  // extern "C"
