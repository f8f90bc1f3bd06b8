// Two-centre NDDO quantities of one atom pair, for device (and host) code, templated on the
// scalar: `double` for energies, `D3` (value + three partials along the displacement) for the
// analytic gradient.
//
// Physics follows pm3-rs (which follows MOPAC):
//   - frame rotation onto the pair axis:        src/integrals.rs:25-59
//   - local multipole integrals (22 / 4 / 1):  src/integrals.rs:289-464 (Dewar-Sabelli-Klopman)
//   - rotation to the molecular frame:          src/integrals.rs:466-552
//   - electron-core attraction (MOPAC spcore):  src/integrals.rs:234-271
//   - Slater overlap, n <= 3 closed forms:      src/overlap.rs:266-507, 763-850
//   - PM3 core-core repulsion:                  src/repulsion.rs:57-120
// Orbital order s, px, py, pz; packed pair index pk(a,b) = max*(max+1)/2 + min.
#pragma once
#include <cmath>

#include "pm3_elements.h"

#if defined(__CUDACC__)
#define PM3_HD __host__ __device__ __forceinline__
#else
#define PM3_HD inline
#endif

namespace pm3gpu {

// ------------------------------------------------------------------------------------ scalars
struct D3 {
  double v, g[3];
};
PM3_HD double vof(double x) { return x; }
PM3_HD double vof(const D3& x) { return x.v; }
template <class S> PM3_HD S mk(double x);
template <> PM3_HD double mk<double>(double x) { return x; }
template <> PM3_HD D3 mk<D3>(double x) { return D3{x, {0.0, 0.0, 0.0}}; }

PM3_HD D3 operator+(const D3& a, const D3& b) { return {a.v + b.v, {a.g[0] + b.g[0], a.g[1] + b.g[1], a.g[2] + b.g[2]}}; }
PM3_HD D3 operator-(const D3& a, const D3& b) { return {a.v - b.v, {a.g[0] - b.g[0], a.g[1] - b.g[1], a.g[2] - b.g[2]}}; }
PM3_HD D3 operator-(const D3& a) { return {-a.v, {-a.g[0], -a.g[1], -a.g[2]}}; }
PM3_HD D3 operator*(const D3& a, const D3& b) {
  return {a.v * b.v, {a.g[0] * b.v + a.v * b.g[0], a.g[1] * b.v + a.v * b.g[1], a.g[2] * b.v + a.v * b.g[2]}};
}
PM3_HD D3 operator+(const D3& a, double b) { return {a.v + b, {a.g[0], a.g[1], a.g[2]}}; }
PM3_HD D3 operator+(double b, const D3& a) { return {a.v + b, {a.g[0], a.g[1], a.g[2]}}; }
PM3_HD D3 operator-(const D3& a, double b) { return {a.v - b, {a.g[0], a.g[1], a.g[2]}}; }
PM3_HD D3 operator-(double b, const D3& a) { return {b - a.v, {-a.g[0], -a.g[1], -a.g[2]}}; }
PM3_HD D3 operator*(const D3& a, double b) { return {a.v * b, {a.g[0] * b, a.g[1] * b, a.g[2] * b}}; }
PM3_HD D3 operator*(double b, const D3& a) { return a * b; }
PM3_HD D3 lift(const D3& a, double f, double df) { return {f, {a.g[0] * df, a.g[1] * df, a.g[2] * df}}; }

// 1/sqrt(x)
PM3_HD double rsq(double x) {
#if defined(__CUDA_ARCH__)
  return rsqrt(x);
#else
  return 1.0 / std::sqrt(x);
#endif
}
PM3_HD D3 rsq(const D3& x) { double r = rsq(x.v); return lift(x, r, -0.5 * r * r * r); }
PM3_HD double sq_rt(double x) { return sqrt(x); }
PM3_HD D3 sq_rt(const D3& x) { double s = sqrt(x.v); return lift(x, s, 0.5 / s); }
PM3_HD double inv(double x) { return 1.0 / x; }
PM3_HD D3 inv(const D3& x) { double r = 1.0 / x.v; return lift(x, r, -r * r); }
PM3_HD double ex(double x) { return exp(x); }
PM3_HD D3 ex(const D3& x) { double e = exp(x.v); return lift(x, e, e); }
PM3_HD double pw(double x, double p) { return pow(x, p); }
PM3_HD D3 pw(const D3& x, double p) { double f = pow(x.v, p); return lift(x, f, p * pow(x.v, p - 1.0)); }
template <class S> PM3_HD S ipow(S x, int n) {
  S r = x;
  for (int i = 1; i < n; ++i) r = r * x;
  return r;
}
PM3_HD double ab(double x) { return fabs(x); }
PM3_HD D3 ab(const D3& x) { return x.v < 0.0 ? -x : x; }

PM3_HD int pk(int a, int b) { return a >= b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; }

// ------------------------------------------------------------------------- frame rotation
// Rows r[0..2], r[3..5], r[6..8] of the rotation taking the unit vector v onto +x: a
// quaternion rotation when v_x >= 0, a Householder reflection otherwise.
template <class S> PM3_HD void frame(const S& vx, const S& vy, const S& vz, S r[9]) {
  if (vof(vx) < 0.0) {
    const S ux = vx - 1.0;
    const S f = inv(ux * ux + vy * vy + vz * vz) * (-2.0);
    r[0] = f * ux * ux + 1.0; r[1] = f * ux * vy; r[2] = f * ux * vz;
    r[3] = f * vy * ux; r[4] = f * vy * vy + 1.0; r[5] = f * vy * vz;
    r[6] = f * vz * ux; r[7] = f * vz * vy; r[8] = f * vz * vz + 1.0;
  } else {
    S qy = vz, qz = -vy, qw = vx + 1.0;
    const S n = rsq(qy * qy + qz * qz + qw * qw);
    qy = qy * n; qz = qz * n; qw = qw * n;
    r[0] = (qy * qy + qz * qz) * (-2.0) + 1.0; r[1] = qz * qw * (-2.0); r[2] = qy * qw * 2.0;
    r[3] = qz * qw * 2.0; r[4] = qz * qz * (-2.0) + 1.0; r[5] = qy * qz * 2.0;
    r[6] = qy * qw * (-2.0); r[7] = qy * qz * 2.0; r[8] = qy * qy * (-2.0) + 1.0;
  }
}

// -------------------------------------------------------------- local multipole integrals
// Multipole description of one side of a pair.
struct Mpole {
  double dd, qq, r0, r1, r2;
};
PM3_HD Mpole ee_pole(const ElemDev& e) { return {e.dd, e.qq, e.rho0, e.rho1, e.rho2}; }
PM3_HD Mpole core_pole(const ElemDev& e) { return {e.ddp2, e.qq_core, e.po1, e.po2, e.po3}; }

// (heavy | s) local integrals: ri[0..3] = (ss|ss), (s pz|ss), (pz pz|ss), (px px|ss).
template <class S> PM3_HD void local4(const Mpole& a, double rho_b, const S& r, S ri[4]) {
  const double h1 = kEv * 0.5, h2 = kEv * 0.25;
  const double da = a.dd, qa = 2.0 * a.qq;
  const double cee = (a.r0 + rho_b) * (a.r0 + rho_b);
  const double cde = (a.r1 + rho_b) * (a.r1 + rho_b);
  const double cqe = (a.r2 + rho_b) * (a.r2 + rho_b);
  const S r2 = r * r;
  const S ee = rsq(r2 + cee) * kEv;
  const S q0 = rsq(r2 + cqe) * h1;
  const S rp = r + da, rm = r - da, sp = r + qa, sm = r - qa;
  ri[0] = ee;
  ri[1] = rsq(rp * rp + cde) * h1 - rsq(rm * rm + cde) * h1;
  ri[2] = ee + rsq(sp * sp + cqe) * h2 + rsq(sm * sm + cqe) * h2 - q0;
  ri[3] = ee + rsq(r2 + qa * qa + cqe) * h1 - q0;
}

// (heavy | heavy) local integrals, the 22 distinct values of the sp-sp multipole model.
template <class S> PM3_HD void local22(const Mpole& a, const Mpole& b, const S& r, S ri[22]) {
  const double h1 = kEv * 0.5, h2 = kEv * 0.25, h3 = kEv * 0.125, h4 = kEv * 0.0625;
  const double da = a.dd, db = b.dd, qa = 2.0 * a.qq, qb = 2.0 * b.qq, ha = a.qq, hb = b.qq;
  auto s2 = [](double x) { return x * x; };
  const double cee = s2(a.r0 + b.r0), cde = s2(a.r1 + b.r0), cqe = s2(a.r2 + b.r0);
  const double ced = s2(a.r0 + b.r1), ceq = s2(a.r0 + b.r2), cdd = s2(a.r1 + b.r1);
  const double cdq = s2(a.r1 + b.r2), cqd = s2(a.r2 + b.r1), cqq = s2(a.r2 + b.r2);
  const S r2 = r * r;
  // 1/sqrt((r+s)^2 + c) for axial point-charge offsets s
  auto ax = [&](double s, double c) { const S t = r + s; return rsq(t * t + c); };
  // 1/sqrt(r^2 + t + c) for a transverse offset with t = (perpendicular distance)^2
  auto tr = [&](double t, double c) { return rsq(r2 + (t + c)); };
  // 1/sqrt((r+s)^2 + t + c): axial and transverse together
  auto at = [&](double s, double t, double c) { const S u = r + s; return rsq(u * u + t + c); };

  const S ee = tr(0.0, cee) * kEv;
  const S dze = ax(-da, cde) * h1 - ax(da, cde) * h1;
  const S qe0 = tr(0.0, cqe) * h1;
  const S qzze = ax(-qa, cqe) * h2 + ax(qa, cqe) * h2 - qe0;
  const S qxxe = tr(qa * qa, cqe) * h1 - qe0;
  const S edz = ax(db, ced) * h1 - ax(-db, ced) * h1;
  const S eq0 = tr(0.0, ceq) * h1;
  const S eqzz = ax(-qb, ceq) * h2 + ax(qb, ceq) * h2 - eq0;
  const S eqxx = tr(qb * qb, ceq) * h1 - eq0;
  const S dq_p = ax(da, cdq) * h2, dq_m = ax(-da, cdq) * h2;
  const S qd_m = ax(-db, cqd) * h2, qd_p = ax(db, cqd) * h2;
  const S qq0 = tr(0.0, cqq) * h2;
  const S qqa = tr(qa * qa, cqq) * h2, qqb = tr(qb * qb, cqq) * h2;
  const S zb_m = ax(-qb, cqq) * h3, zb_p = ax(qb, cqq) * h3;
  const S za_p = ax(qa, cqq) * h3, za_m = ax(-qa, cqq) * h3;

  ri[0] = ee;
  ri[1] = -dze;
  ri[2] = ee + qzze;
  ri[3] = ee + qxxe;
  ri[4] = -edz;
  ri[5] = ax(da - db, cdd) * h2 + ax(-da + db, cdd) * h2 - ax(-da - db, cdd) * h2 - ax(da + db, cdd) * h2;
  ri[6] = tr((da - db) * (da - db), cdd) * h1 - tr((da + db) * (da + db), cdd) * h1;
  ri[7] = -edz + ax(qa - db, cqd) * h3 - ax(qa + db, cqd) * h3 + ax(-qa - db, cqd) * h3 - ax(-qa + db, cqd) * h3 - qd_m + qd_p;
  ri[8] = -edz - qd_m + at(-db, qa * qa, cqd) * h2 + qd_p - at(db, qa * qa, cqd) * h2;
  ri[9] = at(ha, (ha - db) * (ha - db), cqd) * h2 - at(-ha, (ha - db) * (ha - db), cqd) * h2 -
          at(ha, (ha + db) * (ha + db), cqd) * h2 + at(-ha, (ha + db) * (ha + db), cqd) * h2;
  ri[10] = ee + eqzz;
  ri[11] = ee + eqxx;
  ri[12] = -dze + ax(da - qb, cdq) * h3 - ax(-da - qb, cdq) * h3 + ax(da + qb, cdq) * h3 - ax(-da + qb, cdq) * h3 + dq_m - dq_p;
  ri[13] = -dze - dq_p + at(da, qb * qb, cdq) * h2 + dq_m - at(-da, qb * qb, cdq) * h2;
  ri[14] = at(-hb, (da - hb) * (da - hb), cdq) * h2 - at(hb, (da - hb) * (da - hb), cdq) * h2 -
           at(-hb, (da + hb) * (da + hb), cdq) * h2 + at(hb, (da + hb) * (da + hb), cdq) * h2;
  ri[15] = ee + eqzz + qzze + ax(qa - qb, cqq) * h4 + ax(qa + qb, cqq) * h4 + ax(-qa - qb, cqq) * h4 + ax(-qa + qb, cqq) * h4 -
           za_m - za_p - zb_m - zb_p + qq0;
  ri[16] = ee + eqzz + qxxe + at(-qb, qa * qa, cqq) * h3 + at(qb, qa * qa, cqq) * h3 - zb_m - zb_p - qqa + qq0;
  ri[17] = ee + eqxx + qzze + at(qa, qb * qb, cqq) * h3 + at(-qa, qb * qb, cqq) * h3 - za_p - za_m - qqb + qq0;
  const S xx_xx = tr((qa - qb) * (qa - qb), cqq) * h3 + tr((qa + qb) * (qa + qb), cqq) * h3 - qqa - qqb + qq0;
  ri[18] = ee + eqxx + qxxe + xx_xx;
  const double tm = (ha - hb) * (ha - hb), tp = (ha + hb) * (ha + hb);
  ri[19] = at(ha - hb, tm, cqq) * h3 - at(ha + hb, tm, cqq) * h3 - at(-ha - hb, tm, cqq) * h3 + at(-ha + hb, tm, cqq) * h3 -
           at(ha - hb, tp, cqq) * h3 + at(ha + hb, tp, cqq) * h3 + at(-ha - hb, tp, cqq) * h3 - at(-ha + hb, tp, cqq) * h3;
  const S xx_yy = tr(qa * qa + qb * qb, cqq) * h2 - qqa - qqb + qq0;
  ri[20] = ee + eqxx + qxxe + xx_yy;
  ri[21] = (xx_xx - xx_yy) * 0.5;
}

// --------------------------------------------------------------- rotation to molecular frame
// One element W[pk(k,l)][pk(m,n)] (k>=l, m>=n; 0 = s, 1..3 = p) of the rotated heavy-heavy
// table, from the 22 local values and the frame rows R (r0 = R[0..2], r1, r2).
template <class S> PM3_HD S w22(const S ri[22], const S R[9], int kk, int ll, int mm, int nn) {
  const S* r0 = R;
  const S* r1 = R + 3;
  const S* r2 = R + 6;
  const int k = kk - 1, l = ll - 1, m = mm - 1, n = nn - 1;
  if (kk == 0) {
    if (mm == 0) return ri[0];
    if (nn == 0) return ri[4] * r0[m];
    return ri[10] * (r0[m] * r0[n]) + ri[11] * (r1[m] * r1[n] + r2[m] * r2[n]);
  }
  if (ll == 0) {
    if (mm == 0) return ri[1] * r0[k];
    if (nn == 0) return ri[5] * (r0[k] * r0[m]) + ri[6] * (r1[k] * r1[m] + r2[k] * r2[m]);
    const S t0 = r0[k] * r0[m] * r0[n];
    const S t1 = (r1[m] * r1[n] + r2[m] * r2[n]) * r0[k];
    const S t2 = r1[k] * (r1[n] * r0[m] + r1[m] * r0[n]) + r2[k] * (r2[m] * r0[n] + r2[n] * r0[m]);
    return ri[12] * t0 + ri[13] * t1 + ri[14] * t2;
  }
  if (mm == 0) return ri[2] * (r0[k] * r0[l]) + ri[3] * (r1[k] * r1[l] + r2[k] * r2[l]);
  if (nn == 0) {
    const S t0 = r0[k] * r0[l] * r0[m];
    const S t1 = (r1[k] * r1[l] + r2[k] * r2[l]) * r0[m];
    const S t2 = r1[l] * r1[m] + r2[l] * r2[m];
    return ri[7] * t0 + ri[8] * t1 + ri[9] * (r0[k] * t2 + r0[l] * (r1[k] * r1[m] + r2[k] * r2[m]));
  }
  S v = ri[15] * (r0[k] * r0[l] * r0[m] * r0[n]);
  v = v + ri[16] * ((r1[k] * r1[l] + r2[k] * r2[l]) * r0[m] * r0[n]);
  v = v + ri[17] * ((r1[m] * r1[n] + r2[m] * r2[n]) * (r0[k] * r0[l]));
  v = v + ri[18] * (r1[k] * r1[l] * r1[m] * r1[n] + r2[k] * r2[l] * r2[m] * r2[n]);
  const S a1 = r0[m] * (r1[l] * r1[n] + r2[l] * r2[n]);
  const S a2 = r0[n] * (r1[l] * r1[m] + r2[l] * r2[m]);
  const S mix = r0[k] * (a1 + a2) + r0[l] * (r0[m] * (r1[k] * r1[n] + r2[k] * r2[n]) + r0[n] * (r1[k] * r1[m] + r2[k] * r2[m]));
  v = v + ri[19] * mix;
  v = v + ri[20] * (r1[k] * r1[l] * r2[m] * r2[n] + r2[k] * r2[l] * r1[m] * r1[n]);
  v = v + ri[21] * ((r1[k] * r2[l] + r2[k] * r1[l]) * (r1[m] * r2[n] + r2[m] * r1[n]));
  return v;
}

// One element W[pk(k,l)] of a (heavy | s) table.
template <class S> PM3_HD S w4(const S ri[4], const S R[9], int kk, int ll) {
  if (kk == 0) return ri[0];
  const int k = kk - 1;
  if (ll == 0) return ri[1] * R[k];
  const int l = ll - 1;
  return ri[2] * (R[k] * R[l]) + ri[3] * (R[3 + k] * R[3 + l] + R[6 + k] * R[6 + l]);
}

// Unpacked orbital indices of packed index p (0..9).
PM3_HD void unpk(int p, int& hi, int& lo) {
  hi = p >= 6 ? 3 : (p >= 3 ? 2 : (p >= 1 ? 1 : 0));
  lo = p - hi * (hi + 1) / 2;
}

// ------------------------------------------------------------------ electron-core attraction
// Attraction of the AOs of `orb` to the core of `cor` (MOPAC spcore); `d` points from orb to
// cor. Output: packed symmetric 4x4 block (10 values; only [0] for an s-only atom).
template <class S> PM3_HD void core_attraction(const ElemDev& orb, const ElemDev& cor, const S d[3], S out[10]) {
  const S r = sq_rt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const double rho = cor.po9;
  const double c = (orb.po1 + rho) * (orb.po1 + rho);
  out[0] = rsq(r * r + c) * (-cor.core * kEv);
  if (orb.z < 3 || orb.norb < 4) {
    for (int i = 1; i < 10; ++i) out[i] = mk<S>(0.0);
    return;
  }
  const S ir = inv(r);
  S R[9];
  frame(-(d[0] * ir), -(d[1] * ir), -(d[2] * ir), R);
  S ri[4];
  local4(core_pole(orb), rho, r, ri);
  for (int kk = 0; kk < 4; ++kk)
    for (int ll = 0; ll <= kk; ++ll) out[pk(kk, ll)] = w4(ri, R, kk, ll) * (-cor.core);
}

// ------------------------------------------------------------------------------ STO overlap
// A_k(x) = int_1^inf t^k e^{-xt} dt and B_k(x) = int_-1^1 t^k e^{-xt} dt, k = 0..kmax.
template <class S> PM3_HD void aux_a(const S& x, S a[7], int kmax) {
  if (fabs(vof(x)) < 1.0e-12) {
    for (int i = 0; i <= kmax; ++i) a[i] = mk<S>(0.0);
    return;
  }
  const S ix = inv(x);
  a[0] = ex(-x) * ix;
  for (int i = 1; i <= kmax; ++i) a[i] = a[0] + a[i - 1] * ix * (double)i;
}
template <class S> PM3_HD void aux_b(const S& x, S b[7], int kmax) {
  if (fabs(vof(x)) > 3.0) {
    const S ix = inv(x);
    const S ep = ex(x) * ix;
    const S em = ex(-x) * ix * (-1.0);
    b[0] = ep + em;
    for (int i = 1; i <= kmax; ++i) b[i] = ep * ((i & 1) ? -1.0 : 1.0) + em + b[i - 1] * ix * (double)i;
  } else {
    // B_k(x) = 2 sum_{m: k+m even} (-x)^m / (m! (k+m+1)), absolutely convergent
    for (int i = 0; i <= kmax; ++i) b[i] = mk<S>(0.0);
    S term = mk<S>(1.0);
    for (int m = 0; m < 40; ++m) {
      for (int k = (m & 1); k <= kmax; k += 2) b[k] = b[k] + term * (2.0 / (double)(k + m + 1));
      term = term * (-x) * (1.0 / (double)(m + 1));
    }
  }
}

// Local overlaps (s s sigma, p_a s sigma, s p_b sigma, p p sigma, p p pi) for ea the atom with
// the larger principal quantum number. Returns false when no closed form exists.
template <class S> PM3_HD bool overlap_local(const ElemDev& ea, const ElemDev& eb, const S& r, S o[5]) {
  const int na = ea.npq, nb = eb.npq;
  int j = 0;
  if (na == 1 && nb == 1) j = 11;
  else if (na == 2 && nb == 1) j = 21;
  else if (na == 2 && nb == 2) j = 22;
  else if (na == 3 && nb == 1) j = 31;
  else if (na == 3 && nb == 2) j = 32;
  else if (na == 3 && nb == 3) j = 33;
  if (j == 0) return false;
  const double za0 = ea.zs, za1 = ea.zp, zb0 = eb.zs, zb1 = eb.zp;
  double lo = 1.0e300;
  const double sums[4] = {za0 + zb0, za1 + zb0, za0 + zb1, za1 + zb1};
  for (int i = 0; i < 4; ++i)
    if (sums[i] > 0.0 && sums[i] < lo) lo = sums[i];
  for (int i = 0; i < 5; ++i) o[i] = mk<S>(0.0);
  // beyond this the overlap has underflowed while the A/B factors overflow separately
  if (lo < 1.0e300 && vof(r) * (0.5 * lo) > 300.0) return true;
  const int km = (na + nb + 1 < 6) ? na + nb + 1 : 6;
  S a11[7], b11[7];
  aux_a(r * (0.5 * (za0 + zb0)), a11, km);
  aux_b(r * (0.5 * (za0 - zb0)), b11, km);
  const double s3 = sqrt(3.0);
  if (j == 11) {
    o[0] = pw(r * r * (za0 * zb0), 1.5) * (a11[2] * b11[0] - b11[2] * a11[0]) * 0.25;
    return true;
  }
  S a21[7], b21[7];
  aux_a(r * (0.5 * (za1 + zb0)), a21, km);
  aux_b(r * (0.5 * (za1 - zb0)), b21, km);
  if (j == 21) {
    const S r4 = ipow(r, 4);
    o[0] = r4 * (pow(zb0, 1.5) * pow(za0, 2.5)) * (a11[3] * b11[0] - b11[3] * a11[0] + a11[2] * b11[1] - b11[2] * a11[1]) * (1.0 / (s3 * 8.0));
    o[1] = r4 * (pow(zb0, 1.5) * pow(za1, 2.5)) * (a21[2] * b21[0] - b21[2] * a21[0] + a21[3] * b21[1] - b21[3] * a21[1]) * 0.125;
    return true;
  }
  if (j == 31) {
    const S r5 = ipow(r, 5);
    o[0] = r5 * (pow(zb0, 1.5) * pow(za0, 3.5)) *
           (a11[4] * b11[0] + b11[1] * a11[3] * 2.0 - a11[1] * b11[3] * 2.0 - b11[4] * a11[0]) * (1.0 / (sqrt(10.0) * 24.0));
    o[1] = r5 * (pow(zb0, 1.5) * pow(za1, 3.5)) *
           (a21[3] * (b21[0] + b21[2]) - a21[1] * (b21[4] + b21[2]) + b21[1] * (a21[2] + a21[4]) - b21[3] * (a21[2] + a21[0])) *
           (1.0 / (8.0 * sqrt(30.0)));
    return true;
  }
  S a12[7], b12[7], a22[7], b22[7];
  aux_a(r * (0.5 * (za0 + zb1)), a12, km);
  aux_b(r * (0.5 * (za0 - zb1)), b12, km);
  aux_a(r * (0.5 * (za1 + zb1)), a22, km);
  aux_b(r * (0.5 * (za1 - zb1)), b22, km);
  if (j == 22) {
    const S r5 = ipow(r, 5);
    o[0] = r5 * pow(zb0 * za0, 2.5) * (a11[4] * b11[0] + b11[4] * a11[0] - a11[2] * b11[2] * 2.0) * (1.0 / 48.0);
    o[1] = r5 * pow(zb0 * za1, 2.5) *
           (a21[3] * (b21[0] - b21[2]) - a21[1] * (b21[2] - b21[4]) + b21[3] * (a21[0] - a21[2]) - b21[1] * (a21[2] - a21[4])) *
           (1.0 / (16.0 * s3));
    o[2] = r5 * pow(zb1 * za0, 2.5) *
           (a12[3] * (b12[0] - b12[2]) - a12[1] * (b12[2] - b12[4]) - b12[3] * (a12[0] - a12[2]) + b12[1] * (a12[2] - a12[4])) *
           (1.0 / (16.0 * s3));
    const S w = r5 * pow(zb1 * za1, 2.5) * (1.0 / 16.0);
    o[3] = -(w * (b22[2] * (a22[4] + a22[0]) - a22[2] * (b22[4] + b22[0])));
    o[4] = w * (a22[4] * (b22[0] - b22[2]) - b22[4] * (a22[0] - a22[2]) - a22[2] * b22[0] + b22[2] * a22[0]) * 0.5;
    return true;
  }
  if (j == 32) {
    const S r6 = ipow(r, 6);
    o[0] = r6 * (pow(zb0, 2.5) * pow(za0, 3.5)) *
           (a11[5] * b11[0] + b11[1] * a11[4] - b11[2] * a11[3] * 2.0 - a11[2] * b11[3] * 2.0 + b11[4] * a11[1] + b11[5] * a11[0]) *
           (1.0 / (sqrt(30.0) * 48.0));
    o[1] = r6 * (pow(zb0, 2.5) * pow(za1, 3.5)) *
           (a21[4] * b21[0] + b21[1] * a21[5] - b21[3] * a21[3] * 2.0 - a21[2] * b21[2] * 2.0 + a21[1] * b21[5] + a21[0] * b21[4]) *
           (1.0 / (48.0 * sqrt(10.0)));
    o[2] = r6 * (pow(zb1, 2.5) * pow(za0, 3.5)) *
           ((a12[4] * b12[0] - a12[5] * b12[1]) + (a12[3] * b12[1] - a12[4] * b12[2]) * 2.0 -
            (a12[1] * b12[3] - a12[2] * b12[4]) * 2.0 - (a12[0] * b12[4] - a12[1] * b12[5])) *
           (1.0 / (48.0 * sqrt(10.0)));
    o[3] = r6 * (pow(zb1, 2.5) * pow(za1, 3.5)) *
           ((a22[3] * b22[0] - a22[5] * b22[2]) + (a22[2] * b22[1] - a22[4] * b22[3]) - (a22[1] * b22[2] - a22[3] * b22[4]) -
            (a22[0] * b22[3] - a22[2] * b22[5])) *
           (1.0 / (16.0 * sqrt(30.0)));
    o[4] = r6 * (pow(zb1, 2.5) * pow(za1, 3.5)) *
           ((a22[5] - a22[3]) * (b22[0] - b22[2]) + (a22[4] - a22[2]) * (b22[1] - b22[3]) -
            (a22[3] - a22[1]) * (b22[2] - b22[4]) - (a22[2] - a22[0]) * (b22[3] - b22[5])) *
           (1.0 / (32.0 * sqrt(30.0)));
    return true;
  }
  // j == 33
  const S r7 = ipow(r, 7);
  o[0] = r7 * pow(zb0 * za0, 3.5) * (a11[6] * b11[0] - b11[2] * a11[4] * 3.0 + a11[2] * b11[4] * 3.0 - a11[0] * b11[6]) * (1.0 / 1440.0);
  o[1] = r7 * pow(zb0 * za1, 3.5) *
         ((a21[5] * b21[0] + a21[6] * b21[1]) - (a21[4] * b21[1] + a21[5] * b21[2]) - (a21[3] * b21[2] + a21[4] * b21[3]) * 2.0 +
          (a21[2] * b21[3] + a21[3] * b21[4]) * 2.0 + (a21[1] * b21[4] + a21[2] * b21[5]) - (a21[0] * b21[5] + a21[1] * b21[6])) *
         (1.0 / (480.0 * s3));
  o[2] = r7 * pow(zb1 * za0, 3.5) *
         ((a12[5] * b12[0] - a12[6] * b12[1]) + (a12[4] * b12[1] - a12[5] * b12[2]) - (a12[3] * b12[2] - a12[4] * b12[3]) * 2.0 -
          (a12[2] * b12[3] - a12[3] * b12[4]) * 2.0 + (a12[1] * b12[4] - a12[2] * b12[5]) + (a12[0] * b12[5] - a12[1] * b12[6])) *
         (1.0 / (480.0 * s3));
  o[3] = r7 * (pow(zb1, 3.5) * pow(za1, 3.5)) *
         ((a22[4] * b22[0] - a22[6] * b22[2]) - (a22[2] * b22[2] - a22[4] * b22[4]) * 2.0 + (a22[0] * b22[4] - a22[2] * b22[6])) *
         (1.0 / 480.0);
  o[4] = r7 * (pow(zb1, 3.5) * pow(za1, 3.5)) *
         ((a22[6] - a22[4]) * (b22[0] - b22[2]) - (a22[4] - a22[2]) * (b22[2] - b22[4]) * 2.0 + (a22[2] - a22[0]) * (b22[4] - b22[6])) *
         (1.0 / 960.0);
  return true;
}

// Overlap block S[i][j] (row-major 4x4: rows = AOs of `ei`, cols = AOs of `ej`), d = R_j - R_i.
template <class S> PM3_HD bool overlap_block(const ElemDev& ei, const ElemDev& ej, const S d[3], S s[16]) {
  const S r = sq_rt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (vof(r) < 1.0e-8) {
    for (int i = 0; i < 16; ++i) s[i] = mk<S>((i % 5 == 0) ? 1.0 : 0.0);
    return true;
  }
  const bool swap = ei.npq < ej.npq;
  const ElemDev& ea = swap ? ej : ei;
  const ElemDev& eb = swap ? ei : ej;
  S loc[5];
  if (!overlap_local(ea, eb, r, loc)) return false;
  const S ir = inv(r) * (swap ? -1.0 : 1.0);
  S R[9];
  frame(d[0] * ir, d[1] * ir, d[2] * ir, R);
  // columns of R^T are the rows of R; the a->b direction cosines are R[0], R[1], R[2]
  S di[16];
  di[0] = loc[0];
  for (int a = 0; a < 3; ++a) {
    di[(1 + a) * 4] = loc[1] * R[a];
    di[1 + a] = -(loc[2] * R[a]);
  }
  const S m0 = -loc[3], m1 = loc[4];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      di[(1 + a) * 4 + 1 + b] = R[a] * m0 * R[b] + R[3 + a] * m1 * R[3 + b] + R[6 + a] * m1 * R[6 + b];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) s[a * 4 + b] = swap ? di[b * 4 + a] : di[a * 4 + b];
  return true;
}

// -------------------------------------------------------------------------- core-core term
template <class S> PM3_HD S core_core(const ElemDev& ei, const ElemDev& ej, const PairDev& pp, const S& dist) {
  const S ra = dist * kA0;
  const double rho = ei.po9 + ej.po9;
  const S bare = rsq(dist * dist + rho * rho) * (kEv * ei.core * ej.core);
  const double cc = ei.core * ej.core;
  if (pp.has[ei.z][ej.z]) {
    return bare * (ex(ra * (-pp.alpha[ei.z][ej.z])) * (2.0 * pp.x[ei.z][ej.z]) + 1.0);
  }
  const S xi = ex(ra * (-ei.alpha)), xj = ex(ra * (-ej.alpha));
  S scale = xi + xj;
  const int zs = ei.z + ej.z;
  if (zs == 8 || zs == 9) {  // MNDO N-H / O-H adjustment kept by PM3
    if (ei.z == 7 || ei.z == 8) scale = scale + (ra - 1.0) * xi;
    if (ej.z == 7 || ej.z == 8) scale = scale + (ra - 1.0) * xj;
  }
  S e = ab(scale * bare) + bare;
  const S ira = inv(ra);
  for (int g = 0; g < ei.ngauss + ej.ngauss; ++g) {
    const bool first = g < ei.ngauss;
    const int k = first ? g : g - ei.ngauss;
    const double gk = first ? ei.gk[k] : ej.gk[k], gl = first ? ei.gl[k] : ej.gl[k], gm = first ? ei.gm[k] : ej.gm[k];
    const S dl = ra - gm;
    const S axp = dl * dl * gl;
    if (vof(axp) <= 25.0) e = e + ex(-axp) * (cc * gk) * ira;
  }
  return e;
}

}  // namespace pm3gpu
