// PM3 element constants as the GPU library uses them, and their derivation from the raw
// MOPAC parameter table (pm3_param_table.h).
//
// The derivation restates pm3-rs src/params.rs:155-343 (s/p elements only): the multipole
// charge separations dd/qq (params.rs:584-594, MOPAC calpar), the Klopman-Ohno additive terms
// rho0/rho1/rho2 with exactly five secant steps (params.rs:605-649), the isolated-atom energy
// (params.rs:268-289) and the main-group `po`/`ddp` overwrite (params.rs:694-709).
#pragma once
#include <cmath>

#include "pm3_param_table.h"

namespace pm3gpu {

constexpr double kEv = 27.211386245988;             // Hartree in eV (MOPAC 2018 CODATA)
constexpr double kA0 = 0.529177210903;              // Bohr in Angstrom
constexpr double kEvToKcal = 23.06054783061903;     // eV in kcal/mol
constexpr double kAuDipoleToDebye = 2.541746473;    // e*Bohr in Debye
constexpr int kMaxZ = 18;                           // table indexed by Z < 18

// Everything a kernel needs about one element, plain data (lives in global memory on device).
struct ElemDev {
  int z, norb, npq;      // npq: principal quantum number of the s shell (overlap branch)
  int ngauss;
  double uss, upp, zs, zp, bs, bp;
  double gss, gsp, gpp, gp2, hsp;
  double alpha, core;
  // electron-electron multipoles
  double dd, qq, rho0, rho1, rho2;
  // electron-core multipoles (MOPAC spcore uses po(1..3), ddp(2), ddp(3)/sqrt2 and po(9))
  double po1, po2, po3, po9, ddp2, qq_core;
  double occ_s, occ_p, e_isol, eheat_ev, mass;
  double gk[4], gl[4], gm[4];
};

struct PairDev {
  double alpha[kMaxZ][kMaxZ];
  double x[kMaxZ][kMaxZ];
  int has[kMaxZ][kMaxZ];
};

namespace detail {
inline double row_of(int z) { return z <= 2 ? 1.0 : (z <= 10 ? 2.0 : 3.0); }

// Solve H_sp(au) = d/2 - 1/(2 sqrt(4 D1^2 + 1/d^2)) by a secant iteration stopped after
// five steps, as MOPAC does (the truncation is part of the parameterization).
inline double secant_rho1(double hsp_ev, double d1) {
  const double target = std::fmax(hsp_ev, 1.0e-7) / kEv;
  auto f = [d1](double d) { return 0.5 * d - 0.5 / std::sqrt(4.0 * d1 * d1 + 1.0 / (d * d)); };
  double x0 = std::pow(target / (d1 * d1), 1.0 / 3.0);
  double x1 = x0 + 0.04;
  for (int k = 0; k < 5; ++k) {
    const double f0 = f(x0), f1 = f(x1);
    if (std::fabs(f1 - f0) < 1.0e-25) break;
    const double x2 = x0 + (x1 - x0) * (target - f0) / (f1 - f0);
    x0 = x1;
    x1 = x2;
  }
  return 0.5 / x1;
}

// Same for the quadrupole: H_pp(au) = q/4 - 1/(2 sqrt(4 D2^2 + 1/q^2)) + 1/(4 sqrt(8 D2^2 + 1/q^2)).
inline double secant_rho2(double hpp_ev, double d2) {
  const double target = hpp_ev / kEv;
  auto f = [d2](double q) {
    return 0.25 * q - 0.5 / std::sqrt(4.0 * d2 * d2 + 1.0 / (q * q)) + 0.25 / std::sqrt(8.0 * d2 * d2 + 1.0 / (q * q));
  };
  double x0 = std::pow(16.0 * target / (48.0 * d2 * d2 * d2 * d2), 0.2);
  double x1 = x0 + 0.04;
  for (int k = 0; k < 5; ++k) {
    const double f0 = f(x0), f1 = f(x1);
    if (std::fabs(f1 - f0) < 1.0e-25) break;
    const double x2 = x0 + (x1 - x0) * (target - f0) / (f1 - f0);
    x0 = x1;
    x1 = x2;
  }
  return 0.5 / x1;
}
}  // namespace detail

// Fill `out` (indexed by Z) from the raw table; entries with z == 0 are absent elements.
inline void derive_elements(ElemDev out[kMaxZ], PairDev* pairs) {
  for (int z = 0; z < kMaxZ; ++z) out[z] = ElemDev{};
  for (int k = 0; k < PM3_N_RAW_ELEMENTS; ++k) {
    const Pm3RawElement& r = PM3_RAW_ELEMENTS[k];
    if (r.z <= 0 || r.z >= kMaxZ) continue;
    ElemDev e{};
    e.z = r.z;
    e.norb = r.zp > 0.0 ? 4 : 1;
    e.npq = r.npq_s;
    e.uss = r.uss;
    e.upp = r.upp;
    e.zs = r.zs;
    e.zp = r.zp;
    e.bs = r.betas;
    e.bp = r.betap;
    e.gss = r.gss;
    e.gsp = r.gsp;
    e.gpp = r.gpp;
    e.gp2 = r.gp2;
    e.hsp = std::fmax(r.hsp, 1.0e-7);
    e.alpha = r.alp;
    e.core = r.tore;
    e.occ_s = r.ios;
    e.occ_p = r.iop;
    e.eheat_ev = r.eheat_kcal / kEvToKcal;
    e.mass = r.mass;
    e.ngauss = 0;
    for (int g = 0; g < 4; ++g) {
      if (r.gauss[g][0] != 0.0 || r.gauss[g][1] != 0.0) {
        e.gk[e.ngauss] = r.gauss[g][0];
        e.gl[e.ngauss] = r.gauss[g][1];
        e.gm[e.ngauss] = r.gauss[g][2];
        ++e.ngauss;
      }
    }
    e.rho0 = e.gss > 0.0 ? 0.5 * kEv / e.gss : 0.0;
    if (e.norb == 4) {
      const double n = detail::row_of(e.z);
      const double zp = std::fmax(e.zp, 0.3);
      e.dd = (2.0 * n + 1.0) * std::pow(4.0 * e.zs * zp, n + 0.5) / std::pow(e.zs + zp, 2.0 * n + 2.0) / std::sqrt(3.0);
      e.qq = std::sqrt((4.0 * n * n + 6.0 * n + 2.0) / 20.0) / zp;
      e.rho1 = detail::secant_rho1(e.hsp, e.dd);
      e.rho2 = detail::secant_rho2(std::fmax(0.5 * (e.gpp - e.gp2), 0.1), e.qq);
      e.po1 = e.rho0;
      e.po2 = e.rho1;
      e.po3 = e.rho2;
      e.ddp2 = e.dd;
      // MOPAC stores ddp(3) = qq*sqrt(2) and spcore divides it back out.
      e.qq_core = (e.qq * std::sqrt(2.0)) / std::sqrt(2.0);
    } else {
      e.po1 = e.rho0;
    }
    e.po9 = e.rho0;
    // Average-of-configuration isolated-atom energy (MOPAC calpar), hydrogen special-cased.
    if (e.z == 1) {
      e.e_isol = e.uss;
    } else {
      const double s = r.ios, p = r.iop;
      const long kp = (long)p, l = kp < 6 - kp ? kp : 6 - kp;
      const double c_ss = std::fmax(s - 1.0, 0.0);
      const double c_sp = s * p;
      const double c_p2 = (double)((kp * (kp - 1)) / 2) + (double)(l * (l - 1)) / 4.0;
      const double c_pp = -((double)(l * (l - 1))) / 4.0;
      const double c_hsp = -p * s * 0.5;
      e.e_isol = e.uss * s + e.upp * p + e.gss * c_ss + e.gpp * c_pp + e.gsp * c_sp + e.gp2 * c_p2 + e.hsp * c_hsp;
    }
    out[e.z] = e;
  }
  if (pairs) {
    for (int i = 0; i < kMaxZ; ++i)
      for (int j = 0; j < kMaxZ; ++j) {
        pairs->alpha[i][j] = 0.0;
        pairs->x[i][j] = 0.0;
        pairs->has[i][j] = 0;
      }
    for (int k = 0; k < PM3_N_RAW_PAIRS; ++k) {
      const Pm3RawPair& p = PM3_RAW_PAIRS[k];
      if (p.zi >= kMaxZ || p.zj >= kMaxZ) continue;
      // MOPAC reads xfac only when it is non-negligible (repulsion.rs:75-83).
      const int use = std::fabs(p.xfac) > 1.0e-5;
      pairs->alpha[p.zi][p.zj] = pairs->alpha[p.zj][p.zi] = p.alpb < 1.0e-6 ? 1.2 : p.alpb;
      pairs->x[p.zi][p.zj] = pairs->x[p.zj][p.zi] = p.xfac;
      pairs->has[p.zi][p.zj] = pairs->has[p.zj][p.zi] = use;
    }
  }
}

}  // namespace pm3gpu
