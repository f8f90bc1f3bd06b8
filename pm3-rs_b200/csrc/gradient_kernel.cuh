// Closed-form Hellmann-Feynman gradient at fixed converged densities (pm3-rs
// src/gradient.rs:306-599 and src/repulsion.rs:30-49), one thread per atom pair over the pairs
// of every molecule of a batch, forward-mode dual numbers through every integral. Each pair's
// force is added to atom b and subtracted from atom a with FP64 atomics.
#pragma once
#include "pm3_integrals.cuh"

namespace pm3gpu {

struct GradMol {
  int atom0, natom, nao, uhf;
  long long pair0;     // first global pair index of this molecule
  long long dens_off;  // P_tot [, P_alpha, P_beta] in the density buffer
};

struct GradArgs {
  const ElemDev* elem;
  const PairDev* pairs;
  const int* z;
  const double* xyz;
  const int* ao_off;   // first AO of each atom within its molecule
  const GradMol* mols;
  int nmol;
  long long npairs;
  const double* dens;
  double* grad;        // [3 * total atoms], zeroed by the host
};

// dE/d(R_b - R_a) of one ordered pair (a heavy-first), eV/Bohr.
__device__ void pair_gradient(const ElemDev& ea, const ElemDev& eb, const PairDev& pp, const double* ra,
                              const double* rb, int oa, int ob, int n, const double* Pt, const double* Pa,
                              const double* Pb, double f[3]) {
  const bool uhf = Pb != nullptr;
  const int na = ea.norb, nb = eb.norb;
  const D3 dv[3] = {{rb[0] - ra[0], {1.0, 0.0, 0.0}}, {rb[1] - ra[1], {0.0, 1.0, 0.0}}, {rb[2] - ra[2], {0.0, 0.0, 1.0}}};
  f[0] = f[1] = f[2] = 0.0;
  auto add = [&](double coef, const D3& x) {
    f[0] = fma(coef, x.g[0], f[0]);
    f[1] = fma(coef, x.g[1], f[1]);
    f[2] = fma(coef, x.g[2], f[2]);
  };
  {  // resonance: P_ab (beta_i + beta_j) dS_ab (both off-diagonal blocks)
    D3 s[16];
    overlap_block(ea, eb, dv, s);
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < nb; ++j)
        add(Pt[(size_t)(oa + i) * n + ob + j] * ((i ? ea.bp : ea.bs) + (j ? eb.bp : eb.bs)), s[i * 4 + j]);
  }
  {  // electron-core attraction of both atoms
    D3 blk[10];
    core_attraction(ea, eb, dv, blk);
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < na; ++j) add(Pt[(size_t)(oa + i) * n + oa + j], blk[pk(i, j)]);
    const D3 mdv[3] = {-dv[0], -dv[1], -dv[2]};
    core_attraction(eb, ea, mdv, blk);
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j) add(Pt[(size_t)(ob + i) * n + ob + j], blk[pk(i, j)]);
  }
  const D3 r = sq_rt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
  {  // two-electron: (Coulomb - exchange) contracted with dW
    const D3 ir = inv(r);
    D3 R[9];
    frame(-(dv[0] * ir), -(dv[1] * ir), -(dv[2] * ir), R);
    auto coef = [&](int p, int q) {  // sum over the unpacked orbital pairs of p and q
      int ph, pl, qh, ql;
      unpk(p, ph, pl);
      unpk(q, qh, ql);
      double sum = 0.0;
      for (int o1 = 0; o1 < (ph == pl ? 1 : 2); ++o1) {
        const int mu = o1 ? pl : ph, nu = o1 ? ph : pl;
        for (int o2 = 0; o2 < (qh == ql ? 1 : 2); ++o2) {
          const int la = o2 ? ql : qh, si = o2 ? qh : ql;
          const double coul = Pt[(size_t)(oa + mu) * n + oa + nu] * Pt[(size_t)(ob + la) * n + ob + si];
          double exch;
          if (uhf)
            exch = -(Pa[(size_t)(oa + mu) * n + ob + la] * Pa[(size_t)(oa + nu) * n + ob + si] +
                     Pb[(size_t)(oa + mu) * n + ob + la] * Pb[(size_t)(oa + nu) * n + ob + si]);
          else
            exch = -0.5 * Pt[(size_t)(oa + mu) * n + ob + la] * Pt[(size_t)(oa + nu) * n + ob + si];
          sum += coul + exch;
        }
      }
      return sum;
    };
    if (na == 1) {
      const double sr = ea.rho0 + eb.rho0;
      add(coef(0, 0), rsq(r * r + sr * sr) * kEv);
    } else if (nb == 1) {
      D3 ri[4];
      local4(ee_pole(ea), eb.rho0, r, ri);
      for (int kk = 0; kk < 4; ++kk)
        for (int ll = 0; ll <= kk; ++ll) add(coef(pk(kk, ll), 0), w4(ri, R, kk, ll));
    } else {
      D3 ri[22];
      local22(ee_pole(ea), ee_pole(eb), r, ri);
      for (int kk = 0; kk < 4; ++kk)
        for (int ll = 0; ll <= kk; ++ll)
          for (int mm = 0; mm < 4; ++mm)
            for (int nn = 0; nn <= mm; ++nn) add(coef(pk(kk, ll), pk(mm, nn)), w22(ri, R, kk, ll, mm, nn));
    }
  }
  add(1.0, core_core(ea, eb, pp, r));  // core-core repulsion
}

__global__ void __launch_bounds__(128) gradient_kernel(GradArgs g) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < g.npairs; t += stride) {
    int lo = 0, hi = g.nmol - 1;  // molecule with pair0 <= t < next pair0
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (g.mols[mid].pair0 <= t) lo = mid;
      else hi = mid - 1;
    }
    const GradMol& M = g.mols[lo];
    int u, v;
    {
      const int N = M.natom;
      const int loc = (int)(t - M.pair0);
      const double b = 2.0 * N - 1.0;
      int uu = (int)floor((b - sqrt(b * b - 8.0 * loc)) * 0.5);
      if (uu < 0) uu = 0;
      while (uu > 0 && uu * (2 * N - uu - 1) / 2 > loc) --uu;
      while ((uu + 1) * (2 * N - uu - 2) / 2 <= loc) ++uu;
      u = uu;
      v = loc - uu * (2 * N - uu - 1) / 2 + uu + 1;
    }
    const int zu = g.z[M.atom0 + u], zv = g.z[M.atom0 + v];
    const bool hu = g.elem[zu].norb == 4, hv = g.elem[zv].norb == 4;
    const int a = (hu || !hv) ? u : v, b = a == u ? v : u;
    const int ga = M.atom0 + a, gb = M.atom0 + b;
    const size_t nn = (size_t)M.nao * M.nao;
    const double* Pt = g.dens + M.dens_off;
    double f[3];
    pair_gradient(g.elem[g.z[ga]], g.elem[g.z[gb]], *g.pairs, g.xyz + 3 * (size_t)ga, g.xyz + 3 * (size_t)gb,
                  g.ao_off[ga], g.ao_off[gb], M.nao, Pt, M.uhf ? Pt + nn : nullptr, M.uhf ? Pt + 2 * nn : nullptr, f);
    for (int ax = 0; ax < 3; ++ax) {
      atomicAdd(&g.grad[3 * (size_t)gb + ax], f[ax]);
      atomicAdd(&g.grad[3 * (size_t)ga + ax], -f[ax]);
    }
  }
}

}  // namespace pm3gpu
