// One SCF job inside a CTA: guess, the RHF / UHF iteration of pm3-rs (src/scf.rs:1179-1496),
// the closing energy, frontier, properties and (optionally) the analytic gradient
// (src/gradient.rs:306-599, src/repulsion.rs:30-49).
#pragma once
#include "scf_kernel.cuh"

namespace pm3gpu {

// Closed-form Hellmann-Feynman gradient at fixed densities (eV/Bohr), one thread per pair,
// forward-mode dual numbers through every integral.
__device__ void gradient_phase(Ctx& c, const double* Pt, const double* Pa, const double* Pb, double* gout) {
  const KernelArgs& A = *c.A;
  const int n = c.n, N = c.N, tid = threadIdx.x;
  const bool uhf = Pb != nullptr;
  double* g = c.jacc;  // [3N]
  for (int k = tid; k < 3 * N; k += kThreads) g[k] = 0.0;
  __syncthreads();
  const int npairs = N * (N - 1) / 2;
  for (int t = tid; t < npairs; t += kThreads) {
    int u, v;
    pair_uv(N, t, u, v);
    const bool hu = heavy(c, u), hv = heavy(c, v);
    const int a = (hu || !hv) ? u : v, b = a == u ? v : u;
    const ElemDev& ea = A.elem[c.sz[a]];
    const ElemDev& eb = A.elem[c.sz[b]];
    const int na = ea.norb, nb = eb.norb, oa = c.soff[a], ob = c.soff[b];
    const D3 dv[3] = {{c.sxyz[3 * b] - c.sxyz[3 * a], {1.0, 0.0, 0.0}},
                      {c.sxyz[3 * b + 1] - c.sxyz[3 * a + 1], {0.0, 1.0, 0.0}},
                      {c.sxyz[3 * b + 2] - c.sxyz[3 * a + 2], {0.0, 0.0, 1.0}}};
    double f[3] = {0.0, 0.0, 0.0};
    auto add = [&](double coef, const D3& x) {
      f[0] = fma(coef, x.g[0], f[0]);
      f[1] = fma(coef, x.g[1], f[1]);
      f[2] = fma(coef, x.g[2], f[2]);
    };
    {  // resonance: sum P_ab (beta_i + beta_j) dS
      D3 s[16];
      overlap_block(ea, eb, dv, s);
      for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j)
          add(Pt[(size_t)(oa + i) * n + ob + j] * ((i ? ea.bp : ea.bs) + (j ? eb.bp : eb.bs)), s[i * 4 + j]);
    }
    {  // electron-core attraction
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
    {  // two-electron: (Coulomb - exchange) x dW
      const D3 ir = inv(r);
      D3 R[9];
      frame(-(dv[0] * ir), -(dv[1] * ir), -(dv[2] * ir), R);
      auto coef = [&](int p, int q) {  // sum over the unpacked index pairs of p and q
        int ph, pl, qh, ql;
        unpk(p, ph, pl);
        unpk(q, qh, ql);
        double s = 0.0;
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
            s += coul + exch;
          }
        }
        return s;
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
    // core-core term (repulsion.rs:30-49): dE/dd along the same displacement
    add(1.0, core_core(ea, eb, *A.pairs, r));
    for (int ax = 0; ax < 3; ++ax) {
      atomicAdd(&g[3 * b + ax], f[ax]);
      atomicAdd(&g[3 * a + ax], -f[ax]);
    }
  }
  __syncthreads();
  for (int k = tid; k < 3 * N; k += kThreads) gout[k] = g[k];
  __syncthreads();
}

// ------------------------------------------------------------------------------- one job
__device__ void run_job(Ctx& c, int jid) {
  const KernelArgs& A = *c.A;
  c.job = A.jobs[jid];
  const JobDesc& J = c.job;
  c.n = J.nao;
  c.N = J.natom;
  const int n = c.n, tid = threadIdx.x;
  const size_t nn = (size_t)n * n;
  const bool uhf = (J.flags & kJobUhf) != 0;
  const int na = J.n_alpha, nb = J.n_beta;
  JobOut o;
  o.status = 0;
  o.converged = 0;
  o.iterations = 0;
  o.pad = 0;

  setup_job(c);
  o.core = build_core(c);
  if (J.flags & (kJobCoreOnly | kJobFockOnly)) {
    double* io = A.densities + J.dens_off;
    if (J.flags & kJobCoreOnly) {
      for (size_t k = tid; k < nn; k += kThreads) io[k] = c.H[k];
    } else {  // io = [P_tot | P_alpha | P_beta | F_alpha out | F_beta out]
      if (uhf) build_fock(c, io, io + nn, io + 2 * nn, io + 3 * nn, io + 4 * nn);
      else build_fock(c, io, nullptr, nullptr, io + 3 * nn, nullptr);
    }
    __syncthreads();
    if (tid == 0) A.out[jid] = o;
    __syncthreads();
    return;
  }

  // ------------------------------------------------------------------ initial density
  c.cur = 0;
  double* Pa = c.P[0];
  double* Pb = c.Q[0];
  if (J.guess == 2) {  // core-Hamiltonian orbitals, aufbau (scf.rs:929-932, 969-975)
    double* Ap = pack_input(c, c.H, nullptr, 0.0);
    const int kv = uhf ? na : na;  // na >= nb
    eigensolve(c, Ap, n < kv + 1 ? n : kv + 1, kv, c.Vt, c.tri_a + 2 * n, nullptr);
    density(c, c.Vt, na, uhf ? 1.0 : 2.0, Pa, Pa, 0.0);
    if (uhf) density(c, c.Vt, nb, 1.0, Pb, Pb, 0.0);
  } else {
    double fa = 1.0, fb = 0.0;
    if (uhf) {
      const double ne = (double)(na + nb);
      fa = ne > 0.0 ? na / ne : 0.5;
      fb = ne > 0.0 ? nb / ne : 0.5;
    }
    sad_guess(c, Pa, fa, J.guess == 3);
    if (uhf) sad_guess(c, Pb, fb, J.guess == 3);
  }

  // ------------------------------------------------------------------ SCF iteration
  const int depth = J.depth < 2 ? 2 : (J.depth > kMaxDepth ? kMaxDepth : J.depth);
  const bool keep = (J.flags & kJobKeepDens) != 0;
  int len = 0, head = 0;
  double e_old = 0.0, last_change = INFINITY;
  bool converged = false;
  int iterations = 0;
  double* eps_a = c.tri_a + 2 * n;  // eigenvalues of the last iteration (alpha, beta)
  double* eps_b = c.tri_b + 2 * n;
  const int kva = n < na + 1 ? n : na + 1;
  const int kvb = n < nb + 1 ? n : nb + 1;
  const int slot_mats = uhf ? 4 : 3;

  for (int iter = 0; iter < J.max_scf; ++iter) {
    iterations = iter + 1;
    double* Pc = c.P[c.cur];
    double* Qc = c.Q[c.cur];
    double* Pn = c.P[1 - c.cur];
    double* Qn = c.Q[1 - c.cur];
    // history slot of this iteration (drop the oldest entry when full)
    double* Fa = c.F;
    double* Fb = c.G;
    double *Ea = nullptr, *Eb = nullptr, *Dh = nullptr;
    if (J.accel != 0) {
      if (len == depth) {
        if (tid == 0) {
          for (int i = 0; i + 1 < len; ++i)
            for (int j = 0; j + 1 < len; ++j) {
              c.bg[i * kMaxDepth + j] = c.bg[(i + 1) * kMaxDepth + j + 1];
              c.mg[i * kMaxDepth + j] = c.mg[(i + 1) * kMaxDepth + j + 1];
            }
        }
        head = (head + 1) % depth;
        --len;
        __syncthreads();
      }
      const int s = (head + len) % depth;
      double* base = c.hist + (size_t)s * slot_mats * nn;
      Fa = base;
      Ea = base + nn;
      if (uhf) {
        Fb = base + 2 * nn;
        Eb = base + 3 * nn;
      } else {
        Dh = base + 2 * nn;
      }
    }
    double e_elec;
    if (!uhf) {
      build_fock(c, Pc, nullptr, nullptr, Fa, nullptr);
      double part = 0.0;
      for (size_t k = tid; k < nn; k += kThreads) part = fma(Pc[k], c.H[k] + Fa[k], part);
      e_elec = 0.5 * block_sum(part, c.red);
    } else {
      double* Pt = c.Vb + nn;  // scratch right after Vb (slot reserves it)
      for (size_t k = tid; k < nn; k += kThreads) Pt[k] = Pc[k] + Qc[k];
      __syncthreads();
      build_fock(c, Pt, Pc, Qc, Fa, Fb);
      double part = 0.0;
      for (size_t k = tid; k < nn; k += kThreads) part += Pt[k] * c.H[k] + Pc[k] * Fa[k] + Qc[k] * Fb[k];
      e_elec = 0.5 * block_sum(part, c.red);
    }

    // ---- accelerator (scf.rs:1240-1259 RHF; 1398-1413 UHF)
    bool use_hist = false;
    if (J.accel != 0) {
      commutator(c, Fa, Pc, Ea);
      if (uhf) commutator(c, Fb, Qc, Eb);
      if (keep)
        for (size_t k = tid; k < nn; k += kThreads) Dh[k] = Pc[k];
      __syncthreads();
      // new Gram row against the surviving entries l < len, then the new diagonal
      double acc[3 * kMaxDepth + 2];
#pragma unroll
      for (int q = 0; q < 3 * kMaxDepth + 2; ++q) acc[q] = 0.0;
      for (size_t k = tid; k < nn; k += kThreads) {
        const double ea = Ea[k], fa = Fa[k];
        const double eb = uhf ? Eb[k] : 0.0;
        const double dn = keep ? Dh[k] : 0.0;
        acc[3 * kMaxDepth] = fma(ea, ea, acc[3 * kMaxDepth]);
        if (uhf) acc[3 * kMaxDepth] = fma(eb, eb, acc[3 * kMaxDepth]);
        if (keep) acc[3 * kMaxDepth + 1] = fma(dn, fa, acc[3 * kMaxDepth + 1]);
#pragma unroll
        for (int l = 0; l < kMaxDepth; ++l) {
          if (l < len) {
            const double* bl = c.hist + (size_t)((head + l) % depth) * slot_mats * nn;
            double v = bl[nn + k] * ea;
            if (uhf) v = fma(bl[3 * nn + k], eb, v);
            acc[l] += v;
            if (keep) {
              acc[kMaxDepth + l] = fma(dn, bl[k], acc[kMaxDepth + l]);           // <D_new, F_l>
              acc[2 * kMaxDepth + l] = fma(bl[2 * nn + k], fa, acc[2 * kMaxDepth + l]);  // <D_l, F_new>
            }
          }
        }
      }
      block_sums<3 * kMaxDepth + 2>(acc, c.red, c.misc);
      if (tid == 0) {
        for (int l = 0; l < len; ++l) {
          c.bg[l * kMaxDepth + len] = c.misc[l];
          c.bg[len * kMaxDepth + l] = c.misc[l];
          c.mg[len * kMaxDepth + l] = c.misc[kMaxDepth + l];
          c.mg[l * kMaxDepth + len] = c.misc[2 * kMaxDepth + l];
        }
        c.bg[len * kMaxDepth + len] = c.misc[3 * kMaxDepth];
        c.mg[len * kMaxDepth + len] = c.misc[3 * kMaxDepth + 1];
        const int m = len + 1;
        const double err = sqrt(c.misc[3 * kMaxDepth]);
        bool ok;
        if (!uhf && J.accel == 2 && err > J.adiis_switch) {
          ok = keep && m >= 2;
          if (ok) adiis_coeffs(m, c.mg, c.coef);
        } else {
          ok = cdiis_coeffs(m, c.bg, c.coef);
        }
        c.iv[0] = ok ? 1 : 0;
      }
      ++len;
      __syncthreads();
      use_hist = c.iv[0] != 0;
    }

    // ---- diagonalise (level shift for UHF only, scf.rs:1416-1418) and rebuild densities
    double sq_a, sq_b = 0.0;
    {
      double* Ap = n <= A.sm.nsm ? c.Asm : c.Ag;
      const int nt = n * (n + 1) / 2;
      for (int spin = 0; spin < (uhf ? 2 : 1); ++spin) {
        const double* Pproj = spin == 0 ? Pc : Qc;
        const double* Fnew = spin == 0 ? Fa : Fb;
        for (int k = tid; k < nt; k += kThreads) {
          int r = (int)((sqrt(8.0 * k + 1.0) - 1.0) * 0.5);
          while (tri(r + 1) <= k) ++r;
          while (tri(r) > k) --r;
          const int col = k - tri(r);
          const size_t ix = (size_t)r * n + col;
          double v;
          if (use_hist) {
            v = 0.0;
            for (int l = 0; l < len; ++l) {
              const double* bl = c.hist + (size_t)((head + l) % depth) * slot_mats * nn;
              v = fma(c.coef[l], bl[(spin == 0 ? 0 : 2 * nn) + ix], v);
            }
          } else {
            v = Fnew[ix];
          }
          if (uhf && J.shift != 0.0) v += J.shift * ((r == col ? 1.0 : 0.0) - Pproj[ix]);
          Ap[k] = v;
        }
        __syncthreads();
        if (spin == 0) {
          eigensolve(c, Ap, kva, na, c.Vt, eps_a, c.tri_a);
          sq_a = density(c, c.Vt, na, uhf ? 1.0 : 2.0, Pc, Pn, uhf ? J.damping : 0.0);
        } else {
          eigensolve(c, Ap, kvb, nb, c.Vb, eps_b, c.tri_b);
          sq_b = density(c, c.Vb, nb, 1.0, Qc, Qn, J.damping);
        }
      }
    }
    const double dp = uhf ? sqrt(sq_a / (double)nn) + sqrt(sq_b / (double)nn) : sqrt(sq_a / (double)nn);
    const double de = fabs(e_elec - e_old);
    last_change = dp;
    e_old = e_elec;
    c.cur = 1 - c.cur;
    if (iter > 0 && de < J.e_tol && dp < J.p_tol) {
      converged = true;
      break;
    }
  }

  // ------------------------------------------------------- closing energy at the final density
  double* Pf = c.P[c.cur];
  double* Qf = c.Q[c.cur];
  double* Pt = Pf;
  if (!uhf) {
    build_fock(c, Pf, nullptr, nullptr, c.F, nullptr);
    double part = 0.0;
    for (size_t k = tid; k < nn; k += kThreads) part = fma(Pf[k], c.H[k] + c.F[k], part);
    o.electronic = 0.5 * block_sum(part, c.red);
    o.spin_max = 0.0;
  } else {
    Pt = c.Vb + nn;
    double mx = 0.0;
    for (size_t k = tid; k < nn; k += kThreads) {
      Pt[k] = Pf[k] + Qf[k];
      mx = fmax(mx, fabs(Pf[k] - Qf[k]));
    }
    o.spin_max = block_max(mx, c.red);
    build_fock(c, Pt, Pf, Qf, c.F, c.G);
    double part = 0.0;
    for (size_t k = tid; k < nn; k += kThreads) part += Pt[k] * c.H[k] + Pf[k] * c.F[k] + Qf[k] * c.G[k];
    o.electronic = 0.5 * block_sum(part, c.red);
  }
  o.converged = converged ? 1 : 0;
  o.iterations = iterations;
  o.last_change = last_change;
  o.status = converged ? 0 : 4;

  // frontier of the last iteration's orbitals (scf.rs:106-124, 804-822)
  o.has_homo_a = na >= 1;
  o.has_lumo_a = na < n;
  o.homo_a = na >= 1 ? eps_a[na - 1] : 0.0;
  o.lumo_a = na < n ? eps_a[na] : 0.0;
  o.homo = o.homo_a;
  o.lumo = o.lumo_a;
  o.has_homo = o.has_homo_a;
  o.has_lumo = o.has_lumo_a;
  if (uhf) {
    if (nb >= 1) {
      o.homo = o.has_homo ? fmax(o.homo, eps_b[nb - 1]) : eps_b[nb - 1];
      o.has_homo = 1;
    }
    if (nb < n) {
      o.lumo = o.has_lumo ? fmin(o.lumo, eps_b[nb]) : eps_b[nb];
      o.has_lumo = 1;
    }
  }
  o.gap = (o.has_homo && o.has_lumo) ? o.lumo - o.homo : INFINITY;

  properties(c, Pt, o);
  if (J.flags & kJobDensity) {
    double* dst = A.densities + J.dens_off;
    for (size_t k = tid; k < nn; k += kThreads) dst[k] = Pt[k];
  }
  if (J.flags & kJobEps) {
    all_eigenvalues(n, c.tri_a, c.tri_a + n, A.eps + J.eps_off, c.es);
    if (uhf) all_eigenvalues(n, c.tri_b, c.tri_b + n, A.eps + J.eps_off + n, c.es);
  }
  if (J.flags & kJobGrad) gradient_phase(c, Pt, uhf ? Pf : nullptr, uhf ? Qf : nullptr, A.grads + J.grad_off);
  __syncthreads();
  if (tid == 0) A.out[jid] = o;
  __syncthreads();
}

// ----------------------------------------------------------------------- the kernel
__global__ void __launch_bounds__(kThreads, 1) scf_batch_kernel(KernelArgs args) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_job;
  Ctx c;
  c.A = &args;
  const SmemLayout& L = args.sm;
  const int amax = L.amax;
  int* ip = reinterpret_cast<int*>(smem + L.off_int);
  c.sz = ip;
  c.soff = ip + amax;
  c.sprow = ip + 2 * amax;
  c.iv = ip + 3 * amax + 1;
  long long* lp = reinterpret_cast<long long*>(smem + L.off_dbl);
  c.sroff = lp;
  double* dp = reinterpret_cast<double*>(lp + amax);
  c.sxyz = dp;
  dp += 3 * amax;
  c.red = dp;
  dp += 4 * kMaxDepth * kWarps;
  c.misc = dp;
  dp += 4 * kMaxDepth;
  c.bg = dp;
  dp += kMaxDepth * kMaxDepth;
  c.mg = dp;
  dp += kMaxDepth * kMaxDepth;
  c.coef = dp;
  double* ep = reinterpret_cast<double*>(smem + L.off_eig);
  c.es.d = ep;
  c.es.e = ep + kMaxN;
  c.es.e2 = ep + 2 * kMaxN;
  c.es.tau = ep + 3 * kMaxN;
  c.es.v = ep + 4 * kMaxN;
  c.es.p = ep + 5 * kMaxN;
  c.es.lam = ep + 6 * kMaxN;
  c.es.red = c.red;
  c.es.misc = c.misc;
  int* eip = reinterpret_cast<int*>(ep + 7 * kMaxN);
  c.es.blk = eip;
  c.es.nblk = eip + kMaxN + 1;
  c.es.vinfo = eip + kMaxN + 2;
  double* up = reinterpret_cast<double*>(smem + L.off_union);
  c.dpk = up;
  c.jacc = up + 10 * amax;
  c.tile = up;
  c.Asm = up;

  const size_t nn = (size_t)args.nmax * args.nmax;
  double* slot = args.work + (size_t)blockIdx.x * args.slot;
  c.H = slot;
  c.P[0] = slot + nn;
  c.P[1] = slot + 2 * nn;
  c.Q[0] = slot + 3 * nn;
  c.Q[1] = slot + 4 * nn;
  c.F = slot + 5 * nn;
  c.G = slot + 6 * nn;
  c.Vt = slot + 7 * nn;
  c.Vb = slot + 8 * nn;  // followed by one nn of scratch (total density)
  c.Ag = slot + 10 * nn;
  c.tf = slot + 11 * nn;     // 6 nn: eigenvector scratch
  c.hist = slot + 17 * nn;   // 32 nn: accelerator history
  c.tri_a = slot + 49 * nn;
  c.tri_b = c.tri_a + 3 * args.nmax;
  c.W = c.tri_b + 3 * args.nmax;

  for (;;) {
    if (threadIdx.x == 0) s_job = atomicAdd(args.queue, 1);
    __syncthreads();
    const int jid = s_job;
    __syncthreads();
    if (jid >= args.njobs) break;
    run_job(c, jid);
  }
}

inline long long slot_doubles(int nmax, long long wcap) {
  const long long nn = (long long)nmax * nmax;
  return 49 * nn + 6LL * nmax + wcap + 64;
}

}  // namespace pm3gpu
