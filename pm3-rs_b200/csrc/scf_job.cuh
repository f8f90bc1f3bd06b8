// One SCF job inside a CTA: guess, the RHF / UHF iteration of pm3-rs (src/scf.rs:1179-1496),
// the closing energy, frontier, properties and (optionally) the analytic gradient
// (src/gradient.rs:306-599, src/repulsion.rs:30-49).
#pragma once
#include "scf_kernel.cuh"

namespace pm3gpu {

// ------------------------------------------------------------------------------- one job
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait of one thread for *p >= want (about a second at most). False when it ran out.
__device__ __forceinline__ bool wait_at_least(const volatile int* p, int want) {
  for (int i = 0; i < (1 << 22); ++i) {
    if (*p >= want) return true;
    __nanosleep(200);
  }
  return false;
}

__device__ void run_job(Ctx& c, const JobDesc& job, JobOut* out, int kind = -1, int jidx = -1) {
  const KernelArgs& A = *c.A;
  c.job = job;
  c.out = out;
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

  c.tmark = clock64();
  setup_job(c);
  o.core = build_core(c);
  mark(c, kPhCore);
  if (J.flags & (kJobCoreOnly | kJobFockOnly)) {
    double* io = A.densities + J.dens_off;
    if (J.flags & kJobCoreOnly) {
      for (size_t k = tid; k < nn; k += kThreads) io[k] = c.H[k];
    } else {  // io = [P_tot | P_alpha | P_beta | F_alpha out | F_beta out]
      if (uhf) build_fock(c, io, io + nn, io + 2 * nn, io + 3 * nn, io + 4 * nn);
      else build_fock(c, io, nullptr, nullptr, io + 3 * nn, nullptr);
    }
    __syncthreads();
    if (tid == 0) *out = o;
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
  } else if (J.guess == 4) {  // given (learned) density, scaled to the electron count
    const double* G0 = A.guess_dens + J.guess_off;
    double tr = 0.0;
    for (int k = tid; k < n; k += kThreads) tr += G0[(size_t)k * n + k];
    tr = block_sum(tr, c.red);
    const double ne = (double)(na + nb);
    const double sc = tr > 0.0 ? ne / tr : 0.0;
    const double fa = uhf ? (ne > 0.0 ? na / ne : 0.5) : 1.0, fb = ne > 0.0 ? nb / ne : 0.5;
    for (size_t k = tid; k < nn; k += kThreads) {
      const double g = G0[k] * sc;
      Pa[k] = fa * g;
      if (uhf) Pb[k] = fb * g;
    }
    __syncthreads();
    // The prediction is not an idempotent density, and A-DIIS would treat it as one. One
    // Roothaan step turns it into an aufbau density (as the core guess does with H): its Fock
    // matrix, diagonalised, gives the occupied orbitals the iteration starts from.
    if (!uhf) {
      build_fock(c, Pa, nullptr, nullptr, c.F, nullptr);
    } else {
      double* Pt = c.Vb + nn;
      for (size_t k = tid; k < nn; k += kThreads) Pt[k] = Pa[k] + Pb[k];
      __syncthreads();
      build_fock(c, Pt, Pa, Pb, c.F, c.G);
    }
    double* Ap = pack_input(c, c.F, nullptr, 0.0);
    eigensolve(c, Ap, n < na + 1 ? n : na + 1, na, c.Vt, c.tri_a + 2 * n, nullptr);
    density(c, c.Vt, na, uhf ? 1.0 : 2.0, Pa, Pa, 0.0);
    if (uhf) {
      Ap = pack_input(c, c.G, nullptr, 0.0);
      eigensolve(c, Ap, n < nb + 1 ? n : nb + 1, nb, c.Vb, c.tri_b + 2 * n, nullptr);
      density(c, c.Vb, nb, 1.0, Pb, Pb, 0.0);
    }
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

  // An unaccelerated unrestricted job offers its beta spin to an idle CTA: from the first
  // iteration boundary after a helper took the offer, the helper builds F_beta, diagonalises it
  // and forms P_beta on this CTA's workspace while this CTA does the alpha spin.
  HelpRec* hr = (A.help && uhf && J.accel == 0 && kind >= 0) ? A.help + blockIdx.x : nullptr;
  __shared__ int s_pair;  // 1 once the two CTAs run the iterations together
  int gen = 0;
  if (tid == 0) {
    s_pair = 0;
    if (hr) {
      gen = (((volatile HelpRec*)hr)->sg >> 3) + 1;
      hr->kind = kind;
      hr->idx = jidx;
      hr->go = -1;
      hr->hdone = -1;
      __threadfence();
      atomicExch(&hr->sg, gen * 8 + 1);
    }
  }
  __syncthreads();

  for (int iter = 0; iter < J.max_scf; ++iter) {
    iterations = iter + 1;
    if (hr) {  // a helper that took the offer starts with this iteration
      if (tid == 0 && !s_pair && atomicAdd(&hr->sg, 0) == gen * 8 + 2) {
        hr->cur = c.cur;
        hr->go = iter;
        __threadfence();
        // a helper that gave up waiting has set the offer to stop: then this job stays alone
        s_pair = atomicCAS(&hr->sg, gen * 8 + 2, gen * 8 + 3) == gen * 8 + 2 ? 1 : 0;
        if (s_pair) atomicAdd(&A.queue[6], 1);  // jobs that ran paired (reported to the host)
      }
      __syncthreads();
    }
    const bool paired = hr && s_pair;
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
      mark(c, kPhFock);
    } else if (paired) {  // alpha here; the helper builds F_beta and returns its energy part
      double* Pt = c.Vb + nn;
      for (size_t k = tid; k < nn; k += kThreads) Pt[k] = Pc[k] + Qc[k];
      __syncthreads();
      build_fock(c, Pt, Pc, nullptr, Fa, nullptr);
      double part = 0.0;
      for (size_t k = tid; k < nn; k += kThreads) part += Pt[k] * c.H[k] + Pc[k] * Fa[k];
      e_elec = block_sum(part, c.red);  // completed with the helper's part below
      mark(c, kPhFock);
    } else {
      double* Pt = c.Vb + nn;  // scratch right after Vb (slot reserves it)
      for (size_t k = tid; k < nn; k += kThreads) Pt[k] = Pc[k] + Qc[k];
      __syncthreads();
      build_fock(c, Pt, Pc, Qc, Fa, Fb);
      double part = 0.0;
      for (size_t k = tid; k < nn; k += kThreads) part += Pt[k] * c.H[k] + Pc[k] * Fa[k] + Qc[k] * Fb[k];
      e_elec = 0.5 * block_sum(part, c.red);
      mark(c, kPhFock);
    }

    // ---- accelerator (scf.rs:1240-1259 RHF; 1398-1413 UHF)
    bool use_hist = false;
    if (J.accel != 0) {
      commutator(c, Fa, Pc, Ea);
      if (uhf) commutator(c, Fb, Qc, Eb);
      if (keep)
        for (size_t k = tid; k < nn; k += kThreads) Dh[k] = Pc[k];
      __syncthreads();
      mark(c, kPhCommutator);
      // new Gram row against the surviving entries l < len, then the new diagonal
      double acc[3 * kMaxDepth + 2];
#pragma unroll
      for (int q = 0; q < 3 * kMaxDepth + 2; ++q) acc[q] = 0.0;
      // Every product pairs two symmetric (F, D) or two antisymmetric (E) matrices, so the sum
      // over all n^2 elements is the diagonal plus twice the strict lower triangle: half the
      // history reads. Rows go to warps, columns to lanes (coalesced).
      for (int r = tid >> 5; r < n; r += kWarps)
        for (int col = tid & 31; col <= r; col += 32) {
          const size_t k = (size_t)r * n + col;
          const double wgt = col == r ? 1.0 : 2.0;
          const double ea = Ea[k], fa = Fa[k];
          const double eb = uhf ? Eb[k] : 0.0;
          const double dn = keep ? Dh[k] : 0.0;
          double ee = ea * ea;
          if (uhf) ee = fma(eb, eb, ee);
          acc[3 * kMaxDepth] = fma(wgt, ee, acc[3 * kMaxDepth]);
          if (keep) acc[3 * kMaxDepth + 1] = fma(wgt, dn * fa, acc[3 * kMaxDepth + 1]);
#pragma unroll
          for (int l = 0; l < kMaxDepth; ++l) {
            if (l < len) {
              const double* bl = c.hist + (size_t)((head + l) % depth) * slot_mats * nn;
              double v = bl[nn + k] * ea;
              if (uhf) v = fma(bl[3 * nn + k], eb, v);
              acc[l] = fma(wgt, v, acc[l]);
              if (keep) {
                acc[kMaxDepth + l] = fma(wgt, dn * bl[k], acc[kMaxDepth + l]);             // <D_new, F_l>
                acc[2 * kMaxDepth + l] = fma(wgt, bl[2 * nn + k] * fa, acc[2 * kMaxDepth + l]);  // <D_l, F_new>
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
        int mode = 0;
        if (!uhf && J.accel == 2 && err > J.adiis_switch) {
          ok = keep && m >= 2;
          mode = ok ? 1 : 0;  // A-DIIS weights: solved by warp 0 below
        } else {
          ok = cdiis_coeffs(m, c.bg, c.coef);
        }
        c.iv[0] = ok ? 1 : 0;
        c.iv[1] = mode;
      }
      ++len;
      __syncthreads();
      if (c.iv[1] == 1) {  // uniform across the CTA
        if (tid < 32) adiis_coeffs_warp(len, c.mg, c.coef, c.red);
        __syncthreads();
      }
      use_hist = c.iv[0] != 0;
      mark(c, kPhDiisSolve);
    }

    // ---- diagonalise (level shift for UHF only, scf.rs:1416-1418) and rebuild densities
    double sq_a, sq_b = 0.0;
    {
      double* Ap = n <= A.sm.nsm ? c.Asm : c.Ag;
      const double* __restrict__ coef = c.coef;
      const double* __restrict__ hist = c.hist;
      const double shift = J.shift;
      for (int spin = 0; spin < (uhf && !paired ? 2 : 1); ++spin) {
        const double* Pproj = spin == 0 ? Pc : Qc;
        const double* Fnew = spin == 0 ? Fa : Fb;
        // rows to warps, columns to lanes (coalesced reads of the history matrices)
        for (int r = tid >> 5; r < n; r += kWarps)
          for (int col = tid & 31; col <= r; col += 32) {
            const size_t ix = (size_t)r * n + col;
            double v;
            if (use_hist) {
              v = 0.0;
              for (int l = 0; l < len; ++l) {
                const double* bl = hist + (size_t)((head + l) % depth) * slot_mats * nn;
                v = fma(coef[l], bl[(spin == 0 ? 0 : 2 * nn) + ix], v);
              }
            } else {
              v = Fnew[ix];
            }
            if (uhf && shift != 0.0) v += shift * ((r == col ? 1.0 : 0.0) - Pproj[ix]);
            Ap[tri(r) + col] = v;
          }
        __syncthreads();
        if (spin == 0) {
          eigensolve(c, Ap, kva, na, c.Vt, eps_a, c.tri_a, iter > 0, c.tri_a + 3 * n);
          sq_a = density(c, c.Vt, na, uhf ? 1.0 : 2.0, Pc, Pn, uhf ? J.damping : 0.0);
          mark(c, kPhDensity);
        } else {
          eigensolve(c, Ap, kvb, nb, c.Vb, eps_b, c.tri_b, iter > 0, c.tri_b + 3 * n);
          sq_b = density(c, c.Vb, nb, 1.0, Qc, Qn, J.damping);
          mark(c, kPhDensity);
        }
      }
    }
    if (paired) {  // the helper's beta spin of this iteration: energy part and density change
      if (tid == 0) {
        const bool ok = wait_at_least(&((volatile HelpRec*)hr)->hdone, iter);
        if (!ok) atomicExch(&A.queue[3], 1);  // reported by the host as a device error
        __threadfence();
        c.misc[0] = ok ? ((volatile HelpRec*)hr)->part_b[iter & 1] : NAN;
        c.misc[1] = ok ? ((volatile HelpRec*)hr)->sq_b[iter & 1] : NAN;
      }
      __syncthreads();
      e_elec = 0.5 * (e_elec + c.misc[0]);
      sq_b = c.misc[1];
      __syncthreads();
    }
    const double dp = uhf ? sqrt(sq_a / (double)nn) + sqrt(sq_b / (double)nn) : sqrt(sq_a / (double)nn);
    const double de = fabs(e_elec - e_old);
    last_change = dp;
    e_old = e_elec;
    c.cur = 1 - c.cur;
    const bool done = (iter > 0 && de < J.e_tol && dp < J.p_tol) || !(dp == dp);
    if (paired && tid == 0 && !done && iter + 1 < J.max_scf) {  // the helper may run the next iteration
      hr->cur = c.cur;
      __threadfence();
      atomicExch(&hr->go, iter + 1);
    }
    if (iter > 0 && de < J.e_tol && dp < J.p_tol) {
      converged = true;
      break;
    }
    if (!(dp == dp)) break;  // only after a failed pairing wait (NaN), which the host reports
  }
  if (hr && tid == 0) {  // close the offer: stop the helper, or withdraw an offer not yet taken
    if (atomicCAS(&hr->sg, gen * 8 + 1, gen * 8) != gen * 8 + 1) atomicExch(&hr->sg, gen * 8 + 4);
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
  if (J.flags & (kJobDensity | kJobGrad)) {
    double* dst = A.densities + J.dens_off;
    for (size_t k = tid; k < nn; k += kThreads) dst[k] = Pt[k];
    if ((J.flags & kJobGrad) && uhf)
      for (size_t k = tid; k < nn; k += kThreads) {
        dst[nn + k] = Pf[k];
        dst[2 * nn + k] = Qf[k];
      }
  }
  if (J.flags & kJobEps) {
    all_eigenvalues(n, c.tri_a, c.tri_a + n, A.eps + J.eps_off, c.es);
    if (uhf) all_eigenvalues(n, c.tri_b, c.tri_b + n, A.eps + J.eps_off + n, c.es);
  }
  __syncthreads();
  mark(c, kPhFinal);
  if (tid == 0) {
    *out = o;
    if (J.backup >= 0 && !o.converged) {  // learned start failed: the standard-guess pass takes over
      const int base = atomicAdd(&A.queue[1], 1);
      A.rlist[base] = J.backup;
      __threadfence();
      atomicExch(&A.rready[base], 1);
    } else if (J.nrung > 0 && (J.stab == 2 || (J.stab == 1 && o.gap < 6.0))) {
      // stability search (scf.rs:599-715): queue this molecule's rungs for any free CTA
      const int base = atomicAdd(&A.queue[1], J.nrung);
      for (int k = 0; k < J.nrung; ++k) A.rlist[base + k] = J.rung0 + k;
      __threadfence();
      for (int k = 0; k < J.nrung; ++k) atomicExch(&A.rready[base + k], 1);
    }
  }
  __syncthreads();
}

// Workspace pointers of the slot starting at `slot` (layout of slot_doubles).
__device__ __forceinline__ void slot_ptrs(Ctx& c, double* slot, int nmax) {
  const size_t nn = (size_t)nmax * nmax;
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
  c.tri_b = c.tri_a + 4 * nmax;  // per spin: saved tridiagonal (2n), eigenvalues (n), their change (n)
  c.W = c.tri_b + 4 * nmax;
}

// The beta spin of CTA L's unrestricted job (offer generation `mygen`, already taken by this
// CTA), iteration by iteration on L's workspace: F_beta = H + J(P_t) - K(P_beta), its eigensolve
// (warm-started from L's saved beta eigenvalues) and the new P_beta, then the energy part and the
// squared density change for L, which decides convergence. Own shared memory and own scratch
// (packed eigen input, eigenvector scratch, total density) stay with this CTA. Every wait is
// bounded; a wait that runs out raises the launch's error flag.
__device__ __noinline__ void help_job(Ctx& c, int L, int mygen) {
  const KernelArgs& A = *c.A;
  HelpRec* hr = A.help + L;
  volatile HelpRec* vr = hr;
  const int tid = threadIdx.x;
  __shared__ int s_h[2];
  c.tmark = clock64();
  if (tid == 0) {
    int st = 0;
    for (int i = 0; i < (1 << 22) && !st; ++i) {
      const int v = vr->sg;
      if ((v >> 3) != mygen || (v & 7) == 4) st = 4;
      else if ((v & 7) == 3) st = 3;
      else __nanosleep(200);
    }
    if (!st && atomicCAS(&hr->sg, mygen * 8 + 2, mygen * 8 + 4) != mygen * 8 + 2)  // gave up: unless activated
      st = (vr->sg == mygen * 8 + 3) ? 3 : 4;
    __threadfence();
    s_h[0] = st == 3 ? vr->go : -1;
  }
  __syncthreads();
  int iter = s_h[0];
  __syncthreads();
  if (iter < 0) return;
  const JobDesc* tab = vr->kind == 0 ? A.jobs : A.rjobs;
  c.job = tab[vr->idx];
  const JobDesc& J = c.job;
  c.n = J.nao;
  c.N = J.natom;
  const int n = c.n, nb = J.n_beta;
  const size_t nn = (size_t)n * n;
  setup_job(c);
  double* own_vb = c.Vb;
  double* own_vt = c.Vt;
  double* own_ag = c.Ag;
  double* own_tf = c.tf;
  slot_ptrs(c, A.work + (size_t)L * A.slot, A.nmax);  // L's matrices
  c.Vb = own_vb;
  c.Vt = own_vt;
  c.Ag = own_ag;
  c.tf = own_tf;
  double* Pt = own_vb + nn;
  double* eps_b = c.tri_b + 2 * n;
  const int kvb = n < nb + 1 ? n : nb + 1;
  for (;; ++iter) {
    if (tid == 0) {
      int ok = -1;
      for (int i = 0; i < (1 << 22) && ok < 0; ++i) {
        if (vr->go >= iter) ok = 1;
        else {
          const int v = vr->sg;
          if ((v >> 3) != mygen || (v & 7) == 4) ok = 0;
          else __nanosleep(200);
        }
      }
      if (ok < 0) {
        atomicExch(&A.queue[3], 1);
        ok = 0;
      }
      __threadfence();
      s_h[0] = ok;
      s_h[1] = vr->cur;
    }
    __syncthreads();
    const int ok = s_h[0], cur = s_h[1];
    __syncthreads();
    if (!ok) break;
    const double* Pc = c.P[cur];
    double* Qc = c.Q[cur];
    double* Qn = c.Q[1 - cur];
    for (size_t k = tid; k < nn; k += kThreads) Pt[k] = Pc[k] + Qc[k];
    __syncthreads();
    build_fock(c, Pt, Qc, nullptr, c.G, nullptr);
    double part = 0.0;
    for (size_t k = tid; k < nn; k += kThreads) part += Qc[k] * c.G[k];
    part = block_sum(part, c.red);
    mark(c, kPhFock);
    double* Ap = pack_input(c, c.G, Qc, J.shift);
    eigensolve(c, Ap, kvb, nb, c.Vb, eps_b, c.tri_b, iter > 0, c.tri_b + 3 * n);
    const double sq = density(c, c.Vb, nb, 1.0, Qc, Qn, J.damping);
    mark(c, kPhDensity);
    if (tid == 0) {
      hr->part_b[iter & 1] = part;
      hr->sq_b[iter & 1] = sq;
      __threadfence();
      atomicExch(&hr->hdone, iter);
    }
    __syncthreads();
  }
  slot_ptrs(c, A.work + (size_t)blockIdx.x * A.slot, A.nmax);  // back to this CTA's own slot
}

// ----------------------------------------------------------------------- the kernel

__global__ void __launch_bounds__(kThreads, 2) scf_batch_kernel(KernelArgs args) {
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
  const int nm = args.nmax;  // eigen scratch sized for the largest basis of the launch
  c.es.d = ep;
  c.es.e = ep + nm;
  c.es.e2 = ep + 2 * nm;
  c.es.tau = ep + 3 * nm;
  c.es.v = ep + 4 * nm;
  c.es.p = ep + 5 * nm;
  c.es.lam = ep + 6 * nm;
  c.es.red = c.red;
  c.es.misc = c.misc;
  int* eip = reinterpret_cast<int*>(ep + 7 * nm);
  c.es.blk = eip;
  c.es.nblk = eip + nm + 1;
  c.es.vinfo = eip + nm + 2;
  double* up = reinterpret_cast<double*>(smem + L.off_union);
  c.dpk = up;
  c.jacc = up + 10 * amax;
  c.tile = up;
  c.Asm = up;

  slot_ptrs(c, args.work + (size_t)blockIdx.x * args.slot, args.nmax);

  if (args.tjob && threadIdx.x == 0) atomicMin(&args.tjob[args.njobs], globaltimer_ns());
  __shared__ unsigned long long s_ph[kPhases];
  c.ph = s_ph;
  if (threadIdx.x < kPhases) s_ph[threadIdx.x] = 0ULL;
  __syncthreads();
  __shared__ int s_kind, s_hgen;
  int* q = args.queue;
  for (;;) {
    if (threadIdx.x == 0) {
      // Rung jobs first (they are the long ones and only exist once a first pass asked for
      // them), else the next first-pass job. Every wait here is bounded; a handshake that
      // times out raises the error flag instead of hanging.
      int kind = -1, idx = -1, hgen = 0;
      bool first_done = false, waiting = false;
      for (int guard = 0; guard < (1 << 20); ++guard) {
        const int h = atomicAdd(&q[2], 0), t = atomicAdd(&q[1], 0);
        if (h < t) {
          if (atomicCAS(&q[2], h, h + 1) != h) continue;
          bool ok = false;
          for (int spin = 0; spin < (1 << 22); ++spin) {
            if (atomicAdd(&args.rready[h], 0)) {
              ok = true;
              break;
            }
            __nanosleep(64);
          }
          if (ok) {
            kind = 1;
            idx = ((volatile int*)args.rlist)[h];
          } else {
            atomicExch(&q[3], 1);
          }
          break;
        }
        if (!first_done) {
          const int j = atomicAdd(&q[0], 1);
          if (j < args.njobs) {
            kind = 0;
            idx = j;
            break;
          }
          first_done = true;
          continue;
        }
        // No job to take. While first passes are still running they may queue stability rungs
        // (q[4] counts finished first passes); up to max_waiters CTAs stay for them, sleeping
        // between polls, so that late rungs run side by side instead of one after another on the
        // CTA that queued them. The rest exit and free their SM for other work. Bounded by the
        // guard: a CTA that waits too long exits (its rungs still run on the queuing CTA).
        bool offers = false;  // an unrestricted job offering its beta spin: take it
        if (args.help) {
          for (int L = 0; L < (int)gridDim.x && kind < 0; ++L) {
            if (L == (int)blockIdx.x) continue;
            const int v = ((volatile HelpRec*)args.help)[L].sg;
            if ((v & 7) != 1) continue;
            offers = true;
            if (atomicCAS(&args.help[L].sg, v, (v & ~7) | 2) == v) {
              kind = 2;
              idx = L;
              hgen = v >> 3;
            }
          }
          if (kind >= 0) break;
        }
        if (!offers && atomicAdd(&q[4], 0) >= args.njobs) break;
        if (!waiting) {
          if (args.max_waiters <= 0) break;
          if (atomicAdd(&q[5], 1) >= args.max_waiters) {
            atomicSub(&q[5], 1);
            break;
          }
          waiting = true;
        }
        __nanosleep(2000);
      }
      if (waiting) atomicSub(&q[5], 1);
      s_kind = kind;
      s_job = idx;
      s_hgen = hgen;
    }
    __syncthreads();
    const int kind = s_kind, jid = s_job, hg = s_hgen;
    __syncthreads();
    if (kind < 0) break;
    if (kind == 2) {
      help_job(c, jid, hg);
    } else if (kind == 0) {
      run_job(c, args.jobs[jid], args.out + jid, 0, jid);
      if (threadIdx.x == 0) {  // after its rungs (if any) are queued
        __threadfence();
        atomicAdd(&q[4], 1);
        if (args.tjob) args.tjob[jid] = globaltimer_ns();
      }
    } else {
      run_job(c, args.rjobs[jid], args.rout + jid, 1, jid);
    }
  }
  if (args.prof && threadIdx.x < kPhases) atomicAdd(&args.prof[threadIdx.x], s_ph[threadIdx.x]);
}

inline long long slot_doubles(int nmax, long long wcap) {
  const long long nn = (long long)nmax * nmax;
  return 49 * nn + 8LL * nmax + wcap + 64;
}

}  // namespace pm3gpu
