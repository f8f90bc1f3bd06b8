// Persistent batched PM3 SCF: every CTA repeatedly takes the next job (one SCF solve of one
// molecule) from a global work queue and runs the whole calculation for it -- pair
// integrals, H_core, the SCF loop (Fock build, commutator, Pulay CDIIS / A-DIIS, eigensolve,
// density) and the properties of the converged state. Jobs are queued largest first, so the
// tail of the launch is a small molecule.
//
// The per-molecule algorithm is the reference's (pm3-rs src/hamiltonian.rs:191-344,
// src/fock.rs:93-332, src/scf.rs:1039-1693); the stability-search driver that decides
// which jobs to run lives on the host.
#pragma once
#include <cstdint>

#include "cta_blas.cuh"
#include "cta_eigen.cuh"
#include "pm3_integrals.cuh"

namespace pm3gpu {

constexpr int kMaxDepth = 8;  // deepest accelerator history (scf.rs:300)
// Phases of one job, timed with clock64 by thread 0 when profiling is on.
enum Phase : int {
  kPhCore = 0, kPhFock, kPhCommutator, kPhDiisSolve, kPhPack, kPhTridiag, kPhEigval, kPhEigvec, kPhBack,
  kPhDensity, kPhFinal, kPhGradient, kPhases
};

enum JobFlags : int {
  kJobUhf = 1,        // unrestricted iteration
  kJobKeepDens = 2,   // A-DIIS density history
  kJobGrad = 4,       // export the densities the gradient kernel needs (P, and Pa/Pb for UHF)
  kJobDensity = 8,    // export the total density
  kJobEps = 16,       // export all MO energies of the last iteration
  kJobCoreOnly = 32,  // stop after H_core: export H (build_core)
  kJobFockOnly = 64,  // H_core, then F(P) for a given density (build_fock_spin)
};

struct JobDesc {
  int atom0, natom, nao;
  int n_alpha, n_beta;
  int flags;
  int mol;     // molecule index (host bookkeeping)
  int rung0, nrung;  // stability-search jobs of this molecule in the rung table (first pass only)
  int stab;    // 0 no search, 1 search when the frontier gap < 6 eV, 2 always (first pass only)
  int backup;  // rung-table job that repeats this pass from the standard guess if it fails (-1: none)
  int guess;   // 1 SAD, 2 core Hamiltonian, 3 symmetry-broken SAD, 4 given density (learned guess)
  int accel;   // 0 none, 1 CDIIS, 2 A-DIIS -> CDIIS (already combined with use_diis)
  int depth;   // accelerator history length
  int max_scf;
  double e_tol, p_tol, adiis_switch, shift, damping;
  long long charge_off;   // into charges[] (natom values)
  long long dens_off;     // into densities[] (nao^2), when kJobDensity
  long long guess_off;    // into guess_dens[] (nao^2), when guess == 4 (learned initial density)
  long long eps_off;      // into eps[] (2 nao: alpha then beta), when kJobEps
};

struct JobOut {
  int status;        // 0 ok, 4 not converged, 5 linear algebra, 8 unsupported
  int converged, iterations, pad;
  double electronic, core, last_change;
  double homo, lumo;       // frontier over both spins (scf.rs:804-822)
  int has_homo, has_lumo;
  double homo_a, lumo_a;   // alpha-only frontier (a spin-pure UHF rung collapsed to RHF)
  int has_homo_a, has_lumo_a;
  double gap;              // frontier gap used by the stability trigger (scf.rs:106-124)
  double spin_max;         // max |P_alpha - P_beta| (unrestricted jobs)
  double dipole[3];        // Debye
};

// Byte offsets of the dynamic shared-memory carve-up (computed on the host).
struct SmemLayout {
  int amax;      // atoms per molecule this launch supports
  int nsm;       // largest n whose packed matrix lives in shared memory
  int off_int, off_dbl, off_eig, off_union;
  int bytes;
};

struct KernelArgs {
  const ElemDev* elem;
  const PairDev* pairs;
  const int* z;          // [total atoms]
  const double* xyz;     // [3 * total atoms], Bohr
  const JobDesc* jobs;   // first-pass jobs, largest first
  int njobs;
  JobOut* out;
  const JobDesc* rjobs;  // stability-search rung table (all candidates)
  int nrjobs;
  JobOut* rout;          // status stays -1 for rungs that were never enqueued
  int* rlist;            // [nrjobs] rung queue entries (rung table indices)
  int* rready;           // [nrjobs] 1 once rlist[i] is published
  double* charges;
  double* densities;
  const double* guess_dens;  // initial densities of guess-4 jobs
  double* grads;
  double* eps;
  double* work;          // per-CTA slots
  long long slot;        // doubles per slot
  int nmax;              // largest nao of the launch (slot dimension)
  long long wcap;        // doubles reserved for the pair table
  int* queue;            // [0] next first-pass job, [1] rung queue tail, [2] rung queue head, [3] error,
                         // [4] finished first passes, [5] CTAs waiting for late work, [6] jobs paired
  unsigned long long* prof;  // [kPhases] SM cycles per phase, summed over CTAs (null = off)
  SmemLayout sm;
  struct HelpRec* help;  // [grid] per CTA: its unrestricted job's offer of the beta spin (null = off)
  unsigned long long* tjob;  // [njobs + 1] global-timer ns when each first pass ended, [njobs] the start (null = off)
  int max_waiters;       // CTAs that may stay, once the first passes are all taken, for work still to come
};

// One CTA's offer of the beta spin of its unrestricted job to an idle CTA (a "helper"). `sg`
// packs a generation (bits 3..) and a state (bits 0-2): 0 idle, 1 open, 2 taken by a helper,
// 3 active (the two CTAs run the iterations from `go` on together), 4 stop. Each new offer takes a
// new generation, so a helper of an older offer never acts on a newer one.
struct HelpRec {
  int sg;
  int kind, idx;   // the job: 0 first-pass table, 1 rung table
  int go;          // iteration the helper may run next (the leader published its densities for it)
  int cur;         // current density buffer of iteration `go`
  int hdone;       // last iteration the helper has finished
  int pad[2];
  double part_b[2], sq_b[2];  // helper's energy part sum P_beta F_beta and squared density change, by iteration parity
};

// ---------------------------------------------------------------------------- helpers
__device__ __forceinline__ double oc_integral(const ElemDev& e, int a, int b, int c, int d) {
  // One-centre (ab|cd) from Gss..Hsp (fock.rs:244-282).
  if (a == b && c == d) {
    if (a == 0 && c == 0) return e.gss;
    if (a == 0 || c == 0) return e.gsp;
    return a == c ? e.gpp : e.gp2;
  }
  const int ba = min(a, b), bb = max(a, b), kc = min(c, d), kd = max(c, d);
  if (ba == 0 && bb != 0 && kc == 0 && kd != 0 && bb == kd) return e.hsp;
  if (ba != 0 && bb != 0 && ba != bb && ba == kc && bb == kd) return 0.5 * (e.gpp - e.gp2);
  return 0.0;
}

// Per-job context: shared-memory views and global buffers of this CTA's slot.
struct Ctx {
  const KernelArgs* A;
  JobDesc job;
  JobOut* out;
  int n, N;             // AOs, atoms
  // shared
  int* sz;              // [amax] Z of each atom
  int* soff;            // [amax] first AO
  int* sprow;           // [amax+1] prefix of packed sizes
  long long* sroff;     // [amax] pair-table row offsets
  double* sxyz;         // [3 amax]
  double* red;          // reduction scratch
  double* misc;         // broadcast scalars
  double* bg;           // [8*8] <E_i,E_j>
  double* mg;           // [8*8] <D_i,F_j>
  double* coef;         // [kMaxDepth+1]
  int* iv;              // small ints
  double* dpk;          // [amax*10] packed densities (Fock phase)
  double* jacc;         // [amax*10] Coulomb accumulators (Fock phase)
  double* tile;         // GEMM tiles
  double* Asm;          // packed matrix (eigen phase)
  EigenScratch es;
  unsigned long long* ph;  // [kPhases] shared accumulators
  long long tmark;
  // global (slot)
  double *H, *P[2], *Q[2], *F, *G, *Vt, *Vb, *Ag, *tf, *hist, *W, *tri_a, *tri_b;
  int cur;              // which P/Q buffer is current
};

__device__ __forceinline__ void mark(Ctx& c, int phase) {
  if (c.A->prof && threadIdx.x == 0) {
    const long long now = clock64();
    c.ph[phase] += (unsigned long long)(now - c.tmark);
    c.tmark = now;
  }
}

__device__ __forceinline__ bool heavy(const Ctx& c, int a) { return c.A->elem[c.sz[a]].norb == 4; }
__device__ __forceinline__ int psize(const Ctx& c, int a) { return heavy(c, a) ? 10 : 1; }
__device__ __forceinline__ long long woff(const Ctx& c, int u, int v) {
  return c.sroff[u] + (long long)psize(c, u) * (c.sprow[v] - c.sprow[u + 1]);
}
// pair index t -> (u < v)
__device__ __forceinline__ void pair_uv(int N, int t, int& u, int& v) {
  const double b = 2.0 * N - 1.0;
  int uu = (int)floor((b - sqrt(b * b - 8.0 * t)) * 0.5);
  if (uu < 0) uu = 0;
  while (uu > 0 && uu * (2 * N - uu - 1) / 2 > t) --uu;
  while ((uu + 1) * (2 * N - uu - 2) / 2 <= t) ++uu;
  u = uu;
  v = t - uu * (2 * N - uu - 1) / 2 + uu + 1;
}

// ------------------------------------------------------------------ job setup + H_core
__device__ void setup_job(Ctx& c) {
  const KernelArgs& A = *c.A;
  const int tid = threadIdx.x;
  for (int a = tid; a < c.N; a += kThreads) {
    c.sz[a] = A.z[c.job.atom0 + a];
    for (int k = 0; k < 3; ++k) c.sxyz[3 * a + k] = A.xyz[3 * (size_t)(c.job.atom0 + a) + k];
  }
  __syncthreads();
  if (tid == 0) {
    int off = 0, pr = 0;
    for (int a = 0; a < c.N; ++a) {
      c.soff[a] = off;
      off += A.elem[c.sz[a]].norb;
      c.sprow[a] = pr;
      pr += psize(c, a);
    }
    c.sprow[c.N] = pr;
    long long ro = 0;
    for (int a = 0; a < c.N; ++a) {
      c.sroff[a] = ro;
      ro += (long long)psize(c, a) * (pr - c.sprow[a + 1]);
    }
  }
  __syncthreads();
}

// One atom pair of H_core (hamiltonian.rs:191-344): both atoms' electron-core attraction blocks
// (added to their packed diagonal accumulators), the pair table block W in (a, b) orientation (a
// the atom with more orbitals), and the resonance block H_ab = (beta_i + beta_j)/2 S_ij written to
// both triangles of H (row stride n). Returns the pair's core-core energy (repulsion.rs:57-120),
// evaluated with the atoms in the caller's (u, v) order.
__device__ __forceinline__ double core_pair(const ElemDev& ea, const ElemDev& eb, const ElemDev& eu, const ElemDev& ev,
                                            const PairDev& pp, const double* xa, const double* xb, int oa, int ob,
                                            size_t n, double* hacc_a, double* hacc_b, double* w, double* H) {
  const double d[3] = {xb[0] - xa[0], xb[1] - xa[1], xb[2] - xa[2]};
  const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const double dv[3] = {d[0] / r * r, d[1] / r * r, d[2] / r * r};
  const double mdv[3] = {-dv[0], -dv[1], -dv[2]};
  if (hacc_a) {  // null: the caller adds the electron-core blocks per atom itself
    double blk[10];
    core_attraction(ea, eb, dv, blk);
    for (int k = 0; k < (ea.norb == 4 ? 10 : 1); ++k) atomicAdd(&hacc_a[k], blk[k]);
    core_attraction(eb, ea, mdv, blk);
    for (int k = 0; k < (eb.norb == 4 ? 10 : 1); ++k) atomicAdd(&hacc_b[k], blk[k]);
  }
  const double ir = 1.0 / r;
  double R[9];
  frame(-(dv[0] * ir), -(dv[1] * ir), -(dv[2] * ir), R);
  const double rv = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
  if (ea.norb == 1) {
    const double s = ea.rho0 + eb.rho0;
    w[0] = rsq(rv * rv + s * s) * kEv;
  } else if (eb.norb == 1) {
    double ri[4];
    local4(ee_pole(ea), eb.rho0, rv, ri);
    for (int kk = 0; kk < 4; ++kk)
      for (int ll = 0; ll <= kk; ++ll) w[pk(kk, ll)] = w4(ri, R, kk, ll);
  } else {
    double ri[22];
    local22(ee_pole(ea), ee_pole(eb), rv, ri);
    for (int kk = 0; kk < 4; ++kk)
      for (int ll = 0; ll <= kk; ++ll)
        for (int mm = 0; mm < 4; ++mm)
          for (int nn = 0; nn <= mm; ++nn) w[pk(kk, ll) * 10 + pk(mm, nn)] = w22(ri, R, kk, ll, mm, nn);
  }
  double s[16];
  overlap_block(ea, eb, d, s);
  for (int i = 0; i < ea.norb; ++i) {
    const double bi = i == 0 ? ea.bs : ea.bp;
    for (int j = 0; j < eb.norb; ++j) {
      const double bj = j == 0 ? eb.bs : eb.bp;
      const double h = 0.5 * (bi + bj) * s[i * 4 + j];
      H[(size_t)(oa + i) * n + ob + j] = h;
      H[(size_t)(ob + j) * n + oa + i] = h;
    }
  }
  const double dd = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  return core_core(eu, ev, pp, dd);
}

// H_core (hamiltonian.rs:191-344) and the pair table W; returns the core-core energy
// (repulsion.rs:13-27) to every thread.
__device__ double build_core(Ctx& c) {
  const KernelArgs& A = *c.A;
  const int n = c.n, N = c.N, tid = threadIdx.x;
  double* hacc = c.jacc;  // [N*10] diagonal-block accumulators
  for (int k = tid; k < N * 10; k += kThreads) hacc[k] = 0.0;
  __syncthreads();
  double ecc = 0.0;
  const int npairs = N * (N - 1) / 2;
  for (int t = tid; t < npairs; t += kThreads) {
    int u, v;
    pair_uv(N, t, u, v);
    const bool hu = heavy(c, u), hv = heavy(c, v);
    const int a = (hu || !hv) ? u : v, b = a == u ? v : u;
    ecc += core_pair(A.elem[c.sz[a]], A.elem[c.sz[b]], A.elem[c.sz[u]], A.elem[c.sz[v]], *A.pairs, c.sxyz + 3 * a,
                     c.sxyz + 3 * b, c.soff[a], c.soff[b], (size_t)n, hacc + a * 10, hacc + b * 10, c.W + woff(c, u, v),
                     c.H);
  }
  __syncthreads();
  // diagonal blocks: U + sum of electron-core attractions
  for (int k = tid; k < N * 16; k += kThreads) {
    const int a = k >> 4, mu = (k >> 2) & 3, nu = k & 3;
    const ElemDev& e = A.elem[c.sz[a]];
    if (mu >= e.norb || nu >= e.norb) continue;
    double h = hacc[a * 10 + pk(mu, nu)];
    if (mu == nu) h += mu == 0 ? e.uss : e.upp;
    c.H[(size_t)(c.soff[a] + mu) * n + c.soff[a] + nu] = h;
  }
  __syncthreads();
  return block_sum(ecc, c.red);
}

// ------------------------------------------------------------------------ Fock build
// Two-centre part of one atom pair (fock.rs:106-193): Coulomb sums into the atoms' packed
// accumulators and the exchange block F_ab = H_ab - K_ab, written to both triangles. NA / NB are
// the orbital counts of atom a (the heavier one) and b, so every loop has a fixed trip count and
// every array stays in registers. W is the pair's (PA x PB) row-major integral block.
// kJ = false leaves out the two-centre Coulomb sums into jacc (the whole-GPU path adds them per
// atom in a fixed order instead of with atomics).
// SPIN = true builds one spin's Fock matrix of an unrestricted job, F = H + J(Pt) - K(Pa) (the
// first spin of the UHF form alone), for a job whose two spins run on two CTAs.
template <int NA, int NB, bool UHF, bool kJ = true, bool SPIN = false>
__device__ __forceinline__ void fock_pair(int n, int a, int b, int oa, int ob, const double* __restrict__ dpk,
                                          double* jacc, const double* __restrict__ H, const double* __restrict__ w,
                                          const double* Pt, const double* Pa, const double* Pb, double* F, double* G) {
  constexpr int PA = NA == 4 ? 10 : 1, PB = NB == 4 ? 10 : 1;
  if (kJ) {  // Coulomb: J_a[p] += sum_q W[p][q] Pb_q, J_b[q] += sum_p Pa_p W[p][q]
    double db[PB], jb[PB];
#pragma unroll
    for (int q = 0; q < PB; ++q) {
      db[q] = dpk[b * 10 + q];
      jb[q] = 0.0;
    }
#pragma unroll
    for (int p = 0; p < PA; ++p) {
      const double da = dpk[a * 10 + p];
      double acc = 0.0;
#pragma unroll
      for (int q = 0; q < PB; ++q) {
        const double wv = w[p * PB + q];
        acc = fma(db[q], wv, acc);
        jb[q] = fma(da, wv, jb[q]);
      }
      atomicAdd(&jacc[a * 10 + p], acc);
    }
#pragma unroll
    for (int q = 0; q < PB; ++q) atomicAdd(&jacc[b * 10 + q], jb[q]);
  }
  // exchange: K[mu][la] = sum_{nu, si} X[nu][si] (mu nu | la si), one spin at a time
#pragma unroll
  for (int spin = 0; spin < (UHF ? 2 : 1); ++spin) {
    const double* X = (UHF || SPIN) ? (spin == 0 ? Pa : Pb) : Pt;
    const double xs = (UHF || SPIN) ? 1.0 : 0.5;
    double* out = spin == 0 ? F : G;
    double x[NA * NB];
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int j = 0; j < NB; ++j) x[i * NB + j] = xs * X[(size_t)(oa + i) * n + ob + j];
#pragma unroll
    for (int mu = 0; mu < NA; ++mu)
#pragma unroll
      for (int la = 0; la < NB; ++la) {
        double k = 0.0;
#pragma unroll
        for (int nu = 0; nu < NA; ++nu)
#pragma unroll
          for (int si = 0; si < NB; ++si) k = fma(x[nu * NB + si], w[pk(mu, nu) * PB + pk(la, si)], k);
        const double f = H[(size_t)(oa + mu) * n + ob + la] - k;
        out[(size_t)(oa + mu) * n + ob + la] = f;
        out[(size_t)(ob + la) * n + oa + mu] = f;
      }
  }
}

// F = H + J(Pt) - K(Ps) (fock.rs:285-332). Pt = total density; for RHF Ps = Pt/2 (pb == null),
// for UHF two spin Focks F (from Pa) and G (from Pb) are built in one pass.
// With Pa given and Pb null, one spin of an unrestricted job: F = H + J(Pt) - K(Pa) (G unused).
__device__ void build_fock(Ctx& c, const double* Pt, const double* Pa, const double* Pb, double* F, double* G) {
  const KernelArgs& A = *c.A;
  const int n = c.n, N = c.N, tid = threadIdx.x;
  const bool uhf = Pb != nullptr;
  const bool spin1 = !uhf && Pa != nullptr;
  // stage packed atomic densities (fock.rs:93-100) and zero the Coulomb accumulators
  for (int k = tid; k < N * 10; k += kThreads) {
    const int a = k / 10, p = k % 10;
    const int no = A.elem[c.sz[a]].norb;
    c.jacc[k] = 0.0;
    double v = 0.0;
    if (no == 4 || p == 0) {
      int hi, lo;
      unpk(p, hi, lo);
      const int oa = c.soff[a];
      v = Pt[(size_t)(oa + hi) * n + oa + lo];
      if (hi != lo) v *= 2.0;
    }
    c.dpk[k] = v;
  }
  __syncthreads();
  const int npairs = N * (N - 1) / 2;
  {
    const int* __restrict__ sprow = c.sprow;
    const int* __restrict__ soff = c.soff;
    const long long* __restrict__ sroff = c.sroff;
    const double* __restrict__ W = c.W;
    const double* __restrict__ H = c.H;
    const double* __restrict__ dpk = c.dpk;
    double* jacc = c.jacc;
    for (int t = tid; t < npairs; t += kThreads) {
      int u, v;
      pair_uv(N, t, u, v);
      const int su = sprow[u + 1] - sprow[u], sv = sprow[v + 1] - sprow[v];  // packed sizes: 10 sp, 1 s
      const bool hu = su == 10, hv = sv == 10;
      const int a = (hu || !hv) ? u : v, b = a == u ? v : u;
      const double* w = W + sroff[u] + (long long)su * (sprow[v] - sprow[u + 1]);
      const int oa = soff[a], ob = soff[b];
      if (hu && hv) {
        if (uhf) fock_pair<4, 4, true>(n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
        else if (spin1) fock_pair<4, 4, false, true, true>(n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
        else fock_pair<4, 4, false>(n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
      } else if (hu || hv) {
        if (uhf) fock_pair<4, 1, true>(n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
        else if (spin1) fock_pair<4, 1, false, true, true>(n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
        else fock_pair<4, 1, false>(n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
      } else {
        if (uhf) fock_pair<1, 1, true>(n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
        else if (spin1) fock_pair<1, 1, false, true, true>(n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
        else fock_pair<1, 1, false>(n, a, b, oa, ob, dpk, jacc, H, w, Pt, Pa, Pb, F, G);
      }
    }
  }
  __syncthreads();
  // atom-diagonal blocks: H + one-centre J - K + two-centre J
  for (int k = tid; k < N * 16; k += kThreads) {
    const int a = k >> 4, mu = (k >> 2) & 3, nu = k & 3;
    const ElemDev& e = A.elem[c.sz[a]];
    const int no = e.norb;
    if (mu >= no || nu >= no) continue;
    const int oa = c.soff[a];
    double ja = 0.0, ka = 0.0, kb = 0.0;
    for (int la = 0; la < no; ++la)
      for (int si = 0; si < no; ++si) {
        const double coul = oc_integral(e, mu, nu, la, si), exch = oc_integral(e, mu, la, nu, si);
        const size_t ix = (size_t)(oa + la) * n + oa + si;
        ja = fma(Pt[ix], coul, ja);
        if (uhf) {
          ka = fma(Pa[ix], exch, ka);
          kb = fma(Pb[ix], exch, kb);
        } else if (spin1) {
          ka = fma(Pa[ix], exch, ka);
        } else {
          ka = fma(0.5 * Pt[ix], exch, ka);
        }
      }
    const size_t ix = (size_t)(oa + mu) * n + oa + nu;
    const double base = c.H[ix] + c.jacc[a * 10 + pk(mu, nu)] + ja;
    F[ix] = base - ka;
    if (uhf) G[ix] = base - kb;
  }
  __syncthreads();
}

// sum_ij X_ij Y_ij over n x n
__device__ __forceinline__ double fdot(const Ctx& c, const double* X, const double* Y) {
  double s = 0.0;
  const size_t nn = (size_t)c.n * c.n;
  for (size_t k = threadIdx.x; k < nn; k += kThreads) s = fma(X[k], Y[k], s);
  return block_sum(s, c.red);
}

// E = F P - P F into E (scf.rs:1039-1054): one GEMM, then antisymmetrise in place.
__device__ void commutator(Ctx& c, const double* Fm, const double* Pm, double* E) {
  const int n = c.n;
  cta_gemm<false, false>(n, n, n, 1.0, Fm, n, Pm, n, c.tile, false,
                         [&](int i, int j, double v) { E[(size_t)i * n + j] = v; });
  for (int k = threadIdx.x; k < n * n; k += kThreads) {
    const int i = k / n, j = k % n;
    if (j < i) {
      const double lo = E[(size_t)i * n + j], up = E[(size_t)j * n + i];
      E[(size_t)i * n + j] = lo - up;
      E[(size_t)j * n + i] = up - lo;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += kThreads) E[(size_t)i * n + i] = 0.0;
  __syncthreads();
}

// ------------------------------------------------------------ small dense solves (thread 0)
// Pulay coefficients from the Gram matrix (scf.rs:1544-1630); false = singular / unusable.
__host__ __device__ bool cdiis_coeffs(int m, const double* gram, double* x) {
  if (m < 2) return false;
  double scale = 0.0;
  for (int i = 0; i < m * m; ++i) scale = fmax(scale, fabs(gram[(i / m) * kMaxDepth + i % m]));
  if (!(scale > 0.0) || !isfinite(scale)) return false;
  const int dim = m + 1;
  double B[(kMaxDepth + 1) * (kMaxDepth + 1)], rhs[kMaxDepth + 1];
  for (int i = 0; i < dim; ++i) {
    rhs[i] = 0.0;
    for (int j = 0; j < dim; ++j) B[i * dim + j] = 0.0;
  }
  for (int i = 0; i < m; ++i) {
    for (int j = 0; j < m; ++j) B[i * dim + j] = gram[i * kMaxDepth + j] / scale;
    B[i * dim + m] = -1.0;
    B[m * dim + i] = -1.0;
  }
  rhs[m] = -1.0;
  for (int col = 0; col < dim; ++col) {
    int piv = col;
    double best = fabs(B[col * dim + col]);
    for (int r = col + 1; r < dim; ++r)
      if (fabs(B[r * dim + col]) > best) {
        best = fabs(B[r * dim + col]);
        piv = r;
      }
    if (best < 1.0e-12) return false;
    if (piv != col) {
      for (int j = 0; j < dim; ++j) {
        const double t = B[col * dim + j];
        B[col * dim + j] = B[piv * dim + j];
        B[piv * dim + j] = t;
      }
      const double t = rhs[col];
      rhs[col] = rhs[piv];
      rhs[piv] = t;
    }
    for (int r = col + 1; r < dim; ++r) {
      const double f = B[r * dim + col] / B[col * dim + col];
      if (f == 0.0) continue;
      for (int j = col; j < dim; ++j) B[r * dim + j] -= f * B[col * dim + j];
      rhs[r] -= f * rhs[col];
    }
  }
  for (int col = dim - 1; col >= 0; --col) {
    double sum = rhs[col];
    for (int j = col + 1; j < dim; ++j) sum -= B[col * dim + j] * x[j];
    x[col] = sum / B[col * dim + col];
  }
  return true;
}

// A-DIIS weights on the simplex by projected gradient (scf.rs:1152-1172, 1637-1693), one warp:
// lane k owns weight c_k and its gradient component; the Euclidean projection onto the simplex
// sorts the trial point (descending, ties by index, as a stable insertion sort does) and every
// lane runs the reference's serial cumulative-sum scan over the sorted values, so the weights are
// the ones the serial loop produces. `sm` is shared scratch of kMaxDepth * (2 kMaxDepth + 1) doubles.
__device__ void adiis_coeffs_warp(int m, const double* mg, double* out, double* sm) {
  constexpr int K = kMaxDepth;
  const int k = threadIdx.x & 31;
  const int last = m - 1;
  const double mnn = mg[last * K + last];
  double* S = sm;           // [K][K]
  double* T = sm + K * K;   // [K][K] S + S^T, the gradient's matrix (same sums as the reference's)
  double* d = T + K * K;    // [K]
  if (k < m) {
    d[k] = mg[k * K + last] - mnn;
    for (int j = 0; j < m; ++j) S[k * K + j] = mg[k * K + j] - mg[k * K + last] - mg[last * K + j] + mnn;
  }
  __syncwarp();
  if (k < m)
    for (int j = 0; j < m; ++j) T[k * K + j] = S[k * K + j] + S[j * K + k];
  __syncwarp();
  double L = 1.0e-12;
  for (int i = 0; i < m; ++i) {
    double row = 0.0;
    for (int j = 0; j < m; ++j) row += fabs(T[i * K + j]);
    L = fmax(L, row);
  }
  const double lr = 1.0 / L;
  // Every lane runs the whole iteration on the full state in registers (the lanes agree), so the
  // loop needs no shuffles: gradient, trial point, its stable descending order, the reference's
  // cumulative-sum scan for the simplex projection, and the change.
  double c[K];
#pragma unroll
  for (int j = 0; j < K; ++j) c[j] = j == last ? 1.0 : 0.0;
  for (int it = 0; it < 400; ++it) {
    double t[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
      double g = 2.0 * d[q < m ? q : 0];
#pragma unroll
      for (int j = 0; j < K; ++j)
        if (j < m) g += T[q * K + j] * c[j];
      t[q] = q < m ? c[q] - lr * g : 0.0;
    }
    // the trial point sorted descending by a 19-comparator network on a copy (unused entries
    // -inf, so they sort last); ties give equal values in either order, so the cumulative sums,
    // and with them the projection, are those of the reference's stable sort
    double u[K];
#pragma unroll
    for (int q = 0; q < K; ++q) u[q] = q < m ? t[q] : -INFINITY;
    constexpr int kNet[19][2] = {{0, 2}, {1, 3}, {4, 6}, {5, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}, {0, 1}, {2, 3},
                                 {4, 5}, {6, 7}, {2, 4}, {3, 5}, {1, 4}, {3, 6}, {1, 2}, {3, 4}, {5, 6}};
#pragma unroll
    for (int e = 0; e < 19; ++e) {
      const double a = u[kNet[e][0]], b = u[kNet[e][1]];
      u[kNet[e][0]] = fmax(a, b);
      u[kNet[e][1]] = fmin(a, b);
    }
    double css = 0.0, theta = 0.0;
#pragma unroll
    for (int p = 0; p < K; ++p) {
      if (p >= m) break;
      css += u[p];
      const double tt = (css - 1.0) / (double)(p + 1);
      if (u[p] - tt > 0.0) theta = tt;
    }
    double delta = 0.0;
#pragma unroll
    for (int q = 0; q < K; ++q) {
      if (q >= m) break;
      const double pq = fmax(t[q] - theta, 0.0);
      delta += fabs(pq - c[q]);
      c[q] = pq;
    }
    if (delta < 1.0e-12) break;
  }
  if (k < m) {
#pragma unroll
    for (int q = 0; q < K; ++q)
      if (q == k) out[k] = c[q];
  }
  __syncwarp();
}

// ------------------------------------------------------------------- eigensolve + density
// Pack sym(X) [+ shift (I - Pproj)] into the eigen input (shared or global).
__device__ double* pack_input(Ctx& c, const double* X, const double* Pproj, double shift) {
  const int n = c.n;
  double* Ap = n <= c.A->sm.nsm ? c.Asm : c.Ag;
  // rows to warps, columns to lanes (coalesced reads)
  for (int r = threadIdx.x >> 5; r < n; r += kWarps)
    for (int col = threadIdx.x & 31; col <= r; col += 32) {
      double v = X[(size_t)r * n + col];
      if (shift != 0.0) v += shift * ((r == col ? 1.0 : 0.0) - Pproj[(size_t)r * n + col]);
      Ap[tri(r) + col] = v;
    }
  __syncthreads();
  return Ap;
}

// Diagonalise the packed matrix: kval lowest eigenvalues into lam_out, kvec eigenvectors
// into Y (rows). The tridiagonal (d, e) is saved to `tri_save` (2n) for the final MO energies.
// With `warm`, lam_out holds the same eigenvalues from the previous SCF iteration and `dlam`
// their last change; both seed the eigenvalue search and are updated. Without it dlam is reset.
__device__ void eigensolve(Ctx& c, double* Ap, int kval, int kvec, double* Y, double* lam_out, double* tri_save,
                           bool warm = false, double* dlam = nullptr) {
  const int n = c.n;
  mark(c, kPhPack);
  tridiagonalize(n, Ap, c.es);
  if (tri_save && threadIdx.x == 0)
    for (int i = 0; i < n; ++i) {
      tri_save[i] = c.es.d[i];
      tri_save[n + i] = c.es.e[i];
    }
  mark(c, kPhTridiag);
  const bool seeded = warm && dlam != nullptr;
  tridiag_eigenvalues(n, kval, c.es, seeded ? lam_out : nullptr, seeded ? dlam : nullptr);
  for (int j = threadIdx.x; j < kval; j += kThreads) {
    if (dlam) dlam[j] = seeded ? c.es.lam[j] - lam_out[j] : 1.0e30;
    lam_out[j] = c.es.lam[j];
  }
  mark(c, kPhEigval);
  if (kvec > 0) {
    tridiag_vectors(n, kvec, Y, c.tf, c.es);
    mark(c, kPhEigvec);
    back_transform(n, kvec, Ap, Y, c.es);
  }
  __syncthreads();
  mark(c, kPhBack);
}

// Pnew = w Y^T Y (first k rows of Y); returns sum (Pnew - Pold)^2 to all threads. With
// damping lam > 0 the stored value is (1-lam) Pnew + lam Pold (scf.rs:1440-1448); the RMS
// uses the undamped Pnew, as the reference does.
__device__ double density(Ctx& c, const double* Y, int k, double w, const double* Pold, double* Pnew, double damp) {
  const int n = c.n;
  double sq = 0.0;
  if (k == 0) {
    for (int q = threadIdx.x; q < n * n; q += kThreads) {
      const double o = Pold[q];
      sq += o * o;
      Pnew[q] = damp > 0.0 ? damp * o : 0.0;
    }
    __syncthreads();
    return block_sum(sq, c.red);
  }
  cta_gemm<true, false>(n, n, k, w, Y, n, Y, n, c.tile, true, [&](int i, int j, double v) {
    if (i < j) return;
    const size_t ij = (size_t)i * n + j, ji = (size_t)j * n + i;
    const double o = Pold[ij];
    const double dlt = v - o;
    sq += (i == j ? 1.0 : 2.0) * dlt * dlt;
    const double st = damp > 0.0 ? (1.0 - damp) * v + damp * o : v;
    Pnew[ij] = st;
    Pnew[ji] = st;
  });
  return block_sum(sq, c.red);
}

// --------------------------------------------------------------------------- guesses
__device__ void sad_guess(Ctx& c, double* P, double scale, bool tilt) {
  const KernelArgs& A = *c.A;
  const int n = c.n;
  for (size_t k = threadIdx.x; k < (size_t)n * n; k += kThreads) P[k] = 0.0;
  __syncthreads();
  for (int a = threadIdx.x; a < c.N; a += kThreads) {
    const ElemDev& e = A.elem[c.sz[a]];
    const int o = c.soff[a];
    P[(size_t)o * n + o] = e.occ_s * scale;
    if (e.norb == 4)
      for (int k = 1; k < 4; ++k) P[(size_t)(o + k) * n + o + k] = (e.occ_p / 3.0) * scale;
  }
  __syncthreads();
  if (tilt && threadIdx.x == 0) {  // scf.rs:894-916: move 0.2 e from pz to px on the most p-rich atom
    int target = -1;
    double best = 0.0;
    for (int a = 0; a < c.N; ++a) {
      const ElemDev& e = A.elem[c.sz[a]];
      if (e.norb == 4 && e.occ_p > best) {
        best = e.occ_p;
        target = a;
      }
    }
    if (target >= 0) {
      const int o = c.soff[target];
      // the unscaled SAD entries are tilted, then the spin split scales them (scf.rs:951-977)
      const double pz = A.elem[c.sz[target]].occ_p / 3.0;
      const double t = fmin(0.2, pz);
      P[(size_t)(o + 3) * n + o + 3] = (pz - t) * scale;
      P[(size_t)(o + 1) * n + o + 1] = (pz + t) * scale;
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------------------- properties
__device__ void properties(Ctx& c, const double* Pt, JobOut& o) {
  const KernelArgs& A = *c.A;
  const int n = c.n;
  double* q = A.charges + c.job.charge_off;
  for (int a = threadIdx.x; a < c.N; a += kThreads) {
    const ElemDev& e = A.elem[c.sz[a]];
    double pop = 0.0;
    for (int k = 0; k < e.norb; ++k) pop += Pt[(size_t)(c.soff[a] + k) * n + c.soff[a] + k];
    q[a] = e.core - pop;
  }
  // dipole about the centre of mass (dipole.rs:64-144)
  double v[4] = {0, 0, 0, 0};
  for (int a = threadIdx.x; a < c.N; a += kThreads) {
    const double m = A.elem[c.sz[a]].mass;
    v[0] += m;
    for (int k = 0; k < 3; ++k) v[1 + k] += m * c.sxyz[3 * a + k];
  }
  block_sums<4>(v, c.red, c.misc);
  const double mt = c.misc[0];
  double com[3];
  for (int k = 0; k < 3; ++k) com[k] = mt > 0.0 ? c.misc[1 + k] / mt : 0.0;
  double mu[3] = {0, 0, 0};
  for (int a = threadIdx.x; a < c.N; a += kThreads) {
    const ElemDev& e = A.elem[c.sz[a]];
    const int o = c.soff[a];
    double pop = 0.0;
    for (int k = 0; k < e.norb; ++k) pop += Pt[(size_t)(o + k) * n + o + k];
    for (int ax = 0; ax < 3; ++ax) {
      const double disp = c.sxyz[3 * a + ax] - com[ax];
      double el = pop * disp;
      if (e.norb == 4) el += 2.0 * Pt[(size_t)o * n + o + ax + 1] * e.dd;
      mu[ax] += disp * e.core - el;
    }
  }
  block_sums<3>(mu, c.red, c.misc);
  for (int ax = 0; ax < 3; ++ax) o.dipole[ax] = c.misc[ax] * kAuDipoleToDebye;
}

}  // namespace pm3gpu
