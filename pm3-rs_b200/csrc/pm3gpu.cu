// Host side of the pm3gpu C ABI: context, job planning, launches and the stability-search
// driver of run_pm3 (pm3-rs src/scf.rs:450-848).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/pm3gpu.h"
#include "dgemm.cuh"
#include "gradient_kernel.cuh"
#include "large_scf.cuh"
#include "panel_coop.cuh"
#include "guess_mlp.cuh"
#include "scf_job.cuh"
#include "tc_gemm.cuh"

using namespace pm3gpu;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t b) {
    if (b <= bytes && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, b < 256 ? 256 : b);
    if (e == cudaSuccess) bytes = b < 256 ? 256 : b;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

constexpr int kMaxDiisDepthHost = 8;
// Basis size from which a call's only molecule goes to the whole-GPU path by default.
constexpr int kSingleWholeNao = 192;
constexpr int kMaxLargeAtoms = 30000;  // pair indices of the whole-GPU kernels stay in 32 bits
// scf.rs:309-331
int diis_depth(int nao, int mats, int budget_mb) {
  if (budget_mb == 0) return kMaxDiisDepthHost;
  const size_t per = (size_t)mats * nao * nao * 8;
  if (per == 0) return kMaxDiisDepthHost;
  const size_t budget = (size_t)budget_mb * 1024 * 1024;
  return (int)std::min<size_t>(std::max<size_t>(budget / per, 2), kMaxDiisDepthHost);
}
bool diis_depth_fits(int nao, int mats, int budget_mb) {
  return budget_mb == 0 || 2 * (size_t)mats * nao * nao * 8 <= (size_t)budget_mb * 1024 * 1024;
}

struct Rung {
  int guess, accel;
  double shift, damp;
  bool unrestricted;
};

struct LargeBufs;

struct MolPlan {
  bool large = false;  // solved on the whole-GPU path
  int status = 0;
  std::string msg;
  int natom = 0, nao = 0, atom0 = 0;
  int n_alpha = 0, n_beta = 0;
  bool use_uhf = false, steered = false;
  const pm3gpu_options* o = nullptr;
  int first_job = -1;
  std::vector<int> rung_jobs;
  std::vector<Rung> rungs;
};

}  // namespace

// Clears the cached address of the allocation-free path's scratch array on `device`.
void noalloc_forget(int device);

struct pm3gpu_ctx {
  int device = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  std::mutex mu;
  std::string err;
  ElemDev h_elem[kMaxZ];
  PairDev h_pairs;
  DevBuf elem, pairs, z, xyz, jobs, out, charges, dens, grads, eps, work, queue, rq, gmols, aooff, help;
  bool tail_helpers = false;  // idle CTAs take the beta spin of unaccelerated unrestricted jobs
  int tune_goal = 0;           // autotuner: 0 batch time, 1 throughput with batches in flight
  bool record_jobs = false;    // time each first pass's end (the autotuner's throughput goal)
  DevBuf tjob;
  std::vector<unsigned long long> job_ns;  // last launch: first-pass end times, then the start
  int paired = 0;              // jobs of the last call that ran on two CTAs
  int sms = 0, smem_optin = 0, smem_per_sm = 0;
  double timings[7] = {0, 0, 0, 0, 0, 0, 0};
  int launches = 0;
  int last_ctas = 0, last_nsm = 0;  // last batched launch: CTAs per SM, largest basis with its eigen matrix in shared memory
  long long h2d = 0, d2h = 0;  // bytes moved by the last call
  cudaEvent_t ev[6] = {};
  cudaEvent_t kev[2] = {};
  cudaEvent_t gev[2] = {};  // around the learned-guess inference of a batch (timings[6])
  bool profile = false;
  DevBuf prof;
  double phase_cycles[kPhases] = {};
  // whole-GPU path for large molecules
  int large_min = kMaxN + 1;  // molecules with at least this many basis functions
  bool large_set = false;     // large_min set by pm3gpu_set_large_threshold (no single-molecule rule)
  LargeBufs* lbuf = nullptr;
  DevBuf lsel;                // densities of the selected state (P_tot | P_alpha | P_beta)
  double large_ms[16] = {};   // phase times of the last whole-GPU solve (profiling only)
  // autotuner: measured choices per size bucket (autotune.cuh); forced values while it measures
  struct Tune {
    int le;      // bucket: largest basis size it covers
    int choice;  // batch: CTAs per SM (1 or 2); large: 1 cooperative panels, 0 multi-launch
    double ms_a, ms_b;  // measured times of the two candidates (batch: 1 and 2 CTAs; large: coop, multi)
  };
  std::vector<Tune> tune_batch, tune_large;
  int force_ctas = 0, force_coop = -1;
  int precision = PM3GPU_PRECISION_FP64;  // arithmetic of the whole-GPU path's dense products
  bool coop_panels = true;    // Householder panels as cooperative launches (PM3GPU_COOP_PANELS=0: off)
  std::vector<double> ltrace;  // per-iteration record of the last whole-GPU solve (5 per row)
  DevBuf tcbuf[7];             // pm3gpu_split_gemm: A, B (FP64), A hi / lo, B hi / lo, C; tcerr (pm3gpu_dgemm: A, B, C, split-K work)
  bool large_checks = false;   // whole-GPU path: eigen residual of every eigensolve (one more DGEMM)
  std::vector<double> lchecks;  // per-eigensolve checks of the last whole-GPU solve (6 per row)
  // learned initial density: FP32 master parameters, BF16 copy, Adam moments, gradients
  bool has_guess_model = false;
  long long adam_steps = 0;
  DevBuf gp, gpb, gm, gv, gg;
  DevBuf gqmols, gatom, gao, gcoord, gX, gY, gZ[3], gH[3], gdH, gdZ, gT, gM, gidx, gXb, gTb, gMb, gdY, gpart, gguess, gdens;
  DevBuf gwt, gerr;  // inference: transposed hidden weights (tcgen05 B operands), kernel error flag
  DevBuf d3buf;      // post-SCF corrections: inputs, coordination numbers, row energies, scratch, gradients
  void* h_corr = nullptr;  // pinned staging of the corrections' inputs and results
  size_t h_corr_bytes = 0;
  int* h_gerr = nullptr;  // pinned copy of gerr, read after the stream's next synchronisation
};

namespace {

// Choice recorded for the smallest tuned bucket that covers `size`, else `dflt`.
int tune_lookup(const std::vector<pm3gpu_ctx::Tune>& t, int size, int dflt) {
  for (const pm3gpu_ctx::Tune& e : t)
    if (size <= e.le) return e.choice;
  return dflt;
}

// Message of the last failure of a call made without a context (pm3gpu_load_tuning(NULL, ..)),
// per host thread, so that a check without a device can still say what is wrong.
thread_local std::string t_noctx_err;

int fail(pm3gpu_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  else t_noctx_err = msg;
  return code;
}
#define CUDA_TRY(ctx, call)                                                                        \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return fail((ctx), PM3GPU_CUDA_ERROR, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

bool supported(int z) { return z > 0 && z < kMaxZ && [&] {
  for (int k = 0; k < PM3_N_RAW_ELEMENTS; ++k)
    if (PM3_RAW_ELEMENTS[k].z == z) return true;
  return false;
}(); }

// Element z is in the s/p analytic path and present in the context's parameter set.
bool has_elem(const pm3gpu_ctx* c, int z) { return supported(z) && c->h_elem[z].z == z; }

// ---------------------------------------------------------------- parameter sets
// The public pm3gpu_element (the Pm3Element fields of the s/p path) from the context's form.
void elem_to_public(const ElemDev& e, pm3gpu_element& o) {
  std::memset(&o, 0, sizeof(o));
  o.z = e.z;
  o.n_orb = e.norb;
  o.npq = e.npq;
  o.n_gauss = e.ngauss;
  o.u_ss = e.uss;
  o.u_pp = e.upp;
  o.zeta_s = e.zs;
  o.zeta_p = e.zp;
  o.beta_s = e.bs;
  o.beta_p = e.bp;
  o.g_ss = e.gss;
  o.g_sp = e.gsp;
  o.g_pp = e.gpp;
  o.g_p2 = e.gp2;
  o.h_sp = e.hsp;
  o.alpha = e.alpha;
  for (int g = 0; g < e.ngauss && g < 4; ++g) {
    o.gauss[g][0] = e.gk[g];
    o.gauss[g][1] = e.gl[g];
    o.gauss[g][2] = e.gm[g];
  }
  o.core_charge = e.core;
  o.occ_s = e.occ_s;
  o.occ_p = e.occ_p;
  o.eheat_ev = e.eheat_ev;
  o.e_isol = e.e_isol;
  o.mass = e.mass;
  o.dd = e.dd;
  o.qq = e.qq;
  o.rho0 = e.rho0;
  o.rho1 = e.rho1;
  o.rho2 = e.rho2;
  // params.rs:694-709: po(1,2,3,7,9) and ddp(2,3) of a main-group element
  o.po[1] = e.po1;
  o.po[2] = e.po2;
  o.po[3] = e.po3;
  o.po[7] = e.rho0;
  o.po[9] = e.po9;
  if (e.norb == 4) {
    o.ddp[2] = e.ddp2;
    o.ddp[3] = e.qq * std::sqrt(2.0);
  }
}

// The context's form of one public element; false (with the reason) when it is out of range.
bool elem_from_public(const pm3gpu_element& i, ElemDev& e, std::string& why) {
  const std::string tag = "parameter set, Z=" + std::to_string(i.z) + ": ";
  if (!supported(i.z)) {
    why = tag + "element outside the s/p analytic path";
    return false;
  }
  if (i.n_orb != 1 && i.n_orb != 4) {
    why = tag + "n_orb must be 1 or 4";
    return false;
  }
  if (i.npq < 1 || i.npq > 3) {
    why = tag + "npq must be 1, 2 or 3";
    return false;
  }
  if (i.n_gauss < 0 || i.n_gauss > 4) {
    why = tag + "n_gauss must be 0..4";
    return false;
  }
  const double* d = &i.u_ss;
  const double* d_end = reinterpret_cast<const double*>(reinterpret_cast<const char*>(&i) + sizeof(i));
  for (; d < d_end; ++d)
    if (!std::isfinite(*d)) {
      why = tag + "non-finite value";
      return false;
    }
  if (i.n_orb == 4 && (i.zeta_p <= 0.0 || i.dd <= 0.0 || i.qq <= 0.0)) {
    why = tag + "an s/p element needs zeta_p, dd and qq > 0";
    return false;
  }
  if (i.zeta_s <= 0.0 || i.g_ss <= 0.0 || i.rho0 <= 0.0 || i.po[9] <= 0.0 || i.core_charge < 0.0) {
    why = tag + "zeta_s, g_ss, rho0 and po[9] must be > 0 and core_charge >= 0";
    return false;
  }
  e = ElemDev{};
  e.z = i.z;
  e.norb = i.n_orb;
  e.npq = i.npq;
  e.ngauss = i.n_gauss;
  e.uss = i.u_ss;
  e.upp = i.u_pp;
  e.zs = i.zeta_s;
  e.zp = i.zeta_p;
  e.bs = i.beta_s;
  e.bp = i.beta_p;
  e.gss = i.g_ss;
  e.gsp = i.g_sp;
  e.gpp = i.g_pp;
  e.gp2 = i.g_p2;
  e.hsp = i.h_sp;
  e.alpha = i.alpha;
  e.core = i.core_charge;
  e.dd = i.dd;
  e.qq = i.qq;
  e.rho0 = i.rho0;
  e.rho1 = i.rho1;
  e.rho2 = i.rho2;
  e.po1 = i.po[1];
  e.po2 = i.po[2];
  e.po3 = i.po[3];
  e.po9 = i.po[9];
  e.ddp2 = i.ddp[2];
  e.qq_core = i.ddp[3] / std::sqrt(2.0);  // MOPAC spcore divides ddp(3) by sqrt 2
  e.occ_s = i.occ_s;
  e.occ_p = i.occ_p;
  e.e_isol = i.e_isol;
  e.eheat_ev = i.eheat_ev;
  e.mass = i.mass;
  for (int g = 0; g < i.n_gauss; ++g) {
    e.gk[g] = i.gauss[g][0];
    e.gl[g] = i.gauss[g][1];
    e.gm[g] = i.gauss[g][2];
  }
  return true;
}

// Pair table entry as repulsion.rs:75-90 reads it: xfac only when |x| > 1e-5, alpha 1.2 when
// the stored alpb is below 1e-6.
void pair_to_dev(int zi, int zj, double alpb, double xfac, PairDev& P) {
  const int use = std::fabs(xfac) > 1.0e-5;
  P.alpha[zi][zj] = P.alpha[zj][zi] = alpb < 1.0e-6 ? 1.2 : alpb;
  P.x[zi][zj] = P.x[zj][zi] = xfac;
  P.has[zi][zj] = P.has[zj][zi] = use;
}

// Validate one molecule and resolve its electron counts (scf.rs:456-520).
void plan_molecule(const pm3gpu_ctx* c, const int32_t* z, const double* xyz, int natom, const pm3gpu_options* o,
                   MolPlan& m) {
  m.natom = natom;
  m.o = o;
  if (natom < 1) {
    m.status = PM3GPU_INVALID_INPUT;
    m.msg = "molecule has no atoms";
    return;
  }
  if (o->multiplicity < 1) {
    m.status = PM3GPU_INVALID_INPUT;
    m.msg = "multiplicity must be >= 1";
    return;
  }
  if (o->variant < PM3GPU_VARIANT_PM3 || o->variant > PM3GPU_VARIANT_D3H4X) {
    m.status = PM3GPU_INVALID_INPUT;
    m.msg = "method variant outside PM3 / PM3-D3 / PM3-D3H4 / PM3-D3H4X";
    return;
  }
  int nao = 0;
  double core = 0.0;
  for (int a = 0; a < natom; ++a) {
    const int zz = z[a];
    if (supported(zz) && !has_elem(c, zz)) {  // left out of the context's parameter set
      m.status = PM3GPU_MISSING_ELEMENT;
      m.msg = "missing PM3 parameter block for Z=" + std::to_string(zz);
      return;
    }
    if (!supported(zz)) {
      const bool pm3_has = zz >= 1 && zz <= 107 && zz != 87;
      m.status = pm3_has ? PM3GPU_UNSUPPORTED : PM3GPU_MISSING_ELEMENT;
      m.msg = pm3_has ? "Z=" + std::to_string(zz) + " is outside the s/p analytic path of this library"
                      : "missing PM3 parameter block for Z=" + std::to_string(zz);
      return;
    }
    for (int k = 0; k < 3 && xyz; ++k)
      if (!std::isfinite(xyz[3 * a + k])) {
        m.status = PM3GPU_INVALID_INPUT;
        m.msg = "non-finite coordinate";
        return;
      }
    nao += c->h_elem[zz].norb;
    core += c->h_elem[zz].core;
  }
  m.nao = nao;
  const double ne = core - o->charge;
  const long nei = std::lround(ne);
  if (std::fabs(ne - (double)nei) > 1.0e-6 || nei < 0) {
    m.status = PM3GPU_INVALID_INPUT;
    m.msg = "invalid electron count";
    return;
  }
  const long nu = o->multiplicity - 1;
  if (nei - nu < 0 || (nei - nu) % 2 != 0) {
    m.status = PM3GPU_INVALID_INPUT;
    m.msg = "electron count " + std::to_string(nei) + " is incompatible with multiplicity " +
            std::to_string(o->multiplicity) + " (need same parity)";
    return;
  }
  m.n_alpha = (int)((nei + nu) / 2);
  m.n_beta = (int)((nei - nu) / 2);
  if (m.n_alpha > nao) {
    m.status = PM3GPU_INVALID_INPUT;
    m.msg = "more electrons than valence orbitals";
    return;
  }
  if (o->reference == PM3GPU_REF_RHF && m.n_alpha != m.n_beta) {
    m.status = PM3GPU_INVALID_INPUT;
    m.msg = "RHF requested for an open-shell system; use UHF or Auto";
    return;
  }
  m.use_uhf = o->reference == PM3GPU_REF_UHF || (o->reference == PM3GPU_REF_AUTO && m.n_alpha != m.n_beta);
  if (natom > kMaxLargeAtoms) {
    m.status = PM3GPU_UNSUPPORTED;
    m.msg = "molecule exceeds " + std::to_string(kMaxLargeAtoms) + " atoms";
    return;
  }
  m.large = nao >= c->large_min || nao > kMaxN || natom > kMaxN;
  m.steered = o->level_shift_ev != 0.0 || o->damping != 0.0;
}

// run_scf of run_pm3 (scf.rs:531-555) as a job: resolve the accelerator the loop will use.
JobDesc make_job(const MolPlan& m, int guess, int accel, double shift, double damp, bool force_uhf, int extra_flags) {
  const pm3gpu_options& o = *m.o;
  JobDesc j{};
  j.atom0 = m.atom0;
  j.natom = m.natom;
  j.nao = m.nao;
  j.n_alpha = m.n_alpha;
  j.n_beta = m.n_beta;
  const bool uhf = m.use_uhf || force_uhf;
  j.flags = (uhf ? kJobUhf : 0) | extra_flags;
  j.guess = (guess == PM3GPU_GUESS_CORE) ? 2
            : (guess == PM3GPU_GUESS_SYMMETRY_BROKEN ? 3 : (guess == PM3GPU_GUESS_LEARNED ? 4 : 1));
  const bool use_diis = o.use_diis && accel != PM3GPU_ACCEL_NONE;
  if (!uhf) {  // scf.rs:1201-1228
    int a = use_diis ? accel : PM3GPU_ACCEL_NONE;
    bool keep = a == PM3GPU_ACCEL_ADIIS_CDIIS && diis_depth_fits(m.nao, 3, o.scf_memory_mb);
    if (a == PM3GPU_ACCEL_ADIIS_CDIIS && !keep) a = PM3GPU_ACCEL_CDIIS;
    j.accel = a;
    if (keep) j.flags |= kJobKeepDens;
    j.depth = diis_depth(m.nao, keep ? 3 : 2, o.scf_memory_mb);
  } else {  // scf.rs:1369-1374: the unrestricted loop extrapolates only with plain CDIIS
    j.accel = (use_diis && accel == PM3GPU_ACCEL_CDIIS) ? PM3GPU_ACCEL_CDIIS : PM3GPU_ACCEL_NONE;
    j.depth = diis_depth(m.nao, 4, o.scf_memory_mb);
  }
  j.backup = -1;
  j.guess_off = 0;
  j.max_scf = o.max_scf;
  j.e_tol = o.e_tol;
  j.p_tol = o.p_tol;
  j.adiis_switch = o.adiis_switch;
  j.shift = shift;
  j.damping = damp;
  return j;
}

// Stability search of run_pm3 (scf.rs:599-715). The first pass's flag: 0 no search, 1 search
// when its frontier gap is below 6 eV (or it did not converge), 2 search whatever it gives. A
// level shift or damping in the options turns the search off (scf.rs:599-609).
int stability_mode(const MolPlan& p, const pm3gpu_options* o) {
  if (p.steered) return 0;
  if (o->stability == PM3GPU_STABILITY_ALWAYS) return 2;
  return o->stability == PM3GPU_STABILITY_AUTO ? 1 : 0;
}

// The rungs the search tries, in the reference's order, skipping those it skips
// (scf.rs:610-678): restricted rungs for an open shell, the two unrestricted rungs for a closed
// shell (which may end in a spin-pure state). Writes at most 7 to out; returns the count.
int stability_rungs(const MolPlan& p, const pm3gpu_options* o, Rung* out) {
  const int primary = o->guess == PM3GPU_GUESS_CORE ? PM3GPU_GUESS_CORE : PM3GPU_GUESS_SAD;
  const int other = primary == PM3GPU_GUESS_CORE ? PM3GPU_GUESS_SAD : PM3GPU_GUESS_CORE;
  const bool closed = !p.use_uhf;
  const Rung all[7] = {{primary, PM3GPU_ACCEL_NONE, 0.0, 0.0, false},
                       {other, o->accelerator, 0.0, 0.0, false},
                       {other, PM3GPU_ACCEL_NONE, 0.0, 0.0, false},
                       {PM3GPU_GUESS_SYMMETRY_BROKEN, o->accelerator, 0.0, 0.0, false},
                       {PM3GPU_GUESS_SYMMETRY_BROKEN, PM3GPU_ACCEL_NONE, 0.0, 0.0, false},
                       {PM3GPU_GUESS_SYMMETRY_BROKEN, PM3GPU_ACCEL_NONE, -2.0, 0.0, closed},
                       {primary, PM3GPU_ACCEL_CDIIS, 0.0, 0.85, closed}};
  int n = 0;
  for (const Rung& r : all)
    if (r.unrestricted == closed) out[n++] = r;
  return n;
}

// run_pm3's selection (scf.rs:680-715): whether the outcome `cand` of rung `r` replaces the
// current state `cur`. A converged unrestricted rung of a closed shell counts only when it is
// spin-pure, and then as a restricted state (cand_unres cleared, alpha frontier taken).
bool rung_replaces(const Rung& r, JobOut& cand, bool& cand_unres, const JobOut& cur) {
  if (!cand.converged) return false;
  if (r.unrestricted) {
    if (!(cand.spin_max < 1.0e-8)) return false;
    cand_unres = false;
    cand.homo = cand.homo_a;
    cand.lumo = cand.lumo_a;
    cand.has_homo = cand.has_homo_a;
    cand.has_lumo = cand.has_lumo_a;
  }
  return !cur.converged || cand.electronic < cur.electronic - 1.0e-6;
}

long long pair_table_doubles(const pm3gpu_ctx* c, const int32_t* z, int natom) {
  long long s = 0, s2 = 0;
  for (int a = 0; a < natom; ++a) {
    const long long p = c->h_elem[z[a]].norb == 4 ? 10 : 1;
    s += p;
    s2 += p * p;
  }
  return (s * s - s2) / 2;
}

// Static shared memory of scf_batch_kernel (set when a context is created).
int g_scf_static_smem = 1024;

// Shared-memory carve-up of one launch. The packed eigen input lives in shared memory for
// bases up to `nsm` (global memory above). When `naos` is given, the layout is shrunk to let
// two CTAs share an SM as long as at least 90% of the launch's jobs still fit in shared memory.
// ctas: 0 = choose (two CTAs per SM when at least 90% of the batch keeps its packed eigen input
// in the smaller layout), 1 or 2 = the autotuner's measured choice.
SmemLayout make_layout(int amax, int nmax, int optin, int smem_per_sm = 0, const std::vector<int>* naos = nullptr,
                       int ctas = 0) {
  SmemLayout L{};
  L.amax = amax;
  auto align = [](int b) { return (b + 15) & ~15; };
  int off = 0;
  L.off_int = off;
  off += align((3 * amax + 1 + 16) * 4);
  L.off_dbl = off;
  off += align(amax * 8 + (3 * amax + 4 * kMaxDepth * kWarps + 4 * kMaxDepth + 2 * kMaxDepth * kMaxDepth + kMaxDepth + 8) * 8);
  L.off_eig = off;
  off += align(7 * nmax * 8 + (2 * nmax + 2) * 4);
  L.off_union = off;
  const int fixed_union = std::max(20 * amax, 2 * 16 * 65);
  auto fit = [&](int budget) {
    int nsm = nmax;
    for (; nsm > 0; --nsm)
      if (off + std::max(fixed_union, nsm * (nsm + 1) / 2) * 8 <= budget) break;
    return nsm;
  };
  int nsm = fit(optin);
  if (smem_per_sm > 0 && ctas != 1 && (ctas == 2 || (naos && !naos->empty()))) {
    const int budget2 = smem_per_sm / 2 - 1024 - g_scf_static_smem;  // per-CTA reservation, static shared memory
    const int nsm2 = fit(budget2);
    if (nsm2 < nsm && off + fixed_union * 8 <= budget2) {
      if (ctas == 2) {
        nsm = nsm2;
      } else {
        size_t inside = 0;
        for (int v : *naos) inside += v <= nsm2;
        if (inside * 10 >= naos->size() * 9) nsm = nsm2;
      }
    }
  }
  L.nsm = nsm;
  L.bytes = off + std::max(fixed_union, nsm * (nsm + 1) / 2) * 8;
  return L;
}

// Output requests of a whole batch call.
struct Want {
  bool density = false, eps = false, grad = false;
};

// Per-job output bookkeeping: offsets of each job's arrays.
struct Offsets {
  size_t charges = 0, dens = 0, eps = 0;
};

void assign_offsets(JobDesc& j, const Want& w, Offsets& t) {
  j.charge_off = (long long)t.charges;
  t.charges += j.natom;
  const bool uhf = (j.flags & kJobUhf) != 0;
  if (w.density || w.grad) {
    j.flags |= (w.density ? kJobDensity : 0) | (w.grad ? kJobGrad : 0);
    j.dens_off = (long long)t.dens;
    t.dens += (size_t)j.nao * j.nao * ((w.grad && uhf) ? 3 : 1);
  }
  if (w.eps) {
    j.flags |= kJobEps;
    j.eps_off = (long long)t.eps;
    t.eps += 2 * (size_t)j.nao;
  }
}

// One persistent launch: the first-pass jobs (sorted largest first) plus the rung table the
// kernel may enqueue from (scf.rs:599-715). Outputs are read back to the host.
struct LaunchOut {
  std::vector<JobOut> out, rout;
  std::vector<double> charges, dens, eps;
};

int launch_jobs(pm3gpu_ctx* c, const std::vector<JobDesc>& jobs, const std::vector<JobDesc>& rjobs,
                const std::vector<int32_t>& zs, const int32_t* d_z, const double* d_xyz, const Offsets& tot,
                bool read_dens, bool read_eps, LaunchOut& R, const std::vector<double>* dens_in = nullptr) {
  const int nj = (int)jobs.size(), nr = (int)rjobs.size();
  R.out.assign(nj, JobOut{});
  R.rout.assign(nr, JobOut{});
  if (nj == 0) return PM3GPU_OK;
  int nmax = 1, amax = 1;
  long long wcap = 1;
  std::vector<int> naos;
  naos.reserve(jobs.size());
  for (const std::vector<JobDesc>* L : {&jobs, &rjobs})
    for (const JobDesc& j : *L) {
      nmax = std::max(nmax, j.nao);
      amax = std::max(amax, j.natom);
      wcap = std::max(wcap, pair_table_doubles(c, zs.data() + j.atom0, j.natom));
    }
  for (const JobDesc& j : jobs) naos.push_back(j.nao);
  const int ctas = c->force_ctas ? c->force_ctas : tune_lookup(c->tune_batch, nmax, 0);
  const SmemLayout L = make_layout(amax, nmax, c->smem_optin, c->smem_per_sm, &naos, ctas);
  int per_sm = 0;
  CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scf_batch_kernel, kThreads, L.bytes));
  if (per_sm < 1) return fail(c, PM3GPU_RESOURCE_LIMIT, "SCF kernel does not fit on an SM");
  c->last_ctas = per_sm;
  c->last_nsm = L.nsm;
  const long long slot = slot_doubles(nmax, wcap);
  size_t free_b = 0, total_b = 0;
  CUDA_TRY(c, cudaMemGetInfo(&free_b, &total_b));
  long long grid = std::min<long long>(nj + nr, (long long)c->sms * per_sm);
  const size_t budget = (size_t)(0.6 * (double)(free_b + c->work.bytes));
  while (grid > 1 && (size_t)grid * slot * 8 > budget) --grid;
  if ((size_t)grid * slot * 8 > budget) return fail(c, PM3GPU_RESOURCE_LIMIT, "SCF workspace exceeds device memory");
  CUDA_TRY(c, c->work.ensure((size_t)grid * slot * 8));
  CUDA_TRY(c, c->jobs.ensure(sizeof(JobDesc) * (nj + nr)));
  CUDA_TRY(c, c->out.ensure(sizeof(JobOut) * (nj + nr)));
  CUDA_TRY(c, c->rq.ensure(2 * sizeof(int) * std::max(nr, 1)));
  CUDA_TRY(c, c->charges.ensure(8 * std::max<size_t>(tot.charges, 1)));
  CUDA_TRY(c, c->dens.ensure(8 * std::max<size_t>(tot.dens, 1)));
  CUDA_TRY(c, c->eps.ensure(8 * std::max<size_t>(tot.eps, 1)));
  CUDA_TRY(c, c->queue.ensure(64));
  if (c->tail_helpers) CUDA_TRY(c, c->help.ensure(sizeof(HelpRec) * (size_t)grid));
  CUDA_TRY(c, cudaMemcpyAsync(c->jobs.p, jobs.data(), sizeof(JobDesc) * nj, cudaMemcpyHostToDevice, c->stream));
  if (nr)
    CUDA_TRY(c, cudaMemcpyAsync(c->jobs.as<JobDesc>() + nj, rjobs.data(), sizeof(JobDesc) * nr, cudaMemcpyHostToDevice,
                                c->stream));
  if (dens_in && !dens_in->empty())
    CUDA_TRY(c, cudaMemcpyAsync(c->dens.p, dens_in->data(), 8 * dens_in->size(), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->queue.p, 0, 64, c->stream));
  if (c->tail_helpers) CUDA_TRY(c, cudaMemsetAsync(c->help.p, 0, sizeof(HelpRec) * (size_t)grid, c->stream));
  if (c->record_jobs) {
    CUDA_TRY(c, c->tjob.ensure(8 * (size_t)(nj + 1)));
    CUDA_TRY(c, cudaMemsetAsync(c->tjob.p, 0, 8 * (size_t)nj, c->stream));
    CUDA_TRY(c, cudaMemsetAsync(c->tjob.as<unsigned long long>() + nj, 0xff, 8, c->stream));
  }
  CUDA_TRY(c, cudaMemsetAsync(c->rq.p, 0, 2 * sizeof(int) * std::max(nr, 1), c->stream));
  if (nr) CUDA_TRY(c, cudaMemsetAsync(c->out.as<JobOut>() + nj, 0xff, sizeof(JobOut) * nr, c->stream));
  KernelArgs a{};
  a.elem = c->elem.as<ElemDev>();
  a.pairs = c->pairs.as<PairDev>();
  a.z = d_z;
  a.xyz = d_xyz;
  a.jobs = c->jobs.as<JobDesc>();
  a.njobs = nj;
  a.out = c->out.as<JobOut>();
  a.rjobs = c->jobs.as<JobDesc>() + nj;
  a.nrjobs = nr;
  a.rout = c->out.as<JobOut>() + nj;
  a.rlist = c->rq.as<int>();
  a.rready = c->rq.as<int>() + std::max(nr, 1);
  a.charges = c->charges.as<double>();
  a.densities = c->dens.as<double>();
  a.guess_dens = c->gguess.as<double>();
  a.grads = nullptr;
  a.eps = c->eps.as<double>();
  a.work = c->work.as<double>();
  a.slot = slot;
  a.nmax = nmax;
  a.wcap = wcap;
  a.queue = c->queue.as<int>();
  a.prof = nullptr;
  a.help = c->tail_helpers ? c->help.as<HelpRec>() : nullptr;
  // With tail helpers, up to 32 idle CTAs stay for late stability rungs and unrestricted jobs to
  // help; otherwise idle CTAs exit and free their SM for the next batch in flight.
  a.max_waiters = c->tail_helpers ? 32 : 0;
  a.tjob = c->record_jobs ? c->tjob.as<unsigned long long>() : nullptr;
  if (c->profile) {
    CUDA_TRY(c, c->prof.ensure(sizeof(unsigned long long) * kPhases));
    CUDA_TRY(c, cudaMemsetAsync(c->prof.p, 0, sizeof(unsigned long long) * kPhases, c->stream));
    a.prof = c->prof.as<unsigned long long>();
  }
  a.sm = L;
  CUDA_TRY(c, cudaEventRecord(c->kev[0], c->stream));
  scf_batch_kernel<<<(unsigned)grid, kThreads, L.bytes, c->stream>>>(a);
  c->launches += 1;
  CUDA_TRY(c, cudaGetLastError());
  CUDA_TRY(c, cudaEventRecord(c->kev[1], c->stream));
  int qh[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  CUDA_TRY(c, cudaMemcpyAsync(qh, c->queue.p, sizeof(qh), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(R.out.data(), c->out.p, sizeof(JobOut) * nj, cudaMemcpyDeviceToHost, c->stream));
  if (nr)
    CUDA_TRY(c, cudaMemcpyAsync(R.rout.data(), c->out.as<JobOut>() + nj, sizeof(JobOut) * nr, cudaMemcpyDeviceToHost,
                                c->stream));
  R.charges.resize(tot.charges);
  if (tot.charges)
    CUDA_TRY(c, cudaMemcpyAsync(R.charges.data(), c->charges.p, 8 * tot.charges, cudaMemcpyDeviceToHost, c->stream));
  if (read_dens && tot.dens) {
    R.dens.resize(tot.dens);
    CUDA_TRY(c, cudaMemcpyAsync(R.dens.data(), c->dens.p, 8 * tot.dens, cudaMemcpyDeviceToHost, c->stream));
  }
  if (read_eps && tot.eps) {
    R.eps.resize(tot.eps);
    CUDA_TRY(c, cudaMemcpyAsync(R.eps.data(), c->eps.p, 8 * tot.eps, cudaMemcpyDeviceToHost, c->stream));
  }
  if (c->record_jobs) {
    c->job_ns.resize(nj + 1);
    CUDA_TRY(c, cudaMemcpyAsync(c->job_ns.data(), c->tjob.p, 8 * (size_t)(nj + 1), cudaMemcpyDeviceToHost, c->stream));
  }
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (qh[3]) return fail(c, PM3GPU_CUDA_ERROR, "a bounded wait of the batched SCF kernel ran out on the device");
  c->paired += qh[6];
  if (c->profile) {
    unsigned long long ph[kPhases];
    CUDA_TRY(c, cudaMemcpy(ph, c->prof.p, sizeof(ph), cudaMemcpyDeviceToHost));
    for (int k = 0; k < kPhases; ++k) c->phase_cycles[k] += (double)ph[k];
  }
  float kms = 0.f;
  CUDA_TRY(c, cudaEventElapsedTime(&kms, c->kev[0], c->kev[1]));
  c->timings[5] += kms;
  c->h2d += (long long)(sizeof(JobDesc) * (nj + nr) + (dens_in ? 8 * dens_in->size() : 0));
  c->d2h += (long long)(sizeof(JobOut) * (nj + nr) + 8 * tot.charges + (read_dens ? 8 * tot.dens : 0) +
                        (read_eps ? 8 * tot.eps : 0) + sizeof(qh));
  return PM3GPU_OK;
}

// Gradients of the selected states of `mols` (one thread per atom pair of the whole batch).
int launch_gradients(pm3gpu_ctx* c, const std::vector<GradMol>& mols, const std::vector<int32_t>& ao_off,
                     const int32_t* d_z, const double* d_xyz, size_t total_atoms, std::vector<double>& grads,
                     const double* dens = nullptr) {
  grads.assign(3 * total_atoms, 0.0);
  if (mols.empty()) return PM3GPU_OK;
  long long npairs = mols.back().pair0 + (long long)mols.back().natom * (mols.back().natom - 1) / 2;
  CUDA_TRY(c, c->gmols.ensure(sizeof(GradMol) * mols.size()));
  CUDA_TRY(c, c->aooff.ensure(4 * std::max<size_t>(ao_off.size(), 1)));
  CUDA_TRY(c, c->grads.ensure(24 * std::max<size_t>(total_atoms, 1)));
  CUDA_TRY(c, cudaMemcpyAsync(c->gmols.p, mols.data(), sizeof(GradMol) * mols.size(), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->aooff.p, ao_off.data(), 4 * ao_off.size(), cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->grads.p, 0, 24 * total_atoms, c->stream));
  if (npairs > 0) {
    GradArgs g{};
    g.elem = c->elem.as<ElemDev>();
    g.pairs = c->pairs.as<PairDev>();
    g.z = d_z;
    g.xyz = d_xyz;
    g.ao_off = c->aooff.as<int>();
    g.mols = c->gmols.as<GradMol>();
    g.nmol = (int)mols.size();
    g.npairs = npairs;
    g.dens = dens ? dens : c->dens.as<double>();
    g.grad = c->grads.as<double>();
    const long long blocks = std::min<long long>((npairs + 127) / 128, (long long)c->sms * 16);
    gradient_kernel<<<(unsigned)blocks, 128, 0, c->stream>>>(g);
    c->launches += 1;
    CUDA_TRY(c, cudaGetLastError());
  }
  CUDA_TRY(c, cudaMemcpyAsync(grads.data(), c->grads.p, 24 * total_atoms, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->h2d += (long long)(sizeof(GradMol) * mols.size() + 4 * ao_off.size());
  c->d2h += (long long)(24 * total_atoms);
  return PM3GPU_OK;
}

// The DGEMM kernels' shared-memory attribute, set once per device on the first whole-GPU solve or
// pm3gpu_dgemm call (the batched path never launches them). The device must be current.
cudaError_t dgemm_ready(int device) {
  static std::mutex mu;
  static std::vector<char> done;
  std::lock_guard<std::mutex> lk(mu);
  if (device < 0) return cudaErrorInvalidDevice;
  if ((int)done.size() <= device) done.resize(device + 1, 0);
  if (done[device]) return cudaSuccess;
  const cudaError_t e = dg::set_attributes();
  if (e == cudaSuccess) done[device] = 1;
  return e;
}

#include "large_driver.cuh"

// run_pm3 (scf.rs:450-848) for one molecule on the whole-GPU path: the first pass, the
// stability rungs in the reference's order when the search triggers, the same selection, then
// the epilogue and (optionally) the gradient at the selected state.
int run_large(pm3gpu_ctx* c, const MolPlan& p, const int32_t* hz, const int32_t* dz, const double* dxyz,
              const pm3gpu_options* o, const Want& want, pm3gpu_result& Rm, double* charges, double* density,
              double* mo_energies, double* gradient) {
  for (double& t : c->large_ms) t = 0.0;
  c->ltrace.clear();
  c->lchecks.clear();
  CUDA_TRY(c, dgemm_ready(c->device));
  if (!c->lbuf) c->lbuf = new LargeBufs();
  LargeSolver S(c, *c->lbuf);
  double ecc = 0.0;
  int rc = S.setup(hz, dz, dxyz, p.natom, p.nao, &ecc);
  if (rc != PM3GPU_OK) return rc;
  const size_t nn = (size_t)p.nao * p.nao;
  const bool keep_dens = want.density || want.grad;
  auto save = [&](const LargeRun& run) -> int {  // densities of the state that is currently selected
    if (!keep_dens) return PM3GPU_OK;
    CUDA_TRY(c, c->lsel.ensure(8 * nn * (run.uhf ? 3 : 1)));
    CUDA_TRY(c, cudaMemcpyAsync(c->lsel.p, S.final_pt(), 8 * nn, cudaMemcpyDeviceToDevice, c->stream));
    if (run.uhf) {
      CUDA_TRY(c, cudaMemcpyAsync(c->lsel.as<double>() + nn, S.final_pa(), 8 * nn, cudaMemcpyDeviceToDevice, c->stream));
      CUDA_TRY(c, cudaMemcpyAsync(c->lsel.as<double>() + 2 * nn, S.final_pb(), 8 * nn, cudaMemcpyDeviceToDevice,
                                  c->stream));
    }
    return PM3GPU_OK;
  };
  const JobDesc fj = p.steered ? make_job(p, o->guess, o->accelerator, o->level_shift_ev, o->damping, false, 0)
                               : make_job(p, o->guess, o->accelerator, 0.0, 0.0, false, 0);
  LargeRun st;
  CUDA_TRY(c, cudaEventRecord(c->kev[0], c->stream));  // the SCF passes alone (timings[3])
  rc = S.scf(fj, st);
  if (rc != PM3GPU_OK) return rc;
  if ((rc = save(st)) != PM3GPU_OK) return rc;
  bool st_unres = (fj.flags & kJobUhf) != 0;
  const double first_ev = st.o.electronic;
  int paths = 1;
  const int smode = stability_mode(p, o);
  const bool search = smode == 2 || (smode == 1 && st.o.gap < 6.0);
  if (search) {  // scf.rs:610-715
    Rung rungs[7];
    const int nr = stability_rungs(p, o, rungs);
    for (int k = 0; k < nr; ++k) {
      const Rung& r = rungs[k];
      ++paths;
      const JobDesc rj = make_job(p, r.guess, r.accel, r.shift, r.damp, r.unrestricted, 0);
      LargeRun cand;
      if (S.scf(rj, cand) != PM3GPU_OK) continue;
      bool cand_unres = (rj.flags & kJobUhf) != 0;
      if (rung_replaces(r, cand.o, cand_unres, st.o)) {
        st = std::move(cand);
        st_unres = cand_unres;
        if ((rc = save(st)) != PM3GPU_OK) return rc;
      }
    }
  }
  {
    CUDA_TRY(c, cudaEventRecord(c->kev[1], c->stream));
    CUDA_TRY(c, cudaEventSynchronize(c->kev[1]));
    float scf_ms = 0.f;
    CUDA_TRY(c, cudaEventElapsedTime(&scf_ms, c->kev[0], c->kev[1]));
    c->timings[3] += scf_ms;
  }
  double e_isol = 0.0, eheat = 0.0;
  for (int a = 0; a < p.natom; ++a) {
    e_isol += c->h_elem[hz[a]].e_isol;
    eheat += c->h_elem[hz[a]].eheat_ev;
  }
  const JobOut& so = st.o;
  Rm.status = PM3GPU_OK;
  Rm.nao = p.nao;
  Rm.n_occ = p.n_alpha;
  Rm.n_beta = st_unres ? p.n_beta : p.n_alpha;
  Rm.electronic_ev = so.electronic;
  Rm.core_ev = ecc;
  Rm.total_ev = so.electronic + ecc;
  Rm.heat_of_formation_kcal = (Rm.total_ev - e_isol + eheat) * kEvToKcal;
  Rm.iterations = so.iterations;
  Rm.converged = so.converged;
  Rm.unrestricted = st_unres ? 1 : 0;
  Rm.scf_paths_tried = paths;
  Rm.scf_improvement_ev = std::max(first_ev - so.electronic, 0.0);
  Rm.last_change = so.last_change;
  Rm.homo_ev = so.homo;
  Rm.lumo_ev = so.lumo;
  Rm.has_homo = so.has_homo;
  Rm.has_lumo = so.has_lumo;
  for (int k = 0; k < 3; ++k) Rm.dipole_debye[k] = so.dipole[k];
  Rm.dipole_magnitude = std::sqrt(Rm.dipole_debye[0] * Rm.dipole_debye[0] + Rm.dipole_debye[1] * Rm.dipole_debye[1] +
                                  Rm.dipole_debye[2] * Rm.dipole_debye[2]);
  if (!so.converged) {
    Rm.status = PM3GPU_SCF_NOT_CONVERGED;
    char msg[160];
    std::snprintf(msg, sizeof msg, "PM3 SCF did not converge after %d iterations (error=%.3e)", so.iterations,
                  so.last_change);
    c->err = msg;
  }
  if (charges) std::memcpy(charges, st.charges.data(), 8 * (size_t)p.natom);
  if (density && want.density) {
    CUDA_TRY(c, cudaMemcpyAsync(density, c->lsel.p, 8 * nn, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  if (mo_energies && want.eps) {
    std::vector<double> all;
    if ((rc = S.all_eigenvalues(st.tri_a, all)) != PM3GPU_OK) return rc;
    std::memcpy(mo_energies, all.data(), 8 * (size_t)p.nao);
  }
  if (want.grad && gradient && so.converged) {
    std::vector<int32_t> ao_off(p.natom);
    for (int a = 0, off = 0; a < p.natom; ++a) {
      ao_off[a] = off;
      off += c->h_elem[hz[a]].norb;
    }
    GradMol g{};
    g.atom0 = 0;
    g.natom = p.natom;
    g.nao = p.nao;
    g.uhf = st_unres ? 1 : 0;
    if (!st.uhf) g.uhf = 0;
    g.pair0 = 0;
    g.dens_off = 0;
    std::vector<double> gr;
    rc = launch_gradients(c, {g}, ao_off, dz, dxyz, (size_t)p.natom, gr, c->lsel.as<double>());
    if (rc != PM3GPU_OK) return rc;
    std::memcpy(gradient, gr.data(), 24 * (size_t)p.natom);
  }
  return PM3GPU_OK;
}

// ------------------------------------------------------------------ learned initial density
// Feature rows of a set of molecules: per molecule its atoms (self rows) then its pairs a < b.
struct GuessRows {
  std::vector<guess::Mol> mols;
  std::vector<int> atom_mol, ao;  // per atom of the packed batch: molecule, first AO
  long long rows = 0;
  size_t dens_total = 0;
};

void guess_rows(const pm3gpu_ctx* c, const std::vector<int>& atom0, const std::vector<int>& natom,
                const int32_t* h_z_all, int total_atoms, GuessRows& G) {
  G.mols.clear();
  G.atom_mol.assign(total_atoms, 0);
  G.ao.assign(total_atoms, 0);
  G.rows = 0;
  G.dens_total = 0;
  for (size_t m = 0; m < atom0.size(); ++m) {
    guess::Mol M{};
    M.atom0 = atom0[m];
    M.natom = natom[m];
    int off = 0;
    for (int a = 0; a < M.natom; ++a) {
      G.atom_mol[M.atom0 + a] = (int)m;
      G.ao[M.atom0 + a] = off;
      off += c->h_elem[h_z_all[M.atom0 + a]].norb;
    }
    M.nao = off;
    M.row0 = G.rows;
    M.dens_off = (long long)G.dens_total;
    G.rows += M.natom + (long long)M.natom * (M.natom - 1) / 2;
    G.dens_total += (size_t)off * off;
    G.mols.push_back(M);
  }
}

inline int gblocks(long long work, int threads = 256) {
  return (int)std::max<long long>(1, std::min<long long>((work + threads - 1) / threads, 4096));
}

// coordination counts and BF16 feature rows into c->gX
int guess_features(pm3gpu_ctx* c, const GuessRows& G, const int32_t* dz, const double* dxyz, int total_atoms) {
  CUDA_TRY(c, c->gqmols.ensure(sizeof(guess::Mol) * std::max<size_t>(G.mols.size(), 1)));
  CUDA_TRY(c, c->gatom.ensure(4 * (size_t)std::max(total_atoms, 1)));
  CUDA_TRY(c, c->gao.ensure(4 * (size_t)std::max(total_atoms, 1)));
  CUDA_TRY(c, c->gcoord.ensure(4 * (size_t)std::max(total_atoms, 1)));
  CUDA_TRY(c, c->gX.ensure(2 * (size_t)guess::kIn * std::max<long long>(G.rows, 1)));
  CUDA_TRY(c, cudaMemcpyAsync(c->gqmols.p, G.mols.data(), sizeof(guess::Mol) * G.mols.size(), cudaMemcpyHostToDevice,
                              c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->gatom.p, G.atom_mol.data(), 4 * (size_t)total_atoms, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->gao.p, G.ao.data(), 4 * (size_t)total_atoms, cudaMemcpyHostToDevice, c->stream));
  guess::coord_kernel<<<gblocks(total_atoms), 256, 0, c->stream>>>(c->gqmols.as<guess::Mol>(), (int)G.mols.size(),
                                                                 c->gatom.as<int>(), dxyz, total_atoms,
                                                                 c->gcoord.as<float>());
  guess::features_kernel<<<gblocks(G.rows), 256, 0, c->stream>>>(c->gqmols.as<guess::Mol>(), (int)G.mols.size(),
                                                                c->elem.as<ElemDev>(), dz, dxyz, c->gcoord.as<float>(),
                                                                G.rows, c->gX.as<__nv_bfloat16>());
  c->launches += 2;
  CUDA_TRY(c, cudaGetLastError());
  return PM3GPU_OK;
}

template <bool TA, bool TB>
void gemm_bf16(pm3gpu_ctx* c, int M, int N, int K, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb,
               float* C, int ldc, bool acc = false) {
  const dim3 grid((N + guess::kGT - 1) / guess::kGT, (M + guess::kGT - 1) / guess::kGT);
  guess::gemm_bf16_kernel<TA, TB><<<grid, 128, 0, c->stream>>>(M, N, K, A, lda, B, ldb, C, ldc, acc ? 1 : 0);
  ++c->launches;
}

// MLP forward over `rows` feature rows of X (BF16) into Y (rows x kOut, FP32). With `keep`, the
// pre-activations Z and activations H of each hidden layer stay in c->gZ / c->gH (training).
int mlp_forward(pm3gpu_ctx* c, const __nv_bfloat16* X, long long rows, float* Y) {
  using namespace guess;
  const __nv_bfloat16* P = c->gpb.as<__nv_bfloat16>();
  for (int l = 0; l < 3; ++l) {
    CUDA_TRY(c, c->gZ[l].ensure(4 * (size_t)kHid * std::max<long long>(rows, 1)));
    CUDA_TRY(c, c->gH[l].ensure(2 * (size_t)kHid * std::max<long long>(rows, 1)));
  }
  const int woff[3] = {kW1, kW2, kW3}, boff[3] = {kB1, kB2, kB3};
  const __nv_bfloat16* in = X;
  int kin = kIn;
  for (int l = 0; l < 3; ++l) {
    gemm_bf16<false, false>(c, (int)rows, kHid, kin, in, kin, P + woff[l], kHid, c->gZ[l].as<float>(), kHid);
    bias_act_kernel<<<gblocks(rows * kHid), 256, 0, c->stream>>>(c->gZ[l].as<float>(), c->gp.as<float>() + boff[l], kHid,
                                                                 rows, c->gH[l].as<__nv_bfloat16>(), 1);
    ++c->launches;
    in = c->gH[l].as<__nv_bfloat16>();
    kin = kHid;
  }
  gemm_bf16<false, false>(c, (int)rows, kOut, kHid, in, kHid, P + kW4, kOut, Y, kOut);
  bias_act_kernel<<<gblocks(rows * kOut), 256, 0, c->stream>>>(Y, c->gp.as<float>() + kB4, kOut, rows, nullptr, 0);
  ++c->launches;
  CUDA_TRY(c, cudaGetLastError());
  return PM3GPU_OK;
}

// Inference on `rows` feature rows: the three hidden layers on the tcgen05 layer kernel
// (tc::launch_mlp_layer, bias + SiLU in its epilogue), the output layer fused into the last one's
// epilogue; Y = rows x kOut FP32. The rounding points are mlp_forward's (FP32 pre-activations, BF16
// activations); training keeps mlp_forward, whose pre-activations the backward pass needs.
int mlp_infer(pm3gpu_ctx* c, const __nv_bfloat16* X, long long rows, float* Y) {
  using namespace guess;
  if (rows <= 0) return PM3GPU_OK;
  if (rows > (1LL << 30)) return fail(c, PM3GPU_RESOURCE_LIMIT, "learned guess: too many feature rows in one call");
  const __nv_bfloat16* P = c->gpb.as<__nv_bfloat16>();
  const float* pf = c->gp.as<float>();
  CUDA_TRY(c, c->gwt.ensure(2 * (size_t)kHid * (kIn + 2 * kHid)));
  for (int l = 0; l < 2; ++l) CUDA_TRY(c, c->gH[l].ensure(2 * (size_t)kHid * rows));
  __nv_bfloat16* Wt1 = c->gwt.as<__nv_bfloat16>();
  __nv_bfloat16* Wt2 = Wt1 + (size_t)kHid * kIn;
  __nv_bfloat16* Wt3 = Wt2 + (size_t)kHid * kHid;
  transpose_w_kernel<<<64, 256, 0, c->stream>>>(P + kW1, kIn, kHid, Wt1);
  transpose_w_kernel<<<256, 256, 0, c->stream>>>(P + kW2, kHid, kHid, Wt2);
  transpose_w_kernel<<<256, 256, 0, c->stream>>>(P + kW3, kHid, kHid, Wt3);
  CUDA_TRY(c, cudaGetLastError());
  int* err = c->gerr.as<int>();
  __nv_bfloat16* H1 = c->gH[0].as<__nv_bfloat16>();
  __nv_bfloat16* H2 = c->gH[1].as<__nv_bfloat16>();
  const int M = (int)rows;
  if (!tc::launch_mlp_layer(M, kIn, X, Wt1, pf + kB1, H1, nullptr, nullptr, nullptr, err, c->stream) ||
      !tc::launch_mlp_layer(M, kHid, H1, Wt2, pf + kB2, H2, nullptr, nullptr, nullptr, err, c->stream) ||
      !tc::launch_mlp_layer(M, kHid, H2, Wt3, pf + kB3, nullptr, P + kW4, pf + kB4, Y, err, c->stream))
    return fail(c, PM3GPU_CUDA_ERROR, "learned guess: tensor map or kernel attribute of the tcgen05 layers");
  c->launches += 6;
  CUDA_TRY(c, cudaGetLastError());
  return PM3GPU_OK;
}

// Inference over all rows, 2^20 at a time, without blocking the host: the kernels' error flag is
// cleared first and copied to pinned host memory after the last layer; the caller reads it with
// infer_failed() once the stream has been synchronised (a host wait here would hold back the next
// launches while other work occupies the SMs).
int mlp_infer_all(pm3gpu_ctx* c, const __nv_bfloat16* X, long long rows, float* Y) {
  using namespace guess;
  CUDA_TRY(c, c->gerr.ensure(sizeof(int)));
  CUDA_TRY(c, cudaMemsetAsync(c->gerr.p, 0, sizeof(int), c->stream));
  for (long long r0 = 0; r0 < rows; r0 += 1LL << 20) {
    const int rc = mlp_infer(c, X + r0 * kIn, std::min<long long>(1LL << 20, rows - r0), Y + r0 * kOut);
    if (rc != PM3GPU_OK) return rc;
  }
  CUDA_TRY(c, cudaMemcpyAsync(c->h_gerr, c->gerr.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  return PM3GPU_OK;
}
bool infer_failed(pm3gpu_ctx* c) { return *reinterpret_cast<volatile int*>(c->h_gerr) != 0; }

// Forward and backward pass of the network on B rows X (BF16), targets T and masks Mk (FP32):
// loss = inv_count * sum Mk (Y - T)^2 (its partial sums are added into *accum), gradient of
// every parameter into c->gg (layout of the parameter vector). dY, dZ are rounded to BF16 for the
// GEMMs; dH and the parameter gradients are FP32. Needs c->gY, gdY, gdH, gdZ for B rows.
int mlp_loss_grad(pm3gpu_ctx* c, const __nv_bfloat16* X, const float* T, const float* Mk, int B, float inv_count,
                  float* accum) {
  using namespace guess;
  int rc = mlp_forward(c, X, B, c->gY.as<float>());
  if (rc != PM3GPU_OK) return rc;
  float* gg = c->gg.as<float>();
  const __nv_bfloat16* Pb = c->gpb.as<__nv_bfloat16>();
  const int woff[3] = {kW1, kW2, kW3}, boff[3] = {kB1, kB2, kB3};
  loss_kernel<<<gblocks((long long)B * kOut), 256, 0, c->stream>>>(c->gY.as<float>(), T, Mk, (long long)B * kOut,
                                                                    inv_count, c->gdY.as<__nv_bfloat16>(), accum);
  // output layer
  gemm_bf16<true, false>(c, kHid, kOut, B, c->gH[2].as<__nv_bfloat16>(), kHid, c->gdY.as<__nv_bfloat16>(), kOut,
                         gg + kW4, kOut);
  colsum_kernel<<<kOut, 256, 0, c->stream>>>(c->gdY.as<__nv_bfloat16>(), kOut, B, gg + kB4);
  gemm_bf16<false, true>(c, B, kHid, kOut, c->gdY.as<__nv_bfloat16>(), kOut, Pb + kW4, kOut, c->gdH.as<float>(), kHid);
  c->launches += 4;
  // hidden layers, last to first
  for (int l = 2; l >= 0; --l) {
    dact_kernel<<<gblocks((long long)B * kHid), 256, 0, c->stream>>>(c->gdH.as<float>(), c->gZ[l].as<float>(),
                                                                     (long long)B * kHid, c->gdZ.as<__nv_bfloat16>());
    const __nv_bfloat16* in = l > 0 ? c->gH[l - 1].as<__nv_bfloat16>() : X;
    const int kin = l > 0 ? kHid : kIn;
    gemm_bf16<true, false>(c, kin, kHid, B, in, kin, c->gdZ.as<__nv_bfloat16>(), kHid, gg + woff[l], kHid);
    colsum_kernel<<<kHid, 256, 0, c->stream>>>(c->gdZ.as<__nv_bfloat16>(), kHid, B, gg + boff[l]);
    c->launches += 3;
    if (l > 0) {
      gemm_bf16<false, true>(c, B, kHid, kHid, c->gdZ.as<__nv_bfloat16>(), kHid, Pb + woff[l], kHid, c->gdH.as<float>(),
                             kHid);
      ++c->launches;
    }
  }
  CUDA_TRY(c, cudaGetLastError());
  return PM3GPU_OK;
}

// Initial densities of the molecules in G (device buffer c->gguess, G.dens_total doubles).
int guess_infer(pm3gpu_ctx* c, const GuessRows& G, const int32_t* dz, const double* dxyz, int total_atoms) {
  if (!c->has_guess_model) return fail(c, PM3GPU_INVALID_INPUT, "learned guess requested but no model is set");
  int rc = guess_features(c, G, dz, dxyz, total_atoms);
  if (rc != PM3GPU_OK) return rc;
  CUDA_TRY(c, c->gY.ensure(4 * (size_t)guess::kOut * std::max<long long>(G.rows, 1)));
  CUDA_TRY(c, c->gguess.ensure(8 * std::max<size_t>(G.dens_total, 1)));
  rc = mlp_infer_all(c, c->gX.as<__nv_bfloat16>(), G.rows, c->gY.as<float>());
  if (rc != PM3GPU_OK) return rc;
  CUDA_TRY(c, cudaMemsetAsync(c->gguess.p, 0, 8 * G.dens_total, c->stream));
  guess::assemble_kernel<<<gblocks(G.rows), 256, 0, c->stream>>>(c->gqmols.as<guess::Mol>(), (int)G.mols.size(),
                                                                c->elem.as<ElemDev>(), dz, dxyz, c->gao.as<int>(),
                                                                c->gY.as<float>(), G.rows, c->gguess.as<double>());
  ++c->launches;
  CUDA_TRY(c, cudaGetLastError());
  return PM3GPU_OK;
}

struct HostJobResult {
  JobOut o;
  const JobDesc* job = nullptr;
  bool unrestricted = false;
};

// The run_pm3 flow over a batch (scf.rs:450-848): one persistent launch solves every
// molecule and the stability-search rungs its first pass asks for; the host then selects
// each molecule's state exactly as run_pm3 does and forms the epilogue.
#include "d3.cuh"
#include "h4.cuh"
#include "corrections.cuh"

int run_batch(pm3gpu_ctx* c, int n_mol, const int32_t* h_offs, const int32_t* h_z, const double* h_xyz,
              const int32_t* d_z, const double* d_xyz, const pm3gpu_options* opts, int per_mol, const Want& want,
              pm3gpu_result* results, double* charges, double* gradients, double* density, double* mo_energies,
              double* all_dens = nullptr, const size_t* all_dens_off = nullptr) {
  c->launches = 0;
  c->paired = 0;
  c->timings[3] = 0.0;
  c->timings[5] = 0.0;
  c->timings[6] = 0.0;
  bool guess_timed = false;
  c->h2d = c->d2h = 0;
  for (int k = 0; k < kPhases; ++k) c->phase_cycles[k] = 0.0;
  cudaEventRecord(c->ev[0], c->stream);
  const int total_atoms = h_offs[n_mol];
  std::vector<int32_t> zs(h_z, h_z + total_atoms);
  const int32_t* dz = d_z;
  const double* dxyz = d_xyz;
  if (!dz) {
    CUDA_TRY(c, c->z.ensure(4 * (size_t)std::max(total_atoms, 1)));
    CUDA_TRY(c, c->xyz.ensure(24 * (size_t)std::max(total_atoms, 1)));
    CUDA_TRY(c, cudaMemcpyAsync(c->z.p, h_z, 4 * (size_t)total_atoms, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->xyz.p, h_xyz, 24 * (size_t)total_atoms, cudaMemcpyHostToDevice, c->stream));
    dz = c->z.as<int32_t>();
    dxyz = c->xyz.as<double>();
    c->h2d += 28LL * total_atoms;
  }
  cudaEventRecord(c->ev[1], c->stream);
  // post-SCF corrections (scf.rs:740-743) depend on the geometry alone: enqueue them ahead of the SCF
  CorrPlan corr;
  {
    bool offs_ok = true;
    for (int m = 0; m < n_mol; ++m) offs_ok &= h_offs[m + 1] >= h_offs[m];
    if (offs_ok) {
      const int rcc = corrections_for_batch(c, n_mol, h_offs, opts, per_mol, dz, dxyz, want.grad && gradients, corr);
      if (rcc != PM3GPU_OK) return rcc;
    }
  }
  std::vector<MolPlan> plans(n_mol);
  std::vector<JobDesc> jobs, rjobs;
  Offsets tot;
  for (int m = 0; m < n_mol; ++m) {
    MolPlan& p = plans[m];
    p.atom0 = h_offs[m];
    const int na = h_offs[m + 1] - h_offs[m];
    if (na < 0) return fail(c, PM3GPU_INVALID_INPUT, "atom_offsets must be non-decreasing");
    const pm3gpu_options* o = per_mol ? opts + m : opts;
    plan_molecule(c, h_z + p.atom0, h_xyz ? h_xyz + 3 * (size_t)p.atom0 : nullptr, na, o, p);
    // A lone molecule of kSingleWholeNao basis functions or more finishes sooner on all SMs than on
    // the one CTA the batched kernel gives it (n = 204: 47 against 54 ms; n = 252: 62 against 183).
    if (n_mol == 1 && !c->large_set && p.status == PM3GPU_OK && !p.large && p.nao >= kSingleWholeNao &&
        o->guess != PM3GPU_GUESS_LEARNED)
      p.large = true;
    if (p.status != PM3GPU_OK || p.large) continue;  // large molecules: whole-GPU path below
    JobDesc j = p.steered ? make_job(p, o->guess, o->accelerator, o->level_shift_ev, o->damping, false, 0)
                          : make_job(p, o->guess, o->accelerator, 0.0, 0.0, false, 0);
    j.mol = m;
    assign_offsets(j, want, tot);
    // the rungs run_pm3 would try, in its order, skipping those it skips (scf.rs:610-678)
    j.stab = stability_mode(p, o);
    j.rung0 = (int)rjobs.size();
    j.nrung = 0;
    if (j.stab) {
      Rung rungs[7];
      const int nr = stability_rungs(p, o, rungs);
      for (int k = 0; k < nr; ++k) {
        const Rung& r = rungs[k];
        JobDesc rj = make_job(p, r.guess, r.accel, r.shift, r.damp, r.unrestricted, 0);
        rj.mol = m;
        rj.stab = 0;
        rj.nrung = 0;
        assign_offsets(rj, want, tot);
        p.rungs.push_back(r);
        rjobs.push_back(rj);
        ++j.nrung;
      }
    }
    if (j.guess == 4) {  // the same pass from the standard guess, run only if the learned start fails
      JobDesc bj = p.steered ? make_job(p, PM3GPU_GUESS_SAD, o->accelerator, o->level_shift_ev, o->damping, false, 0)
                             : make_job(p, PM3GPU_GUESS_SAD, o->accelerator, 0.0, 0.0, false, 0);
      bj.mol = m;
      bj.stab = j.stab;
      bj.rung0 = j.rung0;
      bj.nrung = j.nrung;
      assign_offsets(bj, want, tot);
      j.backup = (int)rjobs.size();
      rjobs.push_back(bj);
    }
    p.first_job = (int)jobs.size();
    jobs.push_back(j);
  }
  // learned initial densities for the molecules that asked for them
  {
    std::vector<int> la0, lna, lmol;
    for (int m = 0; m < n_mol; ++m) {
      const MolPlan& p = plans[m];
      if (p.status == PM3GPU_OK && !p.large && jobs[p.first_job].guess == 4) {
        la0.push_back(p.atom0);
        lna.push_back(p.natom);
        lmol.push_back(m);
      }
    }
    if (!lmol.empty()) {
      CUDA_TRY(c, cudaEventRecord(c->gev[0], c->stream));
      GuessRows G;
      guess_rows(c, la0, lna, h_z, total_atoms, G);
      const int rg = guess_infer(c, G, dz, dxyz, total_atoms);
      if (rg != PM3GPU_OK) return rg;
      CUDA_TRY(c, cudaEventRecord(c->gev[1], c->stream));
      guess_timed = true;
      for (size_t k = 0; k < lmol.size(); ++k) jobs[plans[lmol[k]].first_job].guess_off = G.mols[k].dens_off;
    }
  }
  // largest first (longest-processing-time order) for the work queue
  std::vector<int> order(jobs.size()), pos(jobs.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return jobs[a].nao > jobs[b].nao; });
  std::vector<JobDesc> sorted(jobs.size());
  for (size_t i = 0; i < order.size(); ++i) {
    sorted[i] = jobs[order[i]];
    pos[order[i]] = (int)i;
  }
  LaunchOut R;
  int rc = launch_jobs(c, sorted, rjobs, zs, dz, dxyz, tot, want.density, want.eps, R);
  if (rc != PM3GPU_OK) return rc;
  if (guess_timed) {  // the launch has synchronised the stream
    if (infer_failed(c)) return fail(c, PM3GPU_CUDA_ERROR, "learned guess: a pipeline wait in the tcgen05 layer kernel ran out");
    float gms = 0.f;
    CUDA_TRY(c, cudaEventElapsedTime(&gms, c->gev[0], c->gev[1]));
    c->timings[6] = gms;
  }
  cudaEventRecord(c->ev[2], c->stream);

  // ---------------------------------------------------------------- selection + epilogue
  std::vector<HostJobResult> chosen(n_mol);
  for (int m = 0; m < n_mol; ++m) {
    MolPlan& p = plans[m];
    pm3gpu_result& Rm = results[m];
    std::memset(&Rm, 0, sizeof(Rm));
    Rm.status = p.status;
    Rm.nao = p.nao;
    if (p.status != PM3GPU_OK) {
      if (c->err.empty() || n_mol == 1) c->err = p.msg;
      continue;
    }
    if (p.large) {
      const pm3gpu_options* o = per_mol ? opts + m : opts;
      const int rl = run_large(c, p, h_z + p.atom0, dz + p.atom0, dxyz + 3 * (size_t)p.atom0, o, want, Rm,
                               charges ? charges + p.atom0 : nullptr, density, mo_energies,
                               (want.grad && gradients) ? gradients + 3 * (size_t)p.atom0 : nullptr);
      if (rl != PM3GPU_OK) {
        Rm.status = rl;
        if (n_mol == 1) return rl;
      }
      continue;
    }
    const JobDesc& fj = jobs[p.first_job];
    HostJobResult st;
    st.o = R.out[pos[p.first_job]];
    st.job = &fj;
    st.unrestricted = (fj.flags & kJobUhf) != 0;
    if (fj.backup >= 0 && !st.o.converged && R.rout[fj.backup].status != -1) {  // learned start failed
      st.o = R.rout[fj.backup];
      st.job = &rjobs[fj.backup];
      st.unrestricted = (st.job->flags & kJobUhf) != 0;
    }
    const double first_ev = st.o.electronic;
    int paths = 1;
    const bool searched = fj.nrung > 0 && R.rout[fj.rung0].status != -1;
    for (int r = 0; searched && r < fj.nrung; ++r) {
      ++paths;
      const JobDesc& rj = rjobs[fj.rung0 + r];
      HostJobResult cand;
      cand.o = R.rout[fj.rung0 + r];
      cand.job = &rj;
      cand.unrestricted = (rj.flags & kJobUhf) != 0;
      if (rung_replaces(p.rungs[r], cand.o, cand.unrestricted, st.o)) st = cand;
    }
    chosen[m] = st;
    double e_isol = 0.0, eheat = 0.0;
    for (int a = 0; a < p.natom; ++a) {
      e_isol += c->h_elem[h_z[p.atom0 + a]].e_isol;
      eheat += c->h_elem[h_z[p.atom0 + a]].eheat_ev;
    }
    Rm.n_occ = p.n_alpha;
    Rm.n_beta = st.unrestricted ? p.n_beta : p.n_alpha;
    Rm.electronic_ev = st.o.electronic;
    Rm.core_ev = st.o.core;
    Rm.total_ev = st.o.electronic + st.o.core;
    Rm.heat_of_formation_kcal = (Rm.total_ev - e_isol + eheat) * kEvToKcal;
    Rm.iterations = st.o.iterations;
    Rm.converged = st.o.converged;
    Rm.unrestricted = st.unrestricted ? 1 : 0;
    Rm.scf_paths_tried = paths;
    Rm.scf_improvement_ev = std::max(first_ev - st.o.electronic, 0.0);
    Rm.last_change = st.o.last_change;
    Rm.homo_ev = st.o.homo;
    Rm.lumo_ev = st.o.lumo;
    Rm.has_homo = st.o.has_homo;
    Rm.has_lumo = st.o.has_lumo;
    for (int k = 0; k < 3; ++k) Rm.dipole_debye[k] = st.o.dipole[k];
    Rm.dipole_magnitude = std::sqrt(Rm.dipole_debye[0] * Rm.dipole_debye[0] + Rm.dipole_debye[1] * Rm.dipole_debye[1] +
                                    Rm.dipole_debye[2] * Rm.dipole_debye[2]);
    if (!st.o.converged) {
      Rm.status = PM3GPU_SCF_NOT_CONVERGED;
      char msg[160];
      std::snprintf(msg, sizeof msg, "PM3 SCF did not converge after %d iterations (error=%.3e)", st.o.iterations,
                    st.o.last_change);
      c->err = msg;
    }
    if (charges) std::memcpy(charges + p.atom0, R.charges.data() + st.job->charge_off, 8 * (size_t)p.natom);
    if (density && want.density) std::memcpy(density, R.dens.data() + st.job->dens_off, 8 * (size_t)p.nao * p.nao);
    if (all_dens && want.density && st.o.converged)
      std::memcpy(all_dens + all_dens_off[m], R.dens.data() + st.job->dens_off, 8 * (size_t)p.nao * p.nao);
    if (mo_energies && want.eps) std::memcpy(mo_energies, R.eps.data() + st.job->eps_off, 8 * (size_t)p.nao);
  }
  // ---------------------------------------------------------------- analytic gradients
  if (want.grad && gradients) {
    std::vector<GradMol> gm;
    std::vector<int32_t> ao_off(total_atoms, 0);
    long long pair0 = 0;
    for (int m = 0; m < n_mol; ++m) {
      const MolPlan& p = plans[m];
      if (p.status != PM3GPU_OK || p.large || !chosen[m].o.converged) continue;
      int off = 0;
      for (int a = 0; a < p.natom; ++a) {
        ao_off[p.atom0 + a] = off;
        off += c->h_elem[h_z[p.atom0 + a]].norb;
      }
      GradMol g{};
      g.atom0 = p.atom0;
      g.natom = p.natom;
      g.nao = p.nao;
      // a collapsed (spin-pure) unrestricted state takes the restricted gradient
      g.uhf = chosen[m].unrestricted ? 1 : 0;
      if ((chosen[m].job->flags & kJobUhf) == 0) g.uhf = 0;
      g.pair0 = pair0;
      g.dens_off = chosen[m].job->dens_off;
      pair0 += (long long)p.natom * (p.natom - 1) / 2;
      gm.push_back(g);
    }
    std::vector<double> gr;
    rc = launch_gradients(c, gm, ao_off, dz, dxyz, (size_t)total_atoms, gr);
    if (rc != PM3GPU_OK) return rc;
    for (int m = 0; m < n_mol; ++m) {
      const MolPlan& p = plans[m];
      if (p.status != PM3GPU_OK || p.large || !chosen[m].o.converged) continue;
      std::memcpy(gradients + 3 * (size_t)p.atom0, gr.data() + 3 * (size_t)p.atom0, 24 * (size_t)p.natom);
    }
  }
  // ---------------------------------------------------------------- post-SCF corrections
  if (corr.any) {
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));  // long done: enqueued ahead of the SCF
    apply_corrections(c, n_mol, h_offs, h_z, corr, results, want.grad ? gradients : nullptr);
  }
  cudaEventRecord(c->ev[3], c->stream);
  cudaEventRecord(c->ev[4], c->stream);
  cudaEventSynchronize(c->ev[4]);
  float ms[4];
  cudaEventElapsedTime(&ms[0], c->ev[0], c->ev[1]);
  cudaEventElapsedTime(&ms[1], c->ev[1], c->ev[2]);
  cudaEventElapsedTime(&ms[2], c->ev[2], c->ev[3]);
  cudaEventElapsedTime(&ms[3], c->ev[0], c->ev[4]);
  c->timings[0] = ms[0];
  c->timings[1] = ms[1];
  c->timings[2] = ms[2];
  c->timings[4] = ms[3];
  return PM3GPU_OK;
}

#include "geom_opt.cuh"
#include "hessian.cuh"

#include "autotune.cuh"

}  // namespace

// ====================================================================== C ABI
extern "C" {

void pm3gpu_default_options(pm3gpu_options* o) {  // scf.rs:259-287
  o->charge = 0.0;
  o->multiplicity = 1;
  o->max_scf = 200;
  o->e_tol = 1.0e-8;
  o->p_tol = 1.0e-7;
  o->use_diis = 1;
  o->accelerator = PM3GPU_ACCEL_ADIIS_CDIIS;
  o->adiis_switch = 0.1;
  o->reference = PM3GPU_REF_AUTO;
  o->guess = PM3GPU_GUESS_AUTO;
  o->stability = PM3GPU_STABILITY_AUTO;
  o->level_shift_ev = 0.0;
  o->damping = 0.0;
  o->scf_memory_mb = 512;
  o->variant = PM3GPU_VARIANT_PM3;
  o->mmok = 0;
}

int pm3gpu_supported_element(int z) { return supported(z) ? 1 : 0; }

int pm3gpu_standard_parameters(pm3gpu_element* elems, int max_elems, int* n_elems, pm3gpu_pair* pairs, int max_pairs,
                               int* n_pairs) {
  if (max_elems < 0 || max_pairs < 0 || (max_elems > 0 && !elems) || (max_pairs > 0 && !pairs))
    return fail(nullptr, PM3GPU_INVALID_INPUT, "bad argument");
  ElemDev el[kMaxZ];
  derive_elements(el, nullptr);
  int ne = 0;
  for (int z = 1; z < kMaxZ; ++z)
    if (supported(z) && el[z].z == z) {
      if (ne < max_elems) elem_to_public(el[z], elems[ne]);
      ++ne;
    }
  int np = 0;
  for (int k = 0; k < PM3_N_RAW_PAIRS; ++k) {
    const Pm3RawPair& r = PM3_RAW_PAIRS[k];
    if (!supported(r.zi) || !supported(r.zj)) continue;
    if (np < max_pairs) pairs[np] = pm3gpu_pair{r.zi, r.zj, r.alpb, r.xfac};
    ++np;
  }
  if (n_elems) *n_elems = ne;
  if (n_pairs) *n_pairs = np;
  return (ne > max_elems || np > max_pairs) ? fail(nullptr, PM3GPU_RESOURCE_LIMIT, "output arrays too small")
                                            : PM3GPU_OK;
}

int pm3gpu_set_parameters(pm3gpu_ctx* c, const pm3gpu_element* elems, int n_elems, const pm3gpu_pair* pairs,
                          int n_pairs) {
  if (!c || n_elems < 0 || n_pairs < 0 || (n_elems > 0 && !elems) || (n_pairs > 0 && !pairs))
    return fail(c, PM3GPU_INVALID_INPUT, "bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  ElemDev el[kMaxZ];
  for (int z = 0; z < kMaxZ; ++z) el[z] = ElemDev{};
  std::string why;
  for (int k = 0; k < n_elems; ++k) {
    ElemDev e;
    if (!elem_from_public(elems[k], e, why)) return fail(c, PM3GPU_INVALID_INPUT, why);
    if (el[e.z].z != 0) return fail(c, PM3GPU_INVALID_INPUT, "parameter set: Z=" + std::to_string(e.z) + " twice");
    el[e.z] = e;
  }
  PairDev P{};
  for (int k = 0; k < n_pairs; ++k) {
    const pm3gpu_pair& q = pairs[k];
    if (!supported(q.zi) || !supported(q.zj) || !std::isfinite(q.alpha) || !std::isfinite(q.x))
      return fail(c, PM3GPU_INVALID_INPUT, "parameter set: bad pair entry " + std::to_string(k));
    pair_to_dev(q.zi, q.zj, q.alpha, q.x, P);
  }
  CUDA_TRY(c, cudaSetDevice(c->device));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  CUDA_TRY(c, cudaMemcpy(c->elem.p, el, sizeof(el), cudaMemcpyHostToDevice));
  CUDA_TRY(c, cudaMemcpy(c->pairs.p, &P, sizeof(PairDev), cudaMemcpyHostToDevice));
  std::memcpy(c->h_elem, el, sizeof(el));
  c->h_pairs = P;
  c->err.clear();
  return PM3GPU_OK;
}

int pm3gpu_result_sizes(int n_atoms, const int32_t* z, int* nao) {
  ElemDev el[kMaxZ];
  derive_elements(el, nullptr);
  int s = 0;
  for (int a = 0; a < n_atoms; ++a) {
    if (!supported(z[a])) {
      if (nao) *nao = -1;
      return -1;
    }
    s += el[z[a]].norb;
  }
  if (nao) *nao = s;
  return s;
}

int pm3gpu_context_create(int device, pm3gpu_ctx** out) {
  if (!out) return PM3GPU_INVALID_INPUT;
  *out = nullptr;
  pm3gpu_ctx* c = new pm3gpu_ctx();
  c->device = device;
  auto bail = [&](cudaError_t e) {
    if (c->h_gerr) cudaFreeHost(c->h_gerr);
  if (c->h_corr) cudaFreeHost(c->h_corr);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    (void)e;
    return PM3GPU_CUDA_ERROR;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return bail(e);
  if ((e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking)) != cudaSuccess) return bail(e);
  c->stream = c->own;
  for (int k = 0; k < 6; ++k)
    if ((e = cudaEventCreate(&c->ev[k])) != cudaSuccess) return bail(e);
  for (int k = 0; k < 2; ++k)
    if ((e = cudaEventCreate(&c->kev[k])) != cudaSuccess || (e = cudaEventCreate(&c->gev[k])) != cudaSuccess)
      return bail(e);
  cudaDeviceProp prop;
  if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) return bail(e);
  c->sms = prop.multiProcessorCount;
  // The dynamic shared-memory limit is an attribute of the kernel for the whole process, not of
  // one context: it is raised once to the most the device allows beside the kernel's static shared
  // memory, so that concurrent contexts never lower it under one another's launches (each launch
  // asks for its own layout's bytes, which make_layout keeps within the same budget).
  cudaFuncAttributes fa{};
  if ((e = cudaFuncGetAttributes(&fa, scf_batch_kernel)) != cudaSuccess) return bail(e);
  c->smem_optin = (int)prop.sharedMemPerBlockOptin - (int)fa.sharedSizeBytes;
  g_scf_static_smem = std::max(512, (int)fa.sharedSizeBytes);
  c->smem_per_sm = (int)prop.sharedMemPerMultiprocessor;
  if ((e = cudaFuncSetAttribute(scf_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, c->smem_optin)) !=
      cudaSuccess)
    return bail(e);
  if ((e = cudaHostAlloc(reinterpret_cast<void**>(&c->h_gerr), sizeof(int), cudaHostAllocDefault)) != cudaSuccess)
    return bail(e);
  *c->h_gerr = 0;
  derive_elements(c->h_elem, &c->h_pairs);
  noalloc_forget(device);
  {
    const char* pe = std::getenv("PM3GPU_PROFILE");
    c->profile = pe && pe[0] && pe[0] != '0';
    const char* pc = std::getenv("PM3GPU_COOP_PANELS");
    c->coop_panels = !(pc && pc[0] == '0');
  }
  if ((e = c->elem.ensure(sizeof(c->h_elem))) != cudaSuccess) return bail(e);
  if ((e = c->pairs.ensure(sizeof(PairDev))) != cudaSuccess) return bail(e);
  if ((e = cudaMemcpy(c->elem.p, c->h_elem, sizeof(c->h_elem), cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e);
  if ((e = cudaMemcpy(c->pairs.p, &c->h_pairs, sizeof(PairDev), cudaMemcpyHostToDevice)) != cudaSuccess) return bail(e);
  *out = c;
  return PM3GPU_OK;
}

void pm3gpu_context_destroy(pm3gpu_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (DevBuf* b : {&c->elem, &c->pairs, &c->z, &c->xyz, &c->jobs, &c->out, &c->charges, &c->dens, &c->grads, &c->eps,
                    &c->work, &c->queue, &c->prof, &c->rq, &c->gmols, &c->aooff, &c->help})
    b->release();
  for (int k = 0; k < 6; ++k)
    if (c->ev[k]) cudaEventDestroy(c->ev[k]);
  for (int k = 0; k < 2; ++k) {
    if (c->kev[k]) cudaEventDestroy(c->kev[k]);
    if (c->gev[k]) cudaEventDestroy(c->gev[k]);
  }
  if (c->lbuf) {
    c->lbuf->release();
    delete c->lbuf;
  }
  c->lsel.release();
  for (DevBuf& b : c->tcbuf) b.release();
  for (DevBuf* b : {&c->gp, &c->gpb, &c->gm, &c->gv, &c->gg, &c->gqmols, &c->gatom, &c->gao, &c->gcoord, &c->gX, &c->gY,
                    &c->gZ[0], &c->gZ[1], &c->gZ[2], &c->gH[0], &c->gH[1], &c->gH[2], &c->gdH, &c->gdZ, &c->gT, &c->gM,
                    &c->gidx, &c->gXb, &c->gTb, &c->gMb, &c->gdY, &c->gpart, &c->gguess, &c->gdens, &c->gwt, &c->gerr,
                    &c->d3buf})
    b->release();
  if (c->h_gerr) cudaFreeHost(c->h_gerr);
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
}

const char* pm3gpu_last_error_message(pm3gpu_ctx* c) { return c ? c->err.c_str() : t_noctx_err.c_str(); }

int pm3gpu_set_stream(pm3gpu_ctx* c, void* stream) {
  if (!c) return PM3GPU_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(c->mu);
  c->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : c->own;
  return PM3GPU_OK;
}

int pm3gpu_single_point(pm3gpu_ctx* c, int n_atoms, const int32_t* z, const double* xyz, const pm3gpu_options* opts,
                        pm3gpu_result* result, double* charges, double* density, double* mo_energies) {
  if (!c || !z || !xyz || !result || !charges) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->err.clear();
  pm3gpu_options d;
  pm3gpu_default_options(&d);
  const int32_t offs[2] = {0, n_atoms};
  Want w;
  w.density = density != nullptr;
  w.eps = mo_energies != nullptr;
  int rc = run_batch(c, 1, offs, z, xyz, nullptr, nullptr, opts ? opts : &d, 0, w, result, charges, nullptr, density,
                     mo_energies);
  if (rc != PM3GPU_OK) {
    result->status = rc;
    return rc;
  }
  return result->status;
}

int pm3gpu_gradient(pm3gpu_ctx* c, int n_atoms, const int32_t* z, const double* xyz, const pm3gpu_options* opts,
                    pm3gpu_result* result, double* charges, double* gradient) {
  if (!c || !z || !xyz || !result || !charges || !gradient) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->err.clear();
  pm3gpu_options d;
  pm3gpu_default_options(&d);
  const int32_t offs[2] = {0, n_atoms};
  Want w;
  w.grad = true;
  int rc = run_batch(c, 1, offs, z, xyz, nullptr, nullptr, opts ? opts : &d, 0, w, result, charges, gradient, nullptr,
                     nullptr);
  if (rc != PM3GPU_OK) {
    result->status = rc;
    return rc;
  }
  return result->status;
}

int pm3gpu_batch(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, const double* xyz,
                 const pm3gpu_options* opts, int per_mol, pm3gpu_result* results, double* charges, double* gradients) {
  if (!c || n_mol < 0 || !offs || !z || !xyz || !results || !charges) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->err.clear();
  pm3gpu_options d;
  pm3gpu_default_options(&d);
  Want w;
  w.grad = gradients != nullptr;
  return run_batch(c, n_mol, offs, z, xyz, nullptr, nullptr, opts ? opts : &d, opts ? per_mol : 0, w, results, charges,
                   gradients, nullptr, nullptr);
}

void pm3gpu_default_opt_options(pm3gpu_opt_options* o) {
  if (!o) return;
  o->max_iter = 200;
  o->gtol = 1.0e-3;
  o->history = 8;
}

int pm3gpu_optimize_batch(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, double* xyz,
                          const pm3gpu_options* opts, const pm3gpu_opt_options* opt, pm3gpu_opt_result* out,
                          double* gradients) {
  if (!c || n_mol < 0 || !offs || !z || !xyz || !out) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  pm3gpu_opt_options o;
  pm3gpu_default_opt_options(&o);
  if (opt) o = *opt;
  if (o.max_iter < 0 || o.history < 0 || !(o.gtol >= 0.0)) return fail(c, PM3GPU_INVALID_INPUT, "bad optimizer options");
  for (int m = 0; m < n_mol; ++m)
    if (offs[m + 1] < offs[m]) return fail(c, PM3GPU_INVALID_INPUT, "atom_offsets must be non-decreasing");
  for (long long k = 0; k < 3LL * offs[n_mol]; ++k)
    if (!std::isfinite(xyz[k])) return fail(c, PM3GPU_INVALID_INPUT, "non-finite coordinate");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->err.clear();
  pm3gpu_options d;
  pm3gpu_default_options(&d);
  return optimize_batch(c, n_mol, offs, z, xyz, opts ? opts : &d, o, out, gradients);
}

int pm3gpu_d3_batch(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, const double* xyz, int d3_set,
                    double* energies, double* gradients) {
  if (!c || n_mol < 0 || !offs || !z || !xyz || !energies) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  if (d3_set != 1 && d3_set != 2) return fail(c, PM3GPU_INVALID_INPUT, "d3_set must be 1 (PM3-D3) or 2 (PM3-D3H4)");
  if (offs[0] != 0) return fail(c, PM3GPU_INVALID_INPUT, "atom_offsets must start at 0");
  for (int m = 0; m < n_mol; ++m)
    if (offs[m + 1] < offs[m]) return fail(c, PM3GPU_INVALID_INPUT, "atom_offsets must be non-decreasing");
  const int total = offs[n_mol];
  for (long long k = 0; k < 3LL * total; ++k)
    if (!std::isfinite(xyz[k])) return fail(c, PM3GPU_INVALID_INPUT, "non-finite coordinate");
  for (int a = 0; a < total; ++a)  // the device tables hold the s/p elements only
    if (!supported(z[a])) return fail(c, PM3GPU_UNSUPPORTED, "unsupported element Z=" + std::to_string(z[a]));
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->err.clear();
  c->launches = 0;
  std::fill(energies, energies + n_mol, 0.0);
  if (gradients) std::fill(gradients, gradients + 3 * (size_t)total, 0.0);
  if (n_mol == 0 || total == 0) return PM3GPU_OK;
  CUDA_TRY(c, c->z.ensure(4 * (size_t)total));
  CUDA_TRY(c, c->xyz.ensure(24 * (size_t)total));
  CUDA_TRY(c, cudaMemcpyAsync(c->z.p, z, 4 * (size_t)total, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->xyz.p, xyz, 24 * (size_t)total, cudaMemcpyHostToDevice, c->stream));
  std::vector<int32_t> set(n_mol, d3_set), var(n_mol, 0);
  std::vector<double> parts(5 * (size_t)n_mol, 0.0);
  const int rc = corrections_batch(c, n_mol, offs, set.data(), var.data(), nullptr, c->z.as<int32_t>(),
                                   c->xyz.as<double>(), parts.data(), gradients);
  for (int m = 0; m < n_mol; ++m) energies[m] = parts[5 * (size_t)m];
  return rc;
}

int pm3gpu_corrections_batch(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, const double* xyz,
                             int variant, double* parts, double* gradients) {
  if (!c || n_mol < 0 || !offs || !z || !xyz || !parts) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  if (variant < PM3GPU_VARIANT_D3 || variant > PM3GPU_VARIANT_D3H4X)
    return fail(c, PM3GPU_INVALID_INPUT, "variant must be PM3-D3, PM3-D3H4 or PM3-D3H4X");
  if (offs[0] != 0) return fail(c, PM3GPU_INVALID_INPUT, "atom_offsets must start at 0");
  for (int m = 0; m < n_mol; ++m)
    if (offs[m + 1] < offs[m]) return fail(c, PM3GPU_INVALID_INPUT, "atom_offsets must be non-decreasing");
  const int total = offs[n_mol];
  for (long long k = 0; k < 3LL * total; ++k)
    if (!std::isfinite(xyz[k])) return fail(c, PM3GPU_INVALID_INPUT, "non-finite coordinate");
  for (int a = 0; a < total; ++a)  // the device tables (D3, covalent radii, X pairs) hold the s/p elements only
    if (!supported(z[a])) return fail(c, PM3GPU_UNSUPPORTED, "unsupported element Z=" + std::to_string(z[a]));
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->err.clear();
  c->launches = 0;
  std::fill(parts, parts + 4 * (size_t)n_mol, 0.0);
  if (gradients) std::fill(gradients, gradients + 3 * (size_t)total, 0.0);
  if (n_mol == 0 || total == 0) return PM3GPU_OK;
  CUDA_TRY(c, c->z.ensure(4 * (size_t)total));
  CUDA_TRY(c, c->xyz.ensure(24 * (size_t)total));
  CUDA_TRY(c, cudaMemcpyAsync(c->z.p, z, 4 * (size_t)total, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->xyz.p, xyz, 24 * (size_t)total, cudaMemcpyHostToDevice, c->stream));
  std::vector<int32_t> set(n_mol, variant == PM3GPU_VARIANT_D3 ? 1 : 2), var(n_mol, variant);
  std::vector<double> p5(5 * (size_t)n_mol, 0.0);
  const int rc = corrections_batch(c, n_mol, offs, set.data(), var.data(), nullptr, c->z.as<int32_t>(),
                                   c->xyz.as<double>(), p5.data(), gradients);
  for (int m = 0; m < n_mol; ++m)
    for (int k = 0; k < 4; ++k) parts[4 * (size_t)m + k] = p5[5 * (size_t)m + k];
  return rc;
}

int pm3gpu_numerical_hessian_batch(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z,
                                   const double* xyz, const pm3gpu_options* opts, double step, double* hessians,
                                   int* status) {
  if (!c || n_mol < 0 || !offs || !z || !xyz || !hessians || !status) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  if (!(step > 0.0) || !std::isfinite(step)) return fail(c, PM3GPU_INVALID_INPUT, "step must be positive and finite");
  for (int m = 0; m < n_mol; ++m)
    if (offs[m + 1] < offs[m]) return fail(c, PM3GPU_INVALID_INPUT, "atom_offsets must be non-decreasing");
  for (long long k = 0; k < 3LL * offs[n_mol]; ++k)
    if (!std::isfinite(xyz[k])) return fail(c, PM3GPU_INVALID_INPUT, "non-finite coordinate");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->err.clear();
  pm3gpu_options d;
  pm3gpu_default_options(&d);
  return hessian_batch(c, n_mol, offs, z, xyz, opts ? opts : &d, step, hessians, status);
}

int pm3gpu_batch_device_inputs(pm3gpu_ctx* c, int n_mol, const int32_t* d_offs, const int32_t* d_z, const double* d_xyz,
                               const int32_t* h_offs, const int32_t* h_z, const pm3gpu_options* opts,
                               pm3gpu_result* results, double* charges, double* gradients) {
  if (!c || n_mol < 0 || !d_z || !d_xyz || !h_offs || !h_z || !results || !charges)
    return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  (void)d_offs;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->err.clear();
  pm3gpu_options d;
  pm3gpu_default_options(&d);
  Want w;
  w.grad = gradients != nullptr;
  return run_batch(c, n_mol, h_offs, h_z, nullptr, d_z, d_xyz, opts ? opts : &d, 0, w, results, charges, gradients,
                   nullptr, nullptr);
}

// build_core (hamiltonian.rs:174-344) and build_fock_spin (fock.rs:285-332) on the GPU, for
// element-by-element checks of the pair-integral and Fock kernels.
static int single_stage(pm3gpu_ctx* c, int n_atoms, const int32_t* z, const double* xyz, int flag, int uhf,
                        std::vector<double>& io, double* core_ev) {
  if (n_atoms < 1 || n_atoms > kMaxN) return fail(c, PM3GPU_INVALID_INPUT, "atom count outside 1..256");
  int nao = 0;
  for (int a = 0; a < n_atoms; ++a) {
    if (!has_elem(c, z[a])) return fail(c, PM3GPU_UNSUPPORTED, "unsupported element Z=" + std::to_string(z[a]));
    for (int k = 0; k < 3; ++k)
      if (!std::isfinite(xyz[3 * a + k])) return fail(c, PM3GPU_INVALID_INPUT, "non-finite coordinate");
    nao += c->h_elem[z[a]].norb;
  }
  if (nao > kMaxN) return fail(c, PM3GPU_UNSUPPORTED, "basis exceeds the per-CTA path");
  JobDesc j{};
  j.natom = n_atoms;
  j.nao = nao;
  j.flags = flag | (uhf ? kJobUhf : 0);
  j.guess = 1;
  j.depth = 2;
  j.dens_off = 0;
  std::vector<int32_t> zs(z, z + n_atoms);
  CUDA_TRY(c, c->z.ensure(4 * (size_t)n_atoms));
  CUDA_TRY(c, c->xyz.ensure(24 * (size_t)n_atoms));
  CUDA_TRY(c, cudaMemcpyAsync(c->z.p, z, 4 * (size_t)n_atoms, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->xyz.p, xyz, 24 * (size_t)n_atoms, cudaMemcpyHostToDevice, c->stream));
  c->launches = 0;
  Offsets tot;
  tot.charges = (size_t)n_atoms;
  tot.dens = io.size();
  LaunchOut R;
  int rc = launch_jobs(c, {j}, {}, zs, c->z.as<int32_t>(), c->xyz.as<double>(), tot, true, false, R, &io);
  if (rc != PM3GPU_OK) return rc;
  io.swap(R.dens);
  if (core_ev) *core_ev = R.out[0].core;
  return PM3GPU_OK;
}

int pm3gpu_core_hamiltonian(pm3gpu_ctx* c, int n_atoms, const int32_t* z, const double* xyz, double* h, double* core_ev) {
  if (!c || !z || !xyz || !h) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->err.clear();
  int nao = 0;
  if (pm3gpu_result_sizes(n_atoms, z, &nao) < 0) return fail(c, PM3GPU_UNSUPPORTED, "unsupported element");
  std::vector<double> io((size_t)nao * nao, 0.0);
  int rc = single_stage(c, n_atoms, z, xyz, kJobCoreOnly, 0, io, core_ev);
  if (rc != PM3GPU_OK) return rc;
  std::memcpy(h, io.data(), 8 * (size_t)nao * nao);
  return PM3GPU_OK;
}

int pm3gpu_fock(pm3gpu_ctx* c, int n_atoms, const int32_t* z, const double* xyz, const double* p_tot,
                const double* p_alpha, const double* p_beta, double* f_alpha, double* f_beta) {
  if (!c || !z || !xyz || !p_tot || !f_alpha) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  const int uhf = (p_alpha && p_beta && f_beta) ? 1 : 0;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaSetDevice(c->device);
  c->err.clear();
  int nao = 0;
  if (pm3gpu_result_sizes(n_atoms, z, &nao) < 0) return fail(c, PM3GPU_UNSUPPORTED, "unsupported element");
  const size_t nn = (size_t)nao * nao;
  std::vector<double> io(5 * nn, 0.0);
  std::memcpy(io.data(), p_tot, 8 * nn);
  if (uhf) {
    std::memcpy(io.data() + nn, p_alpha, 8 * nn);
    std::memcpy(io.data() + 2 * nn, p_beta, 8 * nn);
  }
  int rc = single_stage(c, n_atoms, z, xyz, kJobFockOnly, uhf, io, nullptr);
  if (rc != PM3GPU_OK) return rc;
  std::memcpy(f_alpha, io.data() + 3 * nn, 8 * nn);
  if (uhf) std::memcpy(f_beta, io.data() + 4 * nn, 8 * nn);
  return PM3GPU_OK;
}

int pm3gpu_last_timings(pm3gpu_ctx* c, double* ms, int max_entries) {
  if (!c || !ms) return 0;
  const int k = std::min(max_entries, 7);
  for (int i = 0; i < k; ++i) ms[i] = c->timings[i];
  return k;
}

int pm3gpu_last_kernel_launches(pm3gpu_ctx* c) { return c ? c->launches : 0; }

int pm3gpu_last_launch_layout(pm3gpu_ctx* c, int* ctas_per_sm, int* smem_matrix_n) {
  if (!c) return PM3GPU_INVALID_INPUT;
  if (ctas_per_sm) *ctas_per_sm = c->last_ctas;
  if (smem_matrix_n) *smem_matrix_n = c->last_nsm;
  return PM3GPU_OK;
}

int pm3gpu_last_large_phase_ms(pm3gpu_ctx* c, double* ms, int max_entries) {
  if (!c || !ms) return 0;
  const int k = std::min(max_entries, (int)kLgPhases);
  for (int i = 0; i < k; ++i) ms[i] = c->large_ms[i];
  return c->profile ? k : 0;
}

int pm3gpu_guess_set_params(pm3gpu_ctx* c, const float* params, int n_params) {
  if (!c || !params || n_params != guess::kParams) return fail(c, PM3GPU_INVALID_INPUT, "expected PM3GPU_GUESS_PARAMS floats");
  std::lock_guard<std::mutex> lk(c->mu);
  CUDA_TRY(c, cudaSetDevice(c->device));
  const size_t np = guess::kParams;
  CUDA_TRY(c, c->gp.ensure(4 * np));
  CUDA_TRY(c, c->gpb.ensure(2 * np));
  CUDA_TRY(c, c->gm.ensure(4 * np));
  CUDA_TRY(c, c->gv.ensure(4 * np));
  CUDA_TRY(c, cudaMemcpyAsync(c->gp.p, params, 4 * np, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->gm.p, 0, 4 * np, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->gv.p, 0, 4 * np, c->stream));
  guess::to_bf16_kernel<<<gblocks(np), 256, 0, c->stream>>>(c->gp.as<float>(), (int)np, c->gpb.as<__nv_bfloat16>());
  CUDA_TRY(c, cudaGetLastError());
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->adam_steps = 0;
  c->has_guess_model = true;
  return PM3GPU_OK;
}

int pm3gpu_guess_get_params(pm3gpu_ctx* c, float* params, int n_params) {
  if (!c || !params || n_params != guess::kParams) return fail(c, PM3GPU_INVALID_INPUT, "expected PM3GPU_GUESS_PARAMS floats");
  std::lock_guard<std::mutex> lk(c->mu);
  if (!c->has_guess_model) return fail(c, PM3GPU_INVALID_INPUT, "no learned guess model");
  CUDA_TRY(c, cudaSetDevice(c->device));
  CUDA_TRY(c, cudaMemcpyAsync(params, c->gp.p, 4 * (size_t)guess::kParams, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return PM3GPU_OK;
}

int pm3gpu_guess_predict(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, const double* xyz,
                         float* features, float* outputs) {
  using namespace guess;
  if (!c || n_mol < 1 || !offs || !z || !xyz) return fail(c, PM3GPU_INVALID_INPUT, "bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  CUDA_TRY(c, cudaSetDevice(c->device));
  if (!c->has_guess_model) return fail(c, PM3GPU_INVALID_INPUT, "no learned guess model");
  const int total_atoms = offs[n_mol];
  for (int a = 0; a < total_atoms; ++a)
    if (!has_elem(c, z[a])) return fail(c, PM3GPU_UNSUPPORTED, "unsupported element");
  std::vector<int> a0(n_mol), na(n_mol);
  for (int m = 0; m < n_mol; ++m) {
    a0[m] = offs[m];
    na[m] = offs[m + 1] - offs[m];
  }
  GuessRows G;
  guess_rows(c, a0, na, z, total_atoms, G);
  CUDA_TRY(c, c->z.ensure(4 * (size_t)total_atoms));
  CUDA_TRY(c, c->xyz.ensure(24 * (size_t)total_atoms));
  CUDA_TRY(c, cudaMemcpyAsync(c->z.p, z, 4 * (size_t)total_atoms, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->xyz.p, xyz, 24 * (size_t)total_atoms, cudaMemcpyHostToDevice, c->stream));
  int rc = guess_features(c, G, c->z.as<int32_t>(), c->xyz.as<double>(), total_atoms);
  if (rc != PM3GPU_OK) return rc;
  CUDA_TRY(c, c->gY.ensure(4 * (size_t)kOut * std::max<long long>(G.rows, 1)));
  rc = mlp_infer_all(c, c->gX.as<__nv_bfloat16>(), G.rows, c->gY.as<float>());
  if (rc != PM3GPU_OK) return rc;
  if (outputs)
    CUDA_TRY(c, cudaMemcpyAsync(outputs, c->gY.p, 4 * (size_t)kOut * G.rows, cudaMemcpyDeviceToHost, c->stream));
  std::vector<__nv_bfloat16> xb;
  if (features) {
    xb.resize((size_t)kIn * G.rows);
    CUDA_TRY(c, cudaMemcpyAsync(xb.data(), c->gX.p, 2 * xb.size(), cudaMemcpyDeviceToHost, c->stream));
  }
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (infer_failed(c)) return fail(c, PM3GPU_CUDA_ERROR, "learned guess: a pipeline wait in the tcgen05 layer kernel ran out");
  for (size_t k = 0; k < xb.size(); ++k) features[k] = __bfloat162float(xb[k]);
  return PM3GPU_OK;
}

int pm3gpu_guess_train(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, const double* xyz,
                       const pm3gpu_options* opts, int epochs, int batch, float lr, unsigned seed, float* losses) {
  using namespace guess;
  if (!c || n_mol < 1 || !offs || !z || !xyz || epochs < 0 || batch < 64) return fail(c, PM3GPU_INVALID_INPUT, "bad argument");
  std::unique_lock<std::mutex> lk(c->mu);
  CUDA_TRY(c, cudaSetDevice(c->device));
  c->err.clear();
  pm3gpu_options o;
  if (opts) o = *opts;
  else pm3gpu_default_options(&o);
  if (o.guess == PM3GPU_GUESS_LEARNED) o.guess = PM3GPU_GUESS_AUTO;  // targets come from the plain SCF
  const int total_atoms = offs[n_mol];
  // 1. plain SCF of every molecule, converged densities kept
  std::vector<size_t> doff(n_mol);
  size_t dtot = 0;
  std::vector<int> nao(n_mol);
  for (int m = 0; m < n_mol; ++m) {
    int k = 0;
    for (int a = offs[m]; a < offs[m + 1]; ++a) k += has_elem(c, z[a]) ? c->h_elem[z[a]].norb : 0;
    nao[m] = k;
    doff[m] = dtot;
    dtot += (size_t)k * k;
  }
  std::vector<double> dens(std::max<size_t>(dtot, 1), 0.0);
  std::vector<pm3gpu_result> res(n_mol);
  std::vector<double> q(std::max(total_atoms, 1));
  Want w;
  w.density = true;
  int rc = run_batch(c, n_mol, offs, z, xyz, nullptr, nullptr, &o, 0, w, res.data(), q.data(), nullptr, nullptr, nullptr,
                     dens.data(), doff.data());
  if (rc != PM3GPU_OK) return rc;
  // 2. training rows: the converged molecules below one CTA's size
  std::vector<int> a0, na, keep;
  for (int m = 0; m < n_mol; ++m)
    if (res[m].status == PM3GPU_OK && res[m].converged && nao[m] <= kMaxN) {
      a0.push_back(offs[m]);
      na.push_back(offs[m + 1] - offs[m]);
      keep.push_back(m);
    }
  if (keep.empty()) return fail(c, PM3GPU_INVALID_INPUT, "no converged training molecule");
  GuessRows G;
  guess_rows(c, a0, na, z, total_atoms, G);
  std::vector<double> packed(std::max<size_t>(G.dens_total, 1));
  for (size_t k = 0; k < keep.size(); ++k)
    std::memcpy(packed.data() + G.mols[k].dens_off, dens.data() + doff[keep[k]], 8 * (size_t)G.mols[k].nao * G.mols[k].nao);
  CUDA_TRY(c, c->z.ensure(4 * (size_t)total_atoms));
  CUDA_TRY(c, c->xyz.ensure(24 * (size_t)total_atoms));
  CUDA_TRY(c, cudaMemcpyAsync(c->z.p, z, 4 * (size_t)total_atoms, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->xyz.p, xyz, 24 * (size_t)total_atoms, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, c->gdens.ensure(8 * packed.size()));
  CUDA_TRY(c, cudaMemcpyAsync(c->gdens.p, packed.data(), 8 * packed.size(), cudaMemcpyHostToDevice, c->stream));
  rc = guess_features(c, G, c->z.as<int32_t>(), c->xyz.as<double>(), total_atoms);
  if (rc != PM3GPU_OK) return rc;
  const long long rows = G.rows;
  CUDA_TRY(c, c->gT.ensure(4 * (size_t)kOut * rows));
  CUDA_TRY(c, c->gM.ensure(4 * (size_t)kOut * rows));
  targets_kernel<<<gblocks(rows), 256, 0, c->stream>>>(c->gqmols.as<Mol>(), (int)G.mols.size(), c->elem.as<ElemDev>(),
                                                        c->z.as<int32_t>(), c->xyz.as<double>(), c->gao.as<int>(),
                                                        c->gdens.as<double>(), rows, c->gT.as<float>(), c->gM.as<float>());
  CUDA_TRY(c, cudaGetLastError());
  // masked entries per row on average (normalises the loss gradient)
  double mask_total = 0.0;
  for (size_t k = 0; k < keep.size(); ++k) {
    long long h = 0, l = 0;
    for (int a = 0; a < G.mols[k].natom; ++a) (c->h_elem[z[G.mols[k].atom0 + a]].norb == 4 ? h : l) += 1;
    mask_total += 3.0 * h + l + 5.0 * h * (h - 1) / 2 + 2.0 * h * l + 1.0 * l * (l - 1) / 2;
  }
  const double mask_per_row = mask_total / (double)rows;
  // 3. parameters (Xavier-uniform, seeded) unless the context already has a model
  const size_t np = kParams;
  if (!c->has_guess_model) {
    std::vector<float> init(np, 0.0f);
    std::mt19937 gen(seed);
    auto fill = [&](int off, int fin, int fout) {
      const float lim = std::sqrt(6.0f / (float)(fin + fout));
      std::uniform_real_distribution<float> U(-lim, lim);
      for (int k = 0; k < fin * fout; ++k) init[off + k] = U(gen);
    };
    fill(kW1, kIn, kHid);
    fill(kW2, kHid, kHid);
    fill(kW3, kHid, kHid);
    fill(kW4, kHid, kOut);
    lk.unlock();
    rc = pm3gpu_guess_set_params(c, init.data(), (int)np);
    lk.lock();
    if (rc != PM3GPU_OK) return rc;
  }
  CUDA_TRY(c, c->gg.ensure(4 * np));
  const int B = batch;
  CUDA_TRY(c, c->gidx.ensure(8 * (size_t)rows));
  CUDA_TRY(c, c->gXb.ensure(2 * (size_t)kIn * B));
  CUDA_TRY(c, c->gTb.ensure(4 * (size_t)kOut * B));
  CUDA_TRY(c, c->gMb.ensure(4 * (size_t)kOut * B));
  CUDA_TRY(c, c->gY.ensure(4 * (size_t)kOut * B));
  CUDA_TRY(c, c->gdY.ensure(2 * (size_t)kOut * B));
  CUDA_TRY(c, c->gdH.ensure(4 * (size_t)kHid * B));
  CUDA_TRY(c, c->gdZ.ensure(2 * (size_t)kHid * B));
  CUDA_TRY(c, c->gpart.ensure(4 * 1024));
  CUDA_TRY(c, cudaMemsetAsync(c->gpart.p, 0, 4 * 1024, c->stream));
  std::vector<long long> idx(rows);
  for (long long r = 0; r < rows; ++r) idx[r] = r;
  std::mt19937_64 shuf(seed ^ 0x9e3779b97f4a7c15ull);
  float* gp = c->gp.as<float>();
  float* gg = c->gg.as<float>();
  const int nbatch = (int)(rows / B);
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(idx.begin(), idx.end(), shuf);
    CUDA_TRY(c, cudaMemcpyAsync(c->gidx.p, idx.data(), 8 * (size_t)rows, cudaMemcpyHostToDevice, c->stream));
    float* accum = c->gpart.as<float>() + (ep % 1024);
    for (int bi = 0; bi < nbatch; ++bi) {
      gather_rows_kernel<<<gblocks((long long)B * kIn), 256, 0, c->stream>>>(
          c->gidx.as<long long>() + (size_t)bi * B, B, c->gX.as<__nv_bfloat16>(), c->gT.as<float>(), c->gM.as<float>(),
          c->gXb.as<__nv_bfloat16>(), c->gTb.as<float>(), c->gMb.as<float>());
      rc = mlp_loss_grad(c, c->gXb.as<__nv_bfloat16>(), c->gTb.as<float>(), c->gMb.as<float>(), B,
                         (float)(1.0 / (mask_per_row * B)), accum);
      if (rc != PM3GPU_OK) return rc;
      ++c->adam_steps;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.0f - std::pow(b1, (float)c->adam_steps), c2 = 1.0f - std::pow(b2, (float)c->adam_steps);
      adam_kernel<<<gblocks(np), 256, 0, c->stream>>>(gp, gg, c->gm.as<float>(), c->gv.as<float>(), (int)np, lr, b1, b2,
                                                      c1, c2, c->gpb.as<__nv_bfloat16>());
      CUDA_TRY(c, cudaGetLastError());
    }
    if (losses) {
      float sum = 0.0f;
      CUDA_TRY(c, cudaMemcpyAsync(&sum, accum, 4, cudaMemcpyDeviceToHost, c->stream));
      CUDA_TRY(c, cudaStreamSynchronize(c->stream));
      losses[ep] = (float)(sum / (mask_per_row * (double)nbatch * B));
    }
  }
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return PM3GPU_OK;
}

int pm3gpu_guess_gradients(pm3gpu_ctx* c, int rows, const float* features, const float* targets, const float* mask,
                           float inv_count, float* loss, float* grads) {
  using namespace guess;
  if (!c || rows < 1 || !features || !targets || !mask || !grads || !std::isfinite(inv_count))
    return fail(c, PM3GPU_INVALID_INPUT, "bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  CUDA_TRY(c, cudaSetDevice(c->device));
  c->err.clear();
  if (!c->has_guess_model) return fail(c, PM3GPU_INVALID_INPUT, "no learned guess model");
  c->launches = 0;
  const size_t B = (size_t)rows;
  std::vector<__nv_bfloat16> xb(B * kIn);
  for (size_t k = 0; k < xb.size(); ++k) xb[k] = __float2bfloat16(features[k]);
  CUDA_TRY(c, c->gXb.ensure(2 * kIn * B));
  CUDA_TRY(c, c->gTb.ensure(4 * kOut * B));
  CUDA_TRY(c, c->gMb.ensure(4 * kOut * B));
  CUDA_TRY(c, c->gY.ensure(4 * kOut * B));
  CUDA_TRY(c, c->gdY.ensure(2 * kOut * B));
  CUDA_TRY(c, c->gdH.ensure(4 * kHid * B));
  CUDA_TRY(c, c->gdZ.ensure(2 * kHid * B));
  CUDA_TRY(c, c->gg.ensure(4 * (size_t)kParams));
  CUDA_TRY(c, c->gpart.ensure(4 * 1024));
  CUDA_TRY(c, cudaMemcpyAsync(c->gXb.p, xb.data(), 2 * kIn * B, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->gTb.p, targets, 4 * kOut * B, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(c->gMb.p, mask, 4 * kOut * B, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->gpart.p, 0, 4, c->stream));
  int rc = mlp_loss_grad(c, c->gXb.as<__nv_bfloat16>(), c->gTb.as<float>(), c->gMb.as<float>(), rows, inv_count,
                         c->gpart.as<float>());
  if (rc != PM3GPU_OK) return rc;
  float l = 0.0f;
  CUDA_TRY(c, cudaMemcpyAsync(&l, c->gpart.p, 4, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(grads, c->gg.p, 4 * (size_t)kParams, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (loss) *loss = l * inv_count;
  return PM3GPU_OK;
}

int pm3gpu_autotune(pm3gpu_ctx* c, int n_mol, const int32_t* offs, const int32_t* z, const double* xyz,
                    const pm3gpu_options* opts, const char* cache_path) {
  if (!c || n_mol < 1 || !offs || !z || !xyz) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  CUDA_TRY(c, cudaSetDevice(c->device));
  c->err.clear();
  for (int m = 0; m < n_mol; ++m)
    if (offs[m + 1] < offs[m]) return fail(c, PM3GPU_INVALID_INPUT, "atom offsets must not decrease");
  pm3gpu_options d;
  pm3gpu_default_options(&d);
  int rc = tune_batch_part(c, n_mol, offs, z, xyz, opts ? opts : &d);
  if (rc == PM3GPU_OK) rc = tune_large_part(c, n_mol, offs, z, xyz);
  if (rc == PM3GPU_OK && cache_path) rc = write_tuning(c, cache_path);
  return rc;
}

int pm3gpu_load_tuning(pm3gpu_ctx* c, const char* path) {
  if (!path) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  if (!c) return read_tuning(nullptr, path);  // check the file only
  std::lock_guard<std::mutex> lk(c->mu);
  return read_tuning(c, path);
}

int pm3gpu_tuning_choice(pm3gpu_ctx* c, int kind, int size) {
  if (!c) return -1;
  std::lock_guard<std::mutex> lk(c->mu);
  if (kind == 0) return tune_lookup(c->tune_batch, size, -1);
  if (kind == 1) return tune_lookup(c->tune_large, size, -1);
  return -1;
}

int pm3gpu_set_precision(pm3gpu_ctx* c, int mode) {
  if (!c) return PM3GPU_INVALID_INPUT;
  if (mode != PM3GPU_PRECISION_FP64 && mode != PM3GPU_PRECISION_MIXED)
    return fail(c, PM3GPU_INVALID_INPUT, "precision must be PM3GPU_PRECISION_FP64 or PM3GPU_PRECISION_MIXED");
  std::lock_guard<std::mutex> lk(c->mu);
  c->precision = mode;
  return PM3GPU_OK;
}

int pm3gpu_last_large_trace(pm3gpu_ctx* c, double* rows, int max_rows) {
  if (!c) return 0;
  std::lock_guard<std::mutex> lk(c->mu);
  const int total = (int)(c->ltrace.size() / 5);
  if (rows && max_rows > 0) std::copy_n(c->ltrace.begin(), 5 * (size_t)std::min(total, max_rows), rows);
  return total;
}

int pm3gpu_split_gemm(pm3gpu_ctx* c, int m, int n, int k, const double* a, int lda, const double* b, int ldb,
                      float* out) {
  if (!c || m < 1 || n < 1 || k < 1 || !a || !b || !out || lda < k || ldb < k)
    return fail(c, PM3GPU_INVALID_INPUT, "bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  CUDA_TRY(c, cudaSetDevice(c->device));
  c->err.clear();
  c->launches = 0;
  const int ldp = (k + 7) & ~7;
  DevBuf* B = c->tcbuf;
  CUDA_TRY(c, B[0].ensure(8 * (size_t)m * lda));
  CUDA_TRY(c, B[1].ensure(8 * (size_t)n * ldb));
  for (int q = 0; q < 2; ++q) CUDA_TRY(c, B[2 + q].ensure(2 * (size_t)m * ldp));
  for (int q = 0; q < 2; ++q) CUDA_TRY(c, B[4 + q].ensure(2 * (size_t)n * ldp));
  CUDA_TRY(c, B[6].ensure(4 * (size_t)m * n + 256));
  CUDA_TRY(c, cudaMemcpyAsync(B[0].p, a, 8 * (size_t)m * lda, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(B[1].p, b, 8 * (size_t)n * ldb, cudaMemcpyHostToDevice, c->stream));
  int* derr = reinterpret_cast<int*>(B[6].as<char>() + 4 * (size_t)m * n);
  CUDA_TRY(c, cudaMemsetAsync(derr, 0, sizeof(int), c->stream));
  auto blocks = [](size_t cnt) { return (unsigned)std::min<size_t>((cnt + 255) / 256, 65535); };
  large::split_pad_kernel<<<blocks((size_t)m * ldp), large::kBlock, 0, c->stream>>>(
      B[0].as<double>(), m, k, lda, B[2].as<__nv_bfloat16>(), B[3].as<__nv_bfloat16>(), ldp);
  large::split_pad_kernel<<<blocks((size_t)n * ldp), large::kBlock, 0, c->stream>>>(
      B[1].as<double>(), n, k, ldb, B[4].as<__nv_bfloat16>(), B[5].as<__nv_bfloat16>(), ldp);
  CUDA_TRY(c, cudaGetLastError());
  if (!tc::launch_split_gemm(m, n, k, B[2].as<__nv_bfloat16>(), B[3].as<__nv_bfloat16>(), ldp,
                             B[4].as<__nv_bfloat16>(), B[5].as<__nv_bfloat16>(), ldp, B[6].as<float>(), n, derr,
                             c->stream))
    return fail(c, PM3GPU_CUDA_ERROR, "split-BF16 GEMM: tensor map or kernel attribute could not be set");
  c->launches = 3;
  CUDA_TRY(c, cudaGetLastError());
  int flag = 0;
  CUDA_TRY(c, cudaMemcpyAsync(out, B[6].p, 4 * (size_t)m * n, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(&flag, derr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (flag) return fail(c, PM3GPU_CUDA_ERROR, "split-BF16 GEMM: a pipeline wait in the kernel ran out");
  return PM3GPU_OK;
}

int pm3gpu_dgemm(pm3gpu_ctx* c, int trans_a, int trans_b, int m, int n, int k, double alpha, const double* a, int lda,
                 const double* b, int ldb, double beta, double* cm, int ldc) {
  if (!c || m < 1 || n < 1 || k < 0 || !a || !b || !cm) return fail(c, PM3GPU_INVALID_INPUT, "bad argument");
  const long long ra = trans_a ? k : m, ca = trans_a ? m : k;  // stored shapes, column-major
  const long long rb = trans_b ? n : k, cb = trans_b ? k : n;
  if (lda < std::max<long long>(1, ra) || ldb < std::max<long long>(1, rb) || ldc < m)
    return fail(c, PM3GPU_INVALID_INPUT, "leading dimension below the row count");
  std::lock_guard<std::mutex> lk(c->mu);
  CUDA_TRY(c, cudaSetDevice(c->device));
  c->err.clear();
  CUDA_TRY(c, dgemm_ready(c->device));
  const size_t na = (size_t)lda * std::max<long long>(ca, 1), nb = (size_t)ldb * std::max<long long>(cb, 1),
               nc = (size_t)ldc * n;
  const dg::Plan pl = dg::plan(m, n, k, c->sms);
  DevBuf* B = c->tcbuf;
  CUDA_TRY(c, B[0].ensure(8 * na));
  CUDA_TRY(c, B[1].ensure(8 * nb));
  CUDA_TRY(c, B[2].ensure(8 * nc));
  CUDA_TRY(c, B[3].ensure(8 * std::max<size_t>(pl.work_doubles, 1)));
  CUDA_TRY(c, cudaMemcpyAsync(B[0].p, a, 8 * na, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(B[1].p, b, 8 * nb, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(B[2].p, cm, 8 * nc, cudaMemcpyHostToDevice, c->stream));
  const int r = dg::gemm(c->stream, c->sms, trans_a != 0, trans_b != 0, m, n, k, alpha, B[0].as<double>(), lda,
                         B[1].as<double>(), ldb, beta, B[2].as<double>(), ldc, B[3].as<double>());
  if (r < 0) return fail(c, PM3GPU_CUDA_ERROR, std::string("DGEMM launch: ") + cudaGetErrorString(cudaGetLastError()));
  c->launches = r;
  CUDA_TRY(c, cudaMemcpyAsync(cm, B[2].p, 8 * nc, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return PM3GPU_OK;
}

int pm3gpu_set_tail_helpers(pm3gpu_ctx* c, int on) {
  if (!c) return PM3GPU_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(c->mu);
  c->tail_helpers = on != 0;
  return PM3GPU_OK;
}

int pm3gpu_last_paired_jobs(pm3gpu_ctx* c) { return c ? c->paired : 0; }

int pm3gpu_set_tuning_goal(pm3gpu_ctx* c, int goal) {
  if (!c || (goal != PM3GPU_TUNE_BATCH_TIME && goal != PM3GPU_TUNE_THROUGHPUT)) return fail(c, PM3GPU_INVALID_INPUT, "bad argument");
  std::lock_guard<std::mutex> lk(c->mu);
  c->tune_goal = goal;
  return PM3GPU_OK;
}

int pm3gpu_set_large_checks(pm3gpu_ctx* c, int on) {
  if (!c) return PM3GPU_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(c->mu);
  c->large_checks = on != 0;
  return PM3GPU_OK;
}

int pm3gpu_last_large_checks(pm3gpu_ctx* c, double* rows, int max_rows) {
  if (!c) return 0;
  std::lock_guard<std::mutex> lk(c->mu);
  const int total = (int)(c->lchecks.size() / 6);
  if (rows && max_rows > 0) std::memcpy(rows, c->lchecks.data(), 8 * 6 * (size_t)std::min(total, max_rows));
  return total;
}

int pm3gpu_set_large_threshold(pm3gpu_ctx* c, int nao) {
  if (!c) return PM3GPU_INVALID_INPUT;
  if (nao < 1 || nao > kMaxN + 1) return fail(c, PM3GPU_INVALID_INPUT, "large-path threshold outside 1..257");
  std::lock_guard<std::mutex> lk(c->mu);
  c->large_min = nao;
  c->large_set = true;
  return PM3GPU_OK;
}

int pm3gpu_last_phase_cycles(pm3gpu_ctx* c, double* cycles, int max_entries) {
  if (!c || !cycles) return 0;
  const int k = std::min(max_entries, (int)kPhases);
  for (int i = 0; i < k; ++i) cycles[i] = c->phase_cycles[i];
  return c->profile ? k : 0;
}

int pm3gpu_last_transfer_bytes(pm3gpu_ctx* c, long long* h2d, long long* d2h) {
  if (!c) return PM3GPU_INVALID_INPUT;
  if (h2d) *h2d = c->h2d;
  if (d2h) *d2h = c->d2h;
  return PM3GPU_OK;
}

}  // extern "C"

// ===================================================================== allocation-free single point
// pm3gpu_single_point_noalloc: the run_pm3 single point of pm3gpu_single_point (charges only),
// with every device buffer the SCF kernel needs carved out of one fixed array of this library's
// own device image instead of allocated. Layout of the array for one call (each region starts on a
// 256-byte boundary):
//   [queue: 16 ints][rung list + rung ready flags: 2 x 8 ints][job descriptors: 8]
//   [job outcomes: 8][z: n_atoms int32][xyz: 3 n_atoms][charges: 8 x n_atoms][SCF workspace slots]
// The queue counters and the rung ready flags must be zero when the kernel starts and the rung
// outcomes must read status -1 ("not run"); each call writes both itself before its launch. Nothing
// else in the array needs an initial value: the kernel writes every workspace element before it
// reads it.

static __device__ __align__(256) unsigned char g_noalloc_scratch[PM3GPU_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kNoAllocMaxDevices = 64;
constexpr int kNoAllocMaxJobs = 8;  // the first pass plus the at most seven stability rungs
void* g_noalloc_base[kNoAllocMaxDevices] = {};
std::mutex g_noalloc_setup_mu;

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// Device address of the scratch array on the context's device (which must be current). Resolved
// once per device and cached; the first resolution may also load this library's device code.
// Creating a context on a device clears its entry (noalloc_forget), so that after a device reset
// and a new context the address is looked up again in the new module image.
int noalloc_scratch(pm3gpu_ctx* c, unsigned char** base) {
  if (c->device < 0 || c->device >= kNoAllocMaxDevices)
    return fail(c, PM3GPU_INVALID_INPUT, "device ordinal outside the allocation-free path's table");
  std::lock_guard<std::mutex> lk(g_noalloc_setup_mu);
  if (!g_noalloc_base[c->device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(c, PM3GPU_CUDA_ERROR,
                  std::string("cudaGetSymbolAddress of the allocation-free scratch: ") + cudaGetErrorString(e));
    g_noalloc_base[c->device] = p;
  }
  *base = static_cast<unsigned char*>(g_noalloc_base[c->device]);
  return PM3GPU_OK;
}

}  // namespace

void noalloc_forget(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) return;
  std::lock_guard<std::mutex> lk(g_noalloc_setup_mu);
  g_noalloc_base[device] = nullptr;
}

namespace {

int noalloc_run(pm3gpu_ctx* c, int n_atoms, const int32_t* z, const double* xyz, const pm3gpu_options* o,
                pm3gpu_result* result, double* charges) {
  std::memset(result, 0, sizeof(*result));
  if (n_atoms < 1 || n_atoms > kMaxN)
    return fail(c, PM3GPU_INVALID_INPUT, "atom count outside 1..256 for the allocation-free path");
  if (o->guess == PM3GPU_GUESS_LEARNED)
    return fail(c, PM3GPU_INVALID_INPUT, "the learned guess is not available on the allocation-free path");
  if (o->variant != PM3GPU_VARIANT_PM3 || o->mmok)
    return fail(c, PM3GPU_INVALID_INPUT, "post-SCF corrections are not available on the allocation-free path");
  MolPlan p;
  plan_molecule(c, z, xyz, n_atoms, o, p);
  result->nao = p.nao;
  if (p.status != PM3GPU_OK) {
    c->err = p.msg;
    return p.status;
  }
  // pm3gpu_single_point would run the whole-GPU algorithm, which needs allocations: by the context's
  // threshold, or (none set) by the lone-molecule rule of run_batch
  const bool lone_whole = !c->large_set && p.nao >= kSingleWholeNao && o->guess != PM3GPU_GUESS_LEARNED;
  if (p.large || lone_whole) {
    char msg[220];
    std::snprintf(msg, sizeof msg,
                  "molecule (nao=%d) is at or above the whole-GPU threshold (%d) of a single-molecule call; the "
                  "allocation-free path runs only the one-CTA-per-molecule kernel",
                  p.nao, p.large ? c->large_min : kSingleWholeNao);
    return fail(c, PM3GPU_RESOURCE_LIMIT, msg);
  }
  // the first pass and the stability rungs run_pm3 would try, in its order (scf.rs:599-715)
  JobDesc jobs[kNoAllocMaxJobs];
  Rung rungs[kNoAllocMaxJobs - 1];
  int nr = 0;
  jobs[0] = p.steered ? make_job(p, o->guess, o->accelerator, o->level_shift_ev, o->damping, false, 0)
                      : make_job(p, o->guess, o->accelerator, 0.0, 0.0, false, 0);
  JobDesc& fj = jobs[0];
  fj.mol = 0;
  fj.charge_off = 0;
  fj.stab = stability_mode(p, o);
  if (fj.stab) {
    const int nplan = stability_rungs(p, o, rungs);
    for (int k = 0; k < nplan; ++k) {
      const Rung& r = rungs[k];
      JobDesc rj = make_job(p, r.guess, r.accel, r.shift, r.damp, r.unrestricted, 0);
      rj.mol = 0;
      rj.stab = 0;
      rj.nrung = 0;
      rj.charge_off = (long long)(1 + nr) * n_atoms;
      jobs[1 + nr] = rj;
      ++nr;
    }
  }
  fj.rung0 = 0;
  fj.nrung = nr;
  const int njobs = 1 + nr;

  // carve the scratch array
  const size_t off_queue = 0;
  const size_t off_rq = off_queue + 256;
  const size_t off_jobs = off_rq + 256;
  const size_t off_out = off_jobs + round256(sizeof(JobDesc) * kNoAllocMaxJobs);
  const size_t off_z = off_out + round256(sizeof(JobOut) * kNoAllocMaxJobs);
  const size_t off_xyz = off_z + round256(4 * (size_t)n_atoms);
  const size_t off_q = off_xyz + round256(24 * (size_t)n_atoms);
  const size_t off_work = off_q + round256(8 * (size_t)kNoAllocMaxJobs * n_atoms);
  const long long wcap = std::max(1LL, pair_table_doubles(c, z, n_atoms));
  const long long slot = (slot_doubles(p.nao, wcap) + 31) & ~31LL;  // 256-byte aligned slots
  const size_t slot_bytes = 8 * (size_t)slot;
  const size_t room = PM3GPU_NOALLOC_SCRATCH_BYTES > off_work ? PM3GPU_NOALLOC_SCRATCH_BYTES - off_work : 0;
  if (slot_bytes > room) {
    char msg[200];
    std::snprintf(msg, sizeof msg,
                  "molecule (nao=%d) needs %zu bytes of SCF workspace; the allocation-free path's fixed scratch "
                  "has %zu bytes for it (%d MiB in total)",
                  p.nao, slot_bytes, room, (int)(PM3GPU_NOALLOC_SCRATCH_BYTES >> 20));
    return fail(c, PM3GPU_RESOURCE_LIMIT, msg);
  }
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(c, &base);
  if (rc != PM3GPU_OK) return rc;

  const SmemLayout L = make_layout(n_atoms, p.nao, c->smem_optin);
  int per_sm = 0;
  CUDA_TRY(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scf_batch_kernel, kThreads, L.bytes));
  if (per_sm < 1) return fail(c, PM3GPU_RESOURCE_LIMIT, "SCF kernel does not fit on an SM");
  long long grid = std::min<long long>(njobs, (long long)(room / slot_bytes));
  grid = std::min<long long>(grid, (long long)c->sms * per_sm);

  int* d_queue = reinterpret_cast<int*>(base + off_queue);
  int* d_rq = reinterpret_cast<int*>(base + off_rq);
  JobDesc* d_jobs = reinterpret_cast<JobDesc*>(base + off_jobs);
  JobOut* d_out = reinterpret_cast<JobOut*>(base + off_out);
  int32_t* d_z = reinterpret_cast<int32_t*>(base + off_z);
  double* d_xyz = reinterpret_cast<double*>(base + off_xyz);
  double* d_q = reinterpret_cast<double*>(base + off_q);
  CUDA_TRY(c, cudaMemcpyAsync(d_z, z, 4 * (size_t)n_atoms, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(d_xyz, xyz, 24 * (size_t)n_atoms, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(d_jobs, jobs, sizeof(JobDesc) * njobs, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(c, cudaMemsetAsync(d_queue, 0, 512, c->stream));  // queue counters, rung list and flags
  if (nr) CUDA_TRY(c, cudaMemsetAsync(d_out + 1, 0xff, sizeof(JobOut) * nr, c->stream));

  KernelArgs a{};
  a.elem = c->elem.as<ElemDev>();
  a.pairs = c->pairs.as<PairDev>();
  a.z = d_z;
  a.xyz = d_xyz;
  a.jobs = d_jobs;
  a.njobs = 1;
  a.out = d_out;
  a.rjobs = d_jobs + 1;
  a.nrjobs = nr;
  a.rout = d_out + 1;
  a.rlist = d_rq;
  a.rready = d_rq + kNoAllocMaxJobs;
  a.charges = d_q;
  a.densities = nullptr;
  a.grads = nullptr;
  a.eps = nullptr;
  a.work = reinterpret_cast<double*>(base + off_work);
  a.slot = slot;
  a.nmax = p.nao;
  a.wcap = wcap;
  a.queue = d_queue;
  a.prof = nullptr;
  a.sm = L;
  c->launches = 0;
  scf_batch_kernel<<<(unsigned)grid, kThreads, L.bytes, c->stream>>>(a);
  c->launches = 1;
  CUDA_TRY(c, cudaGetLastError());
  int qh[4] = {0, 0, 0, 0};
  JobOut outs[kNoAllocMaxJobs];
  CUDA_TRY(c, cudaMemcpyAsync(qh, d_queue, sizeof(qh), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(outs, d_out, sizeof(JobOut) * njobs, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (qh[3]) return fail(c, PM3GPU_CUDA_ERROR, "stability-search queue handshake timed out on the device");

  // run_pm3's selection among the first pass and the rungs (scf.rs:680-715)
  JobOut st = outs[0];
  int st_job = 0;
  bool st_unres = (fj.flags & kJobUhf) != 0;
  const double first_ev = st.electronic;
  int paths = 1;
  const bool searched = nr > 0 && outs[1].status != -1;
  for (int r = 0; searched && r < nr; ++r) {
    ++paths;
    JobOut cand = outs[1 + r];
    bool cand_unres = (jobs[1 + r].flags & kJobUhf) != 0;
    if (rung_replaces(rungs[r], cand, cand_unres, st)) {
      st = cand;
      st_job = 1 + r;
      st_unres = cand_unres;
    }
  }
  CUDA_TRY(c, cudaMemcpyAsync(charges, d_q + (size_t)st_job * n_atoms, 8 * (size_t)n_atoms, cudaMemcpyDeviceToHost,
                              c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->h2d = (long long)(28 * (size_t)n_atoms + sizeof(JobDesc) * njobs);
  c->d2h = (long long)(sizeof(qh) + sizeof(JobOut) * njobs + 8 * (size_t)n_atoms);

  double e_isol = 0.0, eheat = 0.0;
  for (int k = 0; k < n_atoms; ++k) {
    e_isol += c->h_elem[z[k]].e_isol;
    eheat += c->h_elem[z[k]].eheat_ev;
  }
  pm3gpu_result& Rm = *result;
  Rm.status = PM3GPU_OK;
  Rm.n_occ = p.n_alpha;
  Rm.n_beta = st_unres ? p.n_beta : p.n_alpha;
  Rm.electronic_ev = st.electronic;
  Rm.core_ev = st.core;
  Rm.total_ev = st.electronic + st.core;
  Rm.heat_of_formation_kcal = (Rm.total_ev - e_isol + eheat) * kEvToKcal;
  Rm.iterations = st.iterations;
  Rm.converged = st.converged;
  Rm.unrestricted = st_unres ? 1 : 0;
  Rm.scf_paths_tried = paths;
  Rm.scf_improvement_ev = std::max(first_ev - st.electronic, 0.0);
  Rm.last_change = st.last_change;
  Rm.homo_ev = st.homo;
  Rm.lumo_ev = st.lumo;
  Rm.has_homo = st.has_homo;
  Rm.has_lumo = st.has_lumo;
  for (int k = 0; k < 3; ++k) Rm.dipole_debye[k] = st.dipole[k];
  Rm.dipole_magnitude = std::sqrt(Rm.dipole_debye[0] * Rm.dipole_debye[0] + Rm.dipole_debye[1] * Rm.dipole_debye[1] +
                                  Rm.dipole_debye[2] * Rm.dipole_debye[2]);
  if (!st.converged) {
    Rm.status = PM3GPU_SCF_NOT_CONVERGED;
    char msg[160];
    std::snprintf(msg, sizeof msg, "PM3 SCF did not converge after %d iterations (error=%.3e)", st.iterations,
                  st.last_change);
    c->err = msg;
  }
  return Rm.status;
}

}  // namespace

extern "C" int pm3gpu_single_point_noalloc(pm3gpu_ctx* c, int n_atoms, const int32_t* z, const double* xyz,
                                           const pm3gpu_options* opts, pm3gpu_result* result, double* charges) {
  if (!c || !z || !xyz || !result || !charges) return fail(c, PM3GPU_INVALID_INPUT, "null argument");
  std::lock_guard<std::mutex> lk(c->mu);
  CUDA_TRY(c, cudaSetDevice(c->device));
  c->err.clear();
  pm3gpu_options d;
  pm3gpu_default_options(&d);
  const int rc = noalloc_run(c, n_atoms, z, xyz, opts ? opts : &d, result, charges);
  if (rc != PM3GPU_OK && result->status == PM3GPU_OK) result->status = rc;
  return rc;
}
