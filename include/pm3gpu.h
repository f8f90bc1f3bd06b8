/*
 * pm3gpu -- B200 (sm_100a) implementation of the molecular PM3 SCF single point of pm3-rs,
 * behind a plain C ABI (no CUDA or torch types in any signature).
 *
 * Reference interfaces each entry point replaces (paths inside the pm3-rs project):
 *   pm3gpu_single_point      run_pm3(&Molecule, &Pm3Parameters, &Pm3Options) -> Result<Pm3Result>
 *                            (src/scf.rs:450), and _native.single_point (src/python.rs:253-296)
 *   pm3gpu_gradient          closed_form_gradient(..) -> GradientResult (src/gradient.rs:201-276),
 *                            and _native.gradient (src/python.rs:299-357)
 *   pm3gpu_batch             the same run_pm3 over many independent molecules in one call
 *                            (no single reference counterpart: the reference loops run_pm3)
 *   pm3gpu_options           Pm3Options molecular fields (src/scf.rs:160-287)
 *   pm3gpu_result            Pm3Result scalar fields (src/scf.rs:353-396)
 *   status codes             Pm3Error variants (src/error.rs:12-47)
 *
 * Units: positions in Bohr; energies in eV; dipole in Debye; gradients in eV/Bohr (the
 * reference's internal units). Matrices are row-major nao x nao doubles.
 *
 * Threading: a context owns one CUDA device, one stream and its workspaces; calls on one
 * context are serialised by an internal lock. Use one context per host thread for concurrency.
 */
#ifndef PM3GPU_H
#define PM3GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (Pm3Error, src/error.rs:12-47). */
#define PM3GPU_OK 0
#define PM3GPU_INVALID_INPUT 1      /* Pm3Error::InvalidInput */
#define PM3GPU_MISSING_ELEMENT 2    /* Pm3Error::MissingElement */
#define PM3GPU_RESOURCE_LIMIT 3     /* Pm3Error::ResourceLimit */
#define PM3GPU_SCF_NOT_CONVERGED 4  /* Pm3Error::ScfNotConverged */
#define PM3GPU_LINALG 5             /* Pm3Error::LinearAlgebra */
#define PM3GPU_CUDA_ERROR 6         /* device or driver failure */
#define PM3GPU_UNSUPPORTED 8        /* outside the s/p analytic path (see pm3gpu_supported_element) */

/* Accelerator / reference / guess / stability enums (src/scf.rs:26-158). */
#define PM3GPU_ACCEL_NONE 0
#define PM3GPU_ACCEL_CDIIS 1
#define PM3GPU_ACCEL_ADIIS_CDIIS 2
#define PM3GPU_REF_AUTO 0
#define PM3GPU_REF_RHF 1
#define PM3GPU_REF_UHF 2
#define PM3GPU_GUESS_AUTO 0
#define PM3GPU_GUESS_SAD 1
#define PM3GPU_GUESS_CORE 2
#define PM3GPU_GUESS_SYMMETRY_BROKEN 3
#define PM3GPU_GUESS_LEARNED 4  /* no reference counterpart: see pm3gpu_guess_train */
#define PM3GPU_STABILITY_OFF 0
#define PM3GPU_STABILITY_AUTO 1
#define PM3GPU_STABILITY_ALWAYS 2
/* Method variants (corrections::Variant, src/corrections/mod.rs:165-191). The variant's post-SCF
 * correction (mod.rs:129-160) joins total_ev and the heat of formation, and its gradient the SCF
 * gradient: PM3-D3 adds Grimme D3 dispersion (src/corrections/d3.rs, D3Params::pm3_d3); PM3-D3H4
 * adds D3 with D3Params::pm3_d3h4, the H4 hydrogen-bond term and the H-H repulsion
 * (src/corrections/h4.rs); PM3-D3H4X adds the halogen-bond term (src/corrections/hx.rs) too. */
#define PM3GPU_VARIANT_PM3 0
#define PM3GPU_VARIANT_D3 1
#define PM3GPU_VARIANT_D3H4 2
#define PM3GPU_VARIANT_D3H4X 3

typedef struct pm3gpu_ctx pm3gpu_ctx;

/* Pm3Options, molecular-path fields (src/scf.rs:160-287). Defaults: pm3gpu_default_options. */
typedef struct {
  double charge;          /* total charge */
  int multiplicity;       /* 2S+1 */
  int max_scf;            /* 200 */
  double e_tol;           /* eV, 1e-8 */
  double p_tol;           /* RMS density change, 1e-7 */
  int use_diis;           /* 1 */
  int accelerator;        /* PM3GPU_ACCEL_* (A-DIIS -> CDIIS) */
  double adiis_switch;    /* 0.1 */
  int reference;          /* PM3GPU_REF_* */
  int guess;              /* PM3GPU_GUESS_* */
  int stability;          /* PM3GPU_STABILITY_* (auto) */
  double level_shift_ev;  /* 0 */
  double damping;         /* 0 */
  int scf_memory_mb;      /* 512: accelerator-history budget (sets the DIIS depth) */
  int variant;            /* PM3GPU_VARIANT_* (Pm3Options::variant, src/scf.rs:184): 0 plain PM3 */
  int mmok;               /* 0; 1 adds MOPAC's MMOK amide torsion term (Pm3Options::mmok, src/scf.rs:193,
                             src/corrections/mmok.rs) on top of the variant's correction */
} pm3gpu_options;

/* Pm3Result scalar fields (src/scf.rs:353-396). Arrays are returned through caller buffers. */
typedef struct {
  int status;                    /* PM3GPU_* for this molecule */
  int nao;
  int n_occ, n_beta;
  double electronic_ev, core_ev, total_ev, heat_of_formation_kcal;
  double dipole_debye[3];
  double dipole_magnitude;
  double homo_ev, lumo_ev;
  int has_homo, has_lumo;
  int iterations;
  int converged;
  int unrestricted;
  int scf_paths_tried;
  double scf_improvement_ev;
  double last_change;            /* RMS density change of the last iteration */
} pm3gpu_result;

void pm3gpu_default_options(pm3gpu_options* opts);

/* 1 when element z is inside the s/p analytic path this library implements. */
int pm3gpu_supported_element(int z);

/* Basis size of a molecule (number of AOs), or -1 on an unsupported element
 * (sizes the caller's density / MO-energy buffers). Replaces Basis::build (src/basis.rs:39). */
int pm3gpu_result_sizes(int n_atoms, const int32_t* z, int* nao);

/* One element of a PM3 parameter set: the fields of Pm3Element (src/params.rs:20-92) that the
 * s/p path reads, raw and derived, exactly as the reference's run_pm3 reads them from
 * &Pm3Parameters (derived values are used as given, not re-derived). Energies in eV, exponents in
 * Bohr^-1, alpha in Angstrom^-1, charge separations and additive terms in Bohr. */
typedef struct {
  int z;            /* atomic number (1..17) */
  int n_orb;        /* 1 (s) or 4 (s, p) */
  int npq;          /* principal quantum number of the valence s shell (Pm3Element::n), 1..3 */
  int n_gauss;      /* core-core Gaussian corrections used, 0..4 */
  double u_ss, u_pp, zeta_s, zeta_p, beta_s, beta_p;
  double g_ss, g_sp, g_pp, g_p2, h_sp;
  double alpha;          /* per-element core-core exponent */
  double gauss[4][3];    /* (K, L, M) of each Gaussian */
  double core_charge, occ_s, occ_p;
  double eheat_ev, e_isol, mass;
  double dd, qq, rho0, rho1, rho2;  /* electron-electron multipoles */
  double ddp[7], po[10];            /* electron-core / core-core terms: ddp[2], ddp[3], po[1..3], po[9] */
} pm3gpu_element;

/* Pairwise core-core parameters PairParams (src/params.rs:104-109), symmetric in (zi, zj). */
typedef struct {
  int zi, zj;
  double alpha, x;
} pm3gpu_pair;

/* Pm3Parameters::standard() (src/params.rs:133-137): the built-in PM3 set for the elements of
 * the s/p path. Writes up to max_elems / max_pairs entries and the counts. */
int pm3gpu_standard_parameters(pm3gpu_element* elems, int max_elems, int* n_elems, pm3gpu_pair* pairs,
                               int max_pairs, int* n_pairs);

/* The &Pm3Parameters argument of run_pm3 (src/scf.rs:450-452; Pm3Calculator::new, src/scf.rs:404-410):
 * replaces the context's parameter set for every later call on it. Elements absent from `elems`
 * are missing (molecules containing them return PM3GPU_MISSING_ELEMENT, as
 * Pm3Parameters::element does, src/params.rs:139-141); pairs absent from `pairs` use the
 * per-element core-core form. Returns PM3GPU_INVALID_INPUT (nothing changed) on an out-of-range
 * or non-finite entry. The learned-guess network is independent of the parameters. */
int pm3gpu_set_parameters(pm3gpu_ctx* ctx, const pm3gpu_element* elems, int n_elems, const pm3gpu_pair* pairs,
                          int n_pairs);

int pm3gpu_context_create(int device, pm3gpu_ctx** out);
void pm3gpu_context_destroy(pm3gpu_ctx* ctx);
/* Message of the last failing call on this context (owned by the context). With ctx = NULL: the
 * message of the last failing context-free call on this host thread (pm3gpu_load_tuning(NULL, ..)). */
const char* pm3gpu_last_error_message(pm3gpu_ctx* ctx);
/* Run subsequent work on an existing CUDA stream (cudaStream_t passed as void*); NULL
 * restores the context's own stream. */
int pm3gpu_set_stream(pm3gpu_ctx* ctx, void* stream);

/* One molecule: run_pm3. charges[n_atoms] required; density[nao*nao] (total density) and
 * mo_energies[nao] (alpha MO energies of the last iteration) may be NULL.
 * Not exported from Pm3Result (src/scf.rs:353-396): mo_coeff and the beta set (mo_coeff_beta,
 * mo_energies_beta, spin_density). The eigensolvers form only the occupied eigenvectors the density
 * needs, so the virtual coefficients of the last iteration do not exist on the device.
 * Returns the molecule's status (also in result->status). */
int pm3gpu_single_point(pm3gpu_ctx* ctx, int n_atoms, const int32_t* z, const double* xyz_bohr,
                        const pm3gpu_options* opts, pm3gpu_result* result, double* charges,
                        double* density, double* mo_energies);

/* Size of the fixed device scratch array behind pm3gpu_single_point_noalloc. */
#define PM3GPU_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)

/* pm3gpu_single_point without any memory allocation in the call. It has no counterpart in the
 * reference, which never runs on a device.
 *
 * Who needs it: a host program that already owns the device memory, such as a framework whose
 * caching allocator has reserved most of HBM (there a library cudaMalloc can fail or force the
 * cache to be released), or a per-step loop (molecular dynamics, geometry optimisation) that
 * cannot pay for cudaMalloc/cudaFree in every step (cudaFree waits for the whole device). This
 * call makes no cudaMalloc, cudaFree or other allocating call, neither does it grow the
 * context's buffers: the SCF kernel's workspace, job table and outputs live in one
 * PM3GPU_NOALLOC_SCRATCH_BYTES array of this library's own device image.
 *
 * Same inputs, options and results as pm3gpu_single_point (host arrays: z[n_atoms],
 * xyz_bohr[3*n_atoms]; charges[n_atoms] out), without the density and MO-energy outputs.
 * Limit: one SCF workspace slot must fit the scratch (about 190 basis functions, e.g. 40 heavy
 * atoms with 30 hydrogens); larger molecules return PM3GPU_RESOURCE_LIMIT with the needed size.
 * The stability-search rungs share the slots that fit and run one after another if only one does.
 * The first call on each device looks up the array's address (and may load this library's device
 * code), so make it before any stream capture begins. A device reset invalidates that address
 * with everything else on the device: create a new context after a reset (creating a context
 * makes the next call look the address up again).
 * The call always runs the one-CTA-per-molecule kernel: a molecule that pm3gpu_single_point sends
 * to the whole-GPU path (pm3gpu_set_large_threshold, or 192+ basis functions when no threshold is
 * set) returns PM3GPU_RESOURCE_LIMIT here, so
 * that the two entry points never run different algorithms on the same input. The caller clears nothing: each call resets
 * the queue counters and flags it needs at zero itself. All contexts of a process on one device
 * share the one array, so calls that overlap in time on that device (two contexts, or two
 * threads on different contexts) race and give wrong results; calls through one context are
 * serialised by the context. The call returns once its results are on the host. */
int pm3gpu_single_point_noalloc(pm3gpu_ctx* ctx, int n_atoms, const int32_t* z, const double* xyz_bohr,
                                const pm3gpu_options* opts, pm3gpu_result* result, double* charges);

/* One molecule: run_pm3 followed by the closed-form Hellmann-Feynman gradient
 * (gradient[3*n_atoms], eV/Bohr) at the converged density. */
int pm3gpu_gradient(pm3gpu_ctx* ctx, int n_atoms, const int32_t* z, const double* xyz_bohr,
                    const pm3gpu_options* opts, pm3gpu_result* result, double* charges,
                    double* gradient);

/* Many independent molecules in one persistent launch. Molecule m owns atoms
 * [atom_offsets[m], atom_offsets[m+1]) of z / xyz_bohr (host arrays). results[n_mol],
 * charges[total atoms] required; gradients[3 * total atoms] optional (NULL = no gradient).
 * opts may be one struct (per_molecule_options = 0) or an array of n_mol structs.
 * Returns PM3GPU_OK when the batch ran (per-molecule outcomes are in results[m].status),
 * or an error that stopped the whole batch. */
int pm3gpu_batch(pm3gpu_ctx* ctx, int n_mol, const int32_t* atom_offsets, const int32_t* z,
                 const double* xyz_bohr, const pm3gpu_options* opts, int per_molecule_options,
                 pm3gpu_result* results, double* charges, double* gradients);

/* Geometry optimisation of many molecules at once: the reference's L-BFGS
 * (src/optimizer.rs:77-221, `optimize` / OptOptions) run per molecule, every energy and gradient
 * from the batched SCF + gradient launch (one launch per round over every molecule's pending
 * geometry: its start or its current line-search trial). Same algorithm and stopping rules: two-loop
 * recursion over the last `history` steps, first step 0.1 / max|g|, uphill guard, backtracking
 * Armijo search (c1 = 1e-4, step halved down to 1e-8; a geometry whose SCF fails is a rejected
 * step), curvature filter s.y > 1e-10, convergence when the largest gradient component is below
 * gtol (eV/Bohr). xyz_bohr holds the starting geometries and receives the final ones;
 * gradients[3 * total atoms] (optional) the final gradients. out[m].status is the start
 * geometry's run_pm3 status when that evaluation failed (the molecule is then left unchanged). */
typedef struct {
  int max_iter;   /* 200 */
  double gtol;    /* 1e-3 eV/Bohr on the largest gradient component */
  int history;    /* 8 */
} pm3gpu_opt_options;
typedef struct {
  int status;                     /* PM3GPU_* of the start geometry's evaluation */
  int converged;                  /* 1 when the largest gradient component fell below gtol */
  int iterations;                 /* the reference's count (OptResult::iterations) */
  int evaluations;                /* energy + gradient evaluations, line-search trials included */
  double energy_ev;               /* total energy at the final geometry */
  double heat_of_formation_kcal;  /* at the final geometry */
  double max_gradient;            /* eV/Bohr, at the final geometry */
} pm3gpu_opt_result;
void pm3gpu_default_opt_options(pm3gpu_opt_options* opt);
int pm3gpu_optimize_batch(pm3gpu_ctx* ctx, int n_mol, const int32_t* atom_offsets, const int32_t* z,
                          double* xyz_bohr, const pm3gpu_options* opts, const pm3gpu_opt_options* opt,
                          pm3gpu_opt_result* out, double* gradients);

/* Cartesian Hessians of many molecules by central differences of the analytic gradient: the
 * reference's numerical_hessian (src/hessian.rs:268-319). Column j of molecule m is
 * (g(x + step e_j) - g(x - step e_j)) / (2 step) with j = 3 * atom + axis, then the matrix is averaged
 * with its transpose. The SCF is tightened as the reference does for second derivatives
 * (src/hessian.rs:169-175: e_tol <= 1e-12 eV, p_tol <= 1e-11, max_scf >= 500). Every displaced
 * geometry of every molecule runs in the batched SCF + gradient launch. hessians receives each
 * molecule's (3 n_m) x (3 n_m) row-major block in eV/Bohr^2, packed molecule after molecule;
 * status[m] is PM3GPU_OK or the run_pm3 status of the molecule's first failing displacement (its
 * block is then zero). step in Bohr (the reference's Python entry points use 1e-3). */
int pm3gpu_numerical_hessian_batch(pm3gpu_ctx* ctx, int n_mol, const int32_t* atom_offsets, const int32_t* z,
                                   const double* xyz_bohr, const pm3gpu_options* opts, double step,
                                   double* hessians, int* status);

/* The D3 dispersion correction alone for many molecules (src/corrections/d3.rs:360-458): d3_set 1 =
 * D3Params::pm3_d3, 2 = D3Params::pm3_d3h4. energies[n_mol] in eV; gradients[3 * total atoms]
 * (optional) in eV/Bohr. */
int pm3gpu_d3_batch(pm3gpu_ctx* ctx, int n_mol, const int32_t* atom_offsets, const int32_t* z,
                    const double* xyz_bohr, int d3_set, double* energies, double* gradients);

/* The whole correction of a variant (PM3GPU_VARIANT_D3 / _D3H4 / _D3H4X) alone for many molecules:
 * the CorrectionEnergies of src/corrections/mod.rs:193-235. parts[4 * n_mol] receives per molecule
 * (D3, H4, H-H repulsion, X) in eV; gradients[3 * total atoms] (optional) the gradient of their sum
 * in eV/Bohr. Both correction-only entries take the s/p elements (pm3gpu_supported_element) and
 * return PM3GPU_UNSUPPORTED for any other. */
int pm3gpu_corrections_batch(pm3gpu_ctx* ctx, int n_mol, const int32_t* atom_offsets, const int32_t* z,
                             const double* xyz_bohr, int variant, double* parts, double* gradients);

/* pm3gpu_batch with z / xyz_bohr / atom_offsets already resident in device memory
 * (device pointers); results, charges and gradients are host buffers as above. */
int pm3gpu_batch_device_inputs(pm3gpu_ctx* ctx, int n_mol, const int32_t* d_atom_offsets,
                               const int32_t* d_z, const double* d_xyz_bohr,
                               const int32_t* h_atom_offsets, const int32_t* h_z,
                               const pm3gpu_options* opts, pm3gpu_result* results,
                               double* charges, double* gradients);

/* H_core of one molecule (hamiltonian.rs:174 build_core): h[nao*nao]; core_ev (optional)
 * receives the core-core repulsion energy (repulsion.rs:13). */
int pm3gpu_core_hamiltonian(pm3gpu_ctx* ctx, int n_atoms, const int32_t* z, const double* xyz_bohr,
                            double* h, double* core_ev);

/* Fock matrix for given densities (fock.rs:285 build_fock_spin / fock.rs:488 build_fock).
 * RHF: p_alpha = p_beta = f_beta = NULL, f_alpha = H + J(P) - K(P/2). UHF: f_alpha from
 * (p_tot, p_alpha), f_beta from (p_tot, p_beta). All nao*nao. */
int pm3gpu_fock(pm3gpu_ctx* ctx, int n_atoms, const int32_t* z, const double* xyz_bohr,
                const double* p_tot, const double* p_alpha, const double* p_beta, double* f_alpha,
                double* f_beta);

/* Phase timings of the last call (milliseconds, CUDA events): [0] upload, [1] the batched launch
 * (first passes and stability rungs of the per-CTA molecules), [2] selection, whole-GPU molecules
 * and gradients, [3] the SCF passes of the whole-GPU molecules alone (first pass and stability
 * rungs, no gradient), [4] total, [5] time inside the batched SCF kernel, [6] the learned-guess
 * inference (features, network, assembly) before the batched launch.
 * Returns the count written. */
int pm3gpu_last_timings(pm3gpu_ctx* ctx, double* ms, int max_entries);

/* SM cycles spent per SCF phase by the last call, summed over CTAs, when the context was
 * created with PM3GPU_PROFILE=1 in the environment (the counterpart of pm3-rs's PM3_TIMING,
 * src/scf.rs:469-485). Phases: 0 integrals + H_core, 1 Fock build + energy, 2 commutator,
 * 3 accelerator solve, 4 extrapolation / packing, 5 tridiagonalisation, 6 eigenvalues,
 * 7 eigenvectors, 8 back-transformation, 9 density, 10 closing energy + properties,
 * 11 gradient. Returns the number of phases written (0 when profiling is off). */
int pm3gpu_last_phase_cycles(pm3gpu_ctx* ctx, double* cycles, int max_entries);

/* Host-to-device and device-to-host bytes moved by the last call. */
int pm3gpu_last_transfer_bytes(pm3gpu_ctx* ctx, long long* h2d, long long* d2h);

/* Number of this library's kernels launched by the last call. */
int pm3gpu_last_kernel_launches(pm3gpu_ctx* ctx);

/* Shape of the last batched SCF launch (no counterpart in the reference): CTAs resident per SM and
 * the largest basis size whose packed eigen matrix stays in shared memory; larger molecules of that
 * launch keep it in global memory until its trailing part fits. */
int pm3gpu_last_launch_layout(pm3gpu_ctx* ctx, int* ctas_per_sm, int* smem_matrix_n);

/* Molecules with at least `nao` basis functions are solved one at a time on the whole GPU
 * (grid-wide integral and Fock kernels, blocked eigensolver, the library's FP64 tensor-core GEMM for
 * the dense products) instead of one CTA each. Default and maximum 257: every molecule beyond one CTA's
 * 256 basis functions; by default a call with a single molecule also sends it there from 192 basis
 * functions, where all SMs beat one CTA (setting a threshold replaces that rule). Lower values send
 * smaller molecules to that path too (one molecule at a time, all SMs on it). Same run_pm3
 * semantics either way (no reference counterpart: the reference has one CPU path). */
int pm3gpu_set_large_threshold(pm3gpu_ctx* ctx, int nao);

/* Autotuner (no counterpart in the reference). Measures, on the caller's sample of molecules
 * (atom_offsets / z / xyz as in pm3gpu_batch), the two launch choices that trade off against each
 * other, and keeps the faster per size bucket in the context: CTAs per SM of the batched SCF
 * launch (bucket: the batch's largest basis size) and, for molecules on the whole-GPU path, the
 * Householder reduction as one cooperative launch per panel or as five launches per column
 * (bucket: basis size). Both variants of each choice give the same results. When cache_path is
 * not NULL the table is written there as JSON; pm3gpu_load_tuning reads such a file into another
 * context (with ctx = NULL it only checks the file and returns its status).
 * pm3gpu_tuning_choice returns the choice a size would get (kind 0: CTAs per SM for a
 * batch whose largest basis is `size`; kind 1: 1 = cooperative panels for basis `size`), or -1
 * when no tuned bucket covers it. */
/* What pm3gpu_autotune minimises for the batched launch: PM3GPU_TUNE_BATCH_TIME (default), the time
 * of one whole batch, tail included (one batch at a time); PM3GPU_TUNE_THROUGHPUT, the time until
 * 90% of the first passes have ended, the rate of the bulk of a batch (batches in flight, where one
 * batch's tail overlaps the next). The times written to the JSON file are of the chosen goal. */
#define PM3GPU_TUNE_BATCH_TIME 0
#define PM3GPU_TUNE_THROUGHPUT 1
int pm3gpu_set_tuning_goal(pm3gpu_ctx* ctx, int goal);
int pm3gpu_autotune(pm3gpu_ctx* ctx, int n_mol, const int32_t* atom_offsets, const int32_t* z,
                    const double* xyz_bohr, const pm3gpu_options* opts, const char* cache_path);
int pm3gpu_load_tuning(pm3gpu_ctx* ctx, const char* path);
int pm3gpu_tuning_choice(pm3gpu_ctx* ctx, int kind, int size);

/* Arithmetic of the whole-GPU path's density and commutator products (no counterpart in the
 * reference, whose products are FP64). PM3GPU_PRECISION_MIXED takes them from split-BF16
 * tensor-core GEMMs (x = hi + lo, products hi*hi + hi*lo + lo*hi, FP32 accumulation) while the
 * density is far from converged, then closes the SCF with FP64 iterations: integrals, Fock build,
 * eigensolver, DIIS solve, energies and gradients stay FP64, and only an FP64 iteration can pass
 * the convergence test. The per-CTA path (n <= 256) is FP64 in both modes. Default FP64.
 * The split products run on a hand-written tcgen05 kernel (see pm3gpu_split_gemm). */
#define PM3GPU_PRECISION_FP64 0
#define PM3GPU_PRECISION_MIXED 1
int pm3gpu_set_precision(pm3gpu_ctx* ctx, int mode);

/* The whole-GPU path's FP64 product by itself (no counterpart in the reference, whose dense
 * products are faer's): C = alpha op(A) op(B) + beta C with the column-major BLAS dgemm contract
 * (op = transpose when trans_a / trans_b is nonzero; A, B, C host arrays with leading dimensions
 * lda, ldb, ldc), computed by the library's FP64 tensor-core (DMMA) GEMM with the tile shape and
 * K split the path would use for these sizes. C is read when beta != 0 and overwritten. */
int pm3gpu_dgemm(pm3gpu_ctx* ctx, int trans_a, int trans_b, int m, int n, int k, double alpha, const double* a, int lda,
                 const double* b, int ldb, double beta, double* c, int ldc);

/* The mixed mode's split-BF16 product by itself (no counterpart in the reference): out (m x n,
 * row-major FP32) = A B^T for A (m x k, leading dimension lda) and B (n x k, ldb), row-major FP64
 * host arrays, each operand split into BF16 hi + lo and the products hi hi + hi lo + lo hi
 * accumulated in FP32 on the tcgen05 tensor cores in one launch. Exposes the kernel the
 * whole-GPU path's mixed mode runs, for checks against an FP64 product. */
int pm3gpu_split_gemm(pm3gpu_ctx* ctx, int m, int n, int k, const double* a, int lda, const double* b, int ldb,
                      float* out);

/* Per-iteration convergence record of the last whole-GPU solve (no counterpart in the
 * reference, whose PM3_TIMING trace, scf.rs:1206-1296, prints phase times only): rows of 5 doubles (pass: 1 = first SCF, 2.. = stability rungs;
 * |dE| in eV, infinite on a pass's first iteration; RMS density change; DIIS error norm
 * ||FP - PF||, 0 without an accelerator; 1 if the iteration ran split-BF16, else 0). Copies at
 * most max_rows rows and returns the total number of rows. */
int pm3gpu_last_large_trace(pm3gpu_ctx* ctx, double* rows, int max_rows);

/* Batched launch (no counterpart in the reference): with on = 1, up to 32 CTAs left without work
 * near the end of a batch stay for stability rungs queued late and take the beta spin of
 * unaccelerated unrestricted jobs still running (the
 * reference's UHF loop without DIIS, src/scf.rs:1319-1496): from the next iteration on, the two
 * CTAs build F_alpha and F_beta, diagonalise and form the two spin densities side by side and
 * exchange energy parts and density changes each iteration (bounded waits). It shortens the tail
 * of a batch (long unrestricted stability rungs, radicals) when one batch runs at a time; with
 * batches overlapping, the idle SMs are better left to the next batch. Same results up to the
 * summation order of the electronic energy. Default off. */
int pm3gpu_set_tail_helpers(pm3gpu_ctx* ctx, int on);
/* Number of jobs of the last call that ran their iterations on two CTAs. */
int pm3gpu_last_paired_jobs(pm3gpu_ctx* ctx);

/* Checks of every eigensolve of the whole-GPU path (no counterpart in the reference, whose
 * eigensolver is faer's, src/linalg.rs:221-263). Each eigensolve orthonormalises the occupied
 * vectors X by Newton-Schulz steps until max |X^T X - I| < 1e-13 (at most 5 steps; a defect still
 * at or above 1e-11 after them returns PM3GPU_LINALG). With pm3gpu_set_large_checks(ctx, 1) each
 * eigensolve also measures max |F X - X diag(eps)| over the occupied pairs (one more n x n x
 * n_occ DGEMM). pm3gpu_last_large_checks copies rows of 6 doubles of the last whole-GPU solve
 * (pass, iteration, spin, orthonormality defect, eigen residual in eV or NaN when not measured,
 * Newton-Schulz steps taken), at most max_rows, and returns the number of rows. */
int pm3gpu_set_large_checks(pm3gpu_ctx* ctx, int on);
int pm3gpu_last_large_checks(pm3gpu_ctx* ctx, double* rows, int max_rows);

/* Learned initial density (no counterpart in the reference). A 3 x 256 BF16 MLP predicts every
 * atom block and atom-pair block of the initial density from element one-hots, 32 Gaussian
 * distance functions (6 A cutoff) and coordination counts; the SCF starts from the aufbau density
 * of that prediction's Fock matrix (guess =
 * PM3GPU_GUESS_LEARNED in the options). The plain SCF has the last word: a molecule that does not
 * converge from the learned start is solved again from the standard guess.
 *
 * pm3gpu_guess_train solves the given molecules with the plain SCF (their options), takes the
 * converged densities as targets and trains the network on the GPU (Adam, minibatches of `batch`
 * rows, `epochs` passes, learning rate `lr`, seeded shuffling and initialisation; continues from
 * the context's current parameters when it has some). losses[epochs] receives the mean masked
 * squared error of each epoch. Parameters: PM3GPU_GUESS_PARAMS floats (W1 b1 W2 b2 W3 b3 W4 b4). */
#define PM3GPU_GUESS_PARAMS 150280
int pm3gpu_guess_train(pm3gpu_ctx* ctx, int n_mol, const int32_t* atom_offsets, const int32_t* z,
                       const double* xyz_bohr, const pm3gpu_options* opts, int epochs, int batch, float lr,
                       unsigned seed, float* losses);
int pm3gpu_guess_set_params(pm3gpu_ctx* ctx, const float* params, int n_params);
/* The network's feature rows (64 floats each, optional) and outputs (8 floats each) for a batch:
 * per molecule its atoms, then its pairs a < b (the atom with more orbitals first in a pair). */
int pm3gpu_guess_predict(pm3gpu_ctx* ctx, int n_mol, const int32_t* atom_offsets, const int32_t* z,
                         const double* xyz_bohr, float* features, float* outputs);
int pm3gpu_guess_get_params(pm3gpu_ctx* ctx, float* params, int n_params);
/* One forward and backward pass of the network at its current parameters, as a training step
 * computes it (no parameter update): rows feature rows (64 floats each, rounded to BF16 on entry),
 * targets and 0/1 masks (8 floats per row). loss = inv_count * sum mask (Y - T)^2; grads
 * receives dloss/dparams (PM3GPU_GUESS_PARAMS floats, the layout of pm3gpu_guess_get_params).
 * Exposes the hand-written backward kernels so they can be checked against a restatement. */
int pm3gpu_guess_gradients(pm3gpu_ctx* ctx, int rows, const float* features, const float* targets,
                           const float* mask, float inv_count, float* loss, float* grads);

/* Wall-clock ms per phase of the last whole-GPU solve (core, Fock, DIIS, tridiagonalise,
 * eigenvalues, eigenvectors, back-transform, orthonormalise, density), when the context was
 * created with PM3GPU_PROFILE=1 (each phase then waits for the stream); returns the count. */
int pm3gpu_last_large_phase_ms(pm3gpu_ctx* ctx, double* ms, int max_entries);

#ifdef __cplusplus
}
#endif
#endif /* PM3GPU_H */
