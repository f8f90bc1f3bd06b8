/*
 * CPU oracle for the molecular PM3 SCF single point of pm3-rs.
 *
 * TEST INFRASTRUCTURE ONLY. This library restates, in C++, the reference's CPU algorithm
 * (pm3-rs 0.2.5: src/params.rs, src/integrals.rs, src/overlap.rs, src/repulsion.rs,
 * src/hamiltonian.rs, src/fock.rs, src/scf.rs, src/dipole.rs, src/gradient.rs) so that the
 * GPU library can be checked against it. Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load it; the product path never does.
 *
 * Units: positions in Bohr, energies in eV (as inside the reference core).
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double charge;
  int multiplicity;
  int max_scf;
  double e_tol;
  double p_tol;
  int use_diis;
  int accelerator;   /* 0 none, 1 CDIIS, 2 A-DIIS -> CDIIS (scf.rs ScfAccelerator) */
  double adiis_switch;
  int reference;     /* 0 auto, 1 RHF, 2 UHF (scf.rs Reference) */
  int guess;         /* 0 auto, 1 SAD, 2 core, 3 symmetry-broken (scf.rs ScfGuess) */
  int stability;     /* 0 off, 1 auto, 2 always (scf.rs ScfStability) */
  double level_shift_ev;
  double damping;
  int scf_memory_mb;
  int variant;       /* 0 PM3, 1 PM3-D3, 2 PM3-D3H4, 3 PM3-D3H4X (corrections::Variant, src/corrections/mod.rs:165-178) */
  int mmok;          /* MOPAC's amide torsion term (Pm3Options::mmok, src/scf.rs:193) */
} oracle_options;

typedef struct {
  double electronic_ev, core_ev, total_ev, heat_of_formation_kcal;
  double dipole_debye[3];
  double homo_ev, lumo_ev;
  int has_homo, has_lumo;
  int iterations, converged, unrestricted, scf_paths_tried;
  double scf_improvement_ev;
  int n_occ, n_beta, nao;
  double last_change;
} oracle_result;

void oracle_default_options(oracle_options* o);

/* Optional LAPACK/BLAS entry points (Fortran ABI: dsyevd_, dgemm_). NULL restores the
 * built-in Jacobi eigensolver and loop GEMMs. */
void oracle_set_lapack(void* dsyevd, void* dgemm);

int oracle_nao(int n_atoms, const int* z);

/* Grimme D3 dispersion of one molecule (src/corrections/d3.rs): d3_set 1 = D3Params::pm3_d3,
 * 2 = D3Params::pm3_d3h4. energy_ev receives the energy (eV); gradient[3n] (eV/Bohr, forward-mode
 * dual numbers as src/gradient.rs:324-357) and cn[n] (coordination numbers) are optional. */
int oracle_d3(int n_atoms, const int* z, const double* xyz_bohr, int d3_set, double* energy_ev, double* gradient,
              double* cn);
/* The post-SCF correction of a method variant (0 none, 1 PM3-D3, 2 PM3-D3H4, 3 PM3-D3H4X;
 * src/corrections/mod.rs:78-160) with the MMOK amide term when mmok is set: parts_ev[5] = (D3, H4,
 * H-H repulsion, X, MMOK) in eV; gradient[3n] (optional) of their sum in eV/Bohr, by dual numbers. */
int oracle_corrections(int n_atoms, const int* z, const double* xyz_bohr, int variant, int mmok, double* parts_ev,
                       double* gradient);
/* getc6 (d3.rs:212-236) for one element pair at the given coordination numbers. */
double oracle_d3_c6(int zi, int zj, double cni, double cnj);

/* Full single point (run_pm3). charges[n_atoms] required; density[nao*nao], mo_energies[nao],
 * gradient[3*n_atoms] (eV/Bohr, closed-form Hellmann-Feynman) are optional (NULL = skip).
 * Returns 0 on success or a status code (1 invalid input, 2 missing element, 4 SCF not
 * converged, 5 linear algebra); err receives a message. */
int oracle_single_point(int n_atoms, const int* z, const double* xyz_bohr,
                        const oracle_options* opt, oracle_result* res, double* charges,
                        double* density, double* mo_energies, double* gradient, char* err,
                        int errlen);

/* One element of a parameter set: the Pm3Element fields of the s/p path (src/params.rs:20-92),
 * raw and derived, used as given. Same layout as the GPU library's pm3gpu_element. */
typedef struct {
  int z, n_orb, npq, n_gauss;
  double u_ss, u_pp, zeta_s, zeta_p, beta_s, beta_p;
  double g_ss, g_sp, g_pp, g_p2, h_sp;
  double alpha;
  double gauss[4][3];
  double core_charge, occ_s, occ_p;
  double eheat_ev, e_isol, mass;
  double dd, qq, rho0, rho1, rho2;
  double ddp[7], po[10];
} oracle_element_params;
typedef struct {
  int zi, zj;
  double alpha, x;
} oracle_pair_params;

/* Replace the parameter set (run_pm3's &Pm3Parameters, src/scf.rs:450-452); elements absent from
 * the set are missing. Returns 0, or 1 on an out-of-range entry. oracle_reset_parameters restores
 * the standard set (Pm3Parameters::standard, src/params.rs:133-137). */
int oracle_set_parameters(const oracle_element_params* elems, int n_elems, const oracle_pair_params* pairs,
                          int n_pairs);
void oracle_reset_parameters(void);

/* Derived element constants: out[0..21] = n_orb, uss, upp, zs, zp, betas, betap, gss, gsp,
 * gpp, gp2, hsp, alpha, core, dd, qq, rho0, rho1, rho2, e_isol, eheat_ev, mass. */
int oracle_element(int z, double* out);

/* One ordered pair (a heavy-first, dvec = R_b - R_a in Bohr): packed two-electron table
 * w[pa*pb] (row-major, pa = na(na+1)/2), electron-core blocks e1b[4*4], e2a[4*4] and the
 * overlap s[4*4] (rows a, cols b). */
int oracle_pair(int za, int zb, const double* dvec, double* w, double* e1b, double* e2a,
                double* s, int* na, int* nb);

int oracle_core_hamiltonian(int n_atoms, const int* z, const double* xyz, double* h);
int oracle_fock(int n_atoms, const int* z, const double* xyz, const double* p_tot,
                const double* p_spin, double* f);
double oracle_core_core(int n_atoms, const int* z, const double* xyz);
/* Hellmann-Feynman gradient at fixed densities (uhf=0: pa/pb ignored). */
int oracle_fixed_density_gradient(int n_atoms, const int* z, const double* xyz,
                                  const double* p_tot, const double* pa, const double* pb,
                                  int uhf, double* grad);
/* Symmetric eigensolver used by the oracle (ascending; vectors as columns, row-major). */
int oracle_eigh(int n, const double* a, double* w, double* v);

#ifdef __cplusplus
}
#endif
