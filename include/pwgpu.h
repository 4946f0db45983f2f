/*
 * pwgpu -- B200 (sm_100a) SCF hot path of a plane-wave Kohn-Sham DFT code,
 * exported as a plain C ABI.
 *
 * The entry points replace, one for one, the per-iteration calls of the
 * reference solver (Ron-Leizrowice/pwdft-rs, paths relative to
 * pwdft/pwdft-core/src/):
 *
 *   pwgpu_set_veff_g   <- the V_eff(G) handed from assemble_v_eff
 *                         (scf/energy.rs:293-301) to the per-k H build
 *                         (scf/driver.rs:459-468)
 *   pwgpu_apply_h      <- H|psi> with H = fill_hamiltonian_with_v_eff
 *                         (scf/potentials.rs:163-190) +
 *                         NonlocalPotential::add_to_hamiltonian
 *                         (potential/nonlocal.rs:432-450), applied
 *                         matrix-free
 *
 * Units are the reference's: eV, Å, e/Å³.  Complex arrays are interleaved
 * (re, im) doubles.  Wavefunction blocks are column-major n_pw x n_bands
 * in the basis order of BasisSet::new (basis.rs:36-63), as faer::Mat.
 *
 * Conventions: every function returns a pwgpu_status (0 = success,
 * negative = error, one code per reference error family); the message of
 * the calling thread's last failure is returned by pwgpu_last_error().
 * The library never aborts the process and never traps the device.
 * Host arrays are borrowed for the duration of a call only; device state
 * is owned by the handle.  A handle is bound to one device and one CUDA
 * stream and must not be used from two threads at once; distinct handles
 * are independent.
 */
#ifndef PWGPU_H
#define PWGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t pwgpu_status;

#define PWGPU_OK 0
#define PWGPU_E_INVALID (-1)          /* PwdftError::InvalidParam / InvalidCrystal */
#define PWGPU_E_CUDA (-2)             /* PwdftError::Gpu */
#define PWGPU_E_OOM (-3)              /* device allocation failed */
#define PWGPU_E_NOT_CONVERGED (-4)    /* PwdftError::ConvergenceFailure */
#define PWGPU_E_TIMEOUT (-5)          /* a bounded device wait ran out */
#define PWGPU_E_NOT_IMPLEMENTED (-6)  /* PwdftError::NotImplemented */
#define PWGPU_E_STATE (-7)            /* call order violated (e.g. no V_eff set) */
#define PWGPU_E_PARSE (-8)            /* PwdftError::Parse (malformed pseudopotential file) */

#define PWGPU_PRECISION_FP64 0  /* plain: every H|psi> stage in FP64 */
#define PWGPU_PRECISION_MIXED 1 /* FFTs and V_eff product in FP32 */

typedef struct pwgpu_handle pwgpu_handle;

/*
 * Per-calculation invariants: the data contract of ScfContext::new
 * (scf/context.rs:102-231).  All pointers are host pointers, read during
 * pwgpu_create only.
 */
typedef struct pwgpu_system {
  int32_t dims[3];             /* FFT grid (FftGrid::new, scf/grid.rs:44-87) */
  int32_t n_pw;                /* basis size (k-independent sphere) */
  const int32_t* miller;       /* n_pw x 3 Miller indices, basis order */
  int32_t n_k;                 /* number of (IBZ) k-points */
  const double* k_weights;     /* n_k, sum 1 */
  const double* kinetic;       /* n_k x n_pw: (hbar^2/2m)|k+G|^2, eV */
  int32_t n_ch;                /* KB channels (atom, projector, m) */
  const double* proj_b;        /* n_k x (n_pw x n_ch) complex, column-major:
                                  B[G,c] = e^{-iG.tau} F(|k+G|) Y_lm / sqrt(Omega)
                                  (nonlocal.rs:311-338) */
  int32_t n_atoms;             /* atoms carrying channels */
  const int32_t* atom_ch_start;/* n_atoms+1: first channel of each atom */
  const double* d_blocks;      /* per atom, the dense nc_a x nc_a block of D
                                  (row-major, eV), concatenated */
  const double* v_local_g;     /* N complex: V_loc(G) on the full grid, G=0 kept */
  const double* g_squared;     /* N: |G|^2, Å^-2 */
  const double* rho_core_r;    /* N: NLCC core density, or NULL */
  int32_t n_sym;               /* symmetry operations (1 = identity only) */
  const int32_t* sym_src;      /* n_sym x N gather map (symmetry/density/g_space.rs) */
  const double* sym_arg;       /* n_sym x N phase arguments 2 pi n.tau */
  double n_electrons;
  double omega;                /* cell volume, Å^3 */
  double e_ewald;              /* eV */
  int32_t nspin;               /* 1 or 2 */
  /* Projectors built on the device (NonlocalPotential::new, potential/nonlocal.rs:190-382),
   * used when proj_b is NULL and n_ch > 0: F_i(|k+G|) = 4 pi int [r beta_i] j_l(|k+G| r) r dr
   * by Simpson on each species' mesh, real Y_lm, e^{-iG.tau}/sqrt(Omega); channels atom by
   * atom, projector by projector, m = 0, +1, -1, ...  atom_ch_start and d_blocks as above. */
  const double* g_cart;         /* n_pw x 3 G vectors (Å^-1), basis order */
  const double* k_cart;         /* n_k x 3 k-points (Å^-1) */
  const double* atom_tau;       /* n_atoms x 3 Cartesian positions (Å) */
  const int32_t* atom_species;  /* n_atoms: species index */
  int32_t n_species;
  const int32_t* species_mesh;  /* n_species radial mesh sizes */
  const double* radial_r;       /* concatenated radial meshes r (Å) */
  const double* radial_rab;     /* concatenated dr/di */
  const int32_t* species_nbeta; /* n_species projector counts */
  const int32_t* beta_l;        /* l of each projector, species by species */
  const double* beta_r;         /* beta_i(r) of each projector on its species' mesh, concatenated */
  /* Local pseudopotential, NLCC core density and start density built on the device
   * (ScfContext::new, scf/context.rs:102-231, with potentials.rs:18-115 and
   * generate_initial_density, scf/initial_density.rs:64-166), used when v_local_g is NULL
   * (rho_core_r must then be NULL too): atom_tau, atom_species, n_species, species_mesh,
   * radial_r and radial_rab as above, for all n_atoms atoms, plus: */
  const double* recip;          /* 3 x 3 reciprocal vectors b1, b2, b3 as rows (Å^-1, 2 pi included) */
  const double* species_zval;   /* n_species valence charges */
  const double* vloc_r;         /* V_loc(r) of each species on its mesh (eV), concatenated */
  const double* core_r;         /* NLCC core charge on the meshes (e/Å^3), concatenated, or NULL */
  const double* rho_atom_r;     /* PP_RHOATOM on the meshes (e/Å), concatenated, or NULL */
  const int32_t* species_flags; /* n_species: bit 0 core charge given, bit 1 rho_atom given */
  double gaussian_sigma;        /* Å: start-density width of species without rho_atom */
} pwgpu_system;

typedef struct pwgpu_options {
  int32_t device;     /* CUDA device ordinal */
  int32_t precision;  /* PWGPU_PRECISION_FP64 or PWGPU_PRECISION_MIXED */
  int32_t lanes;      /* concurrent (spin, k) eigensolves inside pwgpu_scf_run, each on its own
                         stream (the reference's rayon loop over k, driver_spin.rs:356-384);
                         0 = min(nspin * n_k, 8), 1 = one block at a time */
  int32_t gamma_complex;  /* 0: a system with the single k-point Gamma stores its bands as real vectors
                             (psi(-G) = conj psi(G); real subspace algebra, two bands per FFT);
                             1: keep complex bands */
} pwgpu_options;

/* Message of the calling thread's most recent failure ("" if none). */
const char* pwgpu_last_error(void);

/* Library version string. */
const char* pwgpu_version(void);

/* Build a handle: uploads the system, plans the FFTs, sizes scratch.
 * Replaces ScfContext::new's device-facing part (scf/context.rs:102-231). */
pwgpu_status pwgpu_create(const pwgpu_system* sys, const pwgpu_options* opt, pwgpu_handle** out);

/* Release every device allocation of the handle.  NULL is accepted. */
pwgpu_status pwgpu_destroy(pwgpu_handle* h);

/* Set V_eff(G) (N complex, eV) for one spin channel; the library forms
 * V_eff(r) by one unnormalised inverse FFT.  Replaces the V_eff hand-off of
 * scf/driver.rs:427-468. */
pwgpu_status pwgpu_set_veff_g(pwgpu_handle* h, int32_t spin, const double* veff_g);

/* hpsi = H psi for a block of nb bands at k-point ik (host arrays,
 * column-major n_pw x nb, complex).  Equals the dense H of
 * scf/potentials.rs:163-190 + potential/nonlocal.rs:432-450 applied to psi. */
pwgpu_status pwgpu_apply_h(pwgpu_handle* h, int32_t spin, int32_t ik, const double* psi, int32_t nb,
                           double* hpsi);

/* Same on device pointers (leading dimensions in complex elements), on the
 * CUDA stream `stream` (cudaStream_t, NULL = the handle's stream). */
pwgpu_status pwgpu_apply_h_device(pwgpu_handle* h, int32_t spin, int32_t ik, const void* psi_dev, int64_t ldpsi,
                                  int32_t nb, void* hpsi_dev, int64_t ldh, void* stream);

/* pwgpu_apply_h_device on the handle's stream with a CUDA event after every
 * launch; stage_ms[8] / launches[8] receive the summed device time and the
 * launch count per stage: 0..4 the five FFT kernels (z-inverse+scatter,
 * y-inverse, x-inverse*V*x-forward, y-forward, z-forward+gather+kinetic),
 * 5 B^H psi, 6 D apply, 7 B Q.  Diagnostic; no reference counterpart. */
pwgpu_status pwgpu_profile_apply_h(pwgpu_handle* h, int32_t spin, int32_t ik, const void* psi_dev, int64_t ldpsi,
                                   int32_t nb, void* hpsi_dev, int64_t ldh, double* stage_ms, int32_t* launches);

/* Select the arithmetic of subsequent H|psi> calls (PWGPU_PRECISION_*). */
pwgpu_status pwgpu_set_precision(pwgpu_handle* h, int32_t precision);

/* Number of this library's kernel launches since it was loaded (all
 * handles, all threads); library GEMMs (cuBLAS/cuSOLVER) are not counted. */
pwgpu_status pwgpu_kernel_launches(int64_t* count);

/* The CUDA stream (cudaStream_t) a handle runs on, for callers that time or
 * order work against it. */
pwgpu_status pwgpu_get_stream(const pwgpu_handle* h, void** stream);

/* Copy the device projector matrix B of k-point ik (n_pw x n_ch complex,
 * column-major) to the host, whether it was uploaded or built on the device. */
pwgpu_status pwgpu_get_projectors(const pwgpu_handle* h, int32_t ik, double* b);

/* Basis size, grid size and channel count of a handle. */
pwgpu_status pwgpu_get_dims(const pwgpu_handle* h, int32_t* n_pw, int64_t* n_grid, int32_t* n_ch);

/* SCF controls: the fields of ScfParams (scf/mod.rs:228-252) that the
 * unpolarised and spin-polarised loops read, plus the eigensolver and
 * precision controls of the matrix-free form. */
typedef struct pwgpu_scf_params {
  int32_t n_bands;
  int32_t max_iter;
  double conv_threshold;    /* density rms, e/Å^3 (energy.rs:227-235) */
  double energy_threshold;  /* |E_n - E_{n-1}|, eV */
  double mixing_beta;
  int32_t mixing_ndim;
  int32_t mixing_mode;      /* MixingMode (mixing/mod.rs:186-223): 0 Anderson (Plain), 1 Anderson + Kerker,
                               2 Broyden, 3 Broyden + Kerker, 4 Periodic Pulay, 5 Periodic Pulay + Kerker */
  double kerker_q_tf;       /* Å^-1; <= 0 selects the Thomas-Fermi estimate */
  int32_t smearing;         /* 0 Fermi-Dirac, 1 Gaussian, 2 Methfessel-Paxton, 3 cold, 4 fixed */
  double smearing_sigma;    /* eV */
  double diag_tol;          /* eigen-residual floor |H psi - e psi|, eV */
  int32_t diag_max_iter;    /* LOBPCG block steps per SCF step */
  int32_t diag_extra_bands; /* < 0: automatic */
  int32_t precision;        /* PWGPU_PRECISION_* for H|psi> */
  double fp64_switch;       /* mixed: FP64 H|psi> once the density rms < this */
  int32_t verbose;          /* per-iteration line on stderr */
  /* nspin = 2 only (driver_spin.rs:125-167, 400-466): */
  double starting_magnetization; /* atom average of the per-species fractions; rho splits (1 +- m)/2 */
  int32_t fixed_magnetization;   /* 1: tot_magnetization fixes N_up - N_down (one Fermi level per spin) */
  double tot_magnetization;
  int32_t mixing_period;         /* Periodic Pulay: DIIS every period-th step (<= 0: 3) */
  /* Eigen-residual target of an SCF step: max(diag_tol, min(diag_tol_cap,
   * diag_tol_per_drho * last density rms change)) eV; <= 0 selects 3 eV per
   * e/Å^3 and 3e-2 eV. */
  double diag_tol_per_drho;
  double diag_tol_cap;
} pwgpu_scf_params;

/* ScfResult (scf/mod.rs:269-322) scalars. */
typedef struct pwgpu_scf_result {
  double total_energy, harris_foulkes_energy, free_energy, energy_sigma0, entropy_ts;
  double fermi_energy, final_delta;
  double e_band, e_hartree, e_xc, e_vxc, e_ewald;
  int32_t n_iterations, converged, nspin;
  double magnetization;
  int64_t h_applications;   /* band applications of H over the run */
  double max_residual;      /* largest eigen-residual of the last eigensolve */
  /* EnergyComponents (scf/energy.rs:597-670) of the final iteration, eV:
   * sum f w <psi|T|psi>, int rho V_loc dV (V_loc(G = 0) included), sum f w <psi|V_NL|psi>;
   * with e_hartree, e_xc, e_ewald and -entropy_ts they sum to total_energy at self-consistency */
  double e_kinetic, e_local, e_nonlocal;
} pwgpu_scf_result;

/* The start density of a handle created with v_local_g NULL (N doubles, e/Å^3):
 * the superposition of atomic densities of generate_initial_density
 * (scf/initial_density.rs:64-166), built on the device at pwgpu_create.
 * PWGPU_E_STATE for a handle whose local potential came from the caller. */
pwgpu_status pwgpu_initial_density(const pwgpu_handle* h, double* rho_r);

/* Read-back of the device V_loc(G) (N complex) and NLCC core density (N; zeros
 * without one); either pointer may be NULL.  For checking a device build. */
pwgpu_status pwgpu_get_local_potential(const pwgpu_handle* h, double* v_local_g, double* rho_core_r);

/* Run the SCF loop from rho_init_r (N doubles, e/Å^3, the total start
 * density).  Replaces run_scf_unpolarized (scf/driver.rs:266-742) for
 * nspin = 1 and run_scf_spin (scf/driver_spin.rs:114-839) for nspin = 2,
 * with the dense per-k eigensolve replaced by LOBPCG on the device.
 * Outputs may be NULL: eigenvalues nspin x n_k x n_bands (eV; spin up k-points
 * first, as ScfResult::eigenvalues), rho_r_out nspin x N (up then down for
 * nspin = 2), rho_g_basis_out n_pw complex (total rho(G) in basis order, as
 * ScfResult::rho_g).  Returns PWGPU_E_NOT_CONVERGED (result filled) if
 * max_iter is reached. */
pwgpu_status pwgpu_scf_run(pwgpu_handle* h, const pwgpu_scf_params* params, const double* rho_init_r,
                           pwgpu_scf_result* result, double* eigenvalues, double* rho_r_out,
                           double* rho_g_basis_out);

/* Exactly one SCF iteration seeded from a density given as rho(G) on the full
 * FFT grid (N complex, rho(G) = (1/N) sum_r rho(r) e^{-iG.r}, grid order of
 * g_vector_at_dims): replaces run_scf_iter1_from_rho_g_fft
 * (scf/transplant.rs:114-376).  rho_in(r) is the unnormalised inverse
 * transform of the input; V_eff from rho_in, eigenpairs to params->diag_tol
 * from a cold start, occupations, output density, energies and components
 * on the output density; result->final_delta is drho_rms(in, out) and
 * result->converged 0.  nspin = 1 only (PWGPU_E_INVALID otherwise), as the
 * reference.  Outputs may be NULL: eigenvalues n_k x n_bands, rho_r_out N,
 * rho_g_fft_out N complex (the output density on the same grid: a restart
 * point), rho_r_in N (the input density re-materialised). */
pwgpu_status pwgpu_scf_iter1_from_rho_g(pwgpu_handle* h, const pwgpu_scf_params* params,
                                        const double* rho_g_fft_in, pwgpu_scf_result* result,
                                        double* eigenvalues, double* rho_r_out, double* rho_g_fft_out,
                                        double* rho_r_in);

/* Lowest n_bands eigenpairs of H at (spin, ik) for the current V_eff
 * (diagonalize_dispatch, scf/driver.rs:125-184, lowest-n contract of
 * eigensolver/dense.rs:87-98).  psi_in: optional warm start (n_pw x n_bands
 * complex); evals ascending; psi_out optional. */
pwgpu_status pwgpu_eigensolve(pwgpu_handle* h, int32_t spin, int32_t ik, int32_t n_bands, double tol,
                              int32_t max_iter, const double* psi_in, double* evals, double* psi_out,
                              int32_t* iters, double* max_residual);

/* H applied to nb bands of a Gamma-real handle in its packed real form
 * (u = [Re psi(0), sqrt2 Re psi(G_p), sqrt2 Im psi(G_p)] over the half
 * sphere, n_pw reals per band, column-major), at the handle's precision: the
 * operator the Gamma-only eigensolver applies (two bands per complex FFT; in
 * the mixed form the projector products as 3xBF16 tensor-core GEMMs).
 * Diagnostic; the packing itself has no reference counterpart (the
 * reference keeps complex bands), the operator is H of
 * scf/potentials.rs:163-190 + potential/nonlocal.rs:432-450.
 * PWGPU_E_STATE on a handle with complex bands. */
pwgpu_status pwgpu_apply_h_packed(pwgpu_handle* h, int32_t spin, const double* u, int32_t nb, double* hu);

/* The bands of (spin, ik) left on the device by the last pwgpu_scf_run (its
 * final eigensolve) or pwgpu_eigensolve: the first n_bands eigenvectors as
 * complex columns (n_pw x n_bands, column-major, basis order), ascending in
 * energy.  The eigenvector half of diagonalize_dispatch's EigenResult
 * (scf/driver.rs:125-184), which ScfResult does not carry; PWGPU_E_STATE
 * before any solve. */
pwgpu_status pwgpu_get_bands(pwgpu_handle* h, int32_t spin, int32_t ik, int32_t n_bands, double* psi_out);

/* rho(r) = sum_k w_k sum_b occ f |IFFT psi|^2, renormalised to N_el and
 * symmetrised (compute_density, scf/density.rs:41-111, then
 * symmetrize_density_g).  occ: n_k x n_bands; psi: n_k blocks n_pw x n_bands. */
pwgpu_status pwgpu_density(pwgpu_handle* h, int32_t n_bands, const double* occ, const double* psi, double* rho_r);

/* In-place G-space symmetrisation of a real density (symmetry/density/g_space.rs:147-252). */
pwgpu_status pwgpu_symmetrize(pwgpu_handle* h, double* rho_r);

/* V_eff(G) = V_loc + V_H + V_xc from rho (energy.rs:293-358, xc.rs:129-288)
 * and sets it as the H|psi> potential of spin 0; energies[3] = E_H, E_xc,
 * int rho_val v_xc (eV). */
pwgpu_status pwgpu_potentials(pwgpu_handle* h, const double* rho_r, double* veff_g, double* energies);

/* One density-mixing step (Mixer::mix, scf/mixing/mod.rs:281-287):
 * mode as pwgpu_scf_params.mixing_mode (Anderson, mixing/anderson.rs:170-266;
 * modified Broyden, mixing/broyden.rs:140-245; Periodic Pulay,
 * mixing/anderson.rs:294-372 with `period`; each with or without Kerker).
 * channel 0 or 1 selects one of two independent histories on the handle (the
 * CCMX total / magnetisation pair of driver_spin.rs:792-826).  rho_in,
 * rho_out, rho_next: N doubles on the host (rho_next may alias rho_in).
 * Kerker preconditions the residual with G^2/(G^2 + q_tf^2), q_tf in Å^-1
 * (Anderson: <= 0 selects the Thomas-Fermi estimate, kerker.rs:41-49;
 * Broyden and Periodic Pulay always use the estimate).  The first call after
 * pwgpu_mix_reset (or after a change of ndim) starts a new history. */
pwgpu_status pwgpu_mix(pwgpu_handle* h, int32_t channel, int32_t mode, const double* rho_in, const double* rho_out,
                       double* rho_next, double beta, int32_t ndim, int32_t period, double q_tf);
pwgpu_status pwgpu_mix_reset(pwgpu_handle* h);

/* UPF v2 norm-conserving pseudopotential, read on the host by the library:
 * parse_upf_body (pseudopotential/upf/parse.rs:20-135) with the scanning of
 * upf/xml.rs -- each header attribute and data block taken from its first
 * textual occurrence, PP_RHOATOM zero when absent or unreadable, the NLCC
 * core charge read when core_correction="T" (zero when the block is
 * unreadable, empty without it).  Arrays come out in the units of
 * pwgpu_system's radial fields: r and rab in Å, V_loc in eV, r·beta(r)
 * divided by sqrt(Å per bohr), D_ij in eV (n_proj x n_proj, row-major),
 * PP_RHOATOM per Å, core charge in e/Å^3.  A malformed file returns
 * PWGPU_E_PARSE with the reason in pwgpu_last_error(). */
typedef struct pwgpu_upf pwgpu_upf;

typedef struct pwgpu_upf_info {
  char element[8];          /* element symbol, NUL-terminated */
  double z_valence;
  int32_t l_max;
  int32_t n_proj;
  int32_t mesh;             /* radial mesh points */
  int32_t has_nlcc;         /* 1: PWGPU_UPF_NLCC holds mesh values (else none) */
  int32_t has_rho_atom;     /* 1: PP_RHOATOM has a nonzero value */
} pwgpu_upf_info;

#define PWGPU_UPF_R 0        /* mesh */
#define PWGPU_UPF_RAB 1      /* mesh */
#define PWGPU_UPF_LOCAL 2    /* mesh */
#define PWGPU_UPF_BETA 3     /* mesh, projector `index` (0-based) */
#define PWGPU_UPF_DIJ 4      /* n_proj * n_proj */
#define PWGPU_UPF_RHOATOM 5  /* mesh */
#define PWGPU_UPF_NLCC 6     /* mesh when has_nlcc, else 0 */

/* Parse len bytes of UPF text (UpfPseudoPotential::load's body,
 * upf/mod.rs:98-135); *out is freed with pwgpu_upf_free. */
pwgpu_status pwgpu_upf_parse(const char* text, int64_t len, pwgpu_upf** out);
/* Read and parse a UPF file (UpfPseudoPotential::load_from_path, upf/mod.rs:98). */
pwgpu_status pwgpu_upf_load(const char* path, pwgpu_upf** out);
pwgpu_status pwgpu_upf_get_info(const pwgpu_upf* u, pwgpu_upf_info* info);
/* Copy one array (PWGPU_UPF_*) into out, which holds capacity doubles
 * (PWGPU_E_INVALID when it is too small). */
pwgpu_status pwgpu_upf_get_array(const pwgpu_upf* u, int32_t which, int32_t index, double* out, int64_t capacity);
/* Angular momentum of each projector (n_proj ints). */
pwgpu_status pwgpu_upf_get_beta_l(const pwgpu_upf* u, int32_t* l);
/* Free a parsed pseudopotential (NULL is a no-op). */
pwgpu_status pwgpu_upf_free(pwgpu_upf* u);

/* Occupations of a set of eigenvalues, host FP64, no device work:
 * find_fermi_energy / occupation / entropy_ts (scf/smearing.rs:38-252).
 * ev: n_sets x nb (one row per (spin, k) set), weights: n_sets (k weights);
 * smearing as pwgpu_scf_params.smearing; spin_factor 2 (nspin 1) or 1.
 * find_fermi != 0: *fermi_energy receives the level that holds n_electrons;
 * otherwise *fermi_energy is the given level.  occ (n_sets x nb, may be
 * NULL) = spin_factor * f(e); *entropy_ts (may be NULL) = TS, eV. */
pwgpu_status pwgpu_occupations(int32_t n_sets, int32_t nb, const double* ev, const double* weights,
                               double n_electrons, double sigma, int32_t smearing, double spin_factor,
                               int32_t find_fermi, double* fermi_energy, double* occ, double* entropy_ts);

/* Local part of H|psi> (kinetic diagonal + V_eff through the FFT pipeline;
 * no Kleinman-Bylander term) on device pointers, allocating nothing.  No
 * counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code living inside a host framework whose memory manager owns all device
 * memory, and serving loops that cannot afford cudaMalloc's implicit
 * device-wide synchronisation.  The FFT intermediates go to one fixed
 * 32 MiB device array inside the library (held by every GPU that loads
 * it); a grid whose single band needs more than that is rejected with
 * PWGPU_E_INVALID.  The first call on a device looks the array's address
 * up, so make it before any stream capture.  All calls share the array:
 * calls that overlap on the GPU race.  Result equals pwgpu_apply_h_device
 * for a system without projectors. */
pwgpu_status pwgpu_apply_h_local_noalloc(pwgpu_handle* h, int32_t spin, int32_t ik, const void* psi_dev,
                                         int64_t ldpsi, int32_t nb, void* hpsi_dev, int64_t ldh, void* stream);

/* Batched small generalized Hermitian eigensolve H c = e S c (m <= 64,
 * column-major complex, batch consecutive problems): the Rayleigh-Ritz
 * kernel, exposed for testing.  evals batch x nev ascending; C batch x m x nev. */
pwgpu_status pwgpu_small_geneig(int32_t batch, int32_t m, int32_t nev, const double* H, const double* S,
                                double* evals, double* C);

/* Lowest nev eigenpairs of a dense m x m Hermitian (complex_matrix != 0,
 * interleaved complex) or real symmetric matrix, column-major, both triangles
 * given: the subspace eigensolver of the Rayleigh-Ritz step (one thread-block
 * cluster; Householder tridiagonalisation in distributed shared memory,
 * multisection, inverse iteration, back-transform), exposed for testing.
 * Stands in for the dense self_adjoint_eigen of eigensolver/dense.rs:50-98
 * inside the subspace.  w: nev ascending; Z: m x nev eigenvectors.
 * *cluster_ctas (may be NULL) receives the cluster size used, *kernel_ms
 * (may be NULL) the device time of the solve (CUDA events around its one
 * launch).  PWGPU_E_INVALID beyond the supported size (m <= 544 real;
 * complex as shared memory allows). */
pwgpu_status pwgpu_dense_eigh(int32_t m, int32_t nev, int32_t complex_matrix, const double* A, double* w,
                              double* Z, int32_t* cluster_ctas, double* kernel_ms);

/*
 * The eigensolver's orthonormalisation kernel on a host matrix: the
 * Cholesky factor G = R^H R of the Hermitian (complex_matrix != 0,
 * interleaved re/im) or symmetric positive definite q x q matrix G
 * (column-major; upper triangle read) and its inverse.  Writes Ri = R^-1
 * (q x q, zero below the diagonal), rdiag (q entries, may be NULL) = R's
 * diagonal, and *info = 0, or 1 + the first row whose pivot is not positive
 * (LAPACK potrf's count; Ri is then undefined).  cluster_ctas and kernel_ms
 * (may be NULL) as for pwgpu_dense_eigh.  The reference keeps its bases
 * orthonormal inside faer (the Gram-Schmidt of the Krylov-Schur solver,
 * eigensolver/iterative.rs:1-20, and the dense solver's unitary
 * eigenvectors, eigensolver/dense.rs:50-98); this is the Cholesky-QR step of
 * the block eigensolver that replaces them, exposed for testing.
 */
pwgpu_status pwgpu_dense_cholesky_inverse(int32_t q, int32_t complex_matrix, const double* G, double* Ri,
                                          double* rdiag, int32_t* info, int32_t* cluster_ctas, double* kernel_ms);

/*
 * Serving: a job queue in front of pwgpu_scf_run.  No counterpart in the
 * reference (its front door, scf::run_scf at scf/mod.rs:344-402, runs one
 * solve per call); this is the submit/poll seam a service wraps around it.
 * Each worker thread owns one job at a time: it builds a handle for the
 * job's system on the server's device, runs the SCF and releases the
 * handle.  A job starts only when the estimated device footprint of the
 * running jobs plus its own fits the HBM budget (first come, first served:
 * the queue head waits rather than being overtaken); a job larger than the
 * whole budget is refused at submit with PWGPU_E_OOM.
 */
typedef struct pwgpu_server pwgpu_server;

typedef struct pwgpu_server_options {
  int32_t device;            /* CUDA device ordinal */
  int32_t workers;           /* jobs in flight at most; 0 = 4 */
  int32_t precision;         /* pwgpu_options.precision of every job's handle */
  int32_t lanes_per_job;     /* pwgpu_options.lanes of every job's handle; 0 = 2 */
  int64_t hbm_budget_bytes;  /* admission budget; 0 = 80 % of the device memory free at create */
} pwgpu_server_options;

#define PWGPU_JOB_QUEUED 0
#define PWGPU_JOB_RUNNING 1
#define PWGPU_JOB_DONE 2

typedef struct pwgpu_job_info {
  int32_t state;            /* PWGPU_JOB_* */
  pwgpu_status status;      /* the job's pwgpu_scf_run status once done (PWGPU_E_NOT_CONVERGED: result filled) */
  double queue_s;           /* submit -> start, seconds (so far, while queued) */
  double run_s;             /* start -> done, seconds (so far, while running) */
  int64_t footprint_bytes;  /* admission estimate */
} pwgpu_job_info;

typedef struct pwgpu_server_stats {
  int64_t submitted, queued, running, done, failed;
  int64_t bytes_in_use, peak_bytes, budget_bytes;
} pwgpu_server_stats;

pwgpu_status pwgpu_server_create(const pwgpu_server_options* opt, pwgpu_server** out);

/* Stops the workers after their running jobs; queued jobs are dropped. */
pwgpu_status pwgpu_server_destroy(pwgpu_server* s);

/* Queue one SCF: the system, parameters and start density (nspin = the
 * system's; rho_init_r N doubles) are copied, so the caller's arrays are
 * free again on return. */
pwgpu_status pwgpu_server_submit(pwgpu_server* s, const pwgpu_system* sys, const pwgpu_scf_params* params,
                                 const double* rho_init_r, int64_t* job_id);

pwgpu_status pwgpu_server_poll(pwgpu_server* s, int64_t job_id, pwgpu_job_info* info);

/* Wait until job_id is done (PWGPU_E_TIMEOUT after timeout_s seconds). */
pwgpu_status pwgpu_server_wait(pwgpu_server* s, int64_t job_id, double timeout_s, pwgpu_job_info* info);

/* Wait until some finished job has not been collected yet and return its
 * id (each finished job is returned once; PWGPU_E_TIMEOUT after timeout_s). */
pwgpu_status pwgpu_server_wait_any(pwgpu_server* s, double timeout_s, int64_t* job_id);

/* Result of a finished job: the ScfResult scalars, and (when not NULL) the
 * eigenvalues nspin x n_k x n_bands and the job's error message (valid
 * until the job is released). */
pwgpu_status pwgpu_server_result(pwgpu_server* s, int64_t job_id, pwgpu_scf_result* result, double* eigenvalues,
                                 const char** error);

/* Forget a finished job. */
pwgpu_status pwgpu_server_release(pwgpu_server* s, int64_t job_id);

pwgpu_status pwgpu_server_get_stats(pwgpu_server* s, pwgpu_server_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* PWGPU_H */
