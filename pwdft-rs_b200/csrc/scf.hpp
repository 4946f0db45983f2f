// SCF loop on the device: per-k LOBPCG eigensolver (lobpcg.cu), density, G-space
// symmetrisation, Hartree + LDA potentials, energies and Anderson/Kerker
// mixing (scf.cu).
#pragma once

#include <vector>

#include "handle.hpp"

namespace pwgpu {

struct ScfParams {
  int n_bands = 8;
  int max_iter = 100;
  double conv_threshold = 1e-6;     // density rms, e/Å³ (energy.rs:227-235)
  double energy_threshold = 1e-5;   // |E_n - E_{n-1}|, eV
  double mixing_beta = 0.3;
  int mixing_ndim = 8;
  int mixing_mode = 0;              // 0 Anderson, 1 + Kerker, 2 Broyden, 3 + Kerker, 4 Periodic Pulay, 5 + Kerker
  int mixing_period = 3;            // Periodic Pulay: DIIS every period-th step
  double kerker_q_tf = 0.0;         // Å⁻¹; <= 0 selects the Thomas-Fermi estimate
  int smearing = 0;                 // 0 Fermi-Dirac, 1 Gaussian, 2 Methfessel-Paxton, 3 cold, 4 fixed
  double sigma = 0.01;              // eV
  double diag_tol = 1e-8;           // eigen-residual norm floor, eV
  int diag_max_iter = 60;
  int diag_extra_bands = -1;        // < 0: automatic
  int precision = 0;                // 0 FP64, 1 mixed
  double fp64_switch = 1e-6;        // mixed: FP64 H|psi> once delta rho < this
  double diag_tol_per_drho = 3.0;   // eigen-residual target of an SCF step: eV per (e/Å^3) of delta rho
  double diag_tol_cap = 3e-2;       // eV, its loosest value
  int verbose = 0;
  // nspin = 2 (driver_spin.rs:125-167): atom average of the per-species
  // starting_magnetization fractions, and the optional fixed total moment
  double starting_magnetization = 0.0;
  int fixed_magnetization = 0;
  double tot_magnetization = 0.0;
  // one iteration only, eigenpairs to diag_tol from a cold start, reported
  // as a completed run (the transplanted iteration, transplant.rs:114-376)
  int single_step = 0;
};

struct ScfResult {
  double total_energy = 0, harris_foulkes_energy = 0, free_energy = 0, energy_sigma0 = 0, entropy_ts = 0;
  double fermi_energy = 0, final_delta = 0;
  double e_band = 0, e_hartree = 0, e_xc = 0, e_vxc = 0, e_ewald = 0;
  int n_iterations = 0, converged = 0, nspin = 1;
  double magnetization = 0;
  long h_applications = 0;
  double max_residual = 0;
  double e_kinetic = 0, e_local = 0, e_nonlocal = 0;  // EnergyComponents of the final iteration
};

// Whole SCF (driver.rs:266-742 for nspin = 1).  rho_init: N doubles on the
// host (start density).  evals_out: n_k*n_bands (may be null); rho_out: N
// (may be null); rho_g_basis_out: n_pw complex (may be null).
Status scf_run(Handle& h, const ScfParams& p, const double* rho_init, ScfResult& res, double* evals_out,
               double* rho_out, double* rho_g_basis_out);

// One SCF iteration seeded from rho(G) on the full FFT grid (N complex,
// rho(G) = (1/N) sum_r rho(r) e^{-iG.r}): run_scf_iter1_from_rho_g_fft,
// scf/transplant.rs:114-376.  nspin = 1.  rho_in_host (N, the input density
// re-materialised), rho_g_fft_out (N complex, the output density) may be null.
Status scf_iter1_from_rho_g(Handle& h, const ScfParams& p, const double* rho_g_fft_in, ScfResult& res,
                            double* evals_out, double* rho_out_host, double* rho_g_fft_out, double* rho_in_host);

// Pieces exposed through the C-ABI for parity tests.
Status eigensolve_k(Handle& h, int spin, int ik, int n_bands, double tol, int max_iter, const double* psi_in,
                    double* evals, double* psi_out, int* iters, double* max_res, int precision);
// The first n_bands bands of (spin, ik) left on the device by the last SCF
// run or eigensolve, as complex columns (n_pw x n_bands, basis order).
Status bands_to_host(Handle& h, int spin, int ik, int n_bands, double* psi_out);
Status density_from_host(Handle& h, int n_bands, const double* occ, const double* psi_all, double* rho_out);
Status symmetrize_host(Handle& h, double* rho);
Status potentials_host(Handle& h, const double* rho, double* veff_g, double* energies);
// One Anderson/Kerker mixing step on history `channel` (0 or 1), host arrays.
Status mix_host(Handle& h, int channel, int mode, const double* in, const double* out, double* next, double beta,
                int ndim, int period, double q_tf);
Status mix_reset(Handle& h);
// Fermi level (bisection, or *fermi_energy as given), occupations
// spin_factor * f(e) per state and TS, host FP64 (smearing.rs:38-252).
Status occupations_host(int n_sets, int nb, const double* ev, const double* w, double n_electrons, double sigma,
                        int scheme, double spin_factor, bool find_fermi, double* fermi_energy, double* occ,
                        double* ts);

}  // namespace pwgpu
