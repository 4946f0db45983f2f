// Block eigensolver of one (spin, k) Hamiltonian on the device (lobpcg.cu).
#pragma once

#include <vector>

#include "handle.hpp"

namespace pwgpu {

// Ritz block of one (spin, k): persists across SCF iterations.  V and HV hold
// n_pw x 3 nd columns, the current block X (nd), the preconditioned
// residual directions W and the previous-step directions P of the active
// bands.  X is orthonormal on return from the solver.
struct EigVecs {
  double2* V = nullptr;
  double2* HV = nullptr;
  std::vector<double> evals;  // nd Ritz values, ascending
  bool init = false;
};

// Scratch shared by all (spin, k) blocks of one handle.
struct EigWork {
  int nd = 0;
  long n = 0;
  double2* T = nullptr;    // n x nd: preconditioned residuals, then the new X
  double2* HXn = nullptr;  // n x nd: new HX
  double2* Pn = nullptr;   // n x nd: P of the last step (active bands)
  double2* HPn = nullptr;  // n x nd
  double2* Hs = nullptr;   // m x m (m <= 3 nd): subspace matrix, then eigenvectors (cuSOLVER)
  double2* Cs = nullptr;   // m x m: eigenvectors (batched small solver), gathered columns
  double2* G = nullptr;    // m x m: Gram / coupling blocks
  double2* Z = nullptr;    // m x m: coupling block, projection coefficients
  double2* Id = nullptr;   // m x m identity (small solver's overlap)
  double* lam = nullptr;   // m: Ritz values of the last subspace solve
  double* lam0 = nullptr;  // nd: Ritz values the residuals refer to
  double* colsq = nullptr; // 3 nd
  double* partials = nullptr;
  int* idx = nullptr;      // 3 nd
  int* status = nullptr;
  double2* solver_work = nullptr;
  size_t solver_lwork = 0;
  int* info = nullptr;
  double* eigh_work = nullptr;  // scratch of the cluster eigensolver (eigh.cu)
  double2* XX = nullptr;        // nd x nd: X^H HX at the start of a solve
  double* defect = nullptr;     // max |Y^H Y - I| of a Cholesky-QR pass
  size_t eigh_work_len = 0;
};

struct EigStats {
  long happ = 0;     // H|psi> columns applied
  int iters = 0;     // block iterations
  double max_res = 0.0;  // largest residual norm over the first nconv bands, eV
};

Status eig_work_alloc(EigWork& w, long n, int nd);
void eig_work_release(EigWork& w);
Status eig_vecs_alloc(EigVecs& v, long n, int nd);
void eig_vecs_release(EigVecs& v);

// Lowest nd eigenpairs of H(spin, k) until the first nconv residual norms
// |H x - lambda x| fall below tol (eV) or max_iter block steps have run.
// HX is recomputed in FP64 on entry; the search directions W use
// `precision` (0 FP64, 1 mixed).  v0: mean V_eff(r), the preconditioner's
// diagonal shift.
Status lobpcg(Handle& h, EigWork& w, EigVecs& k, int spin, int ik, double v0, double tol, int max_iter, int nconv,
              int precision, EigStats& out);

}  // namespace pwgpu
