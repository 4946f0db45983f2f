// Dense linear-algebra helpers of the Rayleigh-Ritz step (linalg.cu).
#pragma once

#include <cuda_runtime.h>

#include "handle.hpp"

namespace pwgpu {

// Batched small generalized Hermitian eigenproblems (m <= 64): lowest nev
// eigenpairs of H c = lambda S c, ascending; C is S-orthonormal.
// status_dev[b]: 0 ok, 1 S not positive definite, 2 Jacobi sweep cap hit.
Status small_geneig_batched(const double2* H, const double2* S, long ld, long stride, int m, int nev, int batch,
                            double* evals, double2* C, long ldc, long cstride, int* status_dev, cudaStream_t s);
size_t small_geneig_smem(int m);

// One large problem through cuSOLVER zhegvd (H, S overwritten; w ascending,
// eigenvectors in H).
Status large_geneig(Handle& h, double2* Hm, double2* Sm, int m, double* w, cudaStream_t s);

// Lowest nev eigenpairs of the Hermitian (complex) or symmetric (real) m x m
// matrix A (both triangles stored, leading dim lda), one thread-block
// cluster (eigh.cu): w ascending (nev), eigenvectors in Z (m x nev, ld ldz).
// work: eigh_cluster_work_doubles(m, nev) doubles; status_dev (zeroed here)
// becomes 1 if a non-finite value appeared.  A is read only.
size_t eigh_cluster_work_doubles(int m, int nev);
bool eigh_cluster_supported(int m, bool complex_matrix);
int eigh_cluster_size(int m, bool complex_matrix);
Status eigh_cluster(const double* A, long lda, int m, int nev, double* w, double* Z, long ldz, double* work,
                    int* status_dev, cudaStream_t s);
Status eigh_cluster(const double2* A, long lda, int m, int nev, double* w, double2* Z, long ldz, double* work,
                    int* status_dev, cudaStream_t s);

// Cholesky factor and its inverse (chol.cu): G = R^H R for the Hermitian
// (complex) or symmetric (real) positive definite q x q matrix G (column
// major, ld q; upper triangle read, G overwritten as scratch).  Writes
// Ri = R^-1 (q x q, ld q, zero below the diagonal), rdiag[i] = R_ii (rdiag
// may be null) and *info_dev = 0, or 1 + the first row whose pivot is not
// positive (Ri then undefined).  One cluster launch on stream s.
Status chol_inv(double* G, int q, double* Ri, double* rdiag, int* info_dev, cudaStream_t s);
Status chol_inv(double2* G, int q, double2* Ri, double* rdiag, int* info_dev, cudaStream_t s);
int chol_inv_cluster_size(int q, bool complex_matrix);

}  // namespace pwgpu
