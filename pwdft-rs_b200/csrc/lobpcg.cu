// Block eigensolver of one (spin, k) Hamiltonian: locally optimal block
// preconditioned conjugate gradients (LOBPCG) with soft locking, on an
// explicitly orthonormal basis [X | W | P].
//
// Stands in for the dense diagonalisation of the reference's per-k step
// (pwdft-core/src/eigensolver/dense.rs:50-98, the lowest n_bands pairs of the
// full n_pw x n_pw Hamiltonian): H is only applied (apply_h_device, or
// apply_h_real for Gamma-only handles) and the lowest nd Ritz pairs are
// refined until the residual norms of the first nconv fall below tol.
//
// Numerical design:
//  * the basis is orthonormal by construction (block Gram-Schmidt against X,
//    Cholesky-QR inside W and P), so each Rayleigh-Ritz step is a standard
//    Hermitian problem; an ill-conditioned overlap never enters a solve;
//  * H is applied to W after it is orthonormalised, so H W is consistent with
//    W whatever the precision of the product;
//  * H P follows P through the same linear combinations; P columns whose
//    component outside span(X, W) is small (which would amplify the error of
//    the stored H P) are dropped, and the whole P block is dropped when its
//    Cholesky factor shows near dependence;
//  * HX is recomputed in FP64 on entry and the X-(W,P) coupling of the
//    subspace matrix is formed from HX, so reduced-precision products of the
//    search directions only enter through the (small) correction
//    coefficients; the residuals the convergence test reads carry no
//    reduced-precision floor.
//
// The solver is written once for complex bands (double2) and for the real
// packed bands of Gamma-only handles (double): the same steps with real
// GEMMs, Cholesky and symmetric eigensolver.
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <random>
#include <type_traits>
#include <vector>

#include "linalg.hpp"
#include "lobpcg.hpp"

namespace pwgpu {

namespace {

constexpr double kRyToEv = 13.605693122994;
constexpr int kColBlocks = 64;      // partial sums per column reduction
constexpr int kSmallSolveMax = 64;  // subspace size up to which the one-CTA solver runs
// P columns whose component outside span(X, W) is below this fraction of
// their norm are dropped (FP64 / reduced-precision search directions)
constexpr double kPDropFp64 = 1e-5;
constexpr double kPDropMixed = 3e-2;
// A Cholesky-QR pass is skipped when its block is orthonormal to this
// (max |Y^H Y - I|): the second pass of CholQR2 then has nothing to fix.
constexpr double kOrthoSkipTol = 1e-12;

inline unsigned blocks_for(long n, int t = 256) { return (unsigned)std::max<long>(1, (n + t - 1) / t); }

// scalar helpers for double (Gamma-real) and double2 (complex)
__host__ __device__ __forceinline__ double abs2(double x) { return x * x; }
__host__ __device__ __forceinline__ double abs2(double2 x) { return x.x * x.x + x.y * x.y; }
__host__ __device__ __forceinline__ double scl(double x, double s) { return x * s; }
__host__ __device__ __forceinline__ double2 scl(double2 x, double s) { return make_double2(x.x * s, x.y * s); }
__host__ __device__ __forceinline__ double axpy_neg(double hx, double l, double x) { return hx - l * x; }
__host__ __device__ __forceinline__ double2 axpy_neg(double2 hx, double l, double2 x) {
  return make_double2(hx.x - l * x.x, hx.y - l * x.y);
}
__host__ __device__ __forceinline__ double conj_of(double x) { return x; }
__host__ __device__ __forceinline__ double2 conj_of(double2 x) { return make_double2(x.x, -x.y); }
__host__ __device__ __forceinline__ double herm_avg(double a, double b) { return 0.5 * (a + b); }
__host__ __device__ __forceinline__ double2 herm_avg(double2 a, double2 b) {
  return make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
}
template <typename T> __host__ __device__ __forceinline__ T real_scalar(double v);
template <> __host__ __device__ __forceinline__ double real_scalar<double>(double v) { return v; }
template <> __host__ __device__ __forceinline__ double2 real_scalar<double2>(double v) { return make_double2(v, 0.0); }
__host__ __device__ __forceinline__ double real_part(double x) { return x; }
__host__ __device__ __forceinline__ double real_part(double2 x) { return x.x; }

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  v = 0.0;
  if (wid == 0) {
    v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;
}

// Residual R = HX - lambda X, preconditioned into T with the smooth
// denominator 0.5 (1 + x + sqrt(1 + (x-1)^2)) in Ry, x = (|k+G|^2 + v0 -
// lambda)/Ry; per-column partial sums of |R|^2.
template <typename S>
__global__ void k_resid_precond(const S* __restrict__ X, const S* __restrict__ HX, S* __restrict__ T, long ld, int n,
                                const double* __restrict__ lam, const double* __restrict__ kin, double v0,
                                double* __restrict__ partials) {
  __shared__ double sh[32];
  const int col = blockIdx.y;
  const double l = lam[col];
  const S* x = X + (long)col * ld;
  const S* hx = HX + (long)col * ld;
  S* t = T + (long)col * ld;
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const S r = axpy_neg(hx[i], l, x[i]);
    acc += abs2(r);
    const double xx = (kin[i] + v0 - l) / kRyToEv;
    const double den = 0.5 * (1.0 + xx + sqrt(1.0 + (xx - 1.0) * (xx - 1.0))) * kRyToEv;
    t[i] = scl(r, 1.0 / den);
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[(long)col * gridDim.x + blockIdx.x] = acc;
}

template <typename S>
__global__ void k_col_sumsq(const S* __restrict__ X, long ld, int n, double* __restrict__ partials) {
  __shared__ double sh[32];
  const int col = blockIdx.y;
  const S* x = X + (long)col * ld;
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc += abs2(x[i]);
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[(long)col * gridDim.x + blockIdx.x] = acc;
}

// sums[col] = sum of the nblk partials of each column (fixed order)
__global__ void k_col_final(const double* __restrict__ partials, int nblk, int ncols, double* __restrict__ sums) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncols) return;
  double acc = 0.0;
  for (int b = 0; b < nblk; ++b) acc += partials[(long)col * nblk + b];
  sums[col] = acc;
}

// X[:, c] /= sqrt(sumsq[c]) (and Y[:, c] with the same factor when Y != null)
template <typename S>
__global__ void k_scale_cols_invsqrt(S* __restrict__ X, S* __restrict__ Y, long ld, int n,
                                     const double* __restrict__ sumsq) {
  const int col = blockIdx.y;
  const double s = sumsq[col] > 0.0 ? 1.0 / sqrt(sumsq[col]) : 0.0;
  S* x = X + (long)col * ld;
  S* y = Y ? Y + (long)col * ld : nullptr;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = scl(x[i], s);
    if (y) y[i] = scl(y[i], s);
  }
}

// dst[:, c] = src[:, idx[c]] over `rows` rows (src and dst do not overlap)
template <typename S>
__global__ void k_gather_cols(const S* __restrict__ src, long lds, const int* __restrict__ idx, S* __restrict__ dst,
                              long ldd, int rows) {
  const int c = blockIdx.y;
  const S* s = src + (long)idx[c] * lds;
  S* d = dst + (long)c * ldd;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) d[i] = s[i];
}

template <typename S>
__global__ void k_scatter_cols(const S* __restrict__ src, long lds, const int* __restrict__ idx, S* __restrict__ dst,
                               long ldd, int rows) {
  const int c = blockIdx.y;
  const S* s = src + (long)c * lds;
  S* d = dst + (long)idx[c] * ldd;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) d[i] = s[i];
}

// Subspace matrix Hs (m x m, ld m) over the basis [X | B], X holding nd Ritz
// vectors with values lam:  [[diag(lam), Z^H], [Z, (G + G^H)/2]],
// Z = B^H HX (q x nd, ld q), G = B^H HB (q x q, ld q), q = m - nd.  When XX
// (X^H HX, nd x nd, ld nd) is given, X need not be Ritz vectors: the X block
// is (XX + XX^H)/2.
template <typename S>
__global__ void k_assemble_rr(S* __restrict__ Hs, int m, int nd, const double* __restrict__ lam,
                              const S* __restrict__ Z, const S* __restrict__ G, const S* __restrict__ XX = nullptr) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)m * m) return;
  const int r = (int)(t % m), c = (int)(t / m), q = m - nd;
  S v;
  if (r < nd && c < nd) {
    v = XX ? herm_avg(XX[r + (long)c * nd], XX[c + (long)r * nd]) : real_scalar<S>(r == c ? lam[r] : 0.0);
  } else if (c < nd) {
    v = Z[(r - nd) + (long)c * q];
  } else if (r < nd) {
    v = conj_of(Z[(c - nd) + (long)r * q]);
  } else {
    v = herm_avg(G[(r - nd) + (long)(c - nd) * q], G[(c - nd) + (long)(r - nd) * q]);
  }
  Hs[t] = v;
}

template <typename S> __global__ void k_set_identity(S* __restrict__ A, int m) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)m * m) return;
  A[t] = real_scalar<S>((t % m) == (t / m) ? 1.0 : 0.0);
}

// out[i] = Re A[i, i]
template <typename S> __global__ void k_diag_real(const S* __restrict__ A, int ld, int m, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) out[i] = real_part(A[i + (long)i * ld]);
}

// out = max_ij |G_ij - delta_ij| over the q x q Gram matrix (out zeroed by
// the caller; non-negative doubles order like their bit patterns)
__device__ __forceinline__ double defect_of(double g, bool diag) { return fabs(diag ? g - 1.0 : g); }
__device__ __forceinline__ double defect_of(double2 g, bool diag) { return hypot(diag ? g.x - 1.0 : g.x, g.y); }
template <typename S> __global__ void k_gram_defect(const S* __restrict__ G, int q, double* __restrict__ out) {
  double v = 0.0;
  const long nn = (long)q * q;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < nn; t += (long)gridDim.x * blockDim.x) {
    const int r = (int)(t % q), cc = (int)(t / q);
    v = fmax(v, defect_of(G[t], r == cc));
  }
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(out), (unsigned long long)__double_as_longlong(v));
}

// real m x m <-> complex (zero imaginary part), for the one-CTA complex solver
__global__ void k_real_to_complex(const double* __restrict__ a, double2* __restrict__ z, long n) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) z[t] = make_double2(a[t], 0.0);
}
__global__ void k_complex_to_real(const double2* __restrict__ z, double* __restrict__ a, long n) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) a[t] = z[t].x;
}

template <typename T> Status walloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) return fail(kOom, std::string("cudaMalloc (eigensolver): ") + cudaGetErrorString(e));
  return kOk;
}

// ---------------------------------------------------------------------------
// BLAS / LAPACK steps, overloaded on the scalar type
// ---------------------------------------------------------------------------

struct Ctx {
  Handle& h;
  EigWork& w;
  cudaStream_t s;
  long n;
  unsigned gx;
};

Status gemm(Ctx& c, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, const double2* A, long lda,
            const double2* B, long ldb, double2* C, long ldc, double beta_re = 0.0, double alpha_re = 1.0) {
  if (m == 0 || n == 0) return kOk;
  const cuDoubleComplex al = make_cuDoubleComplex(alpha_re, 0.0), be = make_cuDoubleComplex(beta_re, 0.0);
  if (cublasZgemm(c.h.blas, ta, tb, m, n, k, &al, reinterpret_cast<const cuDoubleComplex*>(A), (int)lda,
                  reinterpret_cast<const cuDoubleComplex*>(B), (int)ldb, &be, reinterpret_cast<cuDoubleComplex*>(C),
                  (int)ldc) != CUBLAS_STATUS_SUCCESS)
    return fail(kCuda, "cublasZgemm failed (eigensolver)");
  return kOk;
}

Status gemm(Ctx& c, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, const double* A, long lda,
            const double* B, long ldb, double* C, long ldc, double beta = 0.0, double alpha = 1.0) {
  if (m == 0 || n == 0) return kOk;
  const cublasOperation_t ra = ta == CUBLAS_OP_C ? CUBLAS_OP_T : ta, rb = tb == CUBLAS_OP_C ? CUBLAS_OP_T : tb;
  if (cublasDgemm(c.h.blas, ra, rb, m, n, k, &alpha, A, (int)lda, B, (int)ldb, &beta, C, (int)ldc) !=
      CUBLAS_STATUS_SUCCESS)
    return fail(kCuda, "cublasDgemm failed (eigensolver)");
  return kOk;
}

Status add_shift(Ctx& c, double2* G, double2* Id, int q, double shift) {
  const cuDoubleComplex al = make_cuDoubleComplex(1.0, 0.0), be = make_cuDoubleComplex(shift, 0.0);
  if (cublasZgeam(c.h.blas, CUBLAS_OP_N, CUBLAS_OP_N, q, q, &al, reinterpret_cast<cuDoubleComplex*>(G), q, &be,
                  reinterpret_cast<cuDoubleComplex*>(Id), q, reinterpret_cast<cuDoubleComplex*>(G),
                  q) != CUBLAS_STATUS_SUCCESS)
    return fail(kCuda, "cublasZgeam failed (eigensolver)");
  return kOk;
}
Status add_shift(Ctx& c, double* G, double* Id, int q, double shift) {
  const double al = 1.0;
  if (cublasDgeam(c.h.blas, CUBLAS_OP_N, CUBLAS_OP_N, q, q, &al, G, q, &shift, Id, q, G, q) != CUBLAS_STATUS_SUCCESS)
    return fail(kCuda, "cublasDgeam failed (eigensolver)");
  return kOk;
}

Status ensure_solver_work(Ctx& c, size_t bytes) {
  const size_t lwork = (bytes + sizeof(double2) - 1) / sizeof(double2);
  if (lwork <= c.w.solver_lwork) return kOk;
  if (c.w.solver_work) cudaFree(c.w.solver_work);
  c.w.solver_work = nullptr;
  c.w.solver_lwork = 0;
  PW_CUDA_TRY(cudaMalloc((void**)&c.w.solver_work, lwork * sizeof(double2)));
  c.w.solver_lwork = lwork;
  return kOk;
}

Status ensure_solver(Ctx& c) {
  if (!c.h.solver && cusolverDnCreate(&c.h.solver) != CUSOLVER_STATUS_SUCCESS)
    return fail(kCuda, "cusolverDnCreate failed");
  cusolverDnSetStream(c.h.solver, c.s);
  return kOk;
}

// all eigenpairs of the Hermitian / symmetric m x m matrix A (lower), in place
Status heevd(Ctx& c, double2* A, int m, double* w) {
  int lwork = 0;
  auto* a = reinterpret_cast<cuDoubleComplex*>(A);
  if (cusolverDnZheevd_bufferSize(c.h.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, a, m, w, &lwork) !=
      CUSOLVER_STATUS_SUCCESS)
    return fail(kCuda, "cusolverDnZheevd_bufferSize failed");
  Status r;
  if ((r = ensure_solver_work(c, (size_t)lwork * sizeof(double2))) != kOk) return r;
  if (cusolverDnZheevd(c.h.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, a, m, w,
                       reinterpret_cast<cuDoubleComplex*>(c.w.solver_work), lwork, c.w.info) !=
      CUSOLVER_STATUS_SUCCESS)
    return fail(kCuda, "cusolverDnZheevd failed");
  return kOk;
}
Status heevd(Ctx& c, double* A, int m, double* w) {
  int lwork = 0;
  if (cusolverDnDsyevd_bufferSize(c.h.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, A, m, w, &lwork) !=
      CUSOLVER_STATUS_SUCCESS)
    return fail(kCuda, "cusolverDnDsyevd_bufferSize failed");
  Status r;
  if ((r = ensure_solver_work(c, (size_t)lwork * sizeof(double))) != kOk) return r;
  if (cusolverDnDsyevd(c.h.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, A, m, w,
                       reinterpret_cast<double*>(c.w.solver_work), lwork, c.w.info) != CUSOLVER_STATUS_SUCCESS)
    return fail(kCuda, "cusolverDnDsyevd failed");
  return kOk;
}

// H x for the band type: complex bands through the FFT + projector pipeline,
// packed real bands through the Gamma path
Status apply_op(Handle& h, int spin, int ik, const double2* x, long ld, int nb, double2* hx, int precision,
                cudaStream_t s) {
  return apply_h_device(h, spin, ik, x, ld, nb, hx, ld, precision, s);
}
Status apply_op(Handle& h, int spin, int, const double* x, long ld, int nb, double* hx, int precision,
                cudaStream_t s) {
  return apply_h_real(h, spin, x, ld, nb, hx, ld, precision, s);
}

template <typename T> T* as(double2* p) { return reinterpret_cast<T*>(p); }

// Column sums of squares of Y (q columns) into w.colsq (device); to the
// host too when host != null.
template <typename T> Status col_norms2(Ctx& c, const T* Y, int q, double* host) {
  if (q == 0) return kOk;
  k_col_sumsq<T><<<dim3(c.gx, q), 256, 0, c.s>>>(Y, c.n, (int)c.n, c.w.partials); count_launch();
  k_col_final<<<blocks_for(q), 256, 0, c.s>>>(c.w.partials, (int)c.gx, q, c.w.colsq); count_launch();
  if (host) {
    PW_CUDA_TRY(cudaMemcpyAsync(host, c.w.colsq, q * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    PW_CUDA_TRY(cudaStreamSynchronize(c.s));
  }
  return kOk;
}

// Y -= A (A^H Y), HY -= HA (A^H Y): Y (q columns) projected out of span(A)
// (p orthonormal columns).
template <typename T> Status project_out(Ctx& c, const T* A, const T* HA, int p, T* Y, T* HY, int q) {
  if (p == 0 || q == 0) return kOk;
  Status r;
  T* Z = as<T>(c.w.Z);
  if ((r = gemm(c, CUBLAS_OP_C, CUBLAS_OP_N, p, q, (int)c.n, A, c.n, Y, c.n, Z, p)) != kOk) return r;
  if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)c.n, q, p, A, c.n, Z, p, Y, c.n, 1.0, -1.0)) != kOk) return r;
  if (HY && (r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)c.n, q, p, HA, c.n, Z, p, HY, c.n, 1.0, -1.0)) != kOk)
    return r;
  return kOk;
}

// One Cholesky-QR pass: G = Y^H Y (+ shift I), G = R^H R, Y <- Y R^-1 (and
// HY with the same R).  ok = false when the factorisation broke down (Y is
// left unchanged then).  min_rdiag: smallest diagonal entry of R.  With
// skip_tol > 0 the pass stops after the Gram matrix when Y is already
// orthonormal to skip_tol (max |G - I|; *skipped then true), which saves the
// factorisation and the update products of most second passes.
template <typename T>
Status chol_qr(Ctx& c, T* Y, T* HY, int q, double shift, bool& ok, double* min_rdiag = nullptr,
               double skip_tol = 0.0, bool* skipped = nullptr) {
  ok = true;
  if (skipped) *skipped = false;
  if (q == 0) return kOk;
  Status r;
  T* G = as<T>(c.w.G);
  if ((r = gemm(c, CUBLAS_OP_C, CUBLAS_OP_N, q, q, (int)c.n, Y, c.n, Y, c.n, G, q)) != kOk) return r;
  if (skip_tol > 0.0 && shift == 0.0) {
    PW_CUDA_TRY(cudaMemsetAsync(c.w.defect, 0, sizeof(double), c.s));
    k_gram_defect<T><<<std::min<long>(64, blocks_for((long)q * q)), 256, 0, c.s>>>(G, q, c.w.defect); count_launch();
    double defect = 0.0;
    PW_CUDA_TRY(cudaMemcpyAsync(&defect, c.w.defect, sizeof(double), cudaMemcpyDeviceToHost, c.s));
    PW_CUDA_TRY(cudaStreamSynchronize(c.s));
    if (defect <= skip_tol) {
      if (skipped) *skipped = true;
      if (min_rdiag) *min_rdiag = 1.0;
      return kOk;
    }
  }
  if (shift > 0.0) {
    T* Id = as<T>(c.w.Id);
    k_set_identity<T><<<blocks_for((long)q * q), 256, 0, c.s>>>(Id, q); count_launch();
    if ((r = add_shift(c, G, Id, q, shift)) != kOk) return r;
  }
  // G = R^H R and Ri = R^-1 in one cluster launch (chol.cu; G is
  // overwritten); R's diagonal lands in w.colsq
  T* Ri = as<T>(c.w.Id);
  if ((r = chol_inv(G, q, Ri, c.w.colsq, c.w.info, c.s)) != kOk) return r;
  int info = 0;
  PW_CUDA_TRY(cudaMemcpyAsync(&info, c.w.info, sizeof(int), cudaMemcpyDeviceToHost, c.s));
  std::vector<double> dg;
  if (min_rdiag) {
    dg.resize(q);
    PW_CUDA_TRY(cudaMemcpyAsync(dg.data(), c.w.colsq, q * sizeof(double), cudaMemcpyDeviceToHost, c.s));
  }
  PW_CUDA_TRY(cudaStreamSynchronize(c.s));
  if (info != 0) {
    ok = false;
    return kOk;
  }
  if (min_rdiag) {
    double mn = INFINITY;
    for (double d : dg) mn = std::min(mn, std::fabs(d));
    *min_rdiag = mn;
  }
  // Y <- Y R^-1 as one GEMM with the explicit inverse of the small R (a
  // tall-skinny triangular solve is several times slower than the GEMM);
  // w.T and w.HXn are free whenever a block is orthonormalised
  T* tmp[2] = {as<T>(c.w.T), as<T>(c.w.HXn)};
  T* M[2] = {Y, HY};
  for (int i = 0; i < 2; ++i) {
    if (!M[i]) continue;
    if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)c.n, q, q, M[i], c.n, Ri, q, tmp[i], c.n)) != kOk) return r;
    PW_CUDA_TRY(cudaMemcpyAsync(M[i], tmp[i], c.n * q * sizeof(T), cudaMemcpyDeviceToDevice, c.s));
  }
  return kOk;
}

// Orthonormalise Y (q columns, no H attached): column scaling, then two
// Cholesky-QR passes; a breakdown of the first pass is retried with a small
// diagonal shift, which still yields an orthonormal block after the second
// pass.
template <typename T> Status orthonormalize(Ctx& c, T* Y, int q) {
  if (q == 0) return kOk;
  Status r;
  if ((r = col_norms2(c, (const T*)Y, q, nullptr)) != kOk) return r;
  k_scale_cols_invsqrt<T><<<dim3(c.gx, q), 256, 0, c.s>>>(Y, nullptr, c.n, (int)c.n, c.w.colsq); count_launch();
  bool ok = false, skipped = false;
  // an already orthonormal block (the bands carried over from the previous SCF step) needs no pass
  if ((r = chol_qr(c, Y, (T*)nullptr, q, 0.0, ok, nullptr, kOrthoSkipTol, &skipped)) != kOk) return r;
  if (skipped) return kOk;
  if (!ok) {
    if ((r = chol_qr(c, Y, (T*)nullptr, q, 1e-10 * q, ok)) != kOk) return r;
    if (!ok) return fail(kNotConverged, "eigensolver: search block is numerically rank deficient");
  }
  if ((r = chol_qr(c, Y, (T*)nullptr, q, 0.0, ok, nullptr, kOrthoSkipTol)) != kOk) return r;
  if (!ok) return fail(kNotConverged, "eigensolver: second Cholesky-QR pass broke down");
  return kOk;
}

// Lowest nev eigenpairs of the Hermitian subspace matrix Hs (m x m): values
// into w.lam, vectors into *C (ld m).
template <typename T> Status subspace_eig(Ctx& c, int m, int nev, T** C, bool allow_small = true) {
  Status r;
  T* Hs = as<T>(c.w.Hs);
  if (allow_small && m <= kSmallSolveMax) {
    // one-CTA Cholesky + Jacobi solver (complex; a real symmetric input stays real)
    const double2* Hz = c.w.Hs;
    if (std::is_same<T, double>::value) {
      k_real_to_complex<<<blocks_for((long)m * m), 256, 0, c.s>>>(reinterpret_cast<const double*>(c.w.Hs), c.w.G,
                                                                  (long)m * m); count_launch();
      Hz = c.w.G;
    }
    k_set_identity<double2><<<blocks_for((long)m * m), 256, 0, c.s>>>(c.w.Id, m); count_launch();
    if ((r = small_geneig_batched(Hz, c.w.Id, m, 0, m, nev, 1, c.w.lam, c.w.Cs, m, 0, c.w.status, c.s)) != kOk)
      return r;
    int st = 0;
    PW_CUDA_TRY(cudaMemcpyAsync(&st, c.w.status, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    PW_CUDA_TRY(cudaStreamSynchronize(c.s));
    if (st == 1) return fail(kNotConverged, "eigensolver: subspace solve failed");
    if (std::is_same<T, double>::value) {
      // real parts into Hs (the complex vectors of a real symmetric matrix are real)
      k_complex_to_real<<<blocks_for((long)m * nev), 256, 0, c.s>>>(c.w.Cs, reinterpret_cast<double*>(c.w.Hs),
                                                                    (long)m * nev); count_launch();
      *C = Hs;
    } else {
      *C = as<T>(c.w.Cs);
    }
    return kOk;
  }
  if (eigh_cluster_supported(m, !std::is_same<T, double>::value)) {
    // this project's cluster eigensolver: lowest nev pairs, vectors into Cs
    const size_t need = eigh_cluster_work_doubles(m, nev);
    if (need > c.w.eigh_work_len) {
      if (c.w.eigh_work) cudaFree(c.w.eigh_work);
      c.w.eigh_work = nullptr;
      c.w.eigh_work_len = 0;
      if ((r = walloc(&c.w.eigh_work, need)) != kOk) return r;
      c.w.eigh_work_len = need;
    }
    T* Cv = as<T>(c.w.Cs);
    if ((r = eigh_cluster(Hs, m, m, nev, c.w.lam, Cv, m, c.w.eigh_work, c.w.status, c.s)) != kOk) return r;
    int st = 0;
    PW_CUDA_TRY(cudaMemcpyAsync(&st, c.w.status, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    PW_CUDA_TRY(cudaStreamSynchronize(c.s));
    if (st != 0) return fail(kNotConverged, "eigensolver: subspace eigensolve produced non-finite values");
    *C = Cv;
    return kOk;
  }
  // beyond the cluster solver's size (m > 544, or complex m beyond its shared memory)
  if ((r = ensure_solver(c)) != kOk) return r;
  if ((r = heevd(c, Hs, m, c.w.lam)) != kOk) return r;
  int info = 0;
  PW_CUDA_TRY(cudaMemcpyAsync(&info, c.w.info, sizeof(int), cudaMemcpyDeviceToHost, c.s));
  PW_CUDA_TRY(cudaStreamSynchronize(c.s));
  if (info != 0) return fail(kNotConverged, "eigensolver: subspace eigensolver did not converge");
  *C = Hs;
  return kOk;
}

// Rayleigh-Ritz in span(X) alone (X orthonormal): X <- X C, HX <- HX C.
template <typename T> Status rr_block(Ctx& c, EigVecs& k, int nd) {
  Status r;
  T* X = as<T>(k.V);
  T* HX = as<T>(k.HV);
  T* G = as<T>(c.w.G);
  if ((r = gemm(c, CUBLAS_OP_C, CUBLAS_OP_N, nd, nd, (int)c.n, X, c.n, HX, c.n, G, nd)) != kOk) return r;
  k_assemble_rr<T><<<blocks_for((long)nd * nd), 256, 0, c.s>>>(as<T>(c.w.Hs), nd, 0, c.w.lam0, as<T>(c.w.Z), G);
  count_launch();
  T* C = nullptr;
  if ((r = subspace_eig<T>(c, nd, nd, &C)) != kOk) return r;
  if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)c.n, nd, nd, X, c.n, C, nd, as<T>(c.w.T), c.n)) != kOk) return r;
  if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)c.n, nd, nd, HX, c.n, C, nd, as<T>(c.w.HXn), c.n)) != kOk) return r;
  PW_CUDA_TRY(cudaMemcpyAsync(X, c.w.T, c.n * nd * sizeof(T), cudaMemcpyDeviceToDevice, c.s));
  PW_CUDA_TRY(cudaMemcpyAsync(HX, c.w.HXn, c.n * nd * sizeof(T), cudaMemcpyDeviceToDevice, c.s));
  PW_CUDA_TRY(cudaMemcpyAsync(k.evals.data(), c.w.lam, nd * sizeof(double), cudaMemcpyDeviceToHost, c.s));
  PW_CUDA_TRY(cudaStreamSynchronize(c.s));
  return kOk;
}

// Per-phase CUDA-event timing of the block steps (only when the handle's trace
// flag is set): 0 residual, 1 W, 2 H W, 3 P, 4 subspace matrix, 5 subspace
// solve, 6 update.
struct PhaseTimer {
  static constexpr int kPhases = 7;
  bool on = false;
  cudaEvent_t ev[kPhases + 1] = {};
  double total[kPhases] = {};
  explicit PhaseTimer(bool enable) : on(enable) {
    if (on)
      for (auto& e : ev) cudaEventCreate(&e);
  }
  ~PhaseTimer() {
    if (on)
      for (auto& e : ev) cudaEventDestroy(e);
  }
  void mark(int i, cudaStream_t s) {
    if (on) cudaEventRecord(ev[i], s);
  }
  // after the stream has been synchronised
  void accumulate() {
    if (!on) return;
    for (int i = 0; i < kPhases; ++i) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ev[i], ev[i + 1]) == cudaSuccess) total[i] += ms;
    }
  }
};

inline void noise(double& x, std::mt19937_64& rng, std::uniform_real_distribution<double>& u) { x = 1e-3 * u(rng); }
inline void noise(double2& x, std::mt19937_64& rng, std::uniform_real_distribution<double>& u) {
  const double a = 1e-3 * u(rng);
  x = make_double2(a, 1e-3 * u(rng));
}
inline void add_real(double& x, double v) { x += v; }
inline void add_real(double2& x, double v) { x.x += v; }

template <typename T>
Status lobpcg_t(Handle& h, EigWork& w, EigVecs& k, int spin, int ik, double v0, double tol, int max_iter, int nconv,
                int precision, EigStats& out) {
  const long n = h.n_pw;
  const int nd = w.nd;
  const cudaStream_t s = h.stream;
  cublasSetStream(h.blas, s);
  Ctx c{h, w, s, n, (unsigned)std::min<long>(kColBlocks, blocks_for(n))};
  Status r;
  T* X = as<T>(k.V);
  T* HX = as<T>(k.HV);
  const double* kin = std::is_same<T, double>::value ? h.gam.kin_packed : h.kp[ik].kinetic;
  if (!k.init) {
    // start: unit vectors on the nd lowest kinetic entries plus seeded noise
    std::vector<double> kh(n);
    PW_CUDA_TRY(cudaMemcpyAsync(kh.data(), kin, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    PW_CUDA_TRY(cudaStreamSynchronize(s));
    std::vector<int> order(n);
    for (long i = 0; i < n; ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return kh[a] < kh[b]; });
    std::vector<T> x0((size_t)n * nd);
    std::mt19937_64 rng(20261203ULL + 7919ULL * (ik + 1) + 104729ULL * spin);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    for (size_t i = 0; i < x0.size(); ++i) noise(x0[i], rng, u);
    for (int col = 0; col < nd && col < n; ++col) add_real(x0[(size_t)col * n + order[col]], 1.0);
    PW_CUDA_TRY(cudaMemcpyAsync(X, x0.data(), x0.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    PW_CUDA_TRY(cudaStreamSynchronize(s));
    k.init = true;
  }
  if ((r = orthonormalize(c, X, nd)) != kOk) return r;
  // HX in FP64: the residuals below refer to the full-precision operator
  if ((r = apply_op(h, spin, ik, X, n, nd, HX, 0, s)) != kOk) return r;
  out.happ += nd;
  // The Rayleigh-Ritz of X alone is deferred into the first block step: its
  // subspace matrix takes the full X^H HX block (w.XX), and the residuals of
  // that step use the Rayleigh quotients diag(X^H HX).  Only a solve that
  // stops before any block step rotates X by itself (rr_block).
  T* XX = as<T>(w.XX);
  if ((r = gemm(c, CUBLAS_OP_C, CUBLAS_OP_N, nd, nd, (int)n, X, n, HX, n, XX, nd)) != kOk) return r;
  k_diag_real<T><<<blocks_for(nd), 256, 0, s>>>(XX, nd, nd, w.lam); count_launch();
  PW_CUDA_TRY(cudaMemcpyAsync(k.evals.data(), w.lam, nd * sizeof(double), cudaMemcpyDeviceToHost, s));
  PW_CUDA_TRY(cudaStreamSynchronize(s));
  bool first = true;

  const double p_drop = precision == 0 ? kPDropFp64 : kPDropMixed;
  T* Tb = as<T>(w.T);
  T* Pn = as<T>(w.Pn);
  T* HPn = as<T>(w.HPn);
  std::vector<double> rn(nd), nu0, nu1;
  std::vector<int> act, pband, keep, pk;
  int np = 0;  // columns of Pn / HPn (bands pband)
  out.iters = 0;
  PhaseTimer pt(h.trace);
  for (;;) {
    const auto t0 = std::chrono::steady_clock::now();
    pt.mark(0, s);
    PW_CUDA_TRY(cudaMemcpyAsync(w.lam0, k.evals.data(), nd * sizeof(double), cudaMemcpyHostToDevice, s));
    k_resid_precond<T><<<dim3(c.gx, nd), 256, 0, s>>>(X, HX, Tb, n, (int)n, w.lam0, kin, v0, w.partials);
    count_launch();
    k_col_final<<<blocks_for(nd), 256, 0, s>>>(w.partials, (int)c.gx, nd, w.colsq); count_launch();
    PW_CUDA_TRY(cudaMemcpyAsync(rn.data(), w.colsq, nd * sizeof(double), cudaMemcpyDeviceToHost, s));
    PW_CUDA_TRY(cudaStreamSynchronize(s));
    out.max_res = 0.0;
    for (int b = 0; b < nconv; ++b) out.max_res = std::max(out.max_res, std::sqrt(rn[b]));
    if (out.max_res < tol || out.iters >= max_iter) {
      if (first && (r = rr_block<T>(c, k, nd)) != kOk) return r;
      break;
    }
    // active bands: residual above tol (buffer bands: 10 tol)
    act.clear();
    for (int b = 0; b < nd; ++b)
      if (std::sqrt(rn[b]) > (b < nconv ? tol : 10.0 * tol)) act.push_back(b);
    if ((long)act.size() > n - nd) act.resize((size_t)std::max<long>(0, n - nd));
    const int na = (int)act.size();
    if (na == 0) {
      if (first && (r = rr_block<T>(c, k, nd)) != kOk) return r;
      break;
    }
    T* W = X + n * nd;
    T* HW = HX + n * nd;
    pt.mark(1, s);
    PW_CUDA_TRY(cudaMemcpyAsync(w.idx, act.data(), na * sizeof(int), cudaMemcpyHostToDevice, s));
    k_gather_cols<T><<<dim3(c.gx, na), 256, 0, s>>>(Tb, n, w.idx, W, n, (int)n); count_launch();
    if ((r = project_out(c, (const T*)X, (const T*)nullptr, nd, W, (T*)nullptr, na)) != kOk) return r;
    if ((r = project_out(c, (const T*)X, (const T*)nullptr, nd, W, (T*)nullptr, na)) != kOk) return r;
    if ((r = orthonormalize(c, W, na)) != kOk) return r;
    pt.mark(2, s);
    if ((r = apply_op(h, spin, ik, W, n, na, HW, precision, s)) != kOk) return r;
    out.happ += na;
    pt.mark(3, s);
    // P: previous directions of the bands still active
    int npc = 0;
    pk.clear();
    for (int j = 0, a = 0; j < np; ++j) {
      while (a < na && act[a] < pband[j]) ++a;
      if (a < na && act[a] == pband[j]) pk.push_back(j);
    }
    if ((long)pk.size() > n - nd - na) pk.resize((size_t)std::max<long>(0, n - nd - na));
    T* P = W + n * na;
    T* HP = HW + n * na;
    if (!pk.empty()) {
      npc = (int)pk.size();
      PW_CUDA_TRY(cudaMemcpyAsync(w.idx, pk.data(), npc * sizeof(int), cudaMemcpyHostToDevice, s));
      k_gather_cols<T><<<dim3(c.gx, npc), 256, 0, s>>>(Pn, n, w.idx, P, n, (int)n); count_launch();
      k_gather_cols<T><<<dim3(c.gx, npc), 256, 0, s>>>(HPn, n, w.idx, HP, n, (int)n); count_launch();
      nu0.resize(npc);
      nu1.resize(npc);
      if ((r = col_norms2(c, (const T*)P, npc, nu0.data())) != kOk) return r;
      if ((r = project_out(c, (const T*)X, (const T*)HX, nd, P, HP, npc)) != kOk) return r;
      if ((r = project_out(c, (const T*)W, (const T*)HW, na, P, HP, npc)) != kOk) return r;
      if ((r = col_norms2(c, (const T*)P, npc, nu1.data())) != kOk) return r;
      keep.clear();
      for (int j = 0; j < npc; ++j)
        if (nu1[j] > p_drop * p_drop * nu0[j] && nu1[j] > 0.0) keep.push_back(j);
      if ((int)keep.size() < npc && !keep.empty()) {
        // compact through Pn / HPn (their old contents were consumed above)
        const int nk = (int)keep.size();
        PW_CUDA_TRY(cudaMemcpyAsync(w.idx, keep.data(), nk * sizeof(int), cudaMemcpyHostToDevice, s));
        k_gather_cols<T><<<dim3(c.gx, nk), 256, 0, s>>>(P, n, w.idx, Pn, n, (int)n); count_launch();
        k_gather_cols<T><<<dim3(c.gx, nk), 256, 0, s>>>(HP, n, w.idx, HPn, n, (int)n); count_launch();
        PW_CUDA_TRY(cudaMemcpyAsync(P, Pn, n * nk * sizeof(T), cudaMemcpyDeviceToDevice, s));
        PW_CUDA_TRY(cudaMemcpyAsync(HP, HPn, n * nk * sizeof(T), cudaMemcpyDeviceToDevice, s));
      }
      npc = (int)keep.size();
      if (npc > 0) {
        if ((r = col_norms2(c, (const T*)P, npc, nullptr)) != kOk) return r;
        k_scale_cols_invsqrt<T><<<dim3(c.gx, npc), 256, 0, s>>>(P, HP, n, (int)n, w.colsq); count_launch();
        bool ok = false;
        double rmin = 0.0;
        if ((r = chol_qr(c, P, HP, npc, 0.0, ok, &rmin)) != kOk) return r;
        if (!ok || rmin < p_drop) {
          npc = 0;  // P block nearly dependent: restart without it
        } else if ((r = chol_qr(c, P, HP, npc, 0.0, ok, nullptr, kOrthoSkipTol)) != kOk) {
          return r;
        } else if (!ok) {
          npc = 0;
        }
      }
    }
    const int q = na + npc;
    if (4 * na <= nd && !first) {
      // few active bands: hard locking.  W and P are orthogonal to every
      // column of X, so [X_a | W | P] (X_a the active Ritz vectors) is an
      // orthonormal basis orthogonal to the converged ones; Rayleigh-Ritz in
      // it alone leaves the converged pairs as they are (their coupling to W
      // and P is their residual, below tol) at a third of the subspace size
      pt.mark(4, s);
      const int ms = na + q;
      T* Bx = Tb;                      // [X_a | W | P], n x ms
      T* Bh = as<T>(w.HXn);            // [HX_a | HW | HP]
      PW_CUDA_TRY(cudaMemcpyAsync(w.idx, act.data(), na * sizeof(int), cudaMemcpyHostToDevice, s));
      k_gather_cols<T><<<dim3(c.gx, na), 256, 0, s>>>(X, n, w.idx, Bx, n, (int)n); count_launch();
      k_gather_cols<T><<<dim3(c.gx, na), 256, 0, s>>>(HX, n, w.idx, Bh, n, (int)n); count_launch();
      PW_CUDA_TRY(cudaMemcpyAsync(Bx + n * na, W, n * q * sizeof(T), cudaMemcpyDeviceToDevice, s));
      PW_CUDA_TRY(cudaMemcpyAsync(Bh + n * na, HW, n * q * sizeof(T), cudaMemcpyDeviceToDevice, s));
      std::vector<double> lam_a(na);
      for (int j = 0; j < na; ++j) lam_a[j] = k.evals[act[j]];
      PW_CUDA_TRY(cudaMemcpyAsync(w.lam0, lam_a.data(), na * sizeof(double), cudaMemcpyHostToDevice, s));
      if ((r = gemm(c, CUBLAS_OP_C, CUBLAS_OP_N, q, na, (int)n, W, n, Bh, n, as<T>(w.Z), q)) != kOk) return r;
      if ((r = gemm(c, CUBLAS_OP_C, CUBLAS_OP_N, q, q, (int)n, W, n, HW, n, as<T>(w.G), q)) != kOk) return r;
      k_assemble_rr<T><<<blocks_for((long)ms * ms), 256, 0, s>>>(as<T>(w.Hs), ms, na, w.lam0, as<T>(w.Z),
                                                                  as<T>(w.G));
      count_launch();
      T* C = nullptr;
      pt.mark(5, s);
      if ((r = subspace_eig<T>(c, ms, na, &C, false)) != kOk) return r;
      pt.mark(6, s);
      // new active X, HX into the W, HW columns; new P, HP from the (W, P) rows
      if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, na, ms, Bx, n, C, ms, W, n)) != kOk) return r;
      if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, na, ms, Bh, n, C, ms, HW, n)) != kOk) return r;
      if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, na, q, Bx + n * na, n, C + na, ms, Pn, n)) != kOk) return r;
      if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, na, q, Bh + n * na, n, C + na, ms, HPn, n)) != kOk)
        return r;
      k_scatter_cols<T><<<dim3(c.gx, na), 256, 0, s>>>(W, n, w.idx, X, n, (int)n); count_launch();
      k_scatter_cols<T><<<dim3(c.gx, na), 256, 0, s>>>(HW, n, w.idx, HX, n, (int)n); count_launch();
      PW_CUDA_TRY(cudaMemcpyAsync(lam_a.data(), w.lam, na * sizeof(double), cudaMemcpyDeviceToHost, s));
      PW_CUDA_TRY(cudaStreamSynchronize(s));
      for (int j = 0; j < na; ++j) k.evals[act[j]] = lam_a[j];
      // keep the bands in ascending order (a new active value may pass a converged one)
      std::vector<int> order(nd);
      for (int b = 0; b < nd; ++b) order[b] = b;
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return k.evals[a] < k.evals[b]; });
      bool sorted = true;
      for (int b = 0; b < nd; ++b) sorted = sorted && order[b] == b;
      pband = act;
      if (!sorted) {
        std::vector<int> inv(nd);
        for (int b = 0; b < nd; ++b) inv[order[b]] = b;
        PW_CUDA_TRY(cudaMemcpyAsync(w.idx, order.data(), nd * sizeof(int), cudaMemcpyHostToDevice, s));
        k_gather_cols<T><<<dim3(c.gx, nd), 256, 0, s>>>(X, n, w.idx, Tb, n, (int)n); count_launch();
        k_gather_cols<T><<<dim3(c.gx, nd), 256, 0, s>>>(HX, n, w.idx, as<T>(w.HXn), n, (int)n); count_launch();
        PW_CUDA_TRY(cudaMemcpyAsync(X, Tb, n * nd * sizeof(T), cudaMemcpyDeviceToDevice, s));
        PW_CUDA_TRY(cudaMemcpyAsync(HX, w.HXn, n * nd * sizeof(T), cudaMemcpyDeviceToDevice, s));
        std::vector<double> ev(nd);
        for (int b = 0; b < nd; ++b) ev[b] = k.evals[order[b]];
        std::copy(ev.begin(), ev.end(), k.evals.begin());
        // P columns follow their bands: new band numbers, in ascending order
        std::vector<int> pj(na);
        for (int j = 0; j < na; ++j) pj[j] = j;
        std::sort(pj.begin(), pj.end(), [&](int a, int b) { return inv[act[a]] < inv[act[b]]; });
        for (int j = 0; j < na; ++j) pband[j] = inv[act[pj[j]]];
        PW_CUDA_TRY(cudaMemcpyAsync(w.idx, pj.data(), na * sizeof(int), cudaMemcpyHostToDevice, s));
        k_gather_cols<T><<<dim3(c.gx, na), 256, 0, s>>>(Pn, n, w.idx, Tb, n, (int)n); count_launch();
        k_gather_cols<T><<<dim3(c.gx, na), 256, 0, s>>>(HPn, n, w.idx, as<T>(w.HXn), n, (int)n); count_launch();
        PW_CUDA_TRY(cudaMemcpyAsync(Pn, Tb, n * na * sizeof(T), cudaMemcpyDeviceToDevice, s));
        PW_CUDA_TRY(cudaMemcpyAsync(HPn, w.HXn, n * na * sizeof(T), cudaMemcpyDeviceToDevice, s));
      }
      pt.mark(7, s);
      PW_CUDA_TRY(cudaStreamSynchronize(s));
      pt.accumulate();
      np = na;
      ++out.iters;
      if (h.trace) {
        const double ms_it =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(stderr, "pwgpu lobpcg k=%d it=%d res=%.3e na=%d np=%d hard e0=%.8f e_last=%.8f %.2f ms\n", ik,
                     out.iters, out.max_res, na, npc, k.evals[0], k.evals[nconv - 1], ms_it);
      }
      continue;
    }
    // Rayleigh-Ritz over [X | W | P]
    pt.mark(4, s);
    const int m = nd + q;
    if ((r = gemm(c, CUBLAS_OP_C, CUBLAS_OP_N, q, nd, (int)n, W, n, HX, n, as<T>(w.Z), q)) != kOk) return r;
    if ((r = gemm(c, CUBLAS_OP_C, CUBLAS_OP_N, q, q, (int)n, W, n, HW, n, as<T>(w.G), q)) != kOk) return r;
    k_assemble_rr<T><<<blocks_for((long)m * m), 256, 0, s>>>(as<T>(w.Hs), m, nd, w.lam0, as<T>(w.Z), as<T>(w.G),
                                                            first ? XX : nullptr);
    count_launch();
    first = false;
    T* C = nullptr;
    pt.mark(5, s);
    if ((r = subspace_eig<T>(c, m, nd, &C)) != kOk) return r;
    pt.mark(6, s);
    // new X, HX and new P, HP of the active bands.  T = [W | P] C_wp (C's W, P rows, all nd
    // columns) is the P part of every new X column: P = T(:, active), X = X C_x + T, so the
    // W, P products are formed once (likewise for HX, HP)
    PW_CUDA_TRY(cudaMemcpyAsync(w.idx, act.data(), na * sizeof(int), cudaMemcpyHostToDevice, s));
    T* HXn = as<T>(w.HXn);
    if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, nd, q, W, n, C + nd, m, Tb, n)) != kOk) return r;
    if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, nd, q, HW, n, C + nd, m, HXn, n)) != kOk) return r;
    k_gather_cols<T><<<dim3(c.gx, na), 256, 0, s>>>(Tb, n, w.idx, Pn, n, (int)n); count_launch();
    k_gather_cols<T><<<dim3(c.gx, na), 256, 0, s>>>(HXn, n, w.idx, HPn, n, (int)n); count_launch();
    if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, nd, nd, X, n, C, m, Tb, n, 1.0)) != kOk) return r;
    if ((r = gemm(c, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, nd, nd, HX, n, C, m, HXn, n, 1.0)) != kOk) return r;
    PW_CUDA_TRY(cudaMemcpyAsync(X, Tb, n * nd * sizeof(T), cudaMemcpyDeviceToDevice, s));
    PW_CUDA_TRY(cudaMemcpyAsync(HX, w.HXn, n * nd * sizeof(T), cudaMemcpyDeviceToDevice, s));
    PW_CUDA_TRY(cudaMemcpyAsync(k.evals.data(), w.lam, nd * sizeof(double), cudaMemcpyDeviceToHost, s));
    pt.mark(7, s);
    PW_CUDA_TRY(cudaStreamSynchronize(s));
    pt.accumulate();
    np = na;
    pband = act;
    ++out.iters;
    if (h.trace) {
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      std::fprintf(stderr, "pwgpu lobpcg k=%d it=%d res=%.3e na=%d np=%d e0=%.8f e_last=%.8f %.2f ms\n", ik,
                   out.iters, out.max_res, na, npc, k.evals[0], k.evals[nconv - 1], ms);
    }
  }
  if (pt.on)
    std::fprintf(stderr,
                 "pwgpu lobpcg k=%d phases ms: resid %.2f W %.2f HW %.2f P %.2f matrix %.2f solve %.2f update %.2f\n",
                 ik, pt.total[0], pt.total[1], pt.total[2], pt.total[3], pt.total[4], pt.total[5], pt.total[6]);
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

}  // namespace

// ---------------------------------------------------------------------------
// allocation
// ---------------------------------------------------------------------------

Status eig_work_alloc(EigWork& w, long n, int nd) {
  eig_work_release(w);
  w.nd = nd;
  w.n = n;
  const size_t m = 3 * (size_t)nd;
  Status r;
  for (double2** p : {&w.T, &w.HXn, &w.Pn, &w.HPn})
    if ((r = walloc(p, (size_t)n * nd)) != kOk) return r;
  for (double2** p : {&w.Hs, &w.Cs, &w.G, &w.Z, &w.Id})
    if ((r = walloc(p, m * m)) != kOk) return r;
  if ((r = walloc(&w.XX, (size_t)nd * nd)) != kOk) return r;
  if ((r = walloc(&w.defect, 2)) != kOk) return r;
  if ((r = walloc(&w.lam, m)) != kOk) return r;
  if ((r = walloc(&w.lam0, m)) != kOk) return r;
  if ((r = walloc(&w.colsq, m)) != kOk) return r;
  if ((r = walloc(&w.partials, m * kColBlocks)) != kOk) return r;
  if ((r = walloc(&w.idx, m)) != kOk) return r;
  if ((r = walloc(&w.status, 1)) != kOk) return r;
  if ((r = walloc(&w.info, 1)) != kOk) return r;
  return kOk;
}

void eig_work_release(EigWork& w) {
  auto f = [](void* p) { if (p) cudaFree(p); };
  f(w.T); f(w.HXn); f(w.Pn); f(w.HPn); f(w.Hs); f(w.Cs); f(w.G); f(w.Z); f(w.Id);
  f(w.lam); f(w.lam0); f(w.colsq); f(w.partials); f(w.idx); f(w.status); f(w.solver_work); f(w.info);
  f(w.eigh_work); f(w.XX); f(w.defect);
  w = EigWork();
}

Status eig_vecs_alloc(EigVecs& v, long n, int nd) {
  eig_vecs_release(v);
  Status r;
  if ((r = walloc(&v.V, (size_t)n * 3 * nd)) != kOk) return r;
  if ((r = walloc(&v.HV, (size_t)n * 3 * nd)) != kOk) return r;
  v.evals.assign(nd, 0.0);
  v.init = false;
  return kOk;
}

void eig_vecs_release(EigVecs& v) {
  if (v.V) cudaFree(v.V);
  if (v.HV) cudaFree(v.HV);
  v = EigVecs();
}

// ---------------------------------------------------------------------------
// solver
// ---------------------------------------------------------------------------

Status lobpcg(Handle& h, EigWork& w, EigVecs& k, int spin, int ik, double v0, double tol, int max_iter, int nconv,
              int precision, EigStats& out) {
  if (h.n_pw != w.n || w.nd < 1 || nconv < 1 || nconv > w.nd)
    return fail(kInvalid, "eigensolver: inconsistent block sizes");
  if (h.gam.on) return lobpcg_t<double>(h, w, k, spin, ik, v0, tol, max_iter, nconv, precision, out);
  return lobpcg_t<double2>(h, w, k, spin, ik, v0, tol, max_iter, nconv, precision, out);
}

}  // namespace pwgpu
