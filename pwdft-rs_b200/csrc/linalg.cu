// Dense FP64 linear algebra of the Rayleigh-Ritz step.
//
// Small generalized Hermitian eigenproblems H c = lambda S c (m <= 64) are
// solved one problem per thread block, batched over k-points:
//   S = L L^H (right-looking Cholesky), A = L^{-1} H L^{-H},
//   cyclic complex Jacobi on A with the round-robin pair schedule
//   (m/2 disjoint rotations per step, each a 2x2 unitary
//   [[c, s u], [-s u*, c]], u = A_pq/|A_pq|, t = tan(theta) from
//   zeta = (A_qq - A_pp) / (2|A_pq|)), eigenvalues sorted ascending,
//   C = L^{-H} V.
// Larger problems go to cuSOLVER zhegvd.  Replaces the reference's dense
// self_adjoint_eigen (eigensolver/dense.rs:50-98) inside the subspace.
#include <cusolverDn.h>

#include <algorithm>
#include <mutex>
#include <set>
#include <cmath>
#include <vector>

#include "handle.hpp"
#include "linalg.hpp"

namespace pwgpu {

namespace {

constexpr int kSmallMax = 64;
constexpr int kSweepsMax = 40;

__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cmuld(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }

// One problem per block.  H, S: m x m column-major with leading dim ld, batch
// stride ldb*... (pointer + b*stride).  status[b] = 0 ok, 1 S not positive
// definite, 2 Jacobi did not reach the tolerance within kSweepsMax sweeps.
__global__ void __launch_bounds__(256) k_small_geneig(const double2* __restrict__ H, const double2* __restrict__ S,
                                                     long ld, long stride, int m, int nev, double* __restrict__ evals,
                                                     double2* __restrict__ C, long ldc, long cstride,
                                                     int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* L = reinterpret_cast<double2*>(smem_raw);  // m x m, column-major (S, then L)
  double2* A = L + m * m;                            // m x m
  double2* V = A + m * m;                            // m x m
  double* cs = reinterpret_cast<double*>(V + m * m);  // rotation c, s per pair
  double2* us = reinterpret_cast<double2*>(cs + 2 * (kSmallMax / 2));
  int* order = reinterpret_cast<int*>(us + kSmallMax / 2);
  __shared__ int bad;
  __shared__ double offmax, diagmax;
  const int b = blockIdx.x;
  const int tid = threadIdx.x, T = blockDim.x;
  const double2* Hb = H + b * stride;
  const double2* Sb = S + b * stride;
  if (tid == 0) bad = 0;
  for (int i = tid; i < m * m; i += T) {
    const int r = i % m, c = i / m;
    L[i] = Sb[r + c * ld];
    A[i] = Hb[r + c * ld];
  }
  __syncthreads();
  // Cholesky, lower, in place in L (upper part left as S garbage, unused)
  for (int j = 0; j < m; ++j) {
    if (tid == 0) {
      const double d = L[j + j * m].x;
      if (!(d > 0.0)) bad = 1;
      L[j + j * m] = make_double2(d > 0.0 ? sqrt(d) : 1.0, 0.0);
    }
    __syncthreads();
    const double ljj = L[j + j * m].x;
    for (int i = j + 1 + tid; i < m; i += T) L[i + j * m] = L[i + j * m] * (1.0 / ljj);
    __syncthreads();
    const int rem = m - j - 1;
    for (int t = tid; t < rem * rem; t += T) {
      const int i = j + 1 + t % rem, k = j + 1 + t / rem;
      if (k <= i) L[i + k * m] = L[i + k * m] - cmuld(L[i + j * m], cconj(L[k + j * m]));
    }
    __syncthreads();
  }
  // Y = L^{-1} A (column c by thread c), stored in V
  for (int c = tid; c < m; c += T) {
    for (int i = 0; i < m; ++i) {
      double2 acc = A[i + c * m];
      for (int k = 0; k < i; ++k) acc = acc - cmuld(L[i + k * m], V[k + c * m]);
      V[i + c * m] = acc * (1.0 / L[i + i * m].x);
    }
  }
  __syncthreads();
  // Z = L^{-1} Y^H (column c of Y^H = conj of row c of Y), A = Z^H
  for (int c = tid; c < m; c += T) {
    for (int i = 0; i < m; ++i) {
      double2 acc = cconj(V[c + i * m]);
      for (int k = 0; k < i; ++k) acc = acc - cmuld(L[i + k * m], A[k + c * m]);
      A[i + c * m] = acc * (1.0 / L[i + i * m].x);  // A holds Z temporarily
    }
  }
  __syncthreads();
  for (int i = tid; i < m * m; i += T) {
    const int r = i % m, c = i / m;
    if (r < c) {
      const double2 zrc = A[r + c * m], zcr = A[c + r * m];
      A[r + c * m] = cconj(zcr);
      A[c + r * m] = cconj(zrc);
    } else if (r == c) {
      A[i] = make_double2(A[i].x, 0.0);
    }
  }
  __syncthreads();
  for (int i = tid; i < m * m; i += T) V[i] = make_double2((i % m) == (i / m) ? 1.0 : 0.0, 0.0);
  __syncthreads();
  // cyclic Jacobi, round-robin schedule over an even number of slots
  const int mm = (m + 1) & ~1;  // padded to even; slot m (if odd) is a dummy
  const int npair = mm / 2;
  int sweep = 0;
  for (; sweep < kSweepsMax; ++sweep) {
    if (tid == 0) { offmax = 0.0; diagmax = 0.0; }
    __syncthreads();
    for (int i = tid; i < m * m; i += T) {
      const int r = i % m, c = i / m;
      const double v = sqrt(cabs2(A[i]));
      if (r == c) atomicMax((unsigned long long*)&diagmax, __double_as_longlong(v));
      else atomicMax((unsigned long long*)&offmax, __double_as_longlong(v));
    }
    __syncthreads();
    if (offmax <= 1e-15 * fmax(diagmax, 1e-300)) break;
    for (int step = 0; step < mm - 1; ++step) {
      // pair i: (p, q) from the circle method with slot mm-1 fixed
      for (int i = tid; i < npair; i += T) {
        int p = (i == 0) ? mm - 1 : (step + i) % (mm - 1);
        int q = (step + mm - 1 - i) % (mm - 1);
        if (i == 0) q = step % (mm - 1);
        if (p > q) { const int t = p; p = q; q = t; }
        double c = 1.0, s = 0.0;
        double2 u = make_double2(1.0, 0.0);
        if (q < m) {
          const double2 g = A[p + q * m];
          const double r = sqrt(cabs2(g));
          if (r > 1e-300) {
            const double a = A[p + p * m].x, bq = A[q + q * m].x;
            const double zeta = (bq - a) / (2.0 * r);
            const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
            u = make_double2(g.x / r, g.y / r);
          }
        }
        cs[2 * i] = c;
        cs[2 * i + 1] = s;
        us[i] = u;
        order[2 * i] = p;
        order[2 * i + 1] = q;
      }
      __syncthreads();
      // columns: A <- A U, V <- V U
      for (int t = tid; t < npair * m; t += T) {
        const int i = t / m, k = t % m;
        const int p = order[2 * i], q = order[2 * i + 1];
        if (q >= m) continue;
        const double c = cs[2 * i], s = cs[2 * i + 1];
        const double2 u = us[i];
        const double2 akp = A[k + p * m], akq = A[k + q * m];
        A[k + p * m] = akp * c - cmuld(cconj(u), akq) * s;
        A[k + q * m] = cmuld(u, akp) * s + akq * c;
        const double2 vkp = V[k + p * m], vkq = V[k + q * m];
        V[k + p * m] = vkp * c - cmuld(cconj(u), vkq) * s;
        V[k + q * m] = cmuld(u, vkp) * s + vkq * c;
      }
      __syncthreads();
      // rows: A <- U^H A
      for (int t = tid; t < npair * m; t += T) {
        const int i = t / m, k = t % m;
        const int p = order[2 * i], q = order[2 * i + 1];
        if (q >= m) continue;
        const double c = cs[2 * i], s = cs[2 * i + 1];
        const double2 u = us[i];
        const double2 apk = A[p + k * m], aqk = A[q + k * m];
        A[p + k * m] = apk * c - cmuld(u, aqk) * s;
        A[q + k * m] = cmuld(cconj(u), apk) * s + aqk * c;
      }
      __syncthreads();
      for (int i = tid; i < npair; i += T) {
        const int p = order[2 * i], q = order[2 * i + 1];
        if (q >= m) continue;
        A[p + q * m] = make_double2(0.0, 0.0);
        A[q + p * m] = make_double2(0.0, 0.0);
        A[p + p * m] = make_double2(A[p + p * m].x, 0.0);
        A[q + q * m] = make_double2(A[q + q * m].x, 0.0);
      }
      __syncthreads();
    }
  }
  // sort eigenvalues ascending (rank by counting; ties broken by index)
  for (int i = tid; i < m; i += T) {
    const double ei = A[i + i * m].x;
    int rank = 0;
    for (int j = 0; j < m; ++j) {
      const double ej = A[j + j * m].x;
      if (ej < ei || (ej == ei && j < i)) ++rank;
    }
    order[rank] = i;
  }
  __syncthreads();
  // C = L^{-H} V[:, order[0:nev]]  (back substitution, column per thread)
  double* ev = evals + (long)b * nev;
  double2* Cb = C + b * cstride;
  for (int c = tid; c < nev; c += T) {
    const int src = order[c];
    ev[c] = A[src + src * m].x;
    for (int i = m - 1; i >= 0; --i) {
      double2 acc = V[i + src * m];
      for (int k = i + 1; k < m; ++k) acc = acc - cmuld(cconj(L[k + i * m]), Cb[k + c * ldc]);
      Cb[i + c * ldc] = acc * (1.0 / L[i + i * m].x);
    }
  }
  if (tid == 0) status[b] = bad ? 1 : (sweep >= kSweepsMax ? 2 : 0);
}

}  // namespace

size_t small_geneig_smem(int m) {
  return (size_t)3 * m * m * sizeof(double2) + 2 * (kSmallMax / 2) * sizeof(double) +
         (kSmallMax / 2) * sizeof(double2) + kSmallMax * sizeof(int);
}

Status small_geneig_batched(const double2* H, const double2* S, long ld, long stride, int m, int nev, int batch,
                            double* evals, double2* C, long ldc, long cstride, int* status_dev, cudaStream_t s) {
  if (m < 1 || m > kSmallMax || nev < 1 || nev > m) return fail(kInvalid, "small_geneig: size out of range");
  // the shared-memory opt-in is a per-device attribute; set it once per device
  // (lanes and server workers call this from several host threads)
  {
    static std::mutex mu;
    static std::set<int> done;
    int dev = 0;
    PW_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (!done.count(dev)) {
      PW_CUDA_TRY(cudaFuncSetAttribute((const void*)k_small_geneig, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)small_geneig_smem(kSmallMax)));
      done.insert(dev);
    }
  }
  k_small_geneig<<<batch, 256, small_geneig_smem(m), s>>>(H, S, ld, stride, m, nev, evals, C, ldc, cstride,
                                                          status_dev); count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// Large problems: cuSOLVER zhegvd on copies (H and S are overwritten).
Status large_geneig(Handle& h, double2* Hm, double2* Sm, int m, double* w, cudaStream_t s) {
  if (!h.solver) {
    if (cusolverDnCreate(&h.solver) != CUSOLVER_STATUS_SUCCESS) return fail(kCuda, "cusolverDnCreate failed");
  }
  cusolverDnSetStream(h.solver, s);
  int lwork = 0;
  if (cusolverDnZhegvd_bufferSize(h.solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m,
                                  reinterpret_cast<cuDoubleComplex*>(Hm), m, reinterpret_cast<cuDoubleComplex*>(Sm), m,
                                  w, &lwork) != CUSOLVER_STATUS_SUCCESS)
    return fail(kCuda, "cusolverDnZhegvd_bufferSize failed");
  if ((size_t)lwork > h.solver_work_len) {
    if (h.solver_work) cudaFree(h.solver_work);
    h.solver_work = nullptr;
    PW_CUDA_TRY(cudaMalloc((void**)&h.solver_work, (size_t)lwork * sizeof(double2)));
    h.solver_work_len = lwork;
  }
  if (!h.solver_info) PW_CUDA_TRY(cudaMalloc((void**)&h.solver_info, sizeof(int)));
  if (cusolverDnZhegvd(h.solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m,
                       reinterpret_cast<cuDoubleComplex*>(Hm), m, reinterpret_cast<cuDoubleComplex*>(Sm), m, w,
                       reinterpret_cast<cuDoubleComplex*>(h.solver_work), lwork,
                       h.solver_info) != CUSOLVER_STATUS_SUCCESS)
    return fail(kCuda, "cusolverDnZhegvd failed");
  return kOk;
}

}  // namespace pwgpu
