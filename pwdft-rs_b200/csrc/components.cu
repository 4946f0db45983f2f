// Per-band terms of the energy decomposition at convergence
// (EnergyComponents, scf/energy.rs:597-670):
//   kinetic  t_b = sum_G |c_b(G)|^2 (hbar^2/2m)|k+G|^2   (kinetic_expectation, energy.rs:382-421)
//   nonlocal n_b = <c_b| B D B^H |c_b> = Re sum_ij conj(P_ib) D_ij P_jb, P = B^H c_b
//                                                        (nonlocal_expectation, energy.rs:467-516)
// The reference forms the dense n_pw x n_pw H_NL per k for the second; here
// it is the projection P (one GEMM) and the block-diagonal D, the same
// operator.  On Gamma handles the bands are packed real (u^T u = <c|c> and
// u^2 against the packed kinetic table gives the full-sphere sum) and
// P = B_r^T u carries the factor i of odd-l columns, which cancels in
// conj(P) D P because D couples equal l only.
#include <algorithm>
#include <vector>

#include "handle.hpp"

namespace pwgpu {

namespace {

constexpr int kThreads = 256;

__device__ double block_sum256(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = kThreads / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  return sh[0];
}

// one block per band: out[b] = sum_i |x_ib|^2 kin_i
__global__ void k_band_kinetic_cplx(const double2* __restrict__ x, long ldx, int n, const double* __restrict__ kin,
                                    double* __restrict__ out) {
  __shared__ double sh[kThreads];
  const double2* col = x + (long)blockIdx.x * ldx;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += kThreads) {
    const double2 v = col[i];
    acc += (v.x * v.x + v.y * v.y) * kin[i];
  }
  acc = block_sum256(acc, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = acc;
}

__global__ void k_band_kinetic_real(const double* __restrict__ u, long ldu, int n, const double* __restrict__ kin,
                                    double* __restrict__ out) {
  __shared__ double sh[kThreads];
  const double* col = u + (long)blockIdx.x * ldu;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += kThreads) acc += col[i] * col[i] * kin[i];
  acc = block_sum256(acc, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = acc;
}

// one block per band: out[b] = Re sum_c conj(P_cb) Q_cb with Q = D P
__global__ void k_band_pq_cplx(const double2* __restrict__ P, const double2* __restrict__ Q, int n_ch,
                               double* __restrict__ out) {
  __shared__ double sh[kThreads];
  const long o = (long)blockIdx.x * n_ch;
  double acc = 0.0;
  for (int c = threadIdx.x; c < n_ch; c += kThreads) {
    const double2 p = P[o + c], q = Q[o + c];
    acc += p.x * q.x + p.y * q.y;
  }
  acc = block_sum256(acc, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = acc;
}

__global__ void k_band_pq_real(const double* __restrict__ P, const double* __restrict__ Q, int n_ch,
                               double* __restrict__ out) {
  __shared__ double sh[kThreads];
  const long o = (long)blockIdx.x * n_ch;
  double acc = 0.0;
  for (int c = threadIdx.x; c < n_ch; c += kThreads) acc += P[o + c] * Q[o + c];
  acc = block_sum256(acc, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = acc;
}

}  // namespace

Status band_energy_terms(Handle& h, int ik, const double2* V, long ldv, int nb, double* d_out, double* t_kin,
                         double* t_nl, cudaStream_t s) {
  if (ik < 0 || ik >= h.n_k) return fail(kInvalid, "band_energy_terms: k-point index out of range");
  if (nb <= 0) return kOk;
  if (ldv < h.n_pw) return fail(kInvalid, "band_energy_terms: leading dimension smaller than n_pw");
  if (!d_out) return fail(kInvalid, "band_energy_terms: no scratch");
  const int n = h.n_pw;
  Status r = kOk;
  if (h.gam.on) {
    const double* u = reinterpret_cast<const double*>(V);
    k_band_kinetic_real<<<nb, kThreads, 0, s>>>(u, ldv, n, h.gam.kin_packed, d_out); count_launch();
    if (h.n_ch > 0 && (r = nonlocal_pq_real(h, u, ldv, nb, s)) == kOk) {
      k_band_pq_real<<<nb, kThreads, 0, s>>>(h.gam_p, h.gam_q, h.n_ch, d_out + nb); count_launch();
    }
  } else {
    k_band_kinetic_cplx<<<nb, kThreads, 0, s>>>(V, ldv, n, h.kp[ik].kinetic, d_out); count_launch();
    if (h.n_ch > 0 && (r = nonlocal_pq(h, ik, V, ldv, nb, s)) == kOk) {
      k_band_pq_cplx<<<nb, kThreads, 0, s>>>(h.nl_p, h.nl_q, h.n_ch, d_out + nb); count_launch();
    }
  }
  if (r == kOk && h.n_ch <= 0) {
    cudaError_t e = cudaMemsetAsync(d_out + nb, 0, nb * sizeof(double), s);
    if (e != cudaSuccess) r = fail(kCuda, std::string("band_energy_terms: ") + cudaGetErrorString(e));
  }
  if (r == kOk) {
    std::vector<double> host(2 * (size_t)nb);
    cudaError_t e = cudaMemcpyAsync(host.data(), d_out, host.size() * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      r = fail(kCuda, std::string("band_energy_terms: ") + cudaGetErrorString(e));
    } else {
      std::copy(host.begin(), host.begin() + nb, t_kin);
      std::copy(host.begin() + nb, host.end(), t_nl);
    }
  }
  return r;
}

}  // namespace pwgpu
