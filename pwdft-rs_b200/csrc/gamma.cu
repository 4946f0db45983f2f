// Gamma-only systems with real wavefunctions.
//
// At k = 0 the Hamiltonian of a real potential maps functions with
// psi(-G) = conj(psi(G)) (real in real space) to functions of the same kind,
// and the reference's eigenvectors can be chosen so (its dense H is then
// real symmetric in the cos/sin basis).  A band is stored as the real vector
//   u = [Re psi(0), sqrt2 Re psi(G_1..h), sqrt2 Im psi(G_1..h)]
// over the half sphere G_p > 0 (first nonzero Miller index positive), so
// <a|b> over the full sphere is the real dot product of the packed vectors
// and every subspace GEMM is real (a quarter of the complex flops).
//
// H u: two real bands a, b are packed into one complex full-sphere vector
// c = psi_a + i psi_b; the unchanged local pipeline (hpsi.cu) gives
// H_loc c = H_loc psi_a + i H_loc psi_b, and since both terms are again
// Gamma-real they separate as (x + conj y)/2 and (x - conj y)/(2i) with
// x = (H_loc c)(G), y = (H_loc c)(-G): half the FFTs of the complex form.
// The projector columns of a Gamma system are Gamma-real up to a factor i
// (odd l, whose i^l the reference's B omits); packed as B_r with those
// columns turned by i, B^H psi = B_r^T u (up to the same factors, which
// cancel in B D B^H because D couples equal l only) and B Q packs to B_r Q:
// the nonlocal term is two real GEMMs.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "handle.hpp"

namespace pwgpu {

namespace {

constexpr double kSqrt2 = 1.41421356237309504880;
constexpr double kInvSqrt2 = 0.70710678118654752440;

inline unsigned blocks_for(long n, int t = 256) { return (unsigned)std::max<long>(1, (n + t - 1) / t); }

// point t of the packed index space: t = 0 is G = 0, t = 1..nh the half sphere
// c[:, q] = w_a psi_a + i w_b psi_b for bands a = 2q, b = 2q + 1 (b < nb)
__global__ void k_unpack_pairs(const double* __restrict__ u, long ldu, int nb, double2* __restrict__ c, long ldc,
                               const int* __restrict__ half_idx, const int* __restrict__ half_neg, int zero, int nh,
                               const double* __restrict__ wts) {
  const int q = blockIdx.y;
  const int a = 2 * q, b = 2 * q + 1;
  const bool hb = b < nb;
  const double wa = wts ? wts[a] : 1.0, wb = (hb && wts) ? wts[b] : (hb ? 1.0 : 0.0);
  const double* ua = u + (long)a * ldu;
  const double* ub = u + (long)(hb ? b : a) * ldu;
  double2* cq = c + (long)q * ldc;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= nh; t += gridDim.x * blockDim.x) {
    if (t == 0) {
      cq[zero] = make_double2(wa * ua[0], wb * ub[0]);
      continue;
    }
    const int p = t - 1;
    const double ar = wa * kInvSqrt2 * ua[1 + p], ai = wa * kInvSqrt2 * ua[1 + nh + p];
    const double br = wb * kInvSqrt2 * ub[1 + p], bi = wb * kInvSqrt2 * ub[1 + nh + p];
    cq[half_idx[p]] = make_double2(ar - bi, ai + br);
    cq[half_neg[p]] = make_double2(ar + bi, br - ai);
  }
}

// inverse of k_unpack_pairs for (H c): separate the two real bands and pack
__global__ void k_pack_pairs(const double2* __restrict__ c, long ldc, int nb, double* __restrict__ u, long ldu,
                             const int* __restrict__ half_idx, const int* __restrict__ half_neg, int zero, int nh) {
  const int q = blockIdx.y;
  const int a = 2 * q, b = 2 * q + 1;
  const bool hb = b < nb;
  const double2* cq = c + (long)q * ldc;
  double* ua = u + (long)a * ldu;
  double* ub = hb ? u + (long)b * ldu : nullptr;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= nh; t += gridDim.x * blockDim.x) {
    if (t == 0) {
      const double2 z = cq[zero];
      ua[0] = z.x;
      if (hb) ub[0] = z.y;
      continue;
    }
    const int p = t - 1;
    const double2 x = cq[half_idx[p]], y = cq[half_neg[p]];
    // (H psi_a)(G) = (x + conj y)/2, (H psi_b)(G) = (x - conj y)/(2i)
    ua[1 + p] = kSqrt2 * 0.5 * (x.x + y.x);
    ua[1 + nh + p] = kSqrt2 * 0.5 * (x.y - y.y);
    if (hb) {
      ub[1 + p] = kSqrt2 * 0.5 * (x.y + y.y);
      ub[1 + nh + p] = -kSqrt2 * 0.5 * (x.x - y.x);
    }
  }
}

// single Gamma-real complex columns -> packed real columns; columns with
// rot[c] != 0 are packed as i x (a column with x(-G) = -conj x(G))
__global__ void k_pack_cols(const double2* __restrict__ x, long ldx, double* __restrict__ u, long ldu,
                            const int* __restrict__ half_idx, int zero, int nh, const int* __restrict__ rot) {
  const double2* xc = x + (long)blockIdx.y * ldx;
  double* uc = u + (long)blockIdx.y * ldu;
  const bool r = rot && rot[blockIdx.y];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= nh; t += gridDim.x * blockDim.x) {
    const double2 v0 = xc[t == 0 ? zero : half_idx[t - 1]];
    const double2 v = r ? make_double2(-v0.y, v0.x) : v0;
    if (t == 0) {
      uc[0] = v.x;
      continue;
    }
    uc[t] = kSqrt2 * v.x;
    uc[nh + t] = kSqrt2 * v.y;
  }
}

__global__ void k_unpack_cols(const double* __restrict__ u, long ldu, double2* __restrict__ x, long ldx,
                              const int* __restrict__ half_idx, const int* __restrict__ half_neg, int zero, int nh) {
  const double* uc = u + (long)blockIdx.y * ldu;
  double2* xc = x + (long)blockIdx.y * ldx;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= nh; t += gridDim.x * blockDim.x) {
    if (t == 0) {
      xc[zero] = make_double2(uc[0], 0.0);
      continue;
    }
    const double re = kInvSqrt2 * uc[t], im = kInvSqrt2 * uc[nh + t];
    xc[half_idx[t - 1]] = make_double2(re, im);
    xc[half_neg[t - 1]] = make_double2(re, -im);
  }
}

// Q = D P, real, D block-diagonal over atoms (each block dense, row-major)
__global__ void k_apply_d_real(const double* __restrict__ P, double* __restrict__ Q, int n_ch, int nb,
                               const int* __restrict__ ch_atom, const int* __restrict__ atom_ch_start,
                               const int* __restrict__ d_off, const double* __restrict__ d_vals) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)n_ch * nb) return;
  const int c = (int)(t % n_ch);
  const int b = (int)(t / n_ch);
  const int a = ch_atom[c];
  const int s = atom_ch_start[a];
  const int nc = atom_ch_start[a + 1] - s;
  const double* drow = d_vals + d_off[a] + (long)(c - s) * nc;
  const double* pcol = P + (long)b * n_ch + s;
  double acc = 0.0;
  for (int j = 0; j < nc; ++j) acc += drow[j] * pcol[j];
  Q[(long)b * n_ch + c] = acc;
}

// Gamma symmetry of each projector column c (one block per column):
// out[3c] = max |B(-G) - conj B(G)| with |Im B(0)| (even-l hypothesis),
// out[3c+1] = max |B(-G) + conj B(G)| with |Re B(0)| (odd-l), out[3c+2] = max |B|.
__global__ void k_gamma_check(const double2* __restrict__ B, int n, const int* __restrict__ half_idx,
                              const int* __restrict__ half_neg, int zero, int nh, double* __restrict__ out) {
  __shared__ double sh[3][256];
  const double2* col = B + (long)blockIdx.x * n;
  double de = 0.0, dd = 0.0, bm = 0.0;
  for (int t = threadIdx.x; t <= nh; t += blockDim.x) {
    if (t == 0) {
      const double2 z = col[zero];
      de = fmax(de, fabs(z.y));
      dd = fmax(dd, fabs(z.x));
      bm = fmax(bm, fmax(fabs(z.x), fabs(z.y)));
      continue;
    }
    const double2 x = col[half_idx[t - 1]], y = col[half_neg[t - 1]];
    de = fmax(de, fmax(fabs(x.x - y.x), fabs(x.y + y.y)));
    dd = fmax(dd, fmax(fabs(x.x + y.x), fabs(x.y - y.y)));
    bm = fmax(bm, fmax(fmax(fabs(x.x), fabs(x.y)), fmax(fabs(y.x), fabs(y.y))));
  }
  sh[0][threadIdx.x] = de;
  sh[1][threadIdx.x] = dd;
  sh[2][threadIdx.x] = bm;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] = fmax(sh[q][threadIdx.x], sh[q][threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; ++q) out[3L * blockIdx.x + q] = sh[q][0];
}

template <typename T> Status galloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) return fail(kOom, std::string("cudaMalloc (gamma): ") + cudaGetErrorString(e));
  return kOk;
}

inline int64_t miller_key(int a, int b, int c) {
  return (((int64_t)(a + 2048)) << 24) | (((int64_t)(b + 2048)) << 12) | (int64_t)(c + 2048);
}

inline bool positive(int a, int b, int c) { return a > 0 || (a == 0 && (b > 0 || (b == 0 && c > 0))); }

Status ensure_pairs(Handle& h, int npairs) {
  if (npairs <= h.gam_ccap) return kOk;
  if (h.gam_c1) cudaFree(h.gam_c1);
  if (h.gam_c2) cudaFree(h.gam_c2);
  h.gam_c1 = h.gam_c2 = nullptr;
  h.gam_ccap = 0;
  Status r;
  if ((r = galloc(&h.gam_c1, (size_t)h.n_pw * npairs)) != kOk) return r;
  if ((r = galloc(&h.gam_c2, (size_t)h.n_pw * npairs)) != kOk) return r;
  h.gam_ccap = npairs;
  return kOk;
}

}  // namespace

Status build_gamma(Handle& h, const int* miller, const double* kinetic, const int* atom_ch_start,
                   const double* d_blocks) {
  release_gamma(h);
  if (h.n_k != 1) return kOk;
  const int n = h.n_pw;
  std::unordered_map<int64_t, int> where;
  where.reserve((size_t)n * 2);
  for (int i = 0; i < n; ++i) where[miller_key(miller[3 * i], miller[3 * i + 1], miller[3 * i + 2])] = i;
  int zero = -1;
  std::vector<int> hi, hn;
  for (int i = 0; i < n; ++i) {
    const int a = miller[3 * i], b = miller[3 * i + 1], c = miller[3 * i + 2];
    if (a == 0 && b == 0 && c == 0) {
      zero = i;
      continue;
    }
    if (!positive(a, b, c)) continue;
    auto it = where.find(miller_key(-a, -b, -c));
    if (it == where.end()) return kOk;  // sphere not closed under inversion
    hi.push_back(i);
    hn.push_back(it->second);
  }
  const int nh = (int)hi.size();
  if (zero < 0 || 2 * nh + 1 != n) return kOk;
  // the kinetic term and every projector column must be symmetric under G -> -G
  double kmax = 0.0;
  for (int i = 0; i < n; ++i) kmax = std::max(kmax, std::fabs(kinetic[i]));
  for (int p = 0; p < nh; ++p)
    if (std::fabs(kinetic[hi[p]] - kinetic[hn[p]]) > 1e-12 * std::max(kmax, 1.0)) return kOk;
  // Projector columns: B(-G) = conj B(G) (even l) or -conj B(G) (odd l: the
  // reference's B drops the i^l factor, nonlocal.rs:311-338); the odd ones
  // are packed as i B, which leaves B D B^H unchanged as long as D couples
  // only columns of the same kind (it couples equal l within an atom).
  std::vector<int> rot(std::max(h.n_ch, 1), 0);
  GammaData& g = h.gam;
  Status r;
  if ((r = galloc(&g.half_idx, nh)) != kOk) return r;
  if ((r = galloc(&g.half_neg, nh)) != kOk) return r;
  PW_CUDA_TRY(cudaMemcpy(g.half_idx, hi.data(), nh * sizeof(int), cudaMemcpyHostToDevice));
  PW_CUDA_TRY(cudaMemcpy(g.half_neg, hn.data(), nh * sizeof(int), cudaMemcpyHostToDevice));
  if (h.n_ch > 0) {
    // symmetry of the device-resident B (uploaded or built on the device)
    double* dev = nullptr;
    if ((r = galloc(&dev, 3L * h.n_ch)) != kOk) return r;
    k_gamma_check<<<h.n_ch, 256, 0, h.stream>>>(h.kp[0].b, n, g.half_idx, g.half_neg, zero, nh, dev);
    count_launch();
    std::vector<double> chk(3L * h.n_ch);
    // h.stream is non-blocking: the legacy-stream copy below would not wait for the check
    cudaError_t e = cudaStreamSynchronize(h.stream);
    if (e == cudaSuccess) e = cudaMemcpy(chk.data(), dev, chk.size() * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dev);
    if (e != cudaSuccess) return fail(kCuda, std::string("gamma check: ") + cudaGetErrorString(e));
    double bmax = 0.0;
    for (int c = 0; c < h.n_ch; ++c) bmax = std::max(bmax, chk[3L * c + 2]);
    const double tol = 1e-12 * std::max(bmax, 1e-300);
    for (int c = 0; c < h.n_ch; ++c) {
      const bool even = chk[3L * c] <= tol, odd = chk[3L * c + 1] <= tol;
      if (!even && !odd) {
        release_gamma(h);
        return kOk;
      }
      rot[c] = even ? 0 : 1;
    }
    if (atom_ch_start && d_blocks) {
      long off = 0;
      for (int a = 0; a < h.n_atoms; ++a) {
        const int s0 = atom_ch_start[a], nc = atom_ch_start[a + 1] - s0;
        for (int i = 0; i < nc; ++i)
          for (int j = 0; j < nc; ++j)
            if (d_blocks[off + (long)i * nc + j] != 0.0 && rot[s0 + i] != rot[s0 + j]) {
              release_gamma(h);
              return kOk;
            }
        off += (long)nc * nc;
      }
    }
  }
  if ((r = galloc(&g.kin_packed, n)) != kOk) return r;
  std::vector<double> kp(n);
  kp[0] = kinetic[zero];
  for (int p = 0; p < nh; ++p) kp[1 + p] = kp[1 + nh + p] = kinetic[hi[p]];
  PW_CUDA_TRY(cudaMemcpy(g.kin_packed, kp.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  g.nh = nh;
  g.zero = zero;
  if (h.n_ch > 0) {
    int* rot_dev = nullptr;
    if ((r = galloc(&g.b_real, (size_t)n * h.n_ch)) != kOk) return r;
    if ((r = galloc(&rot_dev, (size_t)h.n_ch)) != kOk) return r;
    PW_CUDA_TRY(cudaMemcpy(rot_dev, rot.data(), h.n_ch * sizeof(int), cudaMemcpyHostToDevice));
    k_pack_cols<<<dim3(blocks_for(nh + 1), h.n_ch), 256, 0, h.stream>>>(h.kp[0].b, n, g.b_real, n, g.half_idx, zero,
                                                                        nh, rot_dev);
    count_launch();
    PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
    cudaFree(rot_dev);
  }
  g.on = true;
  return kOk;
}

void release_gamma(Handle& h) {
  GammaData& g = h.gam;
  auto f = [](void* p) { if (p) cudaFree(p); };
  f(g.half_idx); f(g.half_neg); f(g.kin_packed); f(g.b_real);
  g = GammaData();
  release_gamma_scratch(h);
}

void release_gamma_scratch(Handle& h) {
  auto f = [](void* p) { if (p) cudaFree(p); };
  f(h.gam_c1); f(h.gam_c2); f(h.gam_p); f(h.gam_q);
  h.gam_c1 = h.gam_c2 = nullptr;
  h.gam_p = h.gam_q = nullptr;
  h.gam_ccap = 0;
  h.gam_pcap = 0;
}

Status gamma_pack(Handle& h, const double2* x, long ldx, int ncols, double* u, long ldu, cudaStream_t s) {
  if (!h.gam.on) return fail(kState, "gamma_pack: not a Gamma-real handle");
  if (ncols <= 0) return kOk;
  const GammaData& g = h.gam;
  k_pack_cols<<<dim3(blocks_for(g.nh + 1), ncols), 256, 0, s>>>(x, ldx, u, ldu, g.half_idx, g.zero, g.nh, nullptr);
  count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

Status gamma_unpack(Handle& h, const double* u, long ldu, int ncols, double2* x, long ldx, cudaStream_t s) {
  if (!h.gam.on) return fail(kState, "gamma_unpack: not a Gamma-real handle");
  if (ncols <= 0) return kOk;
  const GammaData& g = h.gam;
  k_unpack_cols<<<dim3(blocks_for(g.nh + 1), ncols), 256, 0, s>>>(u, ldu, x, ldx, g.half_idx, g.half_neg, g.zero,
                                                                  g.nh);
  count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

Status ensure_gamma_pq(Handle& h, int nb) {
  if (nb <= h.gam_pcap) return kOk;
  if (h.gam_p) cudaFree(h.gam_p);
  if (h.gam_q) cudaFree(h.gam_q);
  h.gam_p = h.gam_q = nullptr;
  h.gam_pcap = 0;
  Status r;
  if ((r = galloc(&h.gam_p, (size_t)h.n_ch * nb)) != kOk) return r;
  if ((r = galloc(&h.gam_q, (size_t)h.n_ch * nb)) != kOk) return r;
  h.gam_pcap = nb;
  return kOk;
}

Status apply_d_real(Handle& h, int nb, cudaStream_t s) {
  const long tot = (long)h.n_ch * nb;
  k_apply_d_real<<<blocks_for(tot), 256, 0, s>>>(h.gam_p, h.gam_q, h.n_ch, nb, h.ch_atom, h.atom_ch_start, h.d_off,
                                                 h.d_vals);
  count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

Status nonlocal_pq_real(Handle& h, const double* u, long ldu, int nb, cudaStream_t s) {
  if (!h.gam.on) return fail(kState, "nonlocal_pq_real: not a Gamma-real handle");
  if (h.n_ch <= 0 || nb <= 0) return kOk;
  Status r;
  if ((r = ensure_gamma_pq(h, nb)) != kOk) return r;
  const int n = h.n_pw;
  cublasSetStream(h.blas, s);
  const double one = 1.0, zero = 0.0;
  if (cublasDgemm(h.blas, CUBLAS_OP_T, CUBLAS_OP_N, h.n_ch, nb, n, &one, h.gam.b_real, n, u, (int)ldu, &zero, h.gam_p,
                  h.n_ch) != CUBLAS_STATUS_SUCCESS)
    return fail(kCuda, "cublasDgemm (B^T u) failed");
  return apply_d_real(h, nb, s);
}

Status apply_h_real(Handle& h, int spin, const double* u, long ldu, int nb, double* hu, long ldh, int precision,
                    cudaStream_t s) {
  if (!h.gam.on) return fail(kState, "apply_h_real: not a Gamma-real handle");
  if (nb <= 0) return kOk;
  const GammaData& g = h.gam;
  const int n = h.n_pw;
  const int npairs = (nb + 1) / 2;
  Status r;
  if ((r = ensure_pairs(h, npairs)) != kOk) return r;
  const dim3 grid(std::min<unsigned>(blocks_for(g.nh + 1), 64u), npairs);
  k_unpack_pairs<<<grid, 256, 0, s>>>(u, ldu, nb, h.gam_c1, n, g.half_idx, g.half_neg, g.zero, g.nh, nullptr);
  count_launch();
  if ((r = apply_local_device(h, spin, 0, h.gam_c1, n, npairs, h.gam_c2, n, precision, s)) != kOk) return r;
  k_pack_pairs<<<grid, 256, 0, s>>>(h.gam_c2, n, nb, hu, ldh, g.half_idx, g.half_neg, g.zero, g.nh);
  count_launch();
  if (h.n_ch > 0 && precision == 1 && nl_mixed_eligible(h)) {
    // mixed form: both projector products as 3xBF16 tensor-core GEMMs (every
    // block width: on the four-cell Si64 batch this measured 1 % above
    // keeping the FP64 GEMMs for blocks narrower than 48 or 96 bands)
    if ((r = nonlocal_mixed_real(h, u, ldu, nb, hu, ldh, s)) != kOk) return r;
  } else if (h.n_ch > 0) {
    if ((r = nonlocal_pq_real(h, u, ldu, nb, s)) != kOk) return r;
    const double one = 1.0;
    if (cublasDgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_N, n, nb, h.n_ch, &one, g.b_real, n, h.gam_q, h.n_ch, &one, hu,
                    (int)ldh) != CUBLAS_STATUS_SUCCESS)
      return fail(kCuda, "cublasDgemm (B Q) failed");
  }
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

Status density_accumulate_real(Handle& h, const double* u, long ldu, const std::vector<double>& fw, double* rho,
                               cudaStream_t s) {
  if (!h.gam.on) return fail(kState, "density_accumulate_real: not a Gamma-real handle");
  const int nb = (int)fw.size();
  if (nb == 0) return kOk;
  const GammaData& g = h.gam;
  const int n = h.n_pw;
  const int npairs = (nb + 1) / 2;
  Status r;
  if ((r = ensure_pairs(h, npairs)) != kOk) return r;
  // c = sqrt(f_a) psi_a + i sqrt(f_b) psi_b: |c(r)|^2 = f_a psi_a^2 + f_b psi_b^2
  // for real psi_a(r), psi_b(r); weights go through gam_c2's first column as
  // scratch (nb doubles), the unit weights of the accumulation after them
  std::vector<double> w(nb + npairs);
  for (int b = 0; b < nb; ++b) w[b] = std::sqrt(std::max(fw[b], 0.0));
  for (int q = 0; q < npairs; ++q) w[nb + q] = 1.0;
  double* wdev = reinterpret_cast<double*>(h.gam_c2);
  if ((long)(nb + npairs) > 2L * n * h.gam_ccap) return fail(kInvalid, "density_accumulate_real: scratch too small");
  PW_CUDA_TRY(cudaMemcpyAsync(wdev, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  const dim3 grid(std::min<unsigned>(blocks_for(g.nh + 1), 64u), npairs);
  k_unpack_pairs<<<grid, 256, 0, s>>>(u, ldu, nb, h.gam_c1, n, g.half_idx, g.half_neg, g.zero, g.nh, wdev);
  count_launch();
  // (pageable source: the copy has left w when cudaMemcpyAsync returns)
  return density_accumulate(h, h.gam_c1, n, npairs, wdev + nb, rho, s);
}

}  // namespace pwgpu
