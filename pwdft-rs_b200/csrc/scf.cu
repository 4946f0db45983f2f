// Self-consistent field loop on the device.
//
// Replaces the per-iteration body of run_scf_unpolarized
// (scf/driver.rs:353-735): potentials from rho_in (energy.rs:293-358,
// xc.rs:129-288), per-k eigensolve (dense.rs:50-98 -> LOBPCG here, lobpcg.cu),
// occupations (smearing.rs:38-252, host FP64), density (density.rs:41-111),
// G-space symmetrisation (symmetry/density/g_space.rs:147-252), energies
// (energy.rs:51-235) and Anderson/Kerker mixing (mixing/anderson.rs:158-266,
// kerker.rs:18-49).  Wavefunctions, densities and mixer history stay on the
// device; the host sees eigenvalues, a handful of scalars per iteration and
// the Fermi-level bisection.
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "handle.hpp"
#include "linalg.hpp"
#include "lobpcg.hpp"
#include "scf.hpp"

namespace pwgpu {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kHaToEv = 27.211386245988;
constexpr double kRyToEv = 13.605693122994;
constexpr double kBohrToAng = 0.529177210903;
constexpr double kBohr3ToAng3 = kBohrToAng * kBohrToAng * kBohrToAng;
constexpr double kE2 = 14.399645351950548;
constexpr double kG2Zero = 1e-12;
constexpr double kRhoFloor = 1e-30;
constexpr int kRedBlocks = 512;  // partial sums per reduction (fixed order)

// ---------------------------------------------------------------------------
// deterministic reductions: partials[blockIdx] then one block sums them
// ---------------------------------------------------------------------------

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

// mode 0: sum a; 1: sum a*b; 2: sum (a-b)^2
__global__ void k_reduce(const double* __restrict__ a, const double* __restrict__ b, long n, int mode,
                         double* __restrict__ partials) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double x = a[i];
    if (mode == 0) acc += x;
    else if (mode == 1) acc += x * b[i];
    else { const double d = x - b[i]; acc += d * d; }
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__global__ void k_final_sum(const double* __restrict__ partials, int n, double* __restrict__ out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[i];
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) *out = acc;
}

// Hartree energy partials: sum_{G^2 > thr} |rho(G)|^2 / G^2
__global__ void k_hartree(const double2* __restrict__ rho_g, const double* __restrict__ g2, long n,
                          double2* __restrict__ vh, double fpe2, double* __restrict__ partials) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double q = g2[i];
    const double2 r = rho_g[i];
    if (q > kG2Zero) {
      if (vh) vh[i] = make_double2(r.x * fpe2 / q, r.y * fpe2 / q);
      acc += (r.x * r.x + r.y * r.y) * fpe2 / q;
    } else if (vh) {
      vh[i] = make_double2(0.0, 0.0);
    }
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// PZ81 LDA (xc.rs:129-288), energies per electron and potentials in eV.
__device__ __forceinline__ void pz_rs(double rs, bool pol, double& ec, double& vc) {
  if (rs >= 1.0) {
    const double g = pol ? -0.0843 : -0.1423, b1 = pol ? 1.3981 : 1.0529, b2 = pol ? 0.2611 : 0.3334;
    const double sq = sqrt(rs);
    const double den = 1.0 + b1 * sq + b2 * rs;
    ec = g / den;
    const double dec = -g * (b1 / (2.0 * sq) + b2) / (den * den);
    vc = fma(rs / 3.0, -dec, ec);
  } else {
    const double a = pol ? 0.01555 : 0.0311, b = pol ? -0.0269 : -0.048, c = pol ? 0.0007 : 0.0020,
                 d = pol ? -0.0048 : -0.0116;
    const double lr = log(rs);
    ec = fma(d, rs, fma(c * rs, lr, fma(a, lr, b)));
    const double dec = fma(c, lr + 1.0, a / rs) + d;
    vc = fma(rs / 3.0, -dec, ec);
  }
}

// rho_xc = max(rho + core, 0) (energy.rs:314-324), exc/vxc, and partial sums
// of rho_xc*exc and rho_val*vxc.
__global__ void k_lda(const double* __restrict__ rho, const double* __restrict__ core, long n,
                      double* __restrict__ exc_out, double* __restrict__ vxc_out, double* __restrict__ part_exc,
                      double* __restrict__ part_vxc) {
  __shared__ double sh[32];
  double a1 = 0.0, a2 = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double rv = rho[i];
    const double r = core ? fmax(rv + core[i], 0.0) : rv;
    double exc = 0.0, vxc = 0.0;
    if (r >= kRhoFloor) {
      const double rb = r * kBohr3ToAng3;
      const double ex = -0.75 * cbrt(3.0 * rb / kPi);
      const double vx = (4.0 / 3.0) * ex;
      const double rs = cbrt(3.0 / (4.0 * kPi * rb));
      double ec, vc;
      pz_rs(rs, false, ec, vc);
      exc = (ex + ec) * kHaToEv;
      vxc = (vx + vc) * kHaToEv;
    }
    exc_out[i] = exc;
    vxc_out[i] = vxc;
    a1 += r * exc;
    a2 += rv * vxc;
  }
  a1 = block_sum(a1, sh);
  a2 = block_sum(a2, sh);
  if (threadIdx.x == 0) {
    part_exc[blockIdx.x] = a1;
    part_vxc[blockIdx.x] = a2;
  }
}

__global__ void k_real_to_cplx(const double* __restrict__ r, double2* __restrict__ c, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) c[i] = make_double2(r[i], 0.0);
}

__global__ void k_cplx_real_scaled(const double2* __restrict__ c, double* __restrict__ r, double s, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = c[i].x * s;
}

__global__ void k_scale_cplx(double2* __restrict__ c, double s, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) c[i] = make_double2(c[i].x * s, c[i].y * s);
}

__global__ void k_scale_real(double* __restrict__ r, double s, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] *= s;
}

// V_eff(G) = V_loc(G) + V_H(G) + V_xc(G) (energy.rs:293-301)
__global__ void k_veff_g(const double2* __restrict__ vloc, const double2* __restrict__ vh,
                         const double2* __restrict__ vxc_g, double2* __restrict__ out, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const double2 a = vloc[i], b = vh[i], c = vxc_g[i];
    out[i] = make_double2(a.x + b.x + c.x, a.y + b.y + c.y);
  }
}

__global__ void k_real_part_both(const double2* __restrict__ c, double* __restrict__ r64, float* __restrict__ r32,
                                 long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    r64[i] = c[i].x;
    r32[i] = (float)c[i].x;
  }
}

// rho_sym(n) = (1/N_ops) sum_S e^{-i arg_S(n)} rho(src_S(n))  (g_space.rs:217-243)
__global__ void k_sym_gather(const double2* __restrict__ rg, const int* __restrict__ src,
                             const double* __restrict__ arg, int nops, long n, double2* __restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double re = 0.0, im = 0.0;
  for (int s = 0; s < nops; ++s) {
    const double2 r = rg[src[(long)s * n + i]];
    double sn, cs;
    sincos(arg[(long)s * n + i], &sn, &cs);
    // (cs - i sn) * r
    re += cs * r.x + sn * r.y;
    im += cs * r.y - sn * r.x;
  }
  const double inv = 1.0 / nops;
  out[i] = make_double2(re * inv, im * inv);
}

// Anderson pieces
__global__ void k_sub(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] - b[i];
}

// dot((r_i - r_l), (r_j - r_l)) partials, or dot(r_i - r_l, r_l) when j < 0
__global__ void k_dr_dot(const double* __restrict__ ri, const double* __restrict__ rj, const double* __restrict__ rl,
                         long n, double* __restrict__ partials) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double a = ri[i] - rl[i];
    const double b = rj ? rj[i] - rl[i] : rl[i];
    acc += a * b;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// out = sum_i coef[i] * (hin_i + beta * hres_i)
__global__ void k_mix_combine(const double* const* __restrict__ hin, const double* const* __restrict__ hres,
                              const double* __restrict__ coef, int m, double beta, long n, double* __restrict__ out) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc = 0.0;
  for (int j = 0; j < m; ++j) acc += coef[j] * (hin[j][i] + beta * hres[j][i]);
  out[i] = acc;
}

__global__ void k_mul_real_weights(double2* __restrict__ c, const double* __restrict__ w, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) c[i] = make_double2(c[i].x * w[i], c[i].y * w[i]);
}

inline unsigned blocks_for(long n, int t = 256) { return (unsigned)std::max<long>(1, (n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------------------
// state
// ---------------------------------------------------------------------------

struct ScfState {
  int nd = 0, nb = 0;
  std::vector<EigVecs> ks;  // per (spin, k)
  EigWork ew;
  double *partials = nullptr, *scal = nullptr, *fw = nullptr;
  double *rho_in = nullptr, *rho_out = nullptr, *exc = nullptr, *vxc = nullptr, *rtmp = nullptr;
  double2 *cg = nullptr, *cg2 = nullptr, *vh = nullptr;
  double* kerker_w = nullptr;
  std::vector<double*> hin, hres;
  double** dev_ptrs = nullptr;
  double* dev_coef = nullptr;
  int mix_count = 0;
};

template <typename T> static Status salloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) return fail(kOom, std::string("cudaMalloc (scf): ") + cudaGetErrorString(e));
  return kOk;
}

void release_scf(Handle& h) {
  ScfState* st = h.scf;
  if (!st) return;
  auto f = [](void* p) { if (p) cudaFree(p); };
  for (auto& k : st->ks) eig_vecs_release(k);
  eig_work_release(st->ew);
  f(st->partials); f(st->scal); f(st->fw);
  f(st->rho_in); f(st->rho_out); f(st->exc); f(st->vxc); f(st->rtmp);
  f(st->cg); f(st->cg2); f(st->vh); f(st->kerker_w);
  for (double* p : st->hin) f(p);
  for (double* p : st->hres) f(p);
  f(st->dev_ptrs); f(st->dev_coef);
  delete st;
  h.scf = nullptr;
}

static Status ensure_state(Handle& h, int nb, int nd, int ndim) {
  if (h.scf && h.scf->nd == nd && h.scf->nb == nb && (int)h.scf->hin.size() >= ndim) return kOk;
  release_scf(h);
  ScfState* st = new ScfState();
  h.scf = st;
  st->nd = nd;
  st->nb = nb;
  const long n = h.n_pw, N = h.g.N;
  Status s;
  st->ks.resize((size_t)h.nspin * h.n_k);
  for (auto& k : st->ks)
    if ((s = eig_vecs_alloc(k, n, nd)) != kOk) return s;
  if ((s = eig_work_alloc(st->ew, n, nd)) != kOk) return s;
  if ((s = salloc(&st->partials, (size_t)kRedBlocks * 4)) != kOk) return s;
  if ((s = salloc(&st->scal, 16)) != kOk) return s;
  if ((s = salloc(&st->fw, (size_t)nd)) != kOk) return s;
  if ((s = salloc(&st->rho_in, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->rho_out, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->exc, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->vxc, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->rtmp, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->cg, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->cg2, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->vh, (size_t)N)) != kOk) return s;
  st->hin.assign(ndim, nullptr);
  st->hres.assign(ndim, nullptr);
  for (int i = 0; i < ndim; ++i) {
    if ((s = salloc(&st->hin[i], (size_t)N)) != kOk) return s;
    if ((s = salloc(&st->hres[i], (size_t)N)) != kOk) return s;
  }
  if ((s = salloc(&st->dev_ptrs, (size_t)2 * std::max(ndim, 1))) != kOk) return s;
  if ((s = salloc(&st->dev_coef, (size_t)std::max(ndim, 1))) != kOk) return s;
  return kOk;
}

// Deterministic sum helpers (result copied to the host).
static Status reduce_host(Handle& h, const double* a, const double* b, long n, int mode, double& out) {
  ScfState* st = h.scf;
  const cudaStream_t s = h.stream;
  const unsigned nbk = (unsigned)std::min<long>(kRedBlocks, blocks_for(n));
  k_reduce<<<nbk, 256, 0, s>>>(a, b, n, mode, st->partials); count_launch();
  k_final_sum<<<1, 256, 0, s>>>(st->partials, (int)nbk, st->scal); count_launch();
  PW_CUDA_TRY(cudaMemcpyAsync(&out, st->scal, sizeof(double), cudaMemcpyDeviceToHost, s));
  PW_CUDA_TRY(cudaStreamSynchronize(s));
  return kOk;
}

static Status final_sum_host(Handle& h, int nparts, double& out, int slot = 0) {
  ScfState* st = h.scf;
  k_final_sum<<<1, 256, 0, h.stream>>>(st->partials + (long)slot * kRedBlocks, nparts, st->scal + slot); count_launch();
  PW_CUDA_TRY(cudaMemcpyAsync(&out, st->scal + slot, sizeof(double), cudaMemcpyDeviceToHost, h.stream));
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
  return kOk;
}

// rho(G) = FFT(rho)/N into st->cg
static Status density_to_g(Handle& h, const double* rho) {
  const long N = h.g.N;
  k_real_to_cplx<<<blocks_for(N), 256, 0, h.stream>>>(rho, h.scf->cg, N); count_launch();
  Status s = fft3d_full(h, h.scf->cg, -1, h.stream);
  if (s != kOk) return s;
  k_scale_cplx<<<blocks_for(N), 256, 0, h.stream>>>(h.scf->cg, 1.0 / (double)N, N); count_launch();
  return kOk;
}

struct PotEnergies {
  double e_hartree = 0, e_xc = 0, e_vxc = 0;
};

// Potentials from rho (device): V_eff(G) into st->cg2 (and V_eff(r) into the
// handle's H|psi> arrays when set_hpsi), exc/vxc on the grid, energies.
static Status potentials(Handle& h, const double* rho, bool set_hpsi, PotEnergies& e) {
  ScfState* st = h.scf;
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  Status r = density_to_g(h, rho);
  if (r != kOk) return r;
  const double fpe2 = 4.0 * kPi * kE2;
  const unsigned nbk = (unsigned)std::min<long>(kRedBlocks, blocks_for(N));
  k_hartree<<<nbk, 256, 0, s>>>(st->cg, h.g_squared, N, st->vh, fpe2, st->partials); count_launch();
  double sh = 0.0;
  if ((r = final_sum_host(h, (int)nbk, sh)) != kOk) return r;
  e.e_hartree = sh * 0.5 * h.omega;
  k_lda<<<nbk, 256, 0, s>>>(rho, h.rho_core_r, N, st->exc, st->vxc, st->partials, st->partials + kRedBlocks); count_launch();
  double sx = 0.0, sv = 0.0;
  if ((r = final_sum_host(h, (int)nbk, sx, 0)) != kOk) return r;
  if ((r = final_sum_host(h, (int)nbk, sv, 1)) != kOk) return r;
  const double dv = h.omega / (double)N;
  e.e_xc = sx * dv;
  e.e_vxc = sv * dv;
  // V_xc(G) = FFT(vxc)/N, V_eff(G) = V_loc + V_H + V_xc
  k_real_to_cplx<<<blocks_for(N), 256, 0, s>>>(st->vxc, st->cg2, N); count_launch();
  if ((r = fft3d_full(h, st->cg2, -1, s)) != kOk) return r;
  k_scale_cplx<<<blocks_for(N), 256, 0, s>>>(st->cg2, 1.0 / (double)N, N); count_launch();
  k_veff_g<<<blocks_for(N), 256, 0, s>>>(h.v_local_g, st->vh, st->cg2, st->cg2, N); count_launch();
  if (set_hpsi) {
    PW_CUDA_TRY(cudaMemcpyAsync(h.tmp_grid, st->cg2, N * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    if ((r = fft3d_full(h, h.tmp_grid, +1, s)) != kOk) return r;
    k_real_part_both<<<blocks_for(N), 256, 0, s>>>(h.tmp_grid, h.veff_r[0], h.veff_r32[0], N); count_launch();
  }
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

static Status symmetrize(Handle& h, double* rho) {
  if (h.n_sym <= 1) return kOk;
  ScfState* st = h.scf;
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  k_real_to_cplx<<<blocks_for(N), 256, 0, s>>>(rho, st->cg, N); count_launch();
  Status r = fft3d_full(h, st->cg, -1, s);
  if (r != kOk) return r;
  k_sym_gather<<<blocks_for(N), 256, 0, s>>>(st->cg, h.sym_src, h.sym_arg, h.n_sym, N, st->cg2); count_launch();
  if ((r = fft3d_full(h, st->cg2, +1, s)) != kOk) return r;
  k_cplx_real_scaled<<<blocks_for(N), 256, 0, s>>>(st->cg2, rho, 1.0 / (double)N, N); count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
// occupations (smearing.rs:38-252), host FP64
// ---------------------------------------------------------------------------

static double occ01(int scheme, double e, double ef, double sigma) {
  if (sigma < 1e-15) {
    if (e < ef) return 1.0;
    if (std::fabs(e - ef) < 1e-12) return 0.5;
    return 0.0;
  }
  const double x = (e - ef) / sigma;
  switch (scheme) {
    case 1: return std::erfc(x) / 2.0;
    case 2: return std::fma(0.5 * x, -(std::exp(-x * x) / std::sqrt(kPi)), std::erfc(x) / 2.0);
    case 3: {
      const double a = x + 1.0 / std::sqrt(2.0);
      return std::fma(0.5, std::erfc(a), (1.0 / std::sqrt(2.0 * kPi)) * std::exp(-a * a));
    }
    default:
      if (x > 40.0) return 0.0;
      if (x < -40.0) return 1.0;
      return 1.0 / (1.0 + std::exp(x));
  }
}

static double fermi_level(const std::vector<std::vector<double>>& ev, const std::vector<double>& w, double nel,
                          double sigma, int scheme, double spin_factor) {
  double lo = INFINITY, hi = -INFINITY;
  for (auto& e : ev)
    for (double x : e) { lo = std::min(lo, x); hi = std::max(hi, x); }
  lo -= 10.0 * std::max(sigma, 0.1);
  hi += 10.0 * std::max(sigma, 0.1);
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    double nsum = 0.0;
    for (size_t k = 0; k < ev.size(); ++k) {
      double sk = 0.0;
      for (double x : ev[k]) sk += w[k] * occ01(scheme, x, mid, sigma) * spin_factor;
      nsum += sk;
    }
    if (nsum < nel) lo = mid; else hi = mid;
    if (std::fabs(hi - lo) < 1e-14) break;
  }
  return 0.5 * (lo + hi);
}

static double entropy_ts(const std::vector<std::vector<double>>& ev, const std::vector<double>& w, double ef,
                         double sigma, int scheme, double spin_factor) {
  if (sigma < 1e-15) return 0.0;
  double s = 0.0;
  for (size_t k = 0; k < ev.size(); ++k) {
    for (double e : ev[k]) {
      const double x = (e - ef) / sigma;
      double sw;
      switch (scheme) {
        case 1: sw = std::exp(-x * x) / std::sqrt(kPi); break;
        case 2: sw = std::fma(x, -x, 0.5) * std::exp(-x * x) / std::sqrt(kPi); break;
        case 3: { const double a = x + 1.0 / std::sqrt(2.0); sw = a * std::exp(-a * a) / std::sqrt(kPi); break; }
        default: {
          if (std::fabs(x) > 30.0) { sw = 0.0; break; }
          double f = 1.0 / (1.0 + std::exp(x));
          f = std::min(std::max(f, 1e-30), 1.0 - 1e-30);
          sw = -(f * std::log(f) + (1.0 - f) * std::log(1.0 - f));
        }
      }
      s += w[k] * sw;
    }
  }
  return s * sigma * spin_factor;
}

// partial-pivot LU solve with the 1e-15 singular-pivot fallback (linalg.rs:124-152)
static std::vector<double> solve_small(std::vector<double> a, std::vector<double> b, int n) {
  std::vector<int> piv(n);
  for (int i = 0; i < n; ++i) piv[i] = i;
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(a[r * n + c]) > std::fabs(a[p * n + c])) p = r;
    if (p != c) {
      for (int j = 0; j < n; ++j) std::swap(a[c * n + j], a[p * n + j]);
      std::swap(b[c], b[p]);
    }
    if (std::fabs(a[c * n + c]) < 1e-15) return std::vector<double>(n, 1.0 / (n + 1));
    for (int r = c + 1; r < n; ++r) {
      const double f = a[r * n + c] / a[c * n + c];
      for (int j = c; j < n; ++j) a[r * n + j] -= f * a[c * n + j];
      b[r] -= f * b[c];
    }
  }
  std::vector<double> x(n);
  for (int r = n - 1; r >= 0; --r) {
    double acc = b[r];
    for (int j = r + 1; j < n; ++j) acc -= a[r * n + j] * x[j];
    x[r] = acc / a[r * n + r];
  }
  return x;
}

// Anderson/Kerker mixing: rho_in <- mix(rho_in, rho_out) in place.
static Status mix(Handle& h, const ScfParams& p) {
  ScfState* st = h.scf;
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  const int ndim = p.mixing_ndim;
  // rotate history: slot order oldest .. newest kept in vectors
  if (st->mix_count == ndim) {
    std::rotate(st->hin.begin(), st->hin.begin() + 1, st->hin.end());
    std::rotate(st->hres.begin(), st->hres.begin() + 1, st->hres.end());
    --st->mix_count;
  }
  const int slot = st->mix_count;
  double* res = st->hres[slot];
  k_sub<<<blocks_for(N), 256, 0, s>>>(st->rho_out, st->rho_in, res, N); count_launch();
  if (st->kerker_w) {
    k_real_to_cplx<<<blocks_for(N), 256, 0, s>>>(res, st->cg, N); count_launch();
    Status r = fft3d_full(h, st->cg, -1, s);
    if (r != kOk) return r;
    k_mul_real_weights<<<blocks_for(N), 256, 0, s>>>(st->cg, st->kerker_w, N); count_launch();
    if ((r = fft3d_full(h, st->cg, +1, s)) != kOk) return r;
    k_cplx_real_scaled<<<blocks_for(N), 256, 0, s>>>(st->cg, res, 1.0 / (double)N, N); count_launch();
  }
  PW_CUDA_TRY(cudaMemcpyAsync(st->hin[slot], st->rho_in, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  st->mix_count++;
  const int m = st->mix_count;
  std::vector<double> coef(m, 0.0);
  if (m < 2) {
    coef[0] = 1.0;
  } else {
    const int mm = m - 1;
    const double* rl = st->hres[m - 1];
    std::vector<double> a((size_t)mm * mm), b(mm);
    const unsigned nbk = (unsigned)std::min<long>(kRedBlocks, blocks_for(N));
    for (int i = 0; i < mm; ++i) {
      k_dr_dot<<<nbk, 256, 0, s>>>(st->hres[i], nullptr, rl, N, st->partials); count_launch();
      double v = 0.0;
      Status r = final_sum_host(h, (int)nbk, v);
      if (r != kOk) return r;
      b[i] = -v;
      for (int j = 0; j <= i; ++j) {
        k_dr_dot<<<nbk, 256, 0, s>>>(st->hres[i], st->hres[j], rl, N, st->partials); count_launch();
        if ((r = final_sum_host(h, (int)nbk, v)) != kOk) return r;
        a[(size_t)i * mm + j] = v;
        a[(size_t)j * mm + i] = v;
      }
    }
    std::vector<double> al = solve_small(a, b, mm);
    double sum = 0.0;
    for (int i = 0; i < mm; ++i) { coef[i] = al[i]; sum += al[i]; }
    coef[mm] = 1.0 - sum;
  }
  std::vector<double*> ptrs(2 * m);
  for (int j = 0; j < m; ++j) { ptrs[j] = st->hin[j]; ptrs[m + j] = st->hres[j]; }
  PW_CUDA_TRY(cudaMemcpyAsync(st->dev_ptrs, ptrs.data(), 2 * m * sizeof(double*), cudaMemcpyHostToDevice, s));
  PW_CUDA_TRY(cudaMemcpyAsync(st->dev_coef, coef.data(), m * sizeof(double), cudaMemcpyHostToDevice, s));
  k_mix_combine<<<blocks_for(N), 256, 0, s>>>(st->dev_ptrs, st->dev_ptrs + m, st->dev_coef, m, p.mixing_beta, N,
                                             st->rho_in); count_launch();
  PW_CUDA_TRY(cudaStreamSynchronize(s));
  return kOk;
}

// Density of all k-points (density.rs:41-111): rho_out = renormalised sum,
// then symmetrised.
static Status build_density(Handle& h, const std::vector<std::vector<double>>& occ, const std::vector<double>& w,
                            int spin, double* rho) {
  ScfState* st = h.scf;
  const long N = h.g.N, n = h.n_pw;
  const cudaStream_t s = h.stream;
  PW_CUDA_TRY(cudaMemsetAsync(rho, 0, N * sizeof(double), s));
  std::vector<double> fw;
  for (int ik = 0; ik < h.n_k; ++ik) {
    fw.clear();
    for (double f : occ[ik]) {
      const double v = f * w[ik];
      if (v < 1e-15) break;  // occupations decrease with band energy
      fw.push_back(v);
    }
    if (fw.empty()) continue;
    PW_CUDA_TRY(cudaMemcpyAsync(st->fw, fw.data(), fw.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    Status r = density_accumulate(h, st->ks[(size_t)spin * h.n_k + ik].V, n, (int)fw.size(), st->fw, rho, s);
    if (r != kOk) return r;
    PW_CUDA_TRY(cudaStreamSynchronize(s));
  }
  double tot = 0.0;
  Status r = reduce_host(h, rho, nullptr, N, 0, tot);
  if (r != kOk) return r;
  const double integ = tot * (h.omega / (double)N);
  if (std::fabs(integ) > 1e-15) {
    k_scale_real<<<blocks_for(N), 256, 0, s>>>(rho, h.n_electrons / integ, N);
    count_launch();
  }
  return symmetrize(h, rho);
}

Status scf_run(Handle& h, const ScfParams& p, const double* rho_init, ScfResult& res, double* evals_out,
               double* rho_out_host, double* rho_g_basis_out) {
  if (h.nspin != 1) return fail(kNotImplemented, "scf_run: nspin = 2 is not available in this build");
  if (p.n_bands < 1 || p.n_bands > h.n_pw) return fail(kInvalid, "scf_run: n_bands out of range");
  if (p.mixing_ndim < 1 || p.max_iter < 1) return fail(kInvalid, "scf_run: mixing_ndim and max_iter must be >= 1");
  PW_CUDA_TRY(cudaSetDevice(h.device));
  const int nb = p.n_bands;
  int extra = p.diag_extra_bands >= 0 ? p.diag_extra_bands : std::max(2, nb / 8);
  const int nd = (int)std::min<long>(nb + extra, h.n_pw);
  Status r = ensure_state(h, nb, nd, p.mixing_ndim);
  if (r != kOk) return r;
  ScfState* st = h.scf;
  for (auto& k : st->ks) k.init = false;
  st->mix_count = 0;
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  cublasSetStream(h.blas, s);
  // Kerker weights P(G) = G^2/(G^2 + q^2), P(0) = 0 (kerker.rs:18-49)
  if (p.mixing_mode == 1) {
    double q2 = p.kerker_q_tf * p.kerker_q_tf;
    if (p.kerker_q_tf <= 0.0) {
      const double rb = h.n_electrons / h.omega * kBohr3ToAng3;
      q2 = 4.0 * std::cbrt(3.0 * kPi * kPi * rb) / kPi / (kBohrToAng * kBohrToAng);
    }
    std::vector<double> g2(N), wk(N);
    PW_CUDA_TRY(cudaMemcpy(g2.data(), h.g_squared, N * sizeof(double), cudaMemcpyDeviceToHost));
    for (long i = 0; i < N; ++i) wk[i] = g2[i] < kG2Zero ? 0.0 : g2[i] / (g2[i] + q2);
    if (!st->kerker_w && (r = salloc(&st->kerker_w, (size_t)N)) != kOk) return r;
    PW_CUDA_TRY(cudaMemcpy(st->kerker_w, wk.data(), N * sizeof(double), cudaMemcpyHostToDevice));
  } else if (st->kerker_w) {
    cudaFree(st->kerker_w);
    st->kerker_w = nullptr;
  }
  PW_CUDA_TRY(cudaMemcpyAsync(st->rho_in, rho_init, N * sizeof(double), cudaMemcpyHostToDevice, s));
  std::vector<double> wk(h.n_k);
  for (int k = 0; k < h.n_k; ++k) wk[k] = h.kp[k].weight;
  const double spin_factor = 2.0;
  bool have_prev = false;
  // mixed form: FP64 H|psi> from the first iteration whose input density rms
  // is below fp64_switch, or once the reduced-precision phase stops reducing
  // it (two iterations without a 30 % improvement on the best so far: the
  // precision floor of the FP32/BF16 operator), for the rest of the solve
  bool fp64_locked = p.precision != 1;
  double best_delta = INFINITY;
  int stalled = 0;
  double e_prev = 0.0, last_delta = INFINITY, max_res_all = 0.0;
  long happ = 0;
  std::vector<std::vector<double>> ev(h.n_k), occ(h.n_k);
  for (int iter = 0; iter < p.max_iter; ++iter) {
    PotEnergies ein;
    if ((r = potentials(h, st->rho_in, true, ein)) != kOk) return r;
    if (!fp64_locked && (last_delta < p.fp64_switch || stalled >= 2)) fp64_locked = true;
    const int prec = fp64_locked ? 0 : 1;
    const double tol = std::max(p.diag_tol, std::min(1e-3, 0.1 * (std::isfinite(last_delta) ? last_delta : 1.0)));
    // preconditioner shift: V_eff(G = 0) = mean of V_eff(r)
    double vsum = 0.0;
    if ((r = reduce_host(h, h.veff_r[0], nullptr, N, 0, vsum)) != kOk) return r;
    const double v0 = vsum / (double)N;
    max_res_all = 0.0;
    for (int ik = 0; ik < h.n_k; ++ik) {
      EigStats es;
      if ((r = lobpcg(h, st->ew, st->ks[ik], 0, ik, v0, tol, iter == 0 ? 4 * p.diag_max_iter : p.diag_max_iter, nb,
                      prec, es)) != kOk)
        return r;
      happ += es.happ;
      max_res_all = std::max(max_res_all, es.max_res);
      ev[ik].assign(st->ks[ik].evals.begin(), st->ks[ik].evals.begin() + nb);
    }
    const double ef = fermi_level(ev, wk, h.n_electrons, p.sigma, p.smearing, spin_factor);
    for (int ik = 0; ik < h.n_k; ++ik) {
      occ[ik].resize(nb);
      for (int b = 0; b < nb; ++b) occ[ik][b] = occ01(p.smearing, ev[ik][b], ef, p.sigma) * spin_factor;
    }
    if ((r = build_density(h, occ, wk, 0, st->rho_out)) != kOk) return r;
    double dsq = 0.0;
    if ((r = reduce_host(h, st->rho_in, st->rho_out, N, 2, dsq)) != kOk) return r;
    const double dv = h.omega / (double)N;
    const double delta = std::sqrt(dsq * dv / h.omega);
    last_delta = delta;
    if (!fp64_locked) {
      if (delta < 0.7 * best_delta) {
        best_delta = delta;
        stalled = 0;
      } else {
        ++stalled;
      }
    }
    PotEnergies eout;
    if ((r = potentials(h, st->rho_out, false, eout)) != kOk) return r;
    double e_band = 0.0;
    for (int ik = 0; ik < h.n_k; ++ik) {
      double sk = 0.0;
      for (int b = 0; b < nb; ++b) sk += occ[ik][b] * wk[ik] * ev[ik][b];
      e_band += sk;
    }
    const double ts = entropy_ts(ev, wk, ef, p.sigma, p.smearing, spin_factor);
    const double e_tot = e_band - eout.e_hartree + (eout.e_xc - eout.e_vxc) + h.e_ewald - ts;
    const double e_hf = e_band - ein.e_hartree + (ein.e_xc - ein.e_vxc) + h.e_ewald - ts;
    const double de = have_prev ? std::fabs(e_tot - e_prev) : INFINITY;
    if (p.verbose)
      std::fprintf(stderr, "pwgpu scf iter %3d E=%.10f dE=%.3e drho=%.3e res=%.2e prec=%d happ=%ld\n", iter, e_tot,
                   de, delta, max_res_all, prec, happ);
    const bool conv = delta < p.conv_threshold && have_prev && de < p.energy_threshold;
    e_prev = e_tot;
    have_prev = true;
    if (conv || iter == p.max_iter - 1) {
      res.total_energy = e_tot;
      res.harris_foulkes_energy = e_hf;
      res.free_energy = e_tot;
      res.energy_sigma0 = 0.5 * ((e_tot + ts) + e_tot);
      res.entropy_ts = ts;
      res.fermi_energy = ef;
      res.final_delta = delta;
      res.e_band = e_band;
      res.e_hartree = eout.e_hartree;
      res.e_xc = eout.e_xc;
      res.e_vxc = eout.e_vxc;
      res.e_ewald = h.e_ewald;
      res.n_iterations = iter + 1;
      res.converged = conv ? 1 : 0;
      res.nspin = 1;
      res.h_applications = happ;
      res.max_residual = max_res_all;
      if (evals_out)
        for (int ik = 0; ik < h.n_k; ++ik)
          for (int b = 0; b < nb; ++b) evals_out[(size_t)ik * nb + b] = ev[ik][b];
      if (rho_out_host)
        PW_CUDA_TRY(cudaMemcpyAsync(rho_out_host, st->rho_out, N * sizeof(double), cudaMemcpyDeviceToHost, s));
      if (rho_g_basis_out) {
        if ((r = density_to_g(h, st->rho_out)) != kOk) return r;
        std::vector<int> gf(h.n_pw);
        std::vector<double2> full(N);
        PW_CUDA_TRY(cudaMemcpyAsync(full.data(), st->cg, N * sizeof(double2), cudaMemcpyDeviceToHost, s));
        PW_CUDA_TRY(cudaMemcpyAsync(gf.data(), h.g.g_to_fft, h.n_pw * sizeof(int), cudaMemcpyDeviceToHost, s));
        PW_CUDA_TRY(cudaStreamSynchronize(s));
        for (int i = 0; i < h.n_pw; ++i) {
          rho_g_basis_out[2 * i] = full[gf[i]].x;
          rho_g_basis_out[2 * i + 1] = full[gf[i]].y;
        }
      }
      PW_CUDA_TRY(cudaStreamSynchronize(s));
      return conv ? kOk : fail(kNotConverged, "SCF did not converge within max_iter");
    }
    if ((r = mix(h, p)) != kOk) return r;
  }
  return fail(kNotConverged, "SCF did not converge within max_iter");
}

// ---------------------------------------------------------------------------
// component entry points (host arrays) for parity tests
// ---------------------------------------------------------------------------

Status eigensolve_k(Handle& h, int spin, int ik, int n_bands, double tol, int max_iter, const double* psi_in,
                    double* evals, double* psi_out, int* iters, double* max_res, int precision) {
  if (ik < 0 || ik >= h.n_k || spin < 0 || spin >= h.nspin) return fail(kInvalid, "eigensolve: index out of range");
  if (n_bands < 1 || n_bands > h.n_pw) return fail(kInvalid, "eigensolve: n_bands out of range");
  const int extra = std::max(2, n_bands / 8);
  const int nd = (int)std::min<long>(n_bands + extra, h.n_pw);
  Status r = ensure_state(h, n_bands, nd, 1);
  if (r != kOk) return r;
  ScfState* st = h.scf;
  EigVecs& k = st->ks[(size_t)spin * h.n_k + ik];
  const long n = h.n_pw;
  double vsum = 0.0;
  if ((r = reduce_host(h, h.veff_r[spin], nullptr, h.g.N, 0, vsum)) != kOk) return r;
  const double v0 = vsum / (double)h.g.N;
  k.init = false;
  if (psi_in) {
    // warm start: given n_bands columns, remaining columns from the cold-start recipe
    EigStats e0;
    if ((r = lobpcg(h, st->ew, k, spin, ik, v0, 1e300, 0, n_bands, precision, e0)) != kOk) return r;
    PW_CUDA_TRY(cudaMemcpyAsync(k.V, psi_in, n * n_bands * sizeof(double2), cudaMemcpyHostToDevice, h.stream));
  }
  EigStats es;
  if ((r = lobpcg(h, st->ew, k, spin, ik, v0, tol, max_iter, n_bands, precision, es)) != kOk) return r;
  const int its = es.iters;
  const double mres = es.max_res;
  for (int b = 0; b < n_bands; ++b) evals[b] = k.evals[b];
  if (psi_out)
    PW_CUDA_TRY(cudaMemcpyAsync(psi_out, k.V, n * n_bands * sizeof(double2), cudaMemcpyDeviceToHost, h.stream));
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
  if (iters) *iters = its;
  if (max_res) *max_res = mres;
  if (mres >= tol) return fail(kNotConverged, "eigensolve: residual tolerance not reached within max_iter");
  return kOk;
}

Status density_from_host(Handle& h, int n_bands, const double* occ, const double* psi_all, double* rho_out) {
  if (n_bands < 1 || n_bands > h.n_pw) return fail(kInvalid, "density: n_bands out of range");
  Status r = ensure_state(h, n_bands, n_bands, 1);
  if (r != kOk) return r;
  ScfState* st = h.scf;
  const long n = h.n_pw;
  std::vector<std::vector<double>> oc(h.n_k);
  std::vector<double> wk(h.n_k);
  for (int ik = 0; ik < h.n_k; ++ik) {
    wk[ik] = h.kp[ik].weight;
    oc[ik].assign(occ + (size_t)ik * n_bands, occ + (size_t)(ik + 1) * n_bands);
    PW_CUDA_TRY(cudaMemcpyAsync(st->ks[ik].V, psi_all + (size_t)ik * n * n_bands * 2, n * n_bands * sizeof(double2),
                                cudaMemcpyHostToDevice, h.stream));
  }
  if ((r = build_density(h, oc, wk, 0, st->rho_out)) != kOk) return r;
  PW_CUDA_TRY(cudaMemcpyAsync(rho_out, st->rho_out, h.g.N * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
  return kOk;
}

Status symmetrize_host(Handle& h, double* rho) {
  Status r = ensure_state(h, 1, 1, 1);
  if (r != kOk) return r;
  ScfState* st = h.scf;
  const long N = h.g.N;
  PW_CUDA_TRY(cudaMemcpyAsync(st->rtmp, rho, N * sizeof(double), cudaMemcpyHostToDevice, h.stream));
  if ((r = symmetrize(h, st->rtmp)) != kOk) return r;
  PW_CUDA_TRY(cudaMemcpyAsync(rho, st->rtmp, N * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
  return kOk;
}

Status potentials_host(Handle& h, const double* rho, double* veff_g, double* energies) {
  Status r = ensure_state(h, 1, 1, 1);
  if (r != kOk) return r;
  ScfState* st = h.scf;
  const long N = h.g.N;
  PW_CUDA_TRY(cudaMemcpyAsync(st->rtmp, rho, N * sizeof(double), cudaMemcpyHostToDevice, h.stream));
  PotEnergies e;
  if ((r = potentials(h, st->rtmp, true, e)) != kOk) return r;
  if (veff_g) PW_CUDA_TRY(cudaMemcpyAsync(veff_g, st->cg2, N * sizeof(double2), cudaMemcpyDeviceToHost, h.stream));
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
  if (energies) {
    energies[0] = e.e_hartree;
    energies[1] = e.e_xc;
    energies[2] = e.e_vxc;
  }
  return kOk;
}

}  // namespace pwgpu
