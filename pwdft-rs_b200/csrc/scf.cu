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
#include <atomic>
#include <cmath>
#include <cstdio>
#include <memory>
#include <random>
#include <thread>
#include <vector>

#include "handle.hpp"
#include "linalg.hpp"
#include "lobpcg.hpp"
#include "scf.hpp"

namespace pwgpu {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kHaToEv = 27.211386245988;
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

// Kerker weights P(G) = G^2 / (G^2 + q^2), P = 0 at G^2 < g2_zero (kerker.rs:18-35)
__global__ void k_kerker_weights(const double* __restrict__ g2, long n, double q2, double g2_zero,
                                 double* __restrict__ w) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w[i] = g2[i] < g2_zero ? 0.0 : g2[i] / (g2[i] + q2);
}

__global__ void k_real_part(const double2* __restrict__ c, double* __restrict__ r, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = c[i].x;
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

// All DIIS inner products of one mixing step in one launch.  With
// dr_i = res[i] - res[mm] (i < mm), blockIdx.y = i * (mm + 1) + jj:
// jj = 0 gives dot(dr_i, res[mm]), jj = j + 1 (j <= i) gives dot(dr_i, dr_j);
// partials[blockIdx.y * gridDim.x + blockIdx.x] (fixed summation order).
// With diff = 0 the same slots hold plain products: <v_i, v_j> and
// <v_i, v_mm> (Broyden's <df_i|df_j> and <df_i|R>).
__global__ void k_dr_dots(const double* const* __restrict__ res, int mm, long n, int diff,
                          double* __restrict__ partials) {
  __shared__ double sh[32];
  const int i = blockIdx.y / (mm + 1), jj = blockIdx.y % (mm + 1), j = jj - 1;
  if (j > i) {
    if (threadIdx.x == 0) partials[(long)blockIdx.y * gridDim.x + blockIdx.x] = 0.0;
    return;
  }
  const double* ri = res[i];
  const double* rl = res[mm];
  const double* rj = j >= 0 ? res[j] : nullptr;
  double acc = 0.0;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const double a = diff ? ri[t] - rl[t] : ri[t];
    const double b = rj ? (diff ? rj[t] - rl[t] : rj[t]) : rl[t];
    acc += a * b;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[(long)blockIdx.y * gridDim.x + blockIdx.x] = acc;
}

// Broyden update (broyden.rs:228-245): next = (in - sum_k g_k dv_k) +
// beta (r - sum_k g_k df_k); next may alias in
__global__ void k_broyden_combine(const double* __restrict__ in, const double* __restrict__ r,
                                  const double* const* __restrict__ dv, const double* const* __restrict__ df,
                                  const double* __restrict__ g, int m, double beta, long n, double* next) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double cv = 0.0, cf = 0.0;
  for (int k = 0; k < m; ++k) {
    cv += g[k] * dv[k][i];
    cf += g[k] * df[k][i];
  }
  next[i] = fma(beta, r[i] - cf, in[i] - cv);
}

// sums[c] = sum of the nblk partials of slot c (fixed order)
__global__ void k_slot_sums(const double* __restrict__ partials, int nblk, int nslots, double* __restrict__ sums) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nslots) return;
  double acc = 0.0;
  for (int b = 0; b < nblk; ++b) acc += partials[(long)c * nblk + b];
  sums[c] = acc;
}

// LSDA (xc.rs:374-596): von Barth-Hedin spin interpolation of PZ81 and
// spin-scaled Slater exchange on rho_sigma + core/2 (add_core_density
// clamp when a core is present).  Writes V_xc per channel; partial sums of
// rho_xc_total * exc (rho_xc_total = max(up + down + core, 0)) and of
// up * v_up + down * v_down (driver_spin.rs:572-610).
__global__ void k_lsda(const double* __restrict__ up, const double* __restrict__ dn, const double* __restrict__ core,
                       long n, double* __restrict__ vup_out, double* __restrict__ vdn_out,
                       double* __restrict__ part_exc, double* __restrict__ part_vxc) {
  __shared__ double sh[32];
  double a1 = 0.0, a2 = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double u = up[i], d = dn[i];
    double ru = u, rd = d, rt = u + d;
    if (core) {
      const double c = core[i];
      ru = fmax(u + 0.5 * c, 0.0);
      rd = fmax(d + 0.5 * c, 0.0);
      rt = fmax(u + d + c, 0.0);
    }
    const double rho = ru + rd;
    double exc = 0.0, vu = 0.0, vd = 0.0;
    if (rho >= kRhoFloor) {
      const double rub = ru * kBohr3ToAng3, rdb = rd * kBohr3ToAng3, rb = rho * kBohr3ToAng3;
      const double exu = rub > kRhoFloor ? -0.75 * cbrt(6.0 * rub / kPi) : 0.0;
      const double exd = rdb > kRhoFloor ? -0.75 * cbrt(6.0 * rdb / kPi) : 0.0;
      const double ex = fma(rub, exu, rdb * exd) / rb;
      const double rs = cbrt(3.0 / (4.0 * kPi * rb));
      const double zeta = fmin(fmax((ru - rd) / rho, -1.0), 1.0);
      double ecu, vcu, ecp, vcp;
      pz_rs(rs, false, ecu, vcu);
      pz_rs(rs, true, ecp, vcp);
      const double fden = fma(cbrt(2.0), 2.0, -2.0);
      const double op = fmax(1.0 + zeta, 0.0), om = fmax(1.0 - zeta, 0.0);
      const double cop = cbrt(op), com = cbrt(om);
      const double fz = (cop * op + com * om - 2.0) / fden;
      const double dfz = (4.0 / 3.0) * (cop - com) / fden;
      const double ec = ecu + fz * (ecp - ecu);
      const double vrs = vcu + fz * (vcp - vcu);
      const double dz = dfz * (ecp - ecu);
      exc = (ex + ec) * kHaToEv;
      vu = ((4.0 / 3.0) * exu + fma(1.0 - zeta, dz, vrs)) * kHaToEv;
      vd = ((4.0 / 3.0) * exd + fma(1.0 + zeta, -dz, vrs)) * kHaToEv;
    }
    vup_out[i] = vu;
    vdn_out[i] = vd;
    a1 += rt * exc;
    a2 += u * vu + d * vd;
  }
  a1 = block_sum(a1, sh);
  a2 = block_sum(a2, sh);
  if (threadIdx.x == 0) {
    part_exc[blockIdx.x] = a1;
    part_vxc[blockIdx.x] = a2;
  }
}

// out = a + s * b
__global__ void k_axpy_to(const double* __restrict__ a, const double* __restrict__ b, double s, double* __restrict__ out,
                          long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + s * b[i];
}

// up = (t + m)/2, dn = (t - m)/2 (driver_spin.rs:817-826)
__global__ void k_unmix_spin(const double* __restrict__ t, const double* __restrict__ m, double* __restrict__ up,
                             double* __restrict__ dn, long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  up[i] = 0.5 * (t[i] + m[i]);
  dn[i] = 0.5 * (t[i] - m[i]);
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

// Concurrent slot for the per-(spin, k) eigensolves (the reference runs them
// in parallel over k with rayon, driver_spin.rs:356-384): a shallow view of
// the handle (shared grid maps, projectors and potentials, all read-only
// during the eigensolve phase) with its own stream, BLAS/solver handles,
// H|psi> scratch and eigensolver workspace.
struct Lane {
  Handle view;
  EigWork ew;
};

constexpr int kMaxLanes = 8;

static void release_lane(Lane& L) {
  Handle& v = L.view;
  eig_work_release(L.ew);
  release_nl_mixed(v);
  release_gamma_scratch(v);
  auto f = [](void* p) { if (p) cudaFree(p); };
  f(v.work_a); f(v.work_b); f(v.nl_p); f(v.nl_q); f(v.solver_work); f(v.solver_info);
  if (v.solver) cusolverDnDestroy(v.solver);
  if (v.blas) cublasDestroy(v.blas);
  if (v.stream) cudaStreamDestroy(v.stream);
  v.work_a = v.work_b = nullptr;
  v.nl_p = v.nl_q = nullptr;
  v.solver_work = nullptr;
  v.solver_info = nullptr;
  v.solver = nullptr;
  v.blas = nullptr;
  v.stream = nullptr;
}

static Status create_lane(Handle& h, Lane& L, int nd, int nlanes) {
  L.view = h;  // pointers to the handle's read-only data; lane-owned members reset below
  Handle& v = L.view;
  v.stream = nullptr;
  v.blas = nullptr;
  v.solver = nullptr;
  v.solver_work = nullptr;
  v.solver_work_len = 0;
  v.solver_info = nullptr;
  v.work_a = v.work_b = nullptr;
  v.nl_p = v.nl_q = nullptr;
  v.nl_cap = 0;
  v.nlm = nullptr;
  v.nlm_real = nullptr;
  v.scf = nullptr;
  v.tmp_grid = nullptr;
  v.gam_c1 = v.gam_c2 = nullptr;
  v.gam_ccap = 0;
  v.gam_p = v.gam_q = nullptr;
  v.gam_pcap = 0;
  // lanes share the L2: each keeps a proportionally smaller band chunk
  v.chunk = std::max(4, h.chunk / nlanes);
  PW_CUDA_TRY(cudaStreamCreateWithFlags(&v.stream, cudaStreamNonBlocking));
  if (cublasCreate(&v.blas) != CUBLAS_STATUS_SUCCESS) return fail(kCuda, "cublasCreate failed (lane)");
  cublasSetStream(v.blas, v.stream);
  const GridMaps& g = h.g;
  cudaError_t e = cudaMalloc(&v.work_a, (size_t)v.chunk * g.ncol * g.d[2] * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc(&v.work_b, (size_t)v.chunk * g.Xp * g.d[1] * g.d[2] * sizeof(double2));
  if (e != cudaSuccess) return fail(kOom, std::string("cudaMalloc (lane): ") + cudaGetErrorString(e));
  return eig_work_alloc(L.ew, h.n_pw, nd);
}

// Anderson history of one mixed channel (anderson.rs:170-266): inputs and
// (preconditioned) residuals, oldest first.
// (Broyden: hin / hres hold the input and residual differences dv, df, and
// prev_in / prev_res the previous step's input and residual.)
struct MixHistory {
  std::vector<double*> hin, hres;
  int count = 0;
  int iteration = 0;            // steps taken (Periodic Pulay's period counter)
  bool has_prev = false;        // Broyden: prev_in / prev_res hold a step
  double *prev_in = nullptr, *prev_res = nullptr, *rcur = nullptr;
  double** dev_ptrs = nullptr;  // 2 * ndim + 2
  double* dev_coef = nullptr;   // ndim
};

// Mixer::new (mixing/mod.rs:245-276) kinds and options of one channel
struct MixConfig {
  int kind = 0;        // 0 Anderson, 1 modified Broyden, 2 Periodic Pulay
  bool kerker = false;
  int period = 3;
  double beta = 0.3;
};

struct ScfState {
  int nd = 0, nb = 0, nspin = 1;
  std::vector<EigVecs> ks;  // per (spin, k)
  EigWork ew;
  double *partials = nullptr, *scal = nullptr, *fw = nullptr, *mix_partials = nullptr, *mix_sums = nullptr;
  double* band_terms = nullptr;  // 2 nd: per-band kinetic and nonlocal expectations
  double *rho_in = nullptr, *rho_out = nullptr, *exc = nullptr, *vxc = nullptr, *rtmp = nullptr;
  double2 *cg = nullptr, *cg2 = nullptr, *vh = nullptr;
  double* kerker_w = nullptr;
  // nspin = 2: down-channel densities and V_xc, (total, magnetisation) in/out
  double *rho_in_dn = nullptr, *rho_out_dn = nullptr, *vxc_dn = nullptr;
  double *t_in = nullptr, *t_out = nullptr, *m_in = nullptr, *m_out = nullptr;
  MixHistory mixh[2];  // 0: rho (or rho_up + rho_down), 1: rho_up - rho_down
  int mix_cap = 0;     // history depth mix_partials / mix_sums are sized for
  std::vector<std::unique_ptr<Lane>> lanes;  // empty: one (spin, k) block at a time
};

template <typename T> static Status salloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) return fail(kOom, std::string("cudaMalloc (scf): ") + cudaGetErrorString(e));
  return kOk;
}

static void release_history(MixHistory& mh);

void release_scf(Handle& h) {
  ScfState* st = h.scf;
  if (!st) return;
  auto f = [](void* p) { if (p) cudaFree(p); };
  for (auto& k : st->ks) eig_vecs_release(k);
  eig_work_release(st->ew);
  f(st->partials); f(st->scal); f(st->fw); f(st->band_terms);
  f(st->rho_in); f(st->rho_out); f(st->exc); f(st->vxc); f(st->rtmp);
  f(st->cg); f(st->cg2); f(st->vh); f(st->kerker_w); f(st->mix_partials); f(st->mix_sums);
  f(st->rho_in_dn); f(st->rho_out_dn); f(st->vxc_dn); f(st->t_in); f(st->t_out); f(st->m_in); f(st->m_out);
  for (auto& mh : st->mixh) release_history(mh);
  for (auto& L : st->lanes) release_lane(*L);
  delete st;
  h.scf = nullptr;
}

static void release_history(MixHistory& mh) {
  auto f = [](void* p) { if (p) cudaFree(p); };
  for (double* p : mh.hin) f(p);
  for (double* p : mh.hres) f(p);
  f(mh.dev_ptrs);
  f(mh.dev_coef);
  f(mh.prev_in);
  f(mh.prev_res);
  f(mh.rcur);
  mh = MixHistory();
}

static Status alloc_history(MixHistory& mh, long N, int ndim) {
  release_history(mh);
  Status s;
  mh.hin.assign(ndim, nullptr);
  mh.hres.assign(ndim, nullptr);
  mh.count = 0;
  for (int i = 0; i < ndim; ++i) {
    if ((s = salloc(&mh.hin[i], (size_t)N)) != kOk) return s;
    if ((s = salloc(&mh.hres[i], (size_t)N)) != kOk) return s;
  }
  if ((s = salloc(&mh.dev_ptrs, (size_t)2 * std::max(ndim, 1) + 2)) != kOk) return s;
  if ((s = salloc(&mh.dev_coef, (size_t)std::max(ndim, 1))) != kOk) return s;
  for (double** p : {&mh.prev_in, &mh.prev_res, &mh.rcur})
    if ((s = salloc(p, (size_t)N)) != kOk) return s;
  return kOk;
}

constexpr int kMixBlocks = 128;  // partial sums per DIIS inner product

static Status ensure_state(Handle& h, int nb, int nd, int ndim) {
  if (h.scf && h.scf->nd == nd && h.scf->nb == nb && (int)h.scf->mixh[0].hin.size() == ndim) return kOk;
  release_scf(h);
  ScfState* st = new ScfState();
  h.scf = st;
  st->nd = nd;
  st->nb = nb;
  st->nspin = h.nspin;
  const long n = h.n_pw, N = h.g.N;
  Status s;
  st->ks.resize((size_t)h.nspin * h.n_k);
  for (auto& k : st->ks)
    if ((s = eig_vecs_alloc(k, n, nd)) != kOk) return s;
  if ((s = eig_work_alloc(st->ew, n, nd)) != kOk) return s;
  if ((s = salloc(&st->partials, (size_t)kRedBlocks * 4)) != kOk) return s;
  if ((s = salloc(&st->scal, 16)) != kOk) return s;
  if ((s = salloc(&st->fw, (size_t)nd)) != kOk) return s;
  if ((s = salloc(&st->band_terms, 2 * (size_t)nd)) != kOk) return s;
  if ((s = salloc(&st->rho_in, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->rho_out, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->exc, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->vxc, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->rtmp, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->cg, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->cg2, (size_t)N)) != kOk) return s;
  if ((s = salloc(&st->vh, (size_t)N)) != kOk) return s;
  const size_t nslots = (size_t)std::max(ndim, 1) * (std::max(ndim, 1) + 1);
  if ((s = salloc(&st->mix_partials, nslots * kMixBlocks)) != kOk) return s;
  if ((s = salloc(&st->mix_sums, nslots)) != kOk) return s;
  st->mix_cap = std::max(ndim, 1);
  if ((s = alloc_history(st->mixh[0], N, ndim)) != kOk) return s;
  if (h.nspin == 2) {
    for (double** p : {&st->rho_in_dn, &st->rho_out_dn, &st->vxc_dn, &st->t_in, &st->t_out, &st->m_in, &st->m_out})
      if ((s = salloc(p, (size_t)N)) != kOk) return s;
    if ((s = alloc_history(st->mixh[1], N, ndim)) != kOk) return s;
  }
  const int nitems = h.nspin * h.n_k;
  const int nl = std::min(nitems, h.lanes > 0 ? h.lanes : kMaxLanes);
  if (nl > 1) {
    for (int i = 0; i < nl; ++i) {
      st->lanes.emplace_back(new Lane());
      if ((s = create_lane(h, *st->lanes.back(), nd, nl)) != kOk) return s;
    }
  }
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
    if ((r = veff_zmajor(h, 0, s)) != kOk) return r;
  }
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// E_local = int rho V_loc dV over the given density channels, V_loc(r) the
// unnormalised inverse FFT of V_loc(G) with its G = 0 term (driver.rs:664-668,
// local_pp_energy_grid energy.rs:439-445); uses cg2 and rtmp as scratch.
static Status local_energy(Handle& h, double* const* rho, int nrho, double& e) {
  ScfState* st = h.scf;
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  PW_CUDA_TRY(cudaMemcpyAsync(st->cg2, h.v_local_g, N * sizeof(double2), cudaMemcpyDeviceToDevice, s));
  Status r = fft3d_full(h, st->cg2, +1, s);
  if (r != kOk) return r;
  k_real_part<<<blocks_for(N), 256, 0, s>>>(st->cg2, st->rtmp, N); count_launch();
  e = 0.0;
  for (int c = 0; c < nrho; ++c) {
    double part = 0.0;
    if ((r = reduce_host(h, rho[c], st->rtmp, N, 1, part)) != kOk) return r;
    e += part;
  }
  e *= h.omega / (double)N;
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

Status occupations_host(int n_sets, int nb, const double* ev, const double* w, double n_electrons, double sigma,
                        int scheme, double spin_factor, bool find_fermi, double* fermi_energy, double* occ,
                        double* ts) {
  std::vector<std::vector<double>> e((size_t)n_sets);
  std::vector<double> wk(w, w + n_sets);
  for (int s = 0; s < n_sets; ++s) e[s].assign(ev + (size_t)s * nb, ev + (size_t)(s + 1) * nb);
  const double ef = find_fermi ? fermi_level(e, wk, n_electrons, sigma, scheme, spin_factor) : *fermi_energy;
  if (occ)
    for (int s = 0; s < n_sets; ++s)
      for (int b = 0; b < nb; ++b) occ[(size_t)s * nb + b] = spin_factor * occ01(scheme, e[s][b], ef, sigma);
  if (ts) *ts = entropy_ts(e, wk, ef, sigma, scheme, spin_factor);
  *fermi_energy = ef;
  return kOk;
}

// partial-pivot LU solve with the 1e-15 singular-pivot fallback (linalg.rs:24-50)
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

// mixing_mode: 0 Anderson, 1 Anderson + Kerker, 2 Broyden, 3 Broyden +
// Kerker, 4 Periodic Pulay, 5 Periodic Pulay + Kerker (MixingMode,
// mixing/mod.rs:186-223)
static MixConfig mix_config(int mode, int period, double beta) {
  MixConfig c;
  c.kind = mode / 2;
  c.kerker = (mode % 2) == 1;
  c.period = std::max(1, period);
  c.beta = beta;
  return c;
}

static void reset_history(MixHistory& mh) {
  mh.count = 0;
  mh.iteration = 0;
  mh.has_prev = false;
}

// Kerker-preconditioned residual (kerker.rs:18-35) out - in into res.
static Status residual_into(Handle& h, const double* in, const double* out, double* res, bool kerker) {
  ScfState* st = h.scf;
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  k_sub<<<blocks_for(N), 256, 0, s>>>(out, in, res, N); count_launch();
  if (kerker && st->kerker_w) {
    k_real_to_cplx<<<blocks_for(N), 256, 0, s>>>(res, st->cg, N); count_launch();
    Status r = fft3d_full(h, st->cg, -1, s);
    if (r != kOk) return r;
    k_mul_real_weights<<<blocks_for(N), 256, 0, s>>>(st->cg, st->kerker_w, N); count_launch();
    if ((r = fft3d_full(h, st->cg, +1, s)) != kOk) return r;
    k_cplx_real_scaled<<<blocks_for(N), 256, 0, s>>>(st->cg, res, 1.0 / (double)N, N); count_launch();
  }
  return kOk;
}

// All products of one step in one launch and one host sync: slots
// i * (mm + 1) + jj of st->mix_sums (see k_dr_dots); ptrs = mm + 1 vectors.
static Status dot_table(Handle& h, double* const* ptrs_dev, int mm, int diff, std::vector<double>& sums) {
  ScfState* st = h.scf;
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  const int nslots = mm * (mm + 1);
  const unsigned nbk = (unsigned)std::min<long>(kMixBlocks, blocks_for(N));
  k_dr_dots<<<dim3(nbk, nslots), 256, 0, s>>>(ptrs_dev, mm, N, diff, st->mix_partials); count_launch();
  k_slot_sums<<<blocks_for(nslots), 256, 0, s>>>(st->mix_partials, (int)nbk, nslots, st->mix_sums); count_launch();
  sums.resize(nslots);
  PW_CUDA_TRY(cudaMemcpyAsync(sums.data(), st->mix_sums, nslots * sizeof(double), cudaMemcpyDeviceToHost, s));
  PW_CUDA_TRY(cudaStreamSynchronize(s));
  return kOk;
}

// Anderson history push (AndersonMixer::push_history, anderson.rs:170-190)
static Status push_anderson(Handle& h, MixHistory& mh, const double* in, const double* out, bool kerker) {
  const long N = h.g.N;
  const int ndim = (int)mh.hin.size();
  // rotate history: slot order oldest .. newest kept in vectors
  if (mh.count == ndim) {
    std::rotate(mh.hin.begin(), mh.hin.begin() + 1, mh.hin.end());
    std::rotate(mh.hres.begin(), mh.hres.begin() + 1, mh.hres.end());
    --mh.count;
  }
  const int slot = mh.count;
  Status r = residual_into(h, in, out, mh.hres[slot], kerker);
  if (r != kOk) return r;
  PW_CUDA_TRY(cudaMemcpyAsync(mh.hin[slot], in, N * sizeof(double), cudaMemcpyDeviceToDevice, h.stream));
  mh.count++;
  return kOk;
}

// next = sum_i c_i (in_i + beta res_i) over the Anderson history; DIIS
// coefficients from the residual differences when diis (anderson.rs:192-266),
// the newest entry alone otherwise.
static Status combine_anderson(Handle& h, MixHistory& mh, double beta, bool diis, double* next) {
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  const int m = mh.count;
  std::vector<double*> ptrs(2 * m);
  for (int j = 0; j < m; ++j) { ptrs[j] = mh.hin[j]; ptrs[m + j] = mh.hres[j]; }
  PW_CUDA_TRY(cudaMemcpyAsync(mh.dev_ptrs, ptrs.data(), 2 * m * sizeof(double*), cudaMemcpyHostToDevice, s));
  std::vector<double> coef(m, 0.0);
  if (m < 2 || !diis) {
    coef[m - 1] = 1.0;
  } else {
    const int mm = m - 1;
    std::vector<double> sums;
    Status r = dot_table(h, mh.dev_ptrs + m, mm, 1, sums);
    if (r != kOk) return r;
    std::vector<double> a((size_t)mm * mm), b(mm);
    for (int i = 0; i < mm; ++i) {
      b[i] = -sums[(size_t)i * (mm + 1)];
      for (int j = 0; j <= i; ++j) {
        const double v = sums[(size_t)i * (mm + 1) + j + 1];
        a[(size_t)i * mm + j] = v;
        a[(size_t)j * mm + i] = v;
      }
    }
    std::vector<double> al = solve_small(a, b, mm);
    double sum = 0.0;
    for (int i = 0; i < mm; ++i) { coef[i] = al[i]; sum += al[i]; }
    coef[mm] = 1.0 - sum;
  }
  PW_CUDA_TRY(cudaMemcpyAsync(mh.dev_coef, coef.data(), m * sizeof(double), cudaMemcpyHostToDevice, s));
  k_mix_combine<<<blocks_for(N), 256, 0, s>>>(mh.dev_ptrs, mh.dev_ptrs + m, mh.dev_coef, m, beta, N, next);
  count_launch();
  PW_CUDA_TRY(cudaStreamSynchronize(s));
  return kOk;
}

// Modified Broyden step (BroydenMixer::mix, broyden.rs:140-245).
static Status mix_broyden(Handle& h, MixHistory& mh, const double* in, const double* out, double* next, double beta,
                          bool kerker) {
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  const int ndim = (int)mh.hin.size();
  Status r = residual_into(h, in, out, mh.rcur, kerker);
  if (r != kOk) return r;
  if (mh.has_prev) {
    if (mh.count == ndim) {
      std::rotate(mh.hin.begin(), mh.hin.begin() + 1, mh.hin.end());
      std::rotate(mh.hres.begin(), mh.hres.begin() + 1, mh.hres.end());
      --mh.count;
    }
    const int slot = mh.count++;
    k_sub<<<blocks_for(N), 256, 0, s>>>(in, mh.prev_in, mh.hin[slot], N); count_launch();      // dv
    k_sub<<<blocks_for(N), 256, 0, s>>>(mh.rcur, mh.prev_res, mh.hres[slot], N); count_launch();  // df
  }
  PW_CUDA_TRY(cudaMemcpyAsync(mh.prev_in, in, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  PW_CUDA_TRY(cudaMemcpyAsync(mh.prev_res, mh.rcur, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  mh.has_prev = true;
  const int m = mh.count;
  std::vector<double> g(std::max(m, 1), 0.0);
  // pointers: dv_0..dv_{m-1}, df_0..df_{m-1}, R
  std::vector<double*> ptrs(2 * m + 1);
  for (int j = 0; j < m; ++j) { ptrs[j] = mh.hin[j]; ptrs[m + j] = mh.hres[j]; }
  ptrs[2 * m] = mh.rcur;
  PW_CUDA_TRY(cudaMemcpyAsync(mh.dev_ptrs, ptrs.data(), ptrs.size() * sizeof(double*), cudaMemcpyHostToDevice, s));
  if (m > 0) {
    std::vector<double> sums;
    if ((r = dot_table(h, mh.dev_ptrs + m, m, 0, sums)) != kOk) return r;
    std::vector<double> a((size_t)m * m), w(m);
    for (int i = 0; i < m; ++i) {
      w[i] = sums[(size_t)i * (m + 1)];
      for (int j = 0; j <= i; ++j) {
        const double v = sums[(size_t)i * (m + 1) + j + 1];
        a[(size_t)i * m + j] = v;
        a[(size_t)j * m + i] = v;
      }
    }
    g = solve_small(a, w, m);
  }
  PW_CUDA_TRY(cudaMemcpyAsync(mh.dev_coef, g.data(), std::max(m, 1) * sizeof(double), cudaMemcpyHostToDevice, s));
  k_broyden_combine<<<blocks_for(N), 256, 0, s>>>(in, mh.rcur, mh.dev_ptrs, mh.dev_ptrs + m, mh.dev_coef, m, beta, N,
                                                  next);
  count_launch();
  PW_CUDA_TRY(cudaStreamSynchronize(s));
  return kOk;
}

// One mixing step of one channel (Mixer::mix, mixing/mod.rs:281-287):
// Anderson (anderson.rs:170-266), modified Broyden (broyden.rs:140-245) or
// Periodic Pulay (anderson.rs:353-372: DIIS every period-th step once the
// history holds two entries, linear mixing of the newest entry otherwise);
// Kerker residual preconditioning (kerker.rs:18-35) when cfg.kerker.
// `next` may alias `in`.
static Status mix_channel(Handle& h, MixHistory& mh, const MixConfig& cfg, const double* in, const double* out,
                          double* next) {
  mh.iteration++;
  if (cfg.kind == 1) return mix_broyden(h, mh, in, out, next, cfg.beta, cfg.kerker);
  Status r = push_anderson(h, mh, in, out, cfg.kerker);
  if (r != kOk) return r;
  const bool diis = cfg.kind == 0 || (mh.iteration % std::max(cfg.period, 1) == 0);
  return combine_anderson(h, mh, cfg.beta, diis, next);
}

// Density of all k-points of one spin channel (density.rs:41-111): rho =
// sum renormalised to n_target electrons, then symmetrised.
static Status build_density(Handle& h, const std::vector<std::vector<double>>& occ, const std::vector<double>& w,
                            int spin, double* rho, double n_target) {
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
    const double2* v = st->ks[(size_t)spin * h.n_k + ik].V;
    Status r;
    if (h.gam.on) {
      r = density_accumulate_real(h, reinterpret_cast<const double*>(v), n, fw, rho, s);
    } else {
      // pageable source: the copy has left fw when the call returns, and the
      // device buffer is reused in stream order
      PW_CUDA_TRY(cudaMemcpyAsync(st->fw, fw.data(), fw.size() * sizeof(double), cudaMemcpyHostToDevice, s));
      r = density_accumulate(h, v, n, (int)fw.size(), st->fw, rho, s);
    }
    if (r != kOk) return r;
  }
  double tot = 0.0;
  Status r = reduce_host(h, rho, nullptr, N, 0, tot);
  if (r != kOk) return r;
  const double integ = tot * (h.omega / (double)N);
  if (std::fabs(integ) > 1e-15) {
    k_scale_real<<<blocks_for(N), 256, 0, s>>>(rho, n_target / integ, N);
    count_launch();
  }
  return symmetrize(h, rho);
}

// Eigensolve of every (spin, k) block for the current potentials.  With
// lanes, host threads take blocks from a shared counter and run them on
// their lanes' streams; the potentials on the handle stream are complete
// before any lane starts.
static Status eigensolve_all(Handle& h, const double* v0, double tol, int max_it, int nb, int prec,
                             std::vector<EigStats>& stats) {
  ScfState* st = h.scf;
  const int nk = h.n_k, nitems = h.nspin * nk;
  Status r;
  if (st->lanes.empty()) {
    for (int c = 0; c < nitems; ++c)
      if ((r = lobpcg(h, st->ew, st->ks[c], c / nk, c % nk, v0[c / nk], tol, max_it, nb, prec, stats[c])) != kOk)
        return r;
    return kOk;
  }
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
  const int nl = (int)st->lanes.size();
  std::atomic<int> next{0};
  std::vector<int> codes(nl, kOk);
  std::vector<std::string> msgs(nl);
  auto worker = [&](int li) {
    if (cudaSetDevice(h.device) != cudaSuccess) {
      codes[li] = kCuda;
      msgs[li] = "cudaSetDevice failed (lane)";
      next.store(nitems);
      return;
    }
    Lane& L = *st->lanes[li];
    for (;;) {
      const int c = next.fetch_add(1);
      if (c >= nitems) break;
      const Status rc = lobpcg(L.view, L.ew, st->ks[c], c / nk, c % nk, v0[c / nk], tol, max_it, nb, prec, stats[c]);
      if (rc != kOk) {
        codes[li] = rc;
        msgs[li] = last_error_message();
        next.store(nitems);
        break;
      }
    }
  };
  std::vector<std::thread> th;
  th.reserve(nl);
  for (int li = 0; li < nl; ++li) th.emplace_back(worker, li);
  for (auto& t : th) t.join();
  for (int li = 0; li < nl; ++li)
    if (codes[li] != kOk) return fail(codes[li], msgs[li]);
  return kOk;
}

// Kerker weights P(G) = G^2/(G^2 + q^2), P(0) = 0 (kerker.rs:18-49); q_tf
// <= 0 selects the Thomas-Fermi estimate (auto_q_tf_squared, kerker.rs:41-49).
static Status set_kerker(Handle& h, bool on, double q_tf) {
  ScfState* st = h.scf;
  const long N = h.g.N;
  if (!on) {
    if (st->kerker_w) cudaFree(st->kerker_w);
    st->kerker_w = nullptr;
    return kOk;
  }
  double q2 = q_tf * q_tf;
  if (q_tf <= 0.0) {
    const double rb = h.n_electrons / h.omega * kBohr3ToAng3;
    q2 = 4.0 * std::cbrt(3.0 * kPi * kPi * rb) / kPi / (kBohrToAng * kBohrToAng);
  }
  Status r;
  if (!st->kerker_w && (r = salloc(&st->kerker_w, (size_t)N)) != kOk) return r;
  k_kerker_weights<<<blocks_for(N), 256, 0, h.stream>>>(h.g_squared, N, q2, kG2Zero, st->kerker_w); count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// Potentials of a spin-polarised density (driver_spin.rs:231-328): Hartree
// from rho_up + rho_down, LSDA V_xc per channel on rho_sigma + core/2,
// V_eff_sigma(r) into the handle's H|psi> arrays when set_hpsi; energies
// e_hartree, e_xc = int rho_xc_total eps_xc, e_vxc = int (up v_up + dn v_dn).
static Status potentials_spin(Handle& h, const double* up, const double* dn, bool set_hpsi, PotEnergies& e) {
  ScfState* st = h.scf;
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  k_axpy_to<<<blocks_for(N), 256, 0, s>>>(up, dn, 1.0, st->rtmp, N); count_launch();
  Status r = density_to_g(h, st->rtmp);
  if (r != kOk) return r;
  const double fpe2 = 4.0 * kPi * kE2;
  const unsigned nbk = (unsigned)std::min<long>(kRedBlocks, blocks_for(N));
  k_hartree<<<nbk, 256, 0, s>>>(st->cg, h.g_squared, N, st->vh, fpe2, st->partials); count_launch();
  double sh = 0.0;
  if ((r = final_sum_host(h, (int)nbk, sh)) != kOk) return r;
  e.e_hartree = sh * 0.5 * h.omega;
  k_lsda<<<nbk, 256, 0, s>>>(up, dn, h.rho_core_r, N, st->vxc, st->vxc_dn, st->partials, st->partials + kRedBlocks);
  count_launch();
  double sx = 0.0, sv = 0.0;
  if ((r = final_sum_host(h, (int)nbk, sx, 0)) != kOk) return r;
  if ((r = final_sum_host(h, (int)nbk, sv, 1)) != kOk) return r;
  const double dv = h.omega / (double)N;
  e.e_xc = sx * dv;
  e.e_vxc = sv * dv;
  if (!set_hpsi) return kOk;
  for (int sp = 0; sp < 2; ++sp) {
    k_real_to_cplx<<<blocks_for(N), 256, 0, s>>>(sp == 0 ? st->vxc : st->vxc_dn, st->cg2, N); count_launch();
    if ((r = fft3d_full(h, st->cg2, -1, s)) != kOk) return r;
    k_scale_cplx<<<blocks_for(N), 256, 0, s>>>(st->cg2, 1.0 / (double)N, N); count_launch();
    k_veff_g<<<blocks_for(N), 256, 0, s>>>(h.v_local_g, st->vh, st->cg2, st->cg2, N); count_launch();
    PW_CUDA_TRY(cudaMemcpyAsync(h.tmp_grid, st->cg2, N * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    if ((r = fft3d_full(h, h.tmp_grid, +1, s)) != kOk) return r;
    k_real_part_both<<<blocks_for(N), 256, 0, s>>>(h.tmp_grid, h.veff_r[sp], h.veff_r32[sp], N); count_launch();
    if ((r = veff_zmajor(h, sp, s)) != kOk) return r;
  }
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// Whole SCF loop: run_scf_unpolarized (driver.rs:353-735) for nspin = 1,
// run_scf_spin (driver_spin.rs:114-839) for nspin = 2.  Per iteration:
// potentials of rho_in, per-(spin, k) eigensolve, Fermi level and
// occupations, density per channel (renormalised, symmetrised), density
// change, energies from the output density, Anderson/Kerker mixing (CCMX
// on total and magnetisation for nspin = 2).
Status scf_run(Handle& h, const ScfParams& p, const double* rho_init, ScfResult& res, double* evals_out,
               double* rho_out_host, double* rho_g_basis_out) {
  if (p.n_bands < 1 || p.n_bands > h.n_pw) return fail(kInvalid, "scf_run: n_bands out of range");
  if (p.mixing_ndim < 1 || p.max_iter < 1) return fail(kInvalid, "scf_run: mixing_ndim and max_iter must be >= 1");
  PW_CUDA_TRY(cudaSetDevice(h.device));
  const int nb = p.n_bands, ns = h.nspin, nk = h.n_k;
  int extra = p.diag_extra_bands >= 0 ? p.diag_extra_bands : std::max(2, nb / 8);
  const int nd = (int)std::min<long>(nb + extra, h.n_pw);
  Status r = ensure_state(h, nb, nd, p.mixing_ndim);
  if (r != kOk) return r;
  ScfState* st = h.scf;
  for (auto& k : st->ks) k.init = false;
  for (auto& mh : st->mixh) reset_history(mh);
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  cublasSetStream(h.blas, s);
  const MixConfig mix_tot = mix_config(p.mixing_mode, p.mixing_period, p.mixing_beta);
  MixConfig mix_mag = mix_tot;
  mix_mag.kerker = false;  // Kerker acts on the charge channel only (driver_spin.rs:176-186)
  // q_TF: the user's value for Anderson + Kerker, the estimate for the others
  if ((r = set_kerker(h, mix_tot.kerker, mix_tot.kind == 0 ? p.kerker_q_tf : 0.0)) != kOk) return r;
  double* rin[2] = {st->rho_in, st->rho_in_dn};
  double* rout[2] = {st->rho_out, st->rho_out_dn};
  if (ns == 1) {
    PW_CUDA_TRY(cudaMemcpyAsync(st->rho_in, rho_init, N * sizeof(double), cudaMemcpyHostToDevice, s));
  } else {
    // split the start density by the atom-averaged starting magnetisation
    // (driver_spin.rs:160-167)
    std::vector<double> up(N), dn(N);
    const double m = p.starting_magnetization;
    for (long i = 0; i < N; ++i) {
      up[i] = rho_init[i] * (1.0 + m) / 2.0;
      dn[i] = rho_init[i] * (1.0 - m) / 2.0;
    }
    PW_CUDA_TRY(cudaMemcpy(st->rho_in, up.data(), N * sizeof(double), cudaMemcpyHostToDevice));
    PW_CUDA_TRY(cudaMemcpy(st->rho_in_dn, dn.data(), N * sizeof(double), cudaMemcpyHostToDevice));
  }
  std::vector<double> wk(nk), wk_all;
  for (int k = 0; k < nk; ++k) wk[k] = h.kp[k].weight;
  for (int sp = 0; sp < ns; ++sp) wk_all.insert(wk_all.end(), wk.begin(), wk.end());
  const double spin_factor = ns == 1 ? 2.0 : 1.0;
  bool have_prev = false;
  // mixed form: FP64 H|psi> from the first iteration whose input density rms
  // is below fp64_switch, or once the reduced-precision phase stops reducing
  // it (two iterations without a 30 % improvement on the best so far), for
  // the rest of the solve
  bool fp64_locked = p.precision != 1;
  double best_delta = INFINITY;
  int stalled = 0;
  double e_prev = 0.0, last_delta = INFINITY, max_res_all = 0.0;
  long happ = 0;
  const double dv = h.omega / (double)N;
  std::vector<std::vector<double>> ev((size_t)ns * nk), occ((size_t)ns * nk);
  for (int iter = 0; iter < p.max_iter; ++iter) {
    PotEnergies ein;
    if (ns == 1) r = potentials(h, st->rho_in, true, ein);
    else r = potentials_spin(h, st->rho_in, st->rho_in_dn, true, ein);
    if (r != kOk) return r;
    if (!fp64_locked && (last_delta < p.fp64_switch || stalled >= 2)) fp64_locked = true;
    const int prec = fp64_locked ? 0 : 1;
    // eigen-residual target of this step: the density error it leaves is far
    // below the SCF's own delta rho until the last iterations (measured on
    // the 64-atom cell: 0.1 drho capped at 1e-3 eV took 2.8 s, 3 drho capped
    // at 3e-2 eV 1.4 s, same converged energy within 3e-5 eV; the slope and
    // cap are parameters, since the best pair depends on the system)
    const double tol = p.single_step ? p.diag_tol
                                     : std::max(p.diag_tol, std::min(p.diag_tol_cap, p.diag_tol_per_drho *
                                                (std::isfinite(last_delta) ? last_delta : 1.0)));
    // preconditioner shift: V_eff(G = 0) = mean of V_eff(r)
    double v0[2] = {0.0, 0.0};
    for (int sp = 0; sp < ns; ++sp) {
      double vsum = 0.0;
      if ((r = reduce_host(h, h.veff_r[sp], nullptr, N, 0, vsum)) != kOk) return r;
      v0[sp] = vsum / (double)N;
    }
    const int max_it = (iter == 0 || p.single_step) ? 4 * p.diag_max_iter : p.diag_max_iter;
    std::vector<EigStats> stats((size_t)ns * nk);
    if ((r = eigensolve_all(h, v0, tol, max_it, nb, prec, stats)) != kOk) return r;
    max_res_all = 0.0;
    for (int c = 0; c < ns * nk; ++c) {
      happ += stats[c].happ;
      max_res_all = std::max(max_res_all, stats[c].max_res);
      ev[c].assign(st->ks[c].evals.begin(), st->ks[c].evals.begin() + nb);
    }
    // Fermi level: one over all channels, or one per channel at fixed
    // magnetisation (driver_spin.rs:400-466); the reported level is their mean
    double ef_sp[2];
    double ef;
    if (ns == 2 && p.fixed_magnetization) {
      const std::vector<std::vector<double>> ev_up(ev.begin(), ev.begin() + nk), ev_dn(ev.begin() + nk, ev.end());
      ef_sp[0] = fermi_level(ev_up, wk, 0.5 * (h.n_electrons + p.tot_magnetization), p.sigma, p.smearing, 1.0);
      ef_sp[1] = fermi_level(ev_dn, wk, (h.n_electrons - p.tot_magnetization) / 2.0, p.sigma, p.smearing, 1.0);
      ef = 0.5 * (ef_sp[0] + ef_sp[1]);
    } else {
      ef = fermi_level(ev, wk_all, h.n_electrons, p.sigma, p.smearing, spin_factor);
      ef_sp[0] = ef_sp[1] = ef;
    }
    double nel_sp[2] = {0.0, 0.0};
    for (int sp = 0; sp < ns; ++sp)
      for (int ik = 0; ik < nk; ++ik) {
        auto& o = occ[(size_t)sp * nk + ik];
        const auto& e = ev[(size_t)sp * nk + ik];
        o.resize(nb);
        for (int b = 0; b < nb; ++b) {
          o[b] = occ01(p.smearing, e[b], ef_sp[sp], p.sigma) * spin_factor;
          nel_sp[sp] += o[b] * wk[ik];
        }
      }
    double delta = 0.0;
    for (int sp = 0; sp < ns; ++sp) {
      const std::vector<std::vector<double>> oc(occ.begin() + (size_t)sp * nk, occ.begin() + (size_t)(sp + 1) * nk);
      if ((r = build_density(h, oc, wk, sp, rout[sp], ns == 1 ? h.n_electrons : nel_sp[sp])) != kOk) return r;
      double dsq = 0.0;
      if ((r = reduce_host(h, rin[sp], rout[sp], N, 2, dsq)) != kOk) return r;
      delta = std::max(delta, std::sqrt(dsq * dv / h.omega));
    }
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
    if (ns == 1) r = potentials(h, st->rho_out, false, eout);
    else r = potentials_spin(h, st->rho_out, st->rho_out_dn, false, eout);
    if (r != kOk) return r;
    double e_band = 0.0;
    for (size_t c = 0; c < ev.size(); ++c) {
      double sk = 0.0;
      for (int b = 0; b < nb; ++b) sk += occ[c][b] * wk_all[c] * ev[c][b];
      e_band += sk;
    }
    const double ts = entropy_ts(ev, wk_all, ef, p.sigma, p.smearing, spin_factor);
    const double e_tot = e_band - eout.e_hartree + (eout.e_xc - eout.e_vxc) + h.e_ewald - ts;
    const double e_hf = e_band - ein.e_hartree + (ein.e_xc - ein.e_vxc) + h.e_ewald - ts;
    const double de = have_prev ? std::fabs(e_tot - e_prev) : INFINITY;
    const double mag = ns == 2 ? std::fabs(nel_sp[0] - nel_sp[1]) : 0.0;
    if (p.verbose)
      std::fprintf(stderr, "pwgpu scf iter %3d E=%.10f dE=%.3e drho=%.3e res=%.2e prec=%d happ=%ld%s", iter, e_tot, de,
                   delta, max_res_all, prec, happ, ns == 2 ? "" : "\n");
    if (p.verbose && ns == 2) std::fprintf(stderr, " M=%.6f\n", mag);
    const bool conv = delta < p.conv_threshold && have_prev && de < p.energy_threshold;
    e_prev = e_tot;
    have_prev = true;
    if (conv || iter == p.max_iter - 1 || p.single_step) {
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
      res.nspin = ns;
      res.magnetization = mag;
      res.h_applications = happ;
      res.max_residual = max_res_all;
      // energy decomposition of the final iteration (driver.rs:652-710,
      // driver_spin.rs:715-780): band terms from the last eigenvectors and
      // occupations, the local term from the output density
      {
        std::vector<double> tk(nb), tn(nb);
        double ekin = 0.0, enl = 0.0;
        for (int c = 0; c < ns * nk; ++c) {
          if ((r = band_energy_terms(h, c % nk, st->ks[c].V, h.n_pw, nb, st->band_terms, tk.data(), tn.data(), s)) !=
              kOk)
            return r;
          for (int b = 0; b < nb; ++b) {
            if (occ[c][b] == 0.0) continue;
            ekin += occ[c][b] * wk_all[c] * tk[b];
            enl += occ[c][b] * wk_all[c] * tn[b];
          }
        }
        double eloc = 0.0;
        if ((r = local_energy(h, rout, ns, eloc)) != kOk) return r;
        res.e_kinetic = ekin;
        res.e_local = eloc;
        res.e_nonlocal = enl;
      }
      if (evals_out)
        for (size_t c = 0; c < ev.size(); ++c)
          for (int b = 0; b < nb; ++b) evals_out[c * nb + b] = ev[c][b];
      for (int sp = 0; sp < ns && rho_out_host; ++sp)
        PW_CUDA_TRY(cudaMemcpyAsync(rho_out_host + (size_t)sp * N, rout[sp], N * sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
      if (rho_g_basis_out) {
        const double* tot = st->rho_out;
        if (ns == 2) {
          k_axpy_to<<<blocks_for(N), 256, 0, s>>>(st->rho_out, st->rho_out_dn, 1.0, st->rtmp, N); count_launch();
          tot = st->rtmp;
        }
        if ((r = density_to_g(h, tot)) != kOk) return r;
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
      return (conv || p.single_step) ? kOk : fail(kNotConverged, "SCF did not converge within max_iter");
    }
    if (ns == 1) {
      if ((r = mix_channel(h, st->mixh[0], mix_tot, st->rho_in, st->rho_out, st->rho_in)) != kOk) return r;
    } else {
      // CCMX (driver_spin.rs:792-826): total density with the requested
      // mode, magnetisation with plain Anderson
      k_axpy_to<<<blocks_for(N), 256, 0, s>>>(st->rho_in, st->rho_in_dn, 1.0, st->t_in, N); count_launch();
      k_axpy_to<<<blocks_for(N), 256, 0, s>>>(st->rho_in, st->rho_in_dn, -1.0, st->m_in, N); count_launch();
      k_axpy_to<<<blocks_for(N), 256, 0, s>>>(st->rho_out, st->rho_out_dn, 1.0, st->t_out, N); count_launch();
      k_axpy_to<<<blocks_for(N), 256, 0, s>>>(st->rho_out, st->rho_out_dn, -1.0, st->m_out, N); count_launch();
      if ((r = mix_channel(h, st->mixh[0], mix_tot, st->t_in, st->t_out, st->t_in)) != kOk) return r;
      if ((r = mix_channel(h, st->mixh[1], mix_mag, st->m_in, st->m_out, st->m_in)) != kOk) return r;
      k_unmix_spin<<<blocks_for(N), 256, 0, s>>>(st->t_in, st->m_in, st->rho_in, st->rho_in_dn, N); count_launch();
    }
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
    if (h.gam.on) {
      // complex Gamma-real columns -> packed real bands (through the T scratch)
      PW_CUDA_TRY(cudaMemcpyAsync(st->ew.T, psi_in, n * n_bands * sizeof(double2), cudaMemcpyHostToDevice, h.stream));
      if ((r = gamma_pack(h, st->ew.T, n, n_bands, reinterpret_cast<double*>(k.V), n, h.stream)) != kOk) return r;
    } else {
      PW_CUDA_TRY(cudaMemcpyAsync(k.V, psi_in, n * n_bands * sizeof(double2), cudaMemcpyHostToDevice, h.stream));
    }
  }
  EigStats es;
  if ((r = lobpcg(h, st->ew, k, spin, ik, v0, tol, max_iter, n_bands, precision, es)) != kOk) return r;
  const int its = es.iters;
  const double mres = es.max_res;
  for (int b = 0; b < n_bands; ++b) evals[b] = k.evals[b];
  if (psi_out) {
    const double2* src = k.V;
    if (h.gam.on) {
      if ((r = gamma_unpack(h, reinterpret_cast<const double*>(k.V), n, n_bands, st->ew.T, n, h.stream)) != kOk)
        return r;
      src = st->ew.T;
    }
    PW_CUDA_TRY(cudaMemcpyAsync(psi_out, src, n * n_bands * sizeof(double2), cudaMemcpyDeviceToHost, h.stream));
  }
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
  if (iters) *iters = its;
  if (max_res) *max_res = mres;
  if (mres >= tol) return fail(kNotConverged, "eigensolve: residual tolerance not reached within max_iter");
  return kOk;
}

Status bands_to_host(Handle& h, int spin, int ik, int n_bands, double* psi_out) {
  if (ik < 0 || ik >= h.n_k || spin < 0 || spin >= h.nspin) return fail(kInvalid, "get_bands: index out of range");
  ScfState* st = h.scf;
  if (!st || st->ks.empty() || !st->ks[(size_t)spin * h.n_k + ik].init)
    return fail(kState, "get_bands: no bands on the device (run the SCF or an eigensolve first)");
  if (n_bands < 1 || n_bands > st->nd) return fail(kInvalid, "get_bands: n_bands out of range");
  EigVecs& k = st->ks[(size_t)spin * h.n_k + ik];
  const long n = h.n_pw;
  const double2* src = k.V;
  if (h.gam.on) {
    Status r = gamma_unpack(h, reinterpret_cast<const double*>(k.V), n, n_bands, st->ew.T, n, h.stream);
    if (r != kOk) return r;
    src = st->ew.T;
  }
  PW_CUDA_TRY(cudaMemcpyAsync(psi_out, src, n * n_bands * sizeof(double2), cudaMemcpyDeviceToHost, h.stream));
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
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
    if (h.gam.on) {
      PW_CUDA_TRY(cudaMemcpyAsync(st->ew.T, psi_all + (size_t)ik * n * n_bands * 2, n * n_bands * sizeof(double2),
                                  cudaMemcpyHostToDevice, h.stream));
      if ((r = gamma_pack(h, st->ew.T, n, n_bands, reinterpret_cast<double*>(st->ks[ik].V), n, h.stream)) != kOk)
        return r;
    } else {
      PW_CUDA_TRY(cudaMemcpyAsync(st->ks[ik].V, psi_all + (size_t)ik * n * n_bands * 2,
                                  n * n_bands * sizeof(double2), cudaMemcpyHostToDevice, h.stream));
    }
  }
  if ((r = build_density(h, oc, wk, 0, st->rho_out, h.n_electrons)) != kOk) return r;
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

Status scf_iter1_from_rho_g(Handle& h, const ScfParams& p, const double* rho_g_fft_in, ScfResult& res,
                            double* evals_out, double* rho_out_host, double* rho_g_fft_out, double* rho_in_host) {
  if (h.nspin != 1)
    return fail(kInvalid, "transplanted iteration: nspin = 1 only (transplant.rs:128-133)");
  if (!rho_g_fft_in) return fail(kInvalid, "transplanted iteration: rho_g_fft_in is NULL");
  PW_CUDA_TRY(cudaSetDevice(h.device));
  const long N = h.g.N;
  const cudaStream_t s = h.stream;
  // rho_in(r) = Re sum_G rho(G) e^{iG.r}: the unnormalised inverse transform
  // (transplant.rs:140-148); the iteration re-derives rho(G) from it
  std::vector<double2> grid(N);
  PW_CUDA_TRY(cudaMemcpyAsync(h.tmp_grid, rho_g_fft_in, N * sizeof(double2), cudaMemcpyHostToDevice, s));
  Status r = fft3d_full(h, h.tmp_grid, +1, s);
  if (r != kOk) return r;
  PW_CUDA_TRY(cudaMemcpyAsync(grid.data(), h.tmp_grid, N * sizeof(double2), cudaMemcpyDeviceToHost, s));
  PW_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<double> rin(N);
  for (long i = 0; i < N; ++i) rin[i] = grid[i].x;
  if (rho_in_host) std::copy(rin.begin(), rin.end(), rho_in_host);
  ScfParams q = p;
  q.max_iter = 1;
  q.single_step = 1;
  if ((r = scf_run(h, q, rin.data(), res, evals_out, rho_out_host, nullptr)) != kOk) return r;
  res.converged = 0;
  if (rho_g_fft_out) {
    if ((r = density_to_g(h, h.scf->rho_out)) != kOk) return r;
    PW_CUDA_TRY(cudaMemcpyAsync(rho_g_fft_out, h.scf->cg, N * sizeof(double2), cudaMemcpyDeviceToHost, s));
    PW_CUDA_TRY(cudaStreamSynchronize(s));
  }
  return kOk;
}

Status mix_host(Handle& h, int channel, int mode, const double* in, const double* out, double* next, double beta,
                int ndim, int period, double q_tf) {
  if (channel < 0 || channel > 1) return fail(kInvalid, "mix: channel must be 0 or 1");
  if (mode < 0 || mode > 5) return fail(kInvalid, "mix: unknown mixing mode");
  if (ndim < 1) return fail(kInvalid, "mix: ndim must be >= 1");
  Status r;
  if (!h.scf && (r = ensure_state(h, 1, 1, ndim)) != kOk) return r;
  ScfState* st = h.scf;
  const long N = h.g.N;
  if (ndim > st->mix_cap) {
    cudaFree(st->mix_partials);
    cudaFree(st->mix_sums);
    st->mix_partials = st->mix_sums = nullptr;
    const size_t nslots = (size_t)ndim * (ndim + 1);
    if ((r = salloc(&st->mix_partials, nslots * kMixBlocks)) != kOk) return r;
    if ((r = salloc(&st->mix_sums, nslots)) != kOk) return r;
    st->mix_cap = ndim;
  }
  MixHistory& mh = st->mixh[channel];
  if ((int)mh.hin.size() != ndim && (r = alloc_history(mh, N, ndim)) != kOk) return r;
  const MixConfig cfg = mix_config(mode, period, beta);
  if ((r = set_kerker(h, cfg.kerker, cfg.kind == 0 ? q_tf : 0.0)) != kOk) return r;
  PW_CUDA_TRY(cudaMemcpyAsync(st->rho_in, in, N * sizeof(double), cudaMemcpyHostToDevice, h.stream));
  PW_CUDA_TRY(cudaMemcpyAsync(st->rho_out, out, N * sizeof(double), cudaMemcpyHostToDevice, h.stream));
  if ((r = mix_channel(h, mh, cfg, st->rho_in, st->rho_out, st->rho_in)) != kOk) return r;
  PW_CUDA_TRY(cudaMemcpyAsync(next, st->rho_in, N * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
  return kOk;
}

Status mix_reset(Handle& h) {
  if (h.scf)
    for (auto& mh : h.scf->mixh) reset_history(mh);
  return kOk;
}

}  // namespace pwgpu
