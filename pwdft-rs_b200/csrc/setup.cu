// Kleinman-Bylander projector matrix built on the device (the reference's
// NonlocalPotential::new, potential/nonlocal.rs:190-382):
//
//   B[G, c] = (1/sqrt(Omega)) e^{-i G.tau_a} F_i(|k+G|) Y_lm(k+G)
//   F_i(q)  = 4 pi int [r beta_i(r)] j_l(q r) r dr     (Simpson, nonlocal.rs:566-583)
//
// with the real Y_lm of nonlocal.rs:469-552 (order m = 0, +1, -1, +2, -2,
// ...; the +m slot carries cos(m phi), the -m slot sin(m phi), both times
// sqrt 2; Y_lm = 0 for l > 0 when |k+G| < 1e-9) and channels ordered atom
// by atom, projector by projector, m by m.  Every |k+G| is evaluated
// directly (no interpolation table), so B equals the host construction to
// rounding.
//
// The local part of ScfContext::new on the full FFT grid, from the same
// radial meshes (build_local_device):
//
//   V_loc(G) = sum_s S_s(G) v_s(|G|),  S_s(G) = sum_{a in s} e^{-iG.tau_a}
//   v_s(G)   = (4 pi/Omega) int r^2 [V(r) + Z e^2 erf(r)/r] sinc(Gr) dr
//              - 4 pi Z e^2 e^{-G^2/4} / (Omega G^2)               (G != 0)
//   v_s(0)   = (4 pi/Omega) int r^2 [V(r) + Z e^2 / r] dr           (upf/mod.rs:166-213)
//   rho_core(G) = sum_s S_s(G) (4 pi/Omega) int r^2 rho_c(r) j0(Gr) dr  (potentials.rs:99-115)
//   rho_0(G)    = sum_s S_s(G) (1/Omega) int rho_atom(r) j0(Gr) dr, or
//                 Z e^{-G^2 sigma^2/2} / Omega without PP_RHOATOM  (initial_density.rs:64-166)
//
// rho_core(r) and rho_0(r) are unnormalised inverse transforms (real part);
// rho_0 is clipped at zero and scaled to the electron count.  Each |G| is
// evaluated directly, one warp per grid point.
#include <algorithm>
#include <cmath>
#include <vector>

#include "handle.hpp"

namespace pwgpu {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxL = 3;

// |k+G| with the host's operation order: ((q0 q0 + q1 q1) + q2 q2), no FMA
__device__ __forceinline__ double qnorm(const double* g, const double* k) {
  const double q0 = __dadd_rn(k[0], g[0]), q1 = __dadd_rn(k[1], g[1]), q2 = __dadd_rn(k[2], g[2]);
  return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(q0, q0), __dmul_rn(q1, q1)), __dmul_rn(q2, q2)));
}

// j_l(x): explicit l = 0, 1 and upward recurrence (nonlocal.rs:592-612);
// |x| < 1e-10 gives j_0 = 1, j_l = 0
__device__ __forceinline__ double sph_bessel(int l, double x) {
  if (fabs(x) < 1e-10) return l == 0 ? 1.0 : 0.0;
  double s, c;
  sincos(x, &s, &c);
  const double j0 = s / x;
  if (l == 0) return j0;
  const double j1 = s / (x * x) - c / x;
  if (l == 1) return j1;
  double jm1 = j0, jl = j1;
  for (int n = 1; n < l; ++n) {
    const double jp1 = (2 * n + 1) / x * jl - jm1;
    jm1 = jl;
    jl = jp1;
  }
  return jl;
}

// Simpson weight of point i of an n-point mesh (numerics.rs:24-53 weights;
// the product with rab and the division by 3 are applied by the caller)
__device__ __forceinline__ double simpson_w(int i, int n) {
  if (n < 3) return 3.0;  // plain sum, divided by 3 later
  double w = (i == 0) ? 1.0 : ((i % 2 == 1) ? 4.0 : 2.0);
  if (n % 2 == 1) {
    if (i == n - 1) w = 1.0;
  } else {
    if (i == n - 1) w = 1.25;
    else if (i == n - 2) w += 1.0;
    if (i == n - 3) w -= 0.25;
  }
  return w;
}

// F[p * nq + j] = 4 pi Simpson(beta_p(r) r j_l(q_j r), rab), one warp per (j, p)
__global__ void k_form_factors(const double* __restrict__ gvec, int n_pw, const double* __restrict__ kvec,
                               const double* __restrict__ r, const double* __restrict__ rab, int mesh,
                               const double* __restrict__ beta, const int* __restrict__ lval, int nproj,
                               double* __restrict__ F) {
  const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= (long)n_pw * nproj) return;
  const int j = (int)(warp % n_pw), p = (int)(warp / n_pw);
  const double q = qnorm(gvec + 3L * j, kvec);
  const int l = lval[p];
  const double* b = beta + (long)p * mesh;
  double acc = 0.0;
  for (int i = lane; i < mesh; i += 32) acc += simpson_w(i, mesh) * (b[i] * r[i]) * sph_bessel(l, q * r[i]) * rab[i];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) F[(long)p * n_pw + j] = 4.0 * kPi * (acc / 3.0);
}

// real Y_lm, l <= kMaxL, into y[(l*l + slot)] (slot 0: m = 0, 2m-1: +m, 2m: -m)
__device__ void real_ylm(const double* g, const double* k, int lmax, double* y) {
  const double fpi = 4.0 * kPi;
  const double q0 = __dadd_rn(k[0], g[0]), q1 = __dadd_rn(k[1], g[1]), q2 = __dadd_rn(k[2], g[2]);
  y[0] = sqrt(1.0 / fpi);
  if (lmax == 0) return;
  const double gm = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(q0, q0), __dmul_rn(q1, q1)), __dmul_rn(q2, q2)));
  if (gm < 1e-9) {
    for (int t = 1; t < (lmax + 1) * (lmax + 1); ++t) y[t] = 0.0;
    return;
  }
  const double cost = q2 / gm;
  const double sint = sqrt(fmax(1.0 - cost * cost, 0.0));
  const double phi = atan2(q1, q0);
  double Q[kMaxL + 1][kMaxL + 1];
  Q[0][0] = 1.0;
  Q[1][0] = cost;
  Q[1][1] = -sint / sqrt(2.0);
  const double c1 = sqrt(3.0 / fpi);
  y[1] = c1 * Q[1][0];
  y[2] = c1 * sqrt(2.0) * Q[1][1] * cos(phi);
  y[3] = c1 * sqrt(2.0) * Q[1][1] * sin(phi);
  int lm = 4;
  for (int l = 2; l <= lmax; ++l) {
    const double c = sqrt((2 * l + 1) / fpi);
    for (int m = 0; m < l - 1; ++m) {
      const double llmm = sqrt((double)(l * l - m * m));
      const double llm1 = sqrt((double)((l - 1) * (l - 1) - m * m));
      Q[l][m] = (cost * (2.0 * l - 1.0) * Q[l - 1][m] - llm1 * Q[l - 2][m]) / llmm;
    }
    Q[l][l - 1] = cost * sqrt(2.0 * l - 1.0) * Q[l - 1][l - 1];
    Q[l][l] = -sqrt((2.0 * l - 1.0) / (2.0 * l)) * sint * Q[l - 1][l - 1];
    y[lm] = c * Q[l][0];
    for (int m = 1; m <= l; ++m) {
      y[lm + 2 * m - 1] = c * sqrt(2.0) * Q[l][m] * cos(m * phi);
      y[lm + 2 * m] = c * sqrt(2.0) * Q[l][m] * sin(m * phi);
    }
    lm += 2 * l + 1;
  }
}

// B[G, c] for every channel: one thread per G, channels of atom a from
// column atom_ch_start[a] on, its species' projectors p0 .. p0 + np - 1
__global__ void k_assemble_b(const double* __restrict__ gvec, int n_pw, const double* __restrict__ kvec,
                             const double* __restrict__ tau, const int* __restrict__ atom_species, int n_atoms,
                             const int* __restrict__ species_p0, const int* __restrict__ species_np,
                             const int* __restrict__ lval, const double* __restrict__ F, int lmax,
                             double inv_sqrt_omega, const int* __restrict__ atom_ch_start, double2* __restrict__ B) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_pw) return;
  const double* g = gvec + 3L * j;
  double y[(kMaxL + 1) * (kMaxL + 1)];
  real_ylm(g, kvec, lmax, y);
  for (int a = 0; a < n_atoms; ++a) {
    const double* t = tau + 3L * a;
    const double arg = -__dadd_rn(__dadd_rn(__dmul_rn(g[0], t[0]), __dmul_rn(g[1], t[1])), __dmul_rn(g[2], t[2]));
    double sn, cs;
    sincos(arg, &sn, &cs);
    const int sp = atom_species[a];
    int c = atom_ch_start[a];
    for (int p = species_p0[sp]; p < species_p0[sp] + species_np[sp]; ++p) {
      const int l = lval[p];
      const double scale = inv_sqrt_omega * F[(long)p * n_pw + j];
      for (int mo = 0; mo < 2 * l + 1; ++mo, ++c) {
        const double v = scale * y[l * l + mo];
        B[(long)c * n_pw + j] = make_double2(cs * v, sn * v);
      }
    }
  }
}

// G of flat grid index t with the host's operation order (grid_g_vectors:
// signed Miller index i > n/2 -> i - n; g_c = (f1 b1_c + f2 b2_c) + f3 b3_c)
__device__ __forceinline__ void grid_g(long t, int d0, int d1, int d2, const double* __restrict__ rec, double* g) {
  const int i2 = (int)(t % d2), i1 = (int)((t / d2) % d1), i0 = (int)(t / ((long)d1 * d2));
  const double f1 = i0 > d0 / 2 ? i0 - d0 : i0, f2 = i1 > d1 / 2 ? i1 - d1 : i1, f3 = i2 > d2 / 2 ? i2 - d2 : i2;
  for (int c = 0; c < 3; ++c)
    g[c] = __dadd_rn(__dadd_rn(__dmul_rn(f1, rec[c]), __dmul_rn(f2, rec[3 + c])), __dmul_rn(f3, rec[6 + c]));
}

__device__ __forceinline__ double norm3(const double* g) {
  return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(g[0], g[0]), __dmul_rn(g[1], g[1])), __dmul_rn(g[2], g[2])));
}

// sin(x)/x with the host's small-argument form 1 - x^2/6 below 1e-10
__device__ __forceinline__ double sinc_host(double x) {
  if (x < 1e-10) return 1.0 - x * x / 6.0;
  return sin(x) / x;
}

enum LocalKind { kVloc = 0, kCore = 1, kAtom = 2, kGauss = 3 };

constexpr double kE2 = 14.399645351950548;  // e^2 in eV Angstrom
constexpr double kGZero = 1e-12;             // |G| below which G = 0

// rad[t] = radial transform of one species at |G_t|, one warp per grid point
__global__ void k_local_radial(int kind, long N, int d0, int d1, int d2, const double* __restrict__ rec,
                               const double* __restrict__ r, const double* __restrict__ rab, int mesh,
                               const double* __restrict__ f, double z, double omega, double sigma,
                               double* __restrict__ rad) {
  const long t = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= N) return;
  double g[3];
  grid_g(t, d0, d1, d2, rec, g);
  const double gn = norm3(g);
  const double fpi = 4.0 * kPi;
  if (kind == kGauss) {
    if (lane == 0) {
      const double g2 = __dadd_rn(__dadd_rn(__dmul_rn(g[0], g[0]), __dmul_rn(g[1], g[1])), __dmul_rn(g[2], g[2]));
      rad[t] = z * exp(-0.5 * g2 * sigma * sigma) / omega;
    }
    return;
  }
  double acc = 0.0;
  const bool g0 = gn < kGZero;
  for (int i = lane; i < mesh; i += 32) {
    const double ri = r[i];
    double v;
    if (kind == kVloc) {
      double eor;
      if (g0) eor = 1.0 / fmax(ri, 1e-20);
      else eor = ri < 1e-20 ? 2.0 / sqrt(kPi) : erf(ri) / ri;
      const double vs = f[i] + z * kE2 * eor;
      v = ri * ri * vs * (g0 ? 1.0 : sinc_host(gn * ri));
    } else if (kind == kCore) {
      v = f[i] * (ri * ri) * sinc_host(gn * ri);
    } else {
      v = f[i] * sinc_host(gn * ri);
    }
    acc += simpson_w(i, mesh) * (v * rab[i]);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane != 0) return;
  const double sint = acc / 3.0;
  double out;
  if (kind == kVloc) {
    out = fpi / omega * sint;
    if (!g0) {
      const double g2 = gn * gn;
      out -= fpi * z * kE2 * exp(-g2 / 4.0) / (omega * g2);
    }
  } else if (kind == kCore) {
    out = fpi * sint / omega;
  } else {
    out = sint / omega;
  }
  rad[t] = out;
}

// out[t] = sum_a e^{-iG_t.tau_a} rad[species(a)][t] (species with rad_used 0 skipped)
__global__ void k_structure_sum(long N, int d0, int d1, int d2, const double* __restrict__ rec,
                                const double* __restrict__ tau, const int* __restrict__ atom_species, int n_atoms,
                                const double* __restrict__ rad, const int* __restrict__ used,
                                double2* __restrict__ out) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N) return;
  double g[3];
  grid_g(t, d0, d1, d2, rec, g);
  double re = 0.0, im = 0.0;
  for (int a = 0; a < n_atoms; ++a) {
    const int sp = atom_species[a];
    if (!used[sp]) continue;
    const double* ta = tau + 3L * a;
    const double ph = -__dadd_rn(__dadd_rn(__dmul_rn(g[0], ta[0]), __dmul_rn(g[1], ta[1])), __dmul_rn(g[2], ta[2]));
    double sn, cs;
    sincos(ph, &sn, &cs);
    const double v = rad[(long)sp * N + t];
    re += cs * v;
    im += sn * v;
  }
  out[t] = make_double2(re, im);
}

__global__ void k_real_clip(const double2* __restrict__ c, double* __restrict__ r, long n, int clip) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = (clip && c[i].x < 0.0) ? 0.0 : c[i].x;
}

constexpr int kSumBlocks = 512;

__global__ void k_sum_partials(const double* __restrict__ a, long n, double* __restrict__ partials) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) acc += a[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

__global__ void k_sum_final(double* __restrict__ partials, int n) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[kSumBlocks] = sh[0];
}

__global__ void k_scale_vec(double* __restrict__ a, long n, double f) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] *= f;
}

// sum of a[0..n) (fixed block count: the same order on every call); red
// holds kSumBlocks + 1 doubles
Status device_sum(Handle& h, const double* a, long n, double* red, double& out) {
  k_sum_partials<<<kSumBlocks, 256, 0, h.stream>>>(a, n, red); count_launch();
  k_sum_final<<<1, 256, 0, h.stream>>>(red, kSumBlocks); count_launch();
  PW_CUDA_TRY(cudaMemcpyAsync(&out, red + kSumBlocks, sizeof(double), cudaMemcpyDeviceToHost, h.stream));
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
  return kOk;
}

Status device_scale(Handle& h, double* a, long n, double f) {
  k_scale_vec<<<(unsigned)((n + 255) / 256), 256, 0, h.stream>>>(a, n, f); count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

template <typename T> Status sup_upload(T** dst, const T* src, size_t n) {
  cudaError_t e = cudaMalloc((void**)dst, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess) return fail(kOom, std::string("cudaMalloc (projector build): ") + cudaGetErrorString(e));
  if (src && n) {
    e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(kCuda, std::string("cudaMemcpy (projector build): ") + cudaGetErrorString(e));
  }
  return kOk;
}

}  // namespace

Status build_projectors_device(Handle& h, const ProjectorSource& src) {
  if (h.n_ch <= 0) return kOk;
  if (!src.gvec || !src.kpts || !src.atom_tau || !src.atom_species || src.n_species <= 0 || !src.species_mesh ||
      !src.radial_r || !src.radial_rab || !src.species_nbeta || !src.beta_l || !src.beta_r)
    return fail(kInvalid, "pwgpu_create: proj_b is NULL and the projector radial data is incomplete");
  const int ns = src.n_species, n = h.n_pw;
  std::vector<long> mesh_off(ns + 1, 0), beta_off(ns + 1, 0);
  std::vector<int> p0(ns, 0), np(ns, 0);
  int nproj = 0, lmax = 0;
  for (int s = 0; s < ns; ++s) {
    if (src.species_mesh[s] < 1 || src.species_nbeta[s] < 0)
      return fail(kInvalid, "pwgpu_create: species radial mesh or projector count out of range");
    mesh_off[s + 1] = mesh_off[s] + src.species_mesh[s];
    p0[s] = nproj;
    np[s] = src.species_nbeta[s];
    nproj += np[s];
    beta_off[s + 1] = beta_off[s] + (long)np[s] * src.species_mesh[s];
  }
  for (int p = 0; p < nproj; ++p) {
    if (src.beta_l[p] < 0 || src.beta_l[p] > kMaxL) return fail(kInvalid, "pwgpu_create: projector l must be 0..3");
    lmax = std::max(lmax, src.beta_l[p]);
  }
  // the channel count implied by the atoms must be the handle's
  int nch = 0;
  for (int a = 0; a < h.n_atoms; ++a) {
    const int sp = src.atom_species[a];
    if (sp < 0 || sp >= ns) return fail(kInvalid, "pwgpu_create: atom species index out of range");
    for (int p = p0[sp]; p < p0[sp] + np[sp]; ++p) nch += 2 * src.beta_l[p] + 1;
  }
  if (nch != h.n_ch) return fail(kInvalid, "pwgpu_create: n_ch does not match the projectors of the atoms");
  std::vector<void*> owned;
  auto cleanup = [&]() {
    for (void* p : owned) cudaFree(p);
  };
  Status r = kOk;
  auto up = [&](auto** dst, const auto* srcp, size_t cnt) {
    if (r != kOk) return;
    r = sup_upload(dst, srcp, cnt);
    if (r == kOk) owned.push_back((void*)*dst);
  };
  double *gv = nullptr, *kv = nullptr, *tau = nullptr, *F = nullptr, *rr = nullptr, *rab = nullptr, *beta = nullptr;
  int *sp_dev = nullptr, *p0_dev = nullptr, *np_dev = nullptr, *l_dev = nullptr;
  up(&gv, src.gvec, 3L * n);
  up(&kv, src.kpts, 3L * h.n_k);
  up(&tau, src.atom_tau, 3L * h.n_atoms);
  up(&sp_dev, src.atom_species, (size_t)h.n_atoms);
  up(&p0_dev, p0.data(), (size_t)ns);
  up(&np_dev, np.data(), (size_t)ns);
  up(&l_dev, src.beta_l, (size_t)nproj);
  up(&rr, src.radial_r, (size_t)mesh_off[ns]);
  up(&rab, src.radial_rab, (size_t)mesh_off[ns]);
  up(&beta, src.beta_r, (size_t)beta_off[ns]);
  up(&F, (const double*)nullptr, (size_t)nproj * n);
  if (r != kOk) {
    cleanup();
    return r;
  }
  const double inv_sqrt_omega = 1.0 / std::sqrt(h.omega);
  for (int ik = 0; ik < h.n_k; ++ik) {
    // F_i(|k+G|) of every species' projectors, then B of this k
    for (int s = 0; s < ns; ++s) {
      if (np[s] == 0) continue;
      const long warps = (long)n * np[s];
      k_form_factors<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, h.stream>>>(
          gv, n, kv + 3L * ik, rr + mesh_off[s], rab + mesh_off[s], src.species_mesh[s], beta + beta_off[s],
          l_dev + p0[s], np[s], F + (long)p0[s] * n);
      count_launch();
    }
    k_assemble_b<<<(unsigned)((n + 127) / 128), 128, 0, h.stream>>>(gv, n, kv + 3L * ik, tau, sp_dev, h.n_atoms,
                                                                   p0_dev, np_dev, l_dev, F, lmax, inv_sqrt_omega,
                                                                   h.atom_ch_start, h.kp[ik].b);
    count_launch();
  }
  cudaError_t e = cudaStreamSynchronize(h.stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  cleanup();
  if (e != cudaSuccess) return fail(kCuda, std::string("projector build: ") + cudaGetErrorString(e));
  return kOk;
}

Status build_local_device(Handle& h, const LocalSource& src, double2* v_local_g, double** rho_core_r,
                          double** rho_start) {
  if (src.n_species <= 0 || !src.species_mesh || !src.radial_r || !src.radial_rab || !src.species_zval ||
      !src.vloc_r || !src.species_flags || !src.atom_tau || !src.atom_species || src.n_atoms <= 0 || !src.recip)
    return fail(kInvalid, "pwgpu_create: v_local_g is NULL and the local radial data is incomplete");
  if (!(src.gaussian_sigma > 0.0) || !std::isfinite(src.gaussian_sigma))
    return fail(kInvalid, "pwgpu_create: gaussian_sigma must be positive and finite");
  const int ns = src.n_species;
  const long N = h.g.N;
  std::vector<long> off(ns + 1, 0);
  bool any_core = false, any_atom = false;
  for (int q = 0; q < ns; ++q) {
    if (src.species_mesh[q] < 1) return fail(kInvalid, "pwgpu_create: species radial mesh out of range");
    off[q + 1] = off[q] + src.species_mesh[q];
    any_core = any_core || (src.species_flags[q] & 1);
    any_atom = any_atom || (src.species_flags[q] & 2);
  }
  if (any_core && !src.core_r) return fail(kInvalid, "pwgpu_create: core charge flagged but core_r is NULL");
  if (any_atom && !src.rho_atom_r) return fail(kInvalid, "pwgpu_create: rho_atom flagged but rho_atom_r is NULL");
  for (int a = 0; a < src.n_atoms; ++a)
    if (src.atom_species[a] < 0 || src.atom_species[a] >= ns)
      return fail(kInvalid, "pwgpu_create: atom species index out of range");
  std::vector<void*> owned;
  Status r = kOk;
  auto up = [&](auto** dst, const auto* srcp, size_t cnt) {
    if (r != kOk) return;
    r = sup_upload(dst, srcp, cnt);
    if (r == kOk) owned.push_back((void*)*dst);
  };
  double *rec = nullptr, *rr = nullptr, *rab = nullptr, *vl = nullptr, *cr = nullptr, *ra = nullptr, *tau = nullptr,
         *rad = nullptr, *red = nullptr;
  int *sp = nullptr, *used = nullptr;
  up(&rec, src.recip, 9);
  up(&rr, src.radial_r, (size_t)off[ns]);
  up(&rab, src.radial_rab, (size_t)off[ns]);
  up(&vl, src.vloc_r, (size_t)off[ns]);
  if (any_core) up(&cr, src.core_r, (size_t)off[ns]);
  if (any_atom) up(&ra, src.rho_atom_r, (size_t)off[ns]);
  up(&tau, src.atom_tau, 3L * src.n_atoms);
  up(&sp, src.atom_species, (size_t)src.n_atoms);
  up(&rad, (const double*)nullptr, (size_t)ns * N);
  up(&used, (const int*)nullptr, (size_t)ns);
  up(&red, (const double*)nullptr, 1024);
  auto done = [&](Status st) {
    cudaStreamSynchronize(h.stream);
    for (void* p : owned) cudaFree(p);
    return st;
  };
  if (r != kOk) return done(r);
  const int d0 = h.g.d[0], d1 = h.g.d[1], d2 = h.g.d[2];
  const cudaStream_t s = h.stream;
  const unsigned wblocks = (unsigned)((N * 32 + 255) / 256), tblocks = (unsigned)((N + 255) / 256);
  std::vector<int> use(ns);
  // one structure sum for the given per-species kinds into out
  auto structure = [&](auto kind_of, double2* out) -> Status {
    for (int q = 0; q < ns; ++q) {
      const int kind = kind_of(q);
      use[q] = kind >= 0;
      if (kind < 0) continue;
      const double* f = kind == kVloc ? vl + off[q] : (kind == kCore ? cr + off[q] : (kind == kAtom ? ra + off[q]
                                                                                                   : nullptr));
      k_local_radial<<<wblocks, 256, 0, s>>>(kind, N, d0, d1, d2, rec, rr + off[q], rab + off[q],
                                             src.species_mesh[q], f, src.species_zval[q], h.omega,
                                             src.gaussian_sigma, rad + (long)q * N);
      count_launch();
    }
    PW_CUDA_TRY(cudaMemcpyAsync(used, use.data(), ns * sizeof(int), cudaMemcpyHostToDevice, s));
    k_structure_sum<<<tblocks, 256, 0, s>>>(N, d0, d1, d2, rec, tau, sp, src.n_atoms, rad, used, out);
    count_launch();
    PW_CUDA_TRY(cudaStreamSynchronize(s));  // use[] is reused by the next sum
    return kOk;
  };
  Status st = structure([](int) { return (int)kVloc; }, v_local_g);
  if (st != kOk) return done(st);
  if (any_core) {
    st = structure([&](int q) { return (src.species_flags[q] & 1) ? (int)kCore : -1; }, h.tmp_grid);
    if (st == kOk) st = fft3d_full(h, h.tmp_grid, +1, s);
    if (st == kOk && !*rho_core_r) st = sup_upload(rho_core_r, (const double*)nullptr, (size_t)N);
    if (st != kOk) return done(st);
    k_real_clip<<<tblocks, 256, 0, s>>>(h.tmp_grid, *rho_core_r, N, 0); count_launch();
  }
  if (rho_start) {
    st = structure([&](int q) { return (src.species_flags[q] & 2) ? (int)kAtom : (int)kGauss; }, h.tmp_grid);
    if (st == kOk) st = fft3d_full(h, h.tmp_grid, +1, s);
    if (st == kOk && !*rho_start) st = sup_upload(rho_start, (const double*)nullptr, (size_t)N);
    if (st != kOk) return done(st);
    k_real_clip<<<tblocks, 256, 0, s>>>(h.tmp_grid, *rho_start, N, 1); count_launch();
    // scale to the electron count: int rho dV = N_el (initial_density.rs:128-143)
    double sum = 0.0;
    if ((st = device_sum(h, *rho_start, N, red, sum)) != kOk) return done(st);
    const double integ = sum * (h.omega / (double)N);
    if (integ > 1e-15) {
      if ((st = device_scale(h, *rho_start, N, h.n_electrons / integ)) != kOk) return done(st);
    }
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return done(fail(kCuda, std::string("local potential build: ") + cudaGetErrorString(e)));
  return done(kOk);
}

}  // namespace pwgpu
