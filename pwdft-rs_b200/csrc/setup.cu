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

}  // namespace pwgpu
