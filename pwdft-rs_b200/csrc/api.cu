// C-ABI entry points of libpwgpu (declared in include/pwgpu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "handle.hpp"
#include "linalg.hpp"
#include "scf.hpp"
#include "../../include/pwgpu.h"

struct pwgpu_handle {
  pwgpu::Handle h;
  int precision = 0;
};

namespace pwgpu {

static thread_local std::string t_last_error;

Status fail(int code, const std::string& msg) {
  t_last_error = msg;
  return (Status)code;
}

std::string last_error_message() { return t_last_error; }

template <typename T> static Status upload(T** dst, const T* src, size_t count) {
  const size_t n = std::max<size_t>(count, 1);
  cudaError_t e = cudaMalloc((void**)dst, n * sizeof(T));
  if (e != cudaSuccess) return fail(kOom, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  if (src && count) {
    e = cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(kCuda, std::string("cudaMemcpy: ") + cudaGetErrorString(e));
  }
  return kOk;
}

static void release(Handle& h) {
  release_gamma(h);
  auto f = [](void* p) { if (p) cudaFree(p); };
  GridMaps& g = h.g;
  for (int a = 0; a < 3; ++a) { f(g.tw64[a]); f(g.tw32[a]); }
  f(g.col_start); f(g.pt_ig); f(g.pt_col); f(g.pt_z); f(g.g_to_fft);
  for (auto& k : h.kp) { f(k.kinetic); f(k.b); f(k.b32); }
  h.kp.clear();
  f(h.ch_atom); f(h.atom_ch_start); f(h.d_off); f(h.d_vals);
  f(h.v_local_g); f(h.g_squared); f(h.rho_core_r); f(h.rho_sad); f(h.sym_src); f(h.sym_arg);
  for (int s = 0; s < 2; ++s) { f(h.veff_r[s]); f(h.veff_r32[s]); f(h.veff_rz[s]); f(h.veff_rz32[s]); }
  f(h.work_a); f(h.work_b); f(h.nl_p); f(h.nl_q); f(h.tmp_grid);
  release_scf(h);
  release_nl_mixed(h);
  f(h.solver_work); f(h.solver_info);
  if (h.solver) cusolverDnDestroy(h.solver);
  if (h.blas) cublasDestroy(h.blas);
  if (h.stream) cudaStreamDestroy(h.stream);
  h = Handle();
}

static Status create(const pwgpu_system* s, const pwgpu_options* o, pwgpu_handle* ph) {
  Handle& h = ph->h;
  if (!s || !s->miller || !s->kinetic || !s->k_weights || !s->g_squared)
    return fail(kInvalid, "pwgpu_create: required system array is NULL");
  if (s->n_pw <= 0 || s->n_k <= 0 || s->dims[0] <= 0 || s->dims[1] <= 0 || s->dims[2] <= 0)
    return fail(kInvalid, "pwgpu_create: n_pw, n_k and dims must be positive");
  if (s->dims[0] > 1024 || s->dims[1] > 1024 || s->dims[2] > 1024)
    return fail(kInvalid, "pwgpu_create: FFT grid dimension exceeds MAX_FFT_DIM=1024");
  if (s->nspin != 1 && s->nspin != 2) return fail(kInvalid, "pwgpu_create: nspin must be 1 or 2");
  if (s->n_ch < 0 || (s->n_ch > 0 && (!s->atom_ch_start || !s->d_blocks || s->n_atoms <= 0)))
    return fail(kInvalid, "pwgpu_create: projector arrays missing");
  if (s->n_sym < 0 || (s->n_sym > 1 && (!s->sym_src || !s->sym_arg)))
    return fail(kInvalid, "pwgpu_create: symmetry map missing");
  h.device = o ? o->device : 0;
  h.trace = std::getenv("PWGPU_TRACE") != nullptr;
  ph->precision = o ? o->precision : 0;
  h.lanes = o ? o->lanes : 0;
  if (h.lanes < 0) return fail(kInvalid, "pwgpu_create: lanes must be >= 0");
  PW_CUDA_TRY(cudaSetDevice(h.device));
  h.n_pw = s->n_pw;
  h.n_k = s->n_k;
  h.n_ch = s->n_ch;
  h.n_atoms = s->n_ch > 0 ? s->n_atoms : 0;
  h.nspin = s->nspin;
  h.n_sym = std::max(1, s->n_sym);
  h.n_electrons = s->n_electrons;
  h.omega = s->omega;
  h.e_ewald = s->e_ewald;
  for (int a = 0; a < 3; ++a) h.g.d[a] = s->dims[a];
  PW_CUDA_TRY(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
  if (cublasCreate(&h.blas) != CUBLAS_STATUS_SUCCESS) return fail(kCuda, "cublasCreate failed");
  cublasSetStream(h.blas, h.stream);
  Status st = build_grid_maps(h, s->miller);
  if (st != kOk) return st;
  const long N = h.g.N;
  h.kp.resize(h.n_k);
  for (int k = 0; k < h.n_k; ++k) {
    KPointData& kd = h.kp[k];
    kd.weight = s->k_weights[k];
    if ((st = upload(&kd.kinetic, s->kinetic + (long)k * h.n_pw, h.n_pw)) != kOk) return st;
    if (h.n_ch > 0) {
      // uploaded from the caller, or built on the device below
      const double2* bsrc =
          s->proj_b ? reinterpret_cast<const double2*>(s->proj_b) + (long)k * h.n_pw * h.n_ch : nullptr;
      if ((st = upload(&kd.b, bsrc, (size_t)h.n_pw * h.n_ch)) != kOk) return st;
    }
  }
  if (h.n_ch > 0) {
    std::vector<int> starts(s->atom_ch_start, s->atom_ch_start + h.n_atoms + 1);
    if (starts[0] != 0 || starts[h.n_atoms] != h.n_ch) return fail(kInvalid, "atom_ch_start must span [0, n_ch]");
    std::vector<int> ch_atom(h.n_ch), d_off(h.n_atoms);
    long off = 0;
    for (int a = 0; a < h.n_atoms; ++a) {
      const int nc = starts[a + 1] - starts[a];
      if (nc < 0) return fail(kInvalid, "atom_ch_start must be non-decreasing");
      d_off[a] = (int)off;
      off += (long)nc * nc;
      for (int c = starts[a]; c < starts[a + 1]; ++c) ch_atom[c] = a;
    }
    if ((st = upload(&h.atom_ch_start, starts.data(), starts.size())) != kOk) return st;
    if ((st = upload(&h.ch_atom, ch_atom.data(), ch_atom.size())) != kOk) return st;
    if ((st = upload(&h.d_off, d_off.data(), d_off.size())) != kOk) return st;
    if ((st = upload(&h.d_vals, s->d_blocks, (size_t)off)) != kOk) return st;
    if (!s->proj_b) {
      ProjectorSource src;
      src.gvec = s->g_cart;
      src.kpts = s->k_cart;
      src.atom_tau = s->atom_tau;
      src.atom_species = s->atom_species;
      src.n_species = s->n_species;
      src.species_mesh = s->species_mesh;
      src.radial_r = s->radial_r;
      src.radial_rab = s->radial_rab;
      src.species_nbeta = s->species_nbeta;
      src.beta_l = s->beta_l;
      src.beta_r = s->beta_r;
      if ((st = build_projectors_device(h, src)) != kOk) return st;
    }
  }
  if ((st = upload(&h.g_squared, s->g_squared, (size_t)N)) != kOk) return st;
  if (s->v_local_g) {
    if ((st = upload(&h.v_local_g, reinterpret_cast<const double2*>(s->v_local_g), (size_t)N)) != kOk) return st;
    if (s->rho_core_r && (st = upload(&h.rho_core_r, s->rho_core_r, (size_t)N)) != kOk) return st;
  } else {
    // V_loc(G), the core density and the start density from the radial data
    if (s->rho_core_r) return fail(kInvalid, "pwgpu_create: rho_core_r must be NULL when v_local_g is");
    if ((st = upload<double2>(&h.v_local_g, nullptr, (size_t)N)) != kOk) return st;
    LocalSource ls;
    ls.recip = s->recip;
    ls.atom_tau = s->atom_tau;
    ls.atom_species = s->atom_species;
    ls.n_atoms = s->n_atoms;
    ls.n_species = s->n_species;
    ls.species_mesh = s->species_mesh;
    ls.radial_r = s->radial_r;
    ls.radial_rab = s->radial_rab;
    ls.species_zval = s->species_zval;
    ls.vloc_r = s->vloc_r;
    ls.species_flags = s->species_flags;
    ls.core_r = s->core_r;
    ls.rho_atom_r = s->rho_atom_r;
    ls.gaussian_sigma = s->gaussian_sigma;
    if ((st = build_local_device(h, ls, h.v_local_g, &h.rho_core_r, &h.rho_sad)) != kOk) return st;
  }
  if (h.n_sym > 1) {
    if ((st = upload(&h.sym_src, s->sym_src, (size_t)h.n_sym * N)) != kOk) return st;
    if ((st = upload(&h.sym_arg, s->sym_arg, (size_t)h.n_sym * N)) != kOk) return st;
  }
  for (int sp = 0; sp < h.nspin; ++sp) {
    if ((st = upload<double>(&h.veff_r[sp], nullptr, (size_t)N)) != kOk) return st;
    if ((st = upload<float>(&h.veff_r32[sp], nullptr, (size_t)N)) != kOk) return st;
    if ((st = upload<double>(&h.veff_rz[sp], nullptr, (size_t)N)) != kOk) return st;
    if ((st = upload<float>(&h.veff_rz32[sp], nullptr, (size_t)N)) != kOk) return st;
    PW_CUDA_TRY(cudaMemset(h.veff_r[sp], 0, N * sizeof(double)));
    PW_CUDA_TRY(cudaMemset(h.veff_r32[sp], 0, N * sizeof(float)));
    PW_CUDA_TRY(cudaMemset(h.veff_rz[sp], 0, N * sizeof(double)));
    PW_CUDA_TRY(cudaMemset(h.veff_rz32[sp], 0, N * sizeof(float)));
  }
  // Gamma-only systems run with real wavefunctions unless the caller keeps them complex
  if (!(o && o->gamma_complex) &&
      (st = build_gamma(h, s->miller, s->kinetic, s->atom_ch_start, s->d_blocks)) != kOk)
    return st;
  PW_CUDA_TRY(cudaDeviceSynchronize());
  return kOk;
}

}  // namespace pwgpu

namespace pwgpu {
// Internal state and precision of an opaque handle (for entry points
// defined in other translation units).
Handle* handle_state(pwgpu_handle* ph, int* precision) {
  if (!ph) return nullptr;
  if (precision) *precision = ph->precision;
  return &ph->h;
}
}  // namespace pwgpu

using namespace pwgpu;

extern "C" {

const char* pwgpu_last_error(void) { return t_last_error.c_str(); }

const char* pwgpu_version(void) { return "pwgpu 0.1 (sm_100a)"; }

pwgpu_status pwgpu_create(const pwgpu_system* sys, const pwgpu_options* opt, pwgpu_handle** out) {
  if (!out) return fail(kInvalid, "pwgpu_create: out is NULL");
  *out = nullptr;
  pwgpu_handle* ph = new (std::nothrow) pwgpu_handle();
  if (!ph) return fail(kOom, "pwgpu_create: host allocation failed");
  Status st = create(sys, opt, ph);
  if (st != kOk) {
    release(ph->h);
    delete ph;
    return st;
  }
  *out = ph;
  return kOk;
}

pwgpu_status pwgpu_destroy(pwgpu_handle* ph) {
  if (!ph) return kOk;
  cudaSetDevice(ph->h.device);
  if (ph->h.stream) cudaStreamSynchronize(ph->h.stream);
  release(ph->h);
  delete ph;
  return kOk;
}

pwgpu_status pwgpu_set_veff_g(pwgpu_handle* ph, int32_t spin, const double* veff_g) {
  if (!ph || !veff_g) return fail(kInvalid, "pwgpu_set_veff_g: NULL argument");
  Handle& h = ph->h;
  if (spin < 0 || spin >= h.nspin) return fail(kInvalid, "pwgpu_set_veff_g: spin out of range");
  PW_CUDA_TRY(cudaSetDevice(h.device));
  PW_CUDA_TRY(cudaMemcpyAsync(h.tmp_grid, veff_g, h.g.N * sizeof(double2), cudaMemcpyHostToDevice, h.stream));
  Status st = set_veff_from_g(h, spin, h.tmp_grid, h.stream);
  if (st != kOk) return st;
  PW_CUDA_TRY(cudaStreamSynchronize(h.stream));
  return kOk;
}

pwgpu_status pwgpu_apply_h(pwgpu_handle* ph, int32_t spin, int32_t ik, const double* psi, int32_t nb,
                           double* hpsi) {
  if (!ph || !psi || !hpsi) return fail(kInvalid, "pwgpu_apply_h: NULL argument");
  if (nb < 0) return fail(kInvalid, "pwgpu_apply_h: nb must be non-negative");
  Handle& h = ph->h;
  if (nb == 0) return kOk;
  PW_CUDA_TRY(cudaSetDevice(h.device));
  const size_t bytes = (size_t)h.n_pw * nb * sizeof(double2);
  double2 *dp = nullptr, *dh = nullptr;
  PW_CUDA_TRY(cudaMallocAsync((void**)&dp, bytes, h.stream));
  cudaError_t e = cudaMallocAsync((void**)&dh, bytes, h.stream);
  if (e != cudaSuccess) {
    cudaFreeAsync(dp, h.stream);
    return fail(kOom, "pwgpu_apply_h: device allocation failed");
  }
  Status st = kOk;
  e = cudaMemcpyAsync(dp, psi, bytes, cudaMemcpyHostToDevice, h.stream);
  if (e != cudaSuccess) st = fail(kCuda, cudaGetErrorString(e));
  if (st == kOk) st = apply_h_device(h, spin, ik, dp, h.n_pw, nb, dh, h.n_pw, ph->precision, h.stream);
  if (st == kOk) {
    e = cudaMemcpyAsync(hpsi, dh, bytes, cudaMemcpyDeviceToHost, h.stream);
    if (e != cudaSuccess) st = fail(kCuda, cudaGetErrorString(e));
  }
  cudaFreeAsync(dp, h.stream);
  cudaFreeAsync(dh, h.stream);
  e = cudaStreamSynchronize(h.stream);
  if (st == kOk && e != cudaSuccess) st = fail(kCuda, cudaGetErrorString(e));
  return st;
}

pwgpu_status pwgpu_apply_h_device(pwgpu_handle* ph, int32_t spin, int32_t ik, const void* psi_dev, int64_t ldpsi,
                                  int32_t nb, void* hpsi_dev, int64_t ldh, void* stream) {
  if (!ph || !psi_dev || !hpsi_dev) return fail(kInvalid, "pwgpu_apply_h_device: NULL argument");
  Handle& h = ph->h;
  cudaStream_t s = stream ? (cudaStream_t)stream : h.stream;
  return apply_h_device(h, spin, ik, (const double2*)psi_dev, ldpsi, nb, (double2*)hpsi_dev, ldh, ph->precision, s);
}

pwgpu_status pwgpu_profile_apply_h(pwgpu_handle* ph, int32_t spin, int32_t ik, const void* psi_dev, int64_t ldpsi,
                                   int32_t nb, void* hpsi_dev, int64_t ldh, double* stage_ms, int32_t* launches) {
  if (!ph || !psi_dev || !hpsi_dev || !stage_ms || !launches) return fail(kInvalid, "pwgpu_profile_apply_h: NULL");
  Handle& h = ph->h;
  StageTimer tm;
  Status st = apply_h_device(h, spin, ik, (const double2*)psi_dev, ldpsi, nb, (double2*)hpsi_dev, ldh, ph->precision,
                             h.stream, &tm);
  cudaError_t e = cudaStreamSynchronize(h.stream);
  for (int k = 0; k < 8; ++k) { stage_ms[k] = 0.0; launches[k] = 0; }
  for (size_t i = 1; i < tm.events.size() && st == kOk && e == cudaSuccess; ++i) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, tm.events[i - 1], tm.events[i]);
    const int sg = tm.stage[i];
    if (sg >= 0 && sg < 8) { stage_ms[sg] += ms; launches[sg] += 1; }
  }
  for (cudaEvent_t ev : tm.events) cudaEventDestroy(ev);
  if (st != kOk) return st;
  if (e != cudaSuccess) return fail(kCuda, cudaGetErrorString(e));
  return kOk;
}

pwgpu_status pwgpu_set_precision(pwgpu_handle* ph, int32_t precision) {
  if (!ph) return fail(kInvalid, "pwgpu_set_precision: NULL handle");
  if (precision != 0 && precision != 1) return fail(kInvalid, "pwgpu_set_precision: unknown precision");
  ph->precision = precision;
  return kOk;
}

static Status convert_params(const pwgpu_scf_params* p, ScfParams& q) {
  q.n_bands = p->n_bands;
  q.max_iter = p->max_iter;
  q.conv_threshold = p->conv_threshold;
  q.energy_threshold = p->energy_threshold;
  q.mixing_beta = p->mixing_beta;
  q.mixing_ndim = p->mixing_ndim;
  q.mixing_mode = p->mixing_mode;
  q.kerker_q_tf = p->kerker_q_tf;
  q.smearing = p->smearing;
  q.sigma = p->smearing_sigma;
  q.diag_tol = p->diag_tol > 0.0 ? p->diag_tol : 1e-8;
  q.diag_max_iter = p->diag_max_iter > 0 ? p->diag_max_iter : 60;
  q.diag_extra_bands = p->diag_extra_bands;
  q.precision = p->precision;
  q.fp64_switch = p->fp64_switch;
  q.diag_tol_per_drho = p->diag_tol_per_drho > 0.0 ? p->diag_tol_per_drho : 3.0;
  q.diag_tol_cap = p->diag_tol_cap > 0.0 ? p->diag_tol_cap : 3e-2;
  q.verbose = p->verbose;
  q.starting_magnetization = p->starting_magnetization;
  q.fixed_magnetization = p->fixed_magnetization;
  q.tot_magnetization = p->tot_magnetization;
  if (q.starting_magnetization < -1.0 || q.starting_magnetization > 1.0)
    return fail(kInvalid, "scf params: starting_magnetization must lie in [-1, 1]");
  if (q.smearing < 0 || q.smearing > 4) return fail(kInvalid, "scf params: unknown smearing scheme");
  q.mixing_period = p->mixing_period > 0 ? p->mixing_period : 3;
  if (q.mixing_mode < 0 || q.mixing_mode > 5) return fail(kInvalid, "scf params: unknown mixing mode");
  return kOk;
}

static void copy_result(const ScfResult& r, pwgpu_scf_result* result) {
  result->total_energy = r.total_energy;
  result->harris_foulkes_energy = r.harris_foulkes_energy;
  result->free_energy = r.free_energy;
  result->energy_sigma0 = r.energy_sigma0;
  result->entropy_ts = r.entropy_ts;
  result->fermi_energy = r.fermi_energy;
  result->final_delta = r.final_delta;
  result->e_band = r.e_band;
  result->e_hartree = r.e_hartree;
  result->e_xc = r.e_xc;
  result->e_vxc = r.e_vxc;
  result->e_ewald = r.e_ewald;
  result->n_iterations = r.n_iterations;
  result->converged = r.converged;
  result->nspin = r.nspin;
  result->magnetization = r.magnetization;
  result->h_applications = r.h_applications;
  result->max_residual = r.max_residual;
  result->e_kinetic = r.e_kinetic;
  result->e_local = r.e_local;
  result->e_nonlocal = r.e_nonlocal;
}

pwgpu_status pwgpu_scf_run(pwgpu_handle* ph, const pwgpu_scf_params* p, const double* rho_init_r,
                           pwgpu_scf_result* result, double* eigenvalues, double* rho_r_out,
                           double* rho_g_basis_out) {
  if (!ph || !p || !rho_init_r || !result) return fail(kInvalid, "pwgpu_scf_run: NULL argument");
  ScfParams q;
  Status st = convert_params(p, q);
  if (st != kOk) return st;
  ScfResult r;
  st = scf_run(ph->h, q, rho_init_r, r, eigenvalues, rho_r_out, rho_g_basis_out);
  copy_result(r, result);
  return st;
}

pwgpu_status pwgpu_scf_iter1_from_rho_g(pwgpu_handle* ph, const pwgpu_scf_params* p, const double* rho_g_fft_in,
                                        pwgpu_scf_result* result, double* eigenvalues, double* rho_r_out,
                                        double* rho_g_fft_out, double* rho_r_in) {
  if (!ph || !p || !rho_g_fft_in || !result) return fail(kInvalid, "pwgpu_scf_iter1_from_rho_g: NULL argument");
  ScfParams q;
  Status st = convert_params(p, q);
  if (st != kOk) return st;
  ScfResult r;
  st = scf_iter1_from_rho_g(ph->h, q, rho_g_fft_in, r, eigenvalues, rho_r_out, rho_g_fft_out, rho_r_in);
  copy_result(r, result);
  return st;
}

pwgpu_status pwgpu_eigensolve(pwgpu_handle* ph, int32_t spin, int32_t ik, int32_t n_bands, double tol,
                              int32_t max_iter, const double* psi_in, double* evals, double* psi_out,
                              int32_t* iters, double* max_residual) {
  if (!ph || !evals) return fail(kInvalid, "pwgpu_eigensolve: NULL argument");
  PW_CUDA_TRY(cudaSetDevice(ph->h.device));
  return eigensolve_k(ph->h, spin, ik, n_bands, tol, max_iter, psi_in, evals, psi_out, iters, max_residual,
                      ph->precision);
}

pwgpu_status pwgpu_apply_h_packed(pwgpu_handle* ph, int32_t spin, const double* u, int32_t nb, double* hu) {
  if (!ph || !u || !hu) return fail(kInvalid, "pwgpu_apply_h_packed: NULL argument");
  Handle& h = ph->h;
  if (!h.gam.on) return fail(kState, "pwgpu_apply_h_packed: not a Gamma-real handle");
  if (spin < 0 || spin >= h.nspin) return fail(kInvalid, "pwgpu_apply_h_packed: spin index out of range");
  if (nb <= 0) return kOk;
  PW_CUDA_TRY(cudaSetDevice(h.device));
  const size_t bytes = (size_t)h.n_pw * nb * sizeof(double);
  double *du = nullptr, *dh = nullptr;
  if (cudaMalloc((void**)&du, bytes) != cudaSuccess || cudaMalloc((void**)&dh, bytes) != cudaSuccess) {
    cudaFree(du);
    cudaFree(dh);
    return fail(kOom, "pwgpu_apply_h_packed: allocation failed");
  }
  Status st = kOk;
  cudaError_t e = cudaMemcpyAsync(du, u, bytes, cudaMemcpyHostToDevice, h.stream);
  if (e == cudaSuccess) st = apply_h_real(h, spin, du, h.n_pw, nb, dh, h.n_pw, ph->precision, h.stream);
  if (e == cudaSuccess && st == kOk) e = cudaMemcpyAsync(hu, dh, bytes, cudaMemcpyDeviceToHost, h.stream);
  if (e == cudaSuccess && st == kOk) e = cudaStreamSynchronize(h.stream);
  cudaFree(du);
  cudaFree(dh);
  if (st != kOk) return st;
  if (e != cudaSuccess) return fail(kCuda, std::string("pwgpu_apply_h_packed: ") + cudaGetErrorString(e));
  return kOk;
}

pwgpu_status pwgpu_get_bands(pwgpu_handle* ph, int32_t spin, int32_t ik, int32_t n_bands, double* psi_out) {
  if (!ph || !psi_out) return fail(kInvalid, "pwgpu_get_bands: NULL argument");
  PW_CUDA_TRY(cudaSetDevice(ph->h.device));
  return bands_to_host(ph->h, spin, ik, n_bands, psi_out);
}

pwgpu_status pwgpu_mix(pwgpu_handle* ph, int32_t channel, int32_t mode, const double* rho_in, const double* rho_out,
                       double* rho_next, double beta, int32_t ndim, int32_t period, double q_tf) {
  if (!ph || !rho_in || !rho_out || !rho_next) return fail(kInvalid, "pwgpu_mix: NULL argument");
  PW_CUDA_TRY(cudaSetDevice(ph->h.device));
  return mix_host(ph->h, channel, mode, rho_in, rho_out, rho_next, beta, ndim, period, q_tf);
}

pwgpu_status pwgpu_get_projectors(const pwgpu_handle* ph, int32_t ik, double* b) {
  if (!ph || !b) return fail(kInvalid, "pwgpu_get_projectors: NULL argument");
  const Handle& h = ph->h;
  if (ik < 0 || ik >= h.n_k) return fail(kInvalid, "pwgpu_get_projectors: k-point index out of range");
  if (h.n_ch == 0) return kOk;
  PW_CUDA_TRY(cudaSetDevice(h.device));
  PW_CUDA_TRY(cudaMemcpy(b, h.kp[ik].b, (size_t)h.n_pw * h.n_ch * sizeof(double2), cudaMemcpyDeviceToHost));
  return kOk;
}

pwgpu_status pwgpu_initial_density(const pwgpu_handle* ph, double* rho_r) {
  if (!ph || !rho_r) return fail(kInvalid, "pwgpu_initial_density: NULL argument");
  const Handle& h = ph->h;
  if (!h.rho_sad) return fail(kState, "pwgpu_initial_density: the system was created with v_local_g given");
  PW_CUDA_TRY(cudaSetDevice(h.device));
  PW_CUDA_TRY(cudaMemcpy(rho_r, h.rho_sad, (size_t)h.g.N * sizeof(double), cudaMemcpyDeviceToHost));
  return kOk;
}

pwgpu_status pwgpu_get_local_potential(const pwgpu_handle* ph, double* v_local_g, double* rho_core_r) {
  if (!ph) return fail(kInvalid, "pwgpu_get_local_potential: NULL handle");
  const Handle& h = ph->h;
  PW_CUDA_TRY(cudaSetDevice(h.device));
  if (v_local_g)
    PW_CUDA_TRY(cudaMemcpy(v_local_g, h.v_local_g, (size_t)h.g.N * sizeof(double2), cudaMemcpyDeviceToHost));
  if (rho_core_r) {
    if (h.rho_core_r)
      PW_CUDA_TRY(cudaMemcpy(rho_core_r, h.rho_core_r, (size_t)h.g.N * sizeof(double), cudaMemcpyDeviceToHost));
    else
      std::fill(rho_core_r, rho_core_r + h.g.N, 0.0);
  }
  return kOk;
}

pwgpu_status pwgpu_mix_reset(pwgpu_handle* ph) {
  if (!ph) return fail(kInvalid, "pwgpu_mix_reset: NULL handle");
  return mix_reset(ph->h);
}

pwgpu_status pwgpu_density(pwgpu_handle* ph, int32_t n_bands, const double* occ, const double* psi, double* rho_r) {
  if (!ph || !occ || !psi || !rho_r) return fail(kInvalid, "pwgpu_density: NULL argument");
  PW_CUDA_TRY(cudaSetDevice(ph->h.device));
  return density_from_host(ph->h, n_bands, occ, psi, rho_r);
}

pwgpu_status pwgpu_symmetrize(pwgpu_handle* ph, double* rho_r) {
  if (!ph || !rho_r) return fail(kInvalid, "pwgpu_symmetrize: NULL argument");
  PW_CUDA_TRY(cudaSetDevice(ph->h.device));
  return symmetrize_host(ph->h, rho_r);
}

pwgpu_status pwgpu_potentials(pwgpu_handle* ph, const double* rho_r, double* veff_g, double* energies) {
  if (!ph || !rho_r) return fail(kInvalid, "pwgpu_potentials: NULL argument");
  PW_CUDA_TRY(cudaSetDevice(ph->h.device));
  return potentials_host(ph->h, rho_r, veff_g, energies);
}

pwgpu_status pwgpu_occupations(int32_t n_sets, int32_t nb, const double* ev, const double* weights,
                               double n_electrons, double sigma, int32_t smearing, double spin_factor,
                               int32_t find_fermi, double* fermi_energy, double* occ, double* entropy_ts) {
  if (!ev || !weights || !fermi_energy || n_sets < 1 || nb < 1)
    return fail(kInvalid, "pwgpu_occupations: bad argument");
  if (smearing < 0 || smearing > 4 || !(sigma >= 0.0) || !(spin_factor > 0.0))
    return fail(kInvalid, "pwgpu_occupations: smearing, sigma or spin_factor out of range");
  return occupations_host(n_sets, nb, ev, weights, n_electrons, sigma, smearing, spin_factor, find_fermi != 0,
                          fermi_energy, occ, entropy_ts);
}

pwgpu_status pwgpu_small_geneig(int32_t batch, int32_t m, int32_t nev, const double* H, const double* S,
                                double* evals, double* C) {
  if (!H || !S || !evals || !C || batch < 1) return fail(kInvalid, "pwgpu_small_geneig: bad argument");
  if (m < 1 || m > 64 || nev < 1 || nev > m) return fail(kInvalid, "pwgpu_small_geneig: need 1 <= nev <= m <= 64");
  const size_t mm = (size_t)m * m * batch;
  double2 *dh = nullptr, *ds = nullptr, *dc = nullptr;
  double* de = nullptr;
  int* dst = nullptr;
  Status st = kOk;
  auto cleanup = [&]() { cudaFree(dh); cudaFree(ds); cudaFree(dc); cudaFree(de); cudaFree(dst); };
  if (cudaMalloc((void**)&dh, mm * sizeof(double2)) != cudaSuccess || cudaMalloc((void**)&ds, mm * sizeof(double2)) != cudaSuccess ||
      cudaMalloc((void**)&dc, (size_t)m * nev * batch * sizeof(double2)) != cudaSuccess ||
      cudaMalloc((void**)&de, (size_t)nev * batch * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&dst, batch * sizeof(int)) != cudaSuccess) {
    cleanup();
    return fail(kOom, "pwgpu_small_geneig: allocation failed");
  }
  // the first failing copy, launch or synchronisation ends the call
  cudaError_t e = cudaMemcpy(dh, H, mm * sizeof(double2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(ds, S, mm * sizeof(double2), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cleanup();
    return fail(kCuda, std::string("pwgpu_small_geneig: copy to the device: ") + cudaGetErrorString(e));
  }
  st = small_geneig_batched(dh, ds, m, (long)m * m, m, nev, batch, de, dc, m, (long)m * nev, dst, 0);
  std::vector<int> stat(batch, 0);
  if (st == kOk) {
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(evals, de, (size_t)nev * batch * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(C, dc, (size_t)m * nev * batch * sizeof(double2), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(stat.data(), dst, batch * sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = fail(kCuda, std::string("pwgpu_small_geneig: ") + cudaGetErrorString(e));
  }
  if (st == kOk)
    for (int b = 0; b < batch; ++b)
      if (stat[b] == 1) { st = fail(kInvalid, "pwgpu_small_geneig: S is not positive definite"); break; }
  cleanup();
  return st;
}

pwgpu_status pwgpu_dense_eigh(int32_t m, int32_t nev, int32_t complex_matrix, const double* A, double* w,
                              double* Z, int32_t* cluster_ctas, double* kernel_ms) {
  if (!A || !w || !Z) return fail(kInvalid, "pwgpu_dense_eigh: NULL argument");
  if (m < 1 || nev < 1 || nev > m) return fail(kInvalid, "pwgpu_dense_eigh: need 1 <= nev <= m");
  const bool cpx = complex_matrix != 0;
  if (!eigh_cluster_supported(m, cpx)) return fail(kInvalid, "pwgpu_dense_eigh: m too large for the cluster solver");
  if (cluster_ctas) *cluster_ctas = eigh_cluster_size(m, cpx);
  const size_t es = cpx ? sizeof(double2) : sizeof(double);
  void *da = nullptr, *dz = nullptr;
  double *dw = nullptr, *dwork = nullptr;
  int* dst = nullptr;
  auto cleanup = [&]() { cudaFree(da); cudaFree(dz); cudaFree(dw); cudaFree(dwork); cudaFree(dst); };
  if (cudaMalloc(&da, (size_t)m * m * es) != cudaSuccess || cudaMalloc(&dz, (size_t)m * nev * es) != cudaSuccess ||
      cudaMalloc((void**)&dw, (size_t)nev * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&dwork, eigh_cluster_work_doubles(m, nev) * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&dst, sizeof(int)) != cudaSuccess) {
    cleanup();
    return fail(kOom, "pwgpu_dense_eigh: allocation failed");
  }
  cudaError_t e = cudaMemcpy(da, A, (size_t)m * m * es, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cleanup();
    return fail(kCuda, std::string("pwgpu_dense_eigh: ") + cudaGetErrorString(e));
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (kernel_ms) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
  }
  Status st = cpx ? eigh_cluster(static_cast<const double2*>(da), m, m, nev, dw, static_cast<double2*>(dz), m, dwork,
                                 dst, 0)
                  : eigh_cluster(static_cast<const double*>(da), m, m, nev, dw, static_cast<double*>(dz), m, dwork,
                                 dst, 0);
  if (kernel_ms) {
    cudaEventRecord(e1, 0);
    float ms = 0.f;
    if (cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) *kernel_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  int flag = 0;
  if (st == kOk) {
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(w, dw, (size_t)nev * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(Z, dz, (size_t)m * nev * es, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&flag, dst, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = fail(kCuda, std::string("pwgpu_dense_eigh: ") + cudaGetErrorString(e));
  }
  if (st == kOk && flag != 0) st = fail(kNotConverged, "pwgpu_dense_eigh: non-finite eigenpair");
  cleanup();
  return st;
}

pwgpu_status pwgpu_dense_cholesky_inverse(int32_t q, int32_t complex_matrix, const double* G, double* Ri,
                                          double* rdiag, int32_t* info, int32_t* cluster_ctas, double* kernel_ms) {
  if (!G || !Ri || !info) return fail(kInvalid, "pwgpu_dense_cholesky_inverse: NULL argument");
  if (q < 1) return fail(kInvalid, "pwgpu_dense_cholesky_inverse: need q >= 1");
  const bool cpx = complex_matrix != 0;
  if (cluster_ctas) *cluster_ctas = chol_inv_cluster_size(q, cpx);
  const size_t es = cpx ? sizeof(double2) : sizeof(double);
  const size_t bytes = (size_t)q * q * es;
  void *dg = nullptr, *dr = nullptr;
  double* dd = nullptr;
  int* di = nullptr;
  auto cleanup = [&]() { cudaFree(dg); cudaFree(dr); cudaFree(dd); cudaFree(di); };
  if (cudaMalloc(&dg, bytes) != cudaSuccess || cudaMalloc(&dr, bytes) != cudaSuccess ||
      cudaMalloc((void**)&dd, (size_t)q * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&di, sizeof(int)) != cudaSuccess) {
    cleanup();
    return fail(kOom, "pwgpu_dense_cholesky_inverse: allocation failed");
  }
  cudaError_t e = cudaMemcpy(dg, G, bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cleanup();
    return fail(kCuda, std::string("pwgpu_dense_cholesky_inverse: ") + cudaGetErrorString(e));
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (kernel_ms) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
  }
  Status st = cpx ? chol_inv(static_cast<double2*>(dg), q, static_cast<double2*>(dr), dd, di, 0)
                  : chol_inv(static_cast<double*>(dg), q, static_cast<double*>(dr), dd, di, 0);
  if (kernel_ms) {
    cudaEventRecord(e1, 0);
    float ms = 0.f;
    if (cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) *kernel_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (st == kOk) {
    int inf = 0;
    e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&inf, di, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(Ri, dr, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && rdiag) e = cudaMemcpy(rdiag, dd, (size_t)q * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) st = fail(kCuda, std::string("pwgpu_dense_cholesky_inverse: ") + cudaGetErrorString(e));
    *info = inf;
  }
  cleanup();
  return st;
}

pwgpu_status pwgpu_kernel_launches(int64_t* count) {
  if (!count) return fail(kInvalid, "pwgpu_kernel_launches: NULL argument");
  *count = launch_counter().load();
  return kOk;
}

pwgpu_status pwgpu_get_stream(const pwgpu_handle* ph, void** stream) {
  if (!ph || !stream) return fail(kInvalid, "pwgpu_get_stream: NULL argument");
  *stream = (void*)ph->h.stream;
  return kOk;
}

pwgpu_status pwgpu_get_dims(const pwgpu_handle* ph, int32_t* n_pw, int64_t* n_grid, int32_t* n_ch) {
  if (!ph) return fail(kInvalid, "pwgpu_get_dims: NULL handle");
  if (n_pw) *n_pw = ph->h.n_pw;
  if (n_grid) *n_grid = ph->h.g.N;
  if (n_ch) *n_ch = ph->h.n_ch;
  return kOk;
}

}  // extern "C"
