// Device-resident state of one pwgpu handle: FFT grid plans and sphere
// maps, per-k projector matrices, potentials and scratch buffers.
#pragma once

#include <cublas_v2.h>
#include <cusolverDn.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "pw_common.cuh"

namespace pwgpu {

Status fail(int code, const std::string& msg);  // records the thread's last error, returns code
std::string last_error_message();                // the calling thread's last recorded error

// Sphere <-> grid maps and per-axis FFT plans.  Grid flat index is
// (i0*d1 + i1)*d2 + i2, x slowest, as in the reference's miller_to_idx.
// The sphere occupies |n_i| <= m_i; the "compact" x range holds Xp = 2*m0+1
// planes and the compact y range Yp = 2*m1+1 rows, so the z-direction FFTs
// run only on the Xp*Yp columns that can carry plane-wave coefficients.
struct GridMaps {
  int d[3] = {0, 0, 0};
  long N = 0;
  int m[3] = {0, 0, 0};
  int Xp = 0, Yp = 0, ncol = 0;
  FftPlan plan[3];
  double2* tw64[3] = {nullptr, nullptr, nullptr};
  float2* tw32[3] = {nullptr, nullptr, nullptr};
  // points sorted by column c = (n0+m0)*Yp + (n1+m1), then by basis order
  int* col_start = nullptr;  // ncol+1
  int* pt_ig = nullptr;      // n_pw: basis index of sorted point
  int* pt_col = nullptr;     // n_pw: column of sorted point
  int* pt_z = nullptr;       // n_pw: wrapped z index
  int* g_to_fft = nullptr;   // n_pw (basis order): flat grid index
  // tile widths chosen for the FFT kernels (lines per block)
  int wz = 1, wy = 1, wx = 1;
  int wz32 = 1, wy32 = 1, wx32 = 1;  // FP32 tiles: measured at handle creation
};

struct KPointData {
  double* kinetic = nullptr;    // n_pw
  double2* b = nullptr;         // n_pw x n_ch, column-major
  float2* b32 = nullptr;        // FP32 copy for the mixed form (lazily made)
  double weight = 0.0;
};

// Gamma-only systems: wavefunctions with psi(-G) = conj(psi(G)) stored as
// real vectors of n_pw entries, u = [Re psi(0), sqrt2 Re psi(G_p),
// sqrt2 Im psi(G_p)] over the half sphere G_p > 0 (lexicographic in the
// Miller indices), so complex inner products are real dot products.
struct GammaData {
  bool on = false;
  int nh = 0;                 // half-sphere points; n_pw = 2 nh + 1
  int zero = 0;               // basis index of G = 0
  int* half_idx = nullptr;    // nh: basis index of G_p
  int* half_neg = nullptr;    // nh: basis index of -G_p
  double* kin_packed = nullptr;  // n_pw: |G|^2 term in packed order
  double* b_real = nullptr;      // n_pw x n_ch packed projectors
};

struct Handle {
  int device = 0;
  int n_pw = 0, n_k = 0, n_ch = 0, n_atoms = 0, nspin = 1, n_sym = 0;
  double n_electrons = 0.0, omega = 0.0, e_ewald = 0.0;
  GridMaps g;
  std::vector<KPointData> kp;
  int* ch_atom = nullptr;          // n_ch: atom of channel
  int* atom_ch_start = nullptr;    // n_atoms+1
  int* d_off = nullptr;            // n_atoms: offset of atom block in d_vals
  double* d_vals = nullptr;        // concatenated blocks
  double2* v_local_g = nullptr;    // N
  double* g_squared = nullptr;     // N
  double* rho_core_r = nullptr;    // N or null
  double* rho_sad = nullptr;       // N: start density built on the device, or null
  int* sym_src = nullptr;          // n_sym x N
  double* sym_arg = nullptr;       // n_sym x N
  // effective potential per spin in real space
  double* veff_r[2] = {nullptr, nullptr};
  float* veff_r32[2] = {nullptr, nullptr};
  // the same potential z-major ([z][x][y]): the fused y/x pass reads one z-plane contiguously
  double* veff_rz[2] = {nullptr, nullptr};
  float* veff_rz32[2] = {nullptr, nullptr};
  // H|psi> scratch: band-chunked compact grids (L2-resident per chunk)
  int chunk = 1;
  void* work_a = nullptr;   // chunk * ncol * d2 complex (FP64 size)
  void* work_b = nullptr;   // chunk * Xp * d1 * d2 complex
  double2* nl_p = nullptr;  // n_ch x max_nb
  double2* nl_q = nullptr;
  int nl_cap = 0;
  double2* tmp_grid = nullptr;  // N complex scratch
  cudaStream_t stream = nullptr;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
  double2* solver_work = nullptr;
  size_t solver_work_len = 0;
  int* solver_info = nullptr;
  struct ScfState* scf = nullptr;  // device state of the SCF loop (scf.cu)
  struct NlMixed* nlm = nullptr;   // split projector operands of the mixed form (nl_mixed.cu)
  struct NlMixed* nlm_real = nullptr;  // the same for the packed real projectors of Gamma-real handles
  GammaData gam;
  // per-call scratch of the Gamma path (lane-owned like nl_p / nl_q)
  double2* gam_c1 = nullptr;
  double2* gam_c2 = nullptr;
  long gam_ccap = 0;          // complex pseudo-band columns of gam_c1 / gam_c2
  double* gam_p = nullptr;
  double* gam_q = nullptr;
  int gam_pcap = 0;
  bool trace = false;  // per-iteration eigensolver lines on stderr (PWGPU_TRACE set at create)
  int lanes = 0;       // concurrent (spin, k) eigensolves in the SCF loop; 0 = automatic
  std::string last_error;
};

void release_scf(Handle& h);

// Optional per-launch event trail of an H|psi> call (profiling entry point).
// stage ids: -1 start, 0..4 the five FFT kernels, 5 B^H psi, 6 D apply, 7 B Q.
struct StageTimer {
  std::vector<cudaEvent_t> events;
  std::vector<int> stage;
};

// Records a CUDA event for stage `stage` when t is non-null (hpsi.cu).
void mark(StageTimer* t, int stage, cudaStream_t s);

// Q = D P over the handle's nl_p / nl_q buffers (block-diagonal D).
Status apply_d_blocks(Handle& h, int nb, cudaStream_t s);

// 3xBF16 tensor-core form of the Kleinman-Bylander term, hpsi += B D B^H psi
// (nl_mixed.cu); used by the mixed form when nl_mixed_eligible(h).
bool nl_mixed_eligible(const Handle& h);
Status nonlocal_mixed(Handle& h, int ik, const double2* psi, long ldpsi, int nb, double2* hpsi, long ldh,
                      cudaStream_t s, StageTimer* tm = nullptr);
// The same for packed real bands of a Gamma-real handle: hu += B_r D B_r^T u.
Status nonlocal_mixed_real(Handle& h, const double* u, long ldu, int nb, double* hu, long ldh, cudaStream_t s);
void release_nl_mixed(Handle& h);

// Per-band kinetic and nonlocal expectations of nb columns of V at k-point ik
// (packed real on Gamma handles), into host t_kin and t_nl (components.cu).
// d_out: device scratch of 2 nb doubles.
Status band_energy_terms(Handle& h, int ik, const double2* V, long ldv, int nb, double* d_out, double* t_kin,
                         double* t_nl, cudaStream_t s);

// Grid-map construction and the H|psi> launcher (hpsi.cu).
Status build_grid_maps(Handle& h, const int* miller_host);
Status apply_h_device(Handle& h, int spin, int ik, const double2* psi, long ldpsi, int nb, double2* hpsi,
                      long ldh, int precision, cudaStream_t stream, StageTimer* timer = nullptr);
Status set_veff_from_g(Handle& h, int spin, const double2* veff_g_dev, cudaStream_t stream);
// Refresh the z-major copies (veff_rz, veff_rz32) of veff_r[spin].
Status veff_zmajor(Handle& h, int spin, cudaStream_t stream);
Status ensure_nl_capacity(Handle& h, int nb);
// P = B^H psi into h.nl_p and Q = D P into h.nl_q (FP64), nb columns.
Status nonlocal_pq(Handle& h, int ik, const double2* psi, long ldpsi, int nb, cudaStream_t s,
                   StageTimer* tm = nullptr);

// Local part of H|psi> only (kinetic + V_eff through the FFT pipeline).
Status apply_local_device(Handle& h, int spin, int ik, const double2* psi, long ldpsi, int nb, double2* hpsi,
                          long ldh, int precision, cudaStream_t s, StageTimer* tm = nullptr);

// Radial data for building the projector matrices on the device (setup.cu):
// G and k vectors, atoms, and per species its radial mesh and projectors.
struct ProjectorSource {
  const double* gvec = nullptr;        // n_pw x 3, Å^-1
  const double* kpts = nullptr;        // n_k x 3, Å^-1
  const double* atom_tau = nullptr;    // n_atoms x 3, Å
  const int* atom_species = nullptr;   // n_atoms
  int n_species = 0;
  const int* species_mesh = nullptr;   // n_species
  const double* radial_r = nullptr;    // concatenated meshes
  const double* radial_rab = nullptr;
  const int* species_nbeta = nullptr;  // n_species
  const int* beta_l = nullptr;         // per projector, species by species
  const double* beta_r = nullptr;      // per projector, on its species' mesh
};
// B of every k into h.kp[k].b (allocated by the caller); needs h.atom_ch_start.
Status build_projectors_device(Handle& h, const ProjectorSource& src);

// Radial data for the local pseudopotential, the NLCC core density and the
// start density on the full grid (setup.cu); meshes as in ProjectorSource.
struct LocalSource {
  const double* recip = nullptr;        // 3 x 3: rows b1, b2, b3 (Å^-1)
  const double* atom_tau = nullptr;     // n_atoms x 3, Å
  const int* atom_species = nullptr;    // n_atoms
  int n_atoms = 0;
  int n_species = 0;
  const int* species_mesh = nullptr;
  const double* radial_r = nullptr;
  const double* radial_rab = nullptr;
  const double* species_zval = nullptr;  // n_species
  const double* vloc_r = nullptr;        // concatenated V_loc(r), eV
  const int* species_flags = nullptr;    // bit 0: core charge, bit 1: rho_atom
  const double* core_r = nullptr;        // concatenated, or null
  const double* rho_atom_r = nullptr;    // concatenated, or null
  double gaussian_sigma = 1.0;           // Å
};
// V_loc(G) into v_local_g (N complex, allocated), rho_core(r) into *rho_core_r
// (allocated here when null and a species has a core charge), the start
// density into *rho_start when rho_start is given.  Needs the grid maps.
Status build_local_device(Handle& h, const LocalSource& src, double2* v_local_g, double** rho_core_r,
                          double** rho_start);

// Gamma path (gamma.cu).  build_gamma decides eligibility (one k-point with
// a kinetic term and projectors symmetric under G -> -G) from host data.
Status build_gamma(Handle& h, const int* miller_host, const double* kinetic_host, const int* atom_ch_start_host,
                   const double* d_blocks_host);
void release_gamma(Handle& h);
void release_gamma_scratch(Handle& h);
// H u for nb packed real bands (local pipeline on pairs of bands packed into
// one complex vector, then real projector GEMMs).
Status apply_h_real(Handle& h, int spin, const double* u, long ldu, int nb, double* hu, long ldh, int precision,
                    cudaStream_t s);
// Capacity of the Gamma path's P / Q buffers (n_ch x nb), and Q = D P on them.
Status ensure_gamma_pq(Handle& h, int nb);
Status apply_d_real(Handle& h, int nb, cudaStream_t s);
// P = B_r^T u into h.gam_p and Q = D P into h.gam_q for nb packed real bands.
Status nonlocal_pq_real(Handle& h, const double* u, long ldu, int nb, cudaStream_t s);
// rho += sum_b fw[b] |psi_b(r)|^2 for nb packed real bands (fw on the host).
Status density_accumulate_real(Handle& h, const double* u, long ldu, const std::vector<double>& fw, double* rho,
                               cudaStream_t s);
// packed real <-> complex full-sphere coefficients (Gamma-real columns)
Status gamma_pack(Handle& h, const double2* x, long ldx, int ncols, double* u, long ldu, cudaStream_t s);
Status gamma_unpack(Handle& h, const double* u, long ldu, int ncols, double2* x, long ldx, cudaStream_t s);

// Local part of H|psi> (kinetic + V_eff, no projectors) with the FFT
// intermediates in caller-provided device scratch; fails with kInvalid when
// one band does not fit.
Status local_apply_on_scratch(Handle& h, int spin, int ik, const double2* psi, long ldpsi, int nb, double2* hpsi,
                              long ldh, int precision, cudaStream_t s, void* scratch, size_t scratch_bytes);

// rho(r) += sum_b fw[b] |psi_b(r)|^2 over nb bands (FP64 FFTs); fw on device.
Status density_accumulate(Handle& h, const double2* psi, long ldpsi, int nb, const double* fw_dev, double* rho,
                          cudaStream_t stream);

// 3-D FFT of a full grid (unnormalised), sign -1 forward / +1 inverse,
// in place on device memory (used for potentials and density paths).
Status fft3d_full(Handle& h, double2* data, int sign, cudaStream_t stream);

}  // namespace pwgpu
