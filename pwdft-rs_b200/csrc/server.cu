// Serving front: a job queue with HBM-footprint admission in front of
// pwgpu_scf_run.  Workers are host threads; each runs one job at a time on
// its own handle (own stream, BLAS/solver handles, device state), so jobs
// overlap on the GPU exactly as far as their kernels leave room.
#include <pwgpu.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "handle.hpp"

using pwgpu::fail;
using pwgpu::kInvalid;
using pwgpu::kOk;
using pwgpu::kOom;
using pwgpu::kTimeout;
using pwgpu::Status;

namespace {

using Clock = std::chrono::steady_clock;

double seconds_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}

// Owned copy of a pwgpu_system and its arrays (the caller's are borrowed for
// the submit call only).
struct SystemCopy {
  pwgpu_system sys{};
  std::vector<int32_t> miller, atom_ch_start, sym_src, atom_species, species_mesh, species_nbeta, beta_l, species_flags;
  std::vector<double> k_weights, kinetic, proj_b, d_blocks, v_local_g, g_squared, rho_core, sym_arg, g_cart, k_cart,
      atom_tau, radial_r, radial_rab, beta_r, recip, species_zval, vloc_r, core_r, rho_atom_r;

  Status copy_from(const pwgpu_system& s) {
    if (s.n_pw <= 0 || s.n_k <= 0 || s.dims[0] <= 0 || s.dims[1] <= 0 || s.dims[2] <= 0)
      return fail(kInvalid, "pwgpu_server_submit: n_pw, n_k and dims must be positive");
    if (!s.miller || !s.k_weights || !s.kinetic || !s.g_squared)
      return fail(kInvalid, "pwgpu_server_submit: required system array is NULL");
    if (!s.v_local_g && (!s.recip || !s.species_zval || !s.vloc_r || !s.species_flags || !s.atom_tau ||
                         !s.atom_species || s.n_species <= 0 || !s.species_mesh || !s.radial_r || !s.radial_rab ||
                         s.n_atoms <= 0))
      return fail(kInvalid, "pwgpu_server_submit: local radial data missing");
    if (s.n_ch > 0 && (!s.atom_ch_start || !s.d_blocks || s.n_atoms <= 0))
      return fail(kInvalid, "pwgpu_server_submit: projector arrays missing");
    if (s.n_ch > 0 && !s.proj_b &&
        (!s.g_cart || !s.k_cart || !s.atom_tau || !s.atom_species || s.n_species <= 0 || !s.species_mesh ||
         !s.radial_r || !s.radial_rab || !s.species_nbeta || !s.beta_l || !s.beta_r))
      return fail(kInvalid, "pwgpu_server_submit: projector radial data missing");
    if (s.n_sym > 1 && (!s.sym_src || !s.sym_arg))
      return fail(kInvalid, "pwgpu_server_submit: symmetry map missing");
    const size_t N = (size_t)s.dims[0] * s.dims[1] * s.dims[2];
    const size_t n = (size_t)s.n_pw, nk = (size_t)s.n_k;
    sys = s;
    miller.assign(s.miller, s.miller + 3 * n);
    k_weights.assign(s.k_weights, s.k_weights + nk);
    kinetic.assign(s.kinetic, s.kinetic + nk * n);
    g_squared.assign(s.g_squared, s.g_squared + N);
    sys.miller = miller.data();
    sys.k_weights = k_weights.data();
    sys.kinetic = kinetic.data();
    sys.g_squared = g_squared.data();
    // atoms and species meshes: shared by the projector and local radial forms
    const bool radial = (s.n_ch > 0 && !s.proj_b) || !s.v_local_g;
    size_t mesh_tot = 0;
    if (radial) {
      const int ns = s.n_species;
      atom_tau.assign(s.atom_tau, s.atom_tau + 3L * s.n_atoms);
      atom_species.assign(s.atom_species, s.atom_species + s.n_atoms);
      species_mesh.assign(s.species_mesh, s.species_mesh + ns);
      for (int q = 0; q < ns; ++q) mesh_tot += (size_t)species_mesh[q];
      radial_r.assign(s.radial_r, s.radial_r + mesh_tot);
      radial_rab.assign(s.radial_rab, s.radial_rab + mesh_tot);
      sys.atom_tau = atom_tau.data();
      sys.atom_species = atom_species.data();
      sys.species_mesh = species_mesh.data();
      sys.radial_r = radial_r.data();
      sys.radial_rab = radial_rab.data();
    }
    if (s.v_local_g) {
      v_local_g.assign(s.v_local_g, s.v_local_g + 2 * N);
      sys.v_local_g = v_local_g.data();
    } else {
      const int ns = s.n_species;
      recip.assign(s.recip, s.recip + 9);
      species_zval.assign(s.species_zval, s.species_zval + ns);
      species_flags.assign(s.species_flags, s.species_flags + ns);
      vloc_r.assign(s.vloc_r, s.vloc_r + mesh_tot);
      bool any_core = false, any_atom = false;
      for (int q = 0; q < ns; ++q) {
        any_core = any_core || (species_flags[q] & 1);
        any_atom = any_atom || (species_flags[q] & 2);
      }
      if ((any_core && !s.core_r) || (any_atom && !s.rho_atom_r))
        return fail(kInvalid, "pwgpu_server_submit: flagged core or atomic density missing");
      if (any_core) core_r.assign(s.core_r, s.core_r + mesh_tot);
      if (any_atom) rho_atom_r.assign(s.rho_atom_r, s.rho_atom_r + mesh_tot);
      sys.recip = recip.data();
      sys.species_zval = species_zval.data();
      sys.species_flags = species_flags.data();
      sys.vloc_r = vloc_r.data();
      sys.core_r = any_core ? core_r.data() : nullptr;
      sys.rho_atom_r = any_atom ? rho_atom_r.data() : nullptr;
    }
    if (s.n_ch > 0) {
      if (s.proj_b) {
        proj_b.assign(s.proj_b, s.proj_b + nk * n * (size_t)s.n_ch * 2);
      } else {
        // radial form of the projectors: G and k vectors and betas (atoms and
        // meshes are copied above)
        const int ns = s.n_species;
        g_cart.assign(s.g_cart, s.g_cart + 3 * n);
        k_cart.assign(s.k_cart, s.k_cart + 3 * nk);
        species_nbeta.assign(s.species_nbeta, s.species_nbeta + ns);
        size_t nbeta = 0, beta_tot = 0;
        for (int q = 0; q < ns; ++q) {
          nbeta += (size_t)species_nbeta[q];
          beta_tot += (size_t)species_nbeta[q] * species_mesh[q];
        }
        beta_l.assign(s.beta_l, s.beta_l + nbeta);
        beta_r.assign(s.beta_r, s.beta_r + beta_tot);
        sys.g_cart = g_cart.data();
        sys.k_cart = k_cart.data();
        sys.species_nbeta = species_nbeta.data();
        sys.beta_l = beta_l.data();
        sys.beta_r = beta_r.data();
      }
      atom_ch_start.assign(s.atom_ch_start, s.atom_ch_start + s.n_atoms + 1);
      size_t nd = 0;
      for (int a = 0; a < s.n_atoms; ++a) {
        const long nc = (long)atom_ch_start[a + 1] - atom_ch_start[a];
        if (nc < 0) return fail(kInvalid, "pwgpu_server_submit: atom_ch_start is not ascending");
        nd += (size_t)nc * nc;
      }
      d_blocks.assign(s.d_blocks, s.d_blocks + nd);
      sys.proj_b = s.proj_b ? proj_b.data() : nullptr;
      sys.atom_ch_start = atom_ch_start.data();
      sys.d_blocks = d_blocks.data();
    } else {
      sys.proj_b = nullptr;
      sys.atom_ch_start = nullptr;
      sys.d_blocks = nullptr;
    }
    if (s.rho_core_r) {
      rho_core.assign(s.rho_core_r, s.rho_core_r + N);
      sys.rho_core_r = rho_core.data();
    }
    if (s.n_sym > 1) {
      sym_src.assign(s.sym_src, s.sym_src + (size_t)s.n_sym * N);
      sym_arg.assign(s.sym_arg, s.sym_arg + (size_t)s.n_sym * N);
      sys.sym_src = sym_src.data();
      sys.sym_arg = sym_arg.data();
    } else {
      sys.sym_src = nullptr;
      sys.sym_arg = nullptr;
    }
    return kOk;
  }
};

// Device bytes a job's handle and SCF state will hold (allocation sizes of
// api.cu, hpsi.cu, scf.cu, lobpcg.cu and nl_mixed.cu, rounded up), plus a
// fixed allowance for library workspaces.
int64_t footprint(const pwgpu_system& s, const pwgpu_scf_params& p, int lanes_per_job) {
  const double N = (double)s.dims[0] * s.dims[1] * s.dims[2];
  const double n = s.n_pw, nk = s.n_k, nch = std::max(0, s.n_ch), ns = s.nspin;
  const double nb = p.n_bands;
  const double nd = std::min(n, nb + std::max(2.0, std::floor(nb / 8.0)));
  const double ndim = std::max(1, p.mixing_ndim);
  const double nsym = std::max(1, s.n_sym);
  double b = 0.0;
  b += nk * (8.0 * n + 16.0 * n * nch);                      // kinetic, projectors
  b += 32.0 * N + 12.0 * nsym * N + 12.0 * ns * N + 16.0 * N;  // grids, symmetry map, V_eff, scratch
  const double fft = std::min(96.0e6, 64.0 * 32.0 * N);      // band-chunk FFT intermediates
  b += fft;
  const double eigw = 64.0 * n * nd + 16.0 * 45.0 * nd * nd;  // eigensolver workspace
  b += ns * nk * 96.0 * n * nd + eigw;                      // Ritz blocks [X|W|P], H applied
  const int items = (int)(ns * nk);
  const int lanes = items > 1 ? std::min(items, lanes_per_job > 0 ? lanes_per_job : 8) : 0;
  b += lanes * (eigw + fft / std::max(1, lanes));
  b += 8.0 * N * 16.0 + (ns > 1 ? 56.0 * N : 0.0);           // SCF grids
  b += (ns > 1 ? 2.0 : 1.0) * ndim * 16.0 * N;               // mixing history
  if (nch >= 256 && n >= 4096) b += (1.0 + lanes) * nk * 24.0 * n * nch;  // split projector operands
  return (int64_t)(1.2 * b) + ((int64_t)64 << 20);
}

struct Job {
  int64_t id = 0;
  SystemCopy sys;
  pwgpu_scf_params params{};
  std::vector<double> rho_init;
  int64_t bytes = 0;
  int state = PWGPU_JOB_QUEUED;
  pwgpu_status status = PWGPU_OK;
  std::string error;
  pwgpu_scf_result result{};
  std::vector<double> evals;
  Clock::time_point t_submit, t_start, t_done;
};

}  // namespace

struct pwgpu_server {
  pwgpu_server_options opt{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Job>> queue;
  std::map<int64_t, std::shared_ptr<Job>> jobs;
  std::deque<int64_t> finished;  // done, not yet returned by wait_any
  int64_t budget = 0, in_use = 0, peak = 0, next_id = 1;
  int64_t submitted = 0, running = 0, done = 0, failed = 0;
  bool stop = false;
  std::vector<std::thread> workers;

  bool head_fits() const {
    if (queue.empty()) return false;
    return in_use == 0 || in_use + queue.front()->bytes <= budget;
  }

  void worker_main() {
    cudaSetDevice(opt.device);
    for (;;) {
      std::shared_ptr<Job> job;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || head_fits(); });
        if (stop) return;
        job = queue.front();
        queue.pop_front();
        in_use += job->bytes;
        peak = std::max(peak, in_use);
        job->state = PWGPU_JOB_RUNNING;
        job->t_start = Clock::now();
        ++running;
      }
      pwgpu_options o{opt.device, opt.precision, opt.lanes_per_job > 0 ? opt.lanes_per_job : 2, 0};
      pwgpu_handle* h = nullptr;
      pwgpu_status st = pwgpu_create(&job->sys.sys, &o, &h);
      if (st == PWGPU_OK && job->rho_init.empty()) {
        // start density built on the device with the local potential
        job->rho_init.resize((size_t)job->sys.sys.dims[0] * job->sys.sys.dims[1] * job->sys.sys.dims[2]);
        st = pwgpu_initial_density(h, job->rho_init.data());
      }
      if (st == PWGPU_OK)
        st = pwgpu_scf_run(h, &job->params, job->rho_init.data(), &job->result, job->evals.data(), nullptr, nullptr);
      const std::string err = st == PWGPU_OK ? std::string() : std::string(pwgpu_last_error());
      pwgpu_destroy(h);
      {
        std::lock_guard<std::mutex> lk(mu);
        in_use -= job->bytes;
        job->status = st;
        job->error = err;
        job->state = PWGPU_JOB_DONE;
        job->t_done = Clock::now();
        --running;
        ++done;
        if (st != PWGPU_OK && st != PWGPU_E_NOT_CONVERGED) ++failed;
        finished.push_back(job->id);
        // the owned system is no longer needed once the handle was built
        job->sys = SystemCopy();
        job->rho_init.clear();
        job->rho_init.shrink_to_fit();
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }

  void fill_info(const Job& j, pwgpu_job_info* info) const {
    if (!info) return;
    const auto now = Clock::now();
    info->state = j.state;
    info->status = j.status;
    info->footprint_bytes = j.bytes;
    info->queue_s = seconds_between(j.t_submit, j.state == PWGPU_JOB_QUEUED ? now : j.t_start);
    info->run_s = j.state == PWGPU_JOB_QUEUED ? 0.0
                  : seconds_between(j.t_start, j.state == PWGPU_JOB_DONE ? j.t_done : now);
  }
};

extern "C" {

pwgpu_status pwgpu_server_create(const pwgpu_server_options* opt, pwgpu_server** out) {
  if (!out) return fail(kInvalid, "pwgpu_server_create: NULL output");
  *out = nullptr;
  pwgpu_server_options o = opt ? *opt : pwgpu_server_options{};
  if (o.workers < 0 || o.lanes_per_job < 0 || o.hbm_budget_bytes < 0)
    return fail(kInvalid, "pwgpu_server_create: negative option");
  if (o.workers == 0) o.workers = 4;
  PW_CUDA_TRY(cudaSetDevice(o.device));
  int64_t budget = o.hbm_budget_bytes;
  if (budget == 0) {
    size_t free_b = 0, total_b = 0;
    PW_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    budget = (int64_t)(0.8 * (double)free_b);
  }
  auto* s = new pwgpu_server();
  s->opt = o;
  s->budget = budget;
  for (int i = 0; i < o.workers; ++i) s->workers.emplace_back([s] { s->worker_main(); });
  *out = s;
  return kOk;
}

pwgpu_status pwgpu_server_destroy(pwgpu_server* s) {
  if (!s) return kOk;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->queue.clear();
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  s->cv_done.notify_all();
  delete s;
  return kOk;
}

pwgpu_status pwgpu_server_submit(pwgpu_server* s, const pwgpu_system* sys, const pwgpu_scf_params* params,
                                 const double* rho_init_r, int64_t* job_id) {
  if (!s || !sys || !params || !job_id) return fail(kInvalid, "pwgpu_server_submit: NULL argument");
  if (!rho_init_r && sys->v_local_g)
    return fail(kInvalid, "pwgpu_server_submit: rho_init_r may be NULL only when the local part is built on the device");
  if (sys->nspin != 1 && sys->nspin != 2) return fail(kInvalid, "pwgpu_server_submit: nspin must be 1 or 2");
  if (params->n_bands < 1 || params->n_bands > sys->n_pw)
    return fail(kInvalid, "pwgpu_server_submit: n_bands out of range");
  auto job = std::make_shared<Job>();
  Status st = job->sys.copy_from(*sys);
  if (st != kOk) return st;
  const size_t N = (size_t)sys->dims[0] * sys->dims[1] * sys->dims[2];
  job->params = *params;
  if (rho_init_r) job->rho_init.assign(rho_init_r, rho_init_r + N);
  job->evals.assign((size_t)sys->nspin * sys->n_k * params->n_bands, 0.0);
  job->bytes = footprint(*sys, *params, s->opt.lanes_per_job > 0 ? s->opt.lanes_per_job : 2);
  if (job->bytes > s->budget)
    return fail(kOom, "pwgpu_server_submit: job footprint exceeds the server's HBM budget");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail(pwgpu::kState, "pwgpu_server_submit: server is stopping");
    job->id = s->next_id++;
    job->t_submit = Clock::now();
    s->jobs[job->id] = job;
    s->queue.push_back(job);
    ++s->submitted;
    *job_id = job->id;
  }
  s->cv_work.notify_all();
  return kOk;
}

pwgpu_status pwgpu_server_poll(pwgpu_server* s, int64_t job_id, pwgpu_job_info* info) {
  if (!s) return fail(kInvalid, "pwgpu_server_poll: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(job_id);
  if (it == s->jobs.end()) return fail(kInvalid, "pwgpu_server_poll: unknown job id");
  s->fill_info(*it->second, info);
  return kOk;
}

pwgpu_status pwgpu_server_wait(pwgpu_server* s, int64_t job_id, double timeout_s, pwgpu_job_info* info) {
  if (!s) return fail(kInvalid, "pwgpu_server_wait: NULL server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(job_id);
  if (it == s->jobs.end()) return fail(kInvalid, "pwgpu_server_wait: unknown job id");
  std::shared_ptr<Job> job = it->second;
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(std::max(0.0, timeout_s)),
                                      [&] { return job->state == PWGPU_JOB_DONE; });
  s->fill_info(*job, info);
  return ok ? kOk : fail(kTimeout, "pwgpu_server_wait: job not done within the timeout");
}

pwgpu_status pwgpu_server_wait_any(pwgpu_server* s, double timeout_s, int64_t* job_id) {
  if (!s || !job_id) return fail(kInvalid, "pwgpu_server_wait_any: NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(std::max(0.0, timeout_s)),
                                      [&] { return !s->finished.empty(); });
  if (!ok) return fail(kTimeout, "pwgpu_server_wait_any: no job finished within the timeout");
  *job_id = s->finished.front();
  s->finished.pop_front();
  return kOk;
}

pwgpu_status pwgpu_server_result(pwgpu_server* s, int64_t job_id, pwgpu_scf_result* result, double* eigenvalues,
                                 const char** error) {
  if (!s) return fail(kInvalid, "pwgpu_server_result: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(job_id);
  if (it == s->jobs.end()) return fail(kInvalid, "pwgpu_server_result: unknown job id");
  const Job& j = *it->second;
  if (j.state != PWGPU_JOB_DONE) return fail(pwgpu::kState, "pwgpu_server_result: job not done");
  if (result) *result = j.result;
  if (eigenvalues) std::memcpy(eigenvalues, j.evals.data(), j.evals.size() * sizeof(double));
  if (error) *error = j.error.c_str();
  return kOk;
}

pwgpu_status pwgpu_server_release(pwgpu_server* s, int64_t job_id) {
  if (!s) return fail(kInvalid, "pwgpu_server_release: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(job_id);
  if (it == s->jobs.end()) return fail(kInvalid, "pwgpu_server_release: unknown job id");
  if (it->second->state != PWGPU_JOB_DONE) return fail(pwgpu::kState, "pwgpu_server_release: job not done");
  s->jobs.erase(it);
  return kOk;
}

pwgpu_status pwgpu_server_get_stats(pwgpu_server* s, pwgpu_server_stats* st) {
  if (!s || !st) return fail(kInvalid, "pwgpu_server_get_stats: NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  st->submitted = s->submitted;
  st->queued = (int64_t)s->queue.size();
  st->running = s->running;
  st->done = s->done;
  st->failed = s->failed;
  st->bytes_in_use = s->in_use;
  st->peak_bytes = s->peak;
  st->budget_bytes = s->budget;
  return kOk;
}

}  // extern "C"
