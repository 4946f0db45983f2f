// Allocation-free variant of the local H|psi> apply.
//
// Some callers cannot call cudaMalloc: code embedded in a host framework
// whose memory manager owns all device memory and forbids raw driver
// allocations, and latency-critical serving loops where cudaMalloc's
// implicit device-wide synchronisation would stall every other stream.
// pwgpu_apply_h_local_noalloc gives them the local part of H|psi> (kinetic
// + V_eff through the sphere-pruned FFT pipeline) with its FFT
// intermediates in one fixed, file-scope device array instead of memory the
// call allocates.  The array is kNoAllocScratchBytes (32 MiB); every GPU
// that loads the library holds it until the process exits.
//
// The host cannot pass the array's name to a kernel: in host code that name
// is a host-side stand-in, not a device address.  The first call on each
// device (with that device current) looks the address up with
// cudaGetSymbolAddress and caches it together with the device's current
// context; that first call should therefore come before any stream capture.
// A later call that finds a different context (after cudaDeviceReset, or a
// reset of the primary context, the module is loaded again) looks the
// address up again.  The call makes the handle's device current for its
// duration and restores the caller's current device before it returns.
// Every call shares the array and leaves the
// last call's intermediates in it; each call writes every scratch element
// it reads before reading it, so nothing has to start at zero.  Calls whose
// executions overlap on the GPU (other streams, other threads) race on the
// array and must be serialised by the caller.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "handle.hpp"
#include "../../include/pwgpu.h"

namespace pwgpu {

Handle* handle_state(pwgpu_handle* ph, int* precision);

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};
CUcontext g_scratch_ctx[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);

// The calling thread's current driver context (through the runtime's driver
// entry point, so the library needs no link against the driver library).
Status current_context(CUcontext* ctx) {
  static CtxGetCurrentFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
      return fail(kCuda, "cuCtxGetCurrent entry point not found");
    fn = reinterpret_cast<CtxGetCurrentFn>(p);
  }
  if (fn(ctx) != CUDA_SUCCESS) return fail(kCuda, "cuCtxGetCurrent failed");
  return kOk;
}

// Device address of g_noalloc_scratch on `device`, which is current: looked
// up once per device and context.
Status scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return fail(kInvalid, "device ordinal out of range for the fixed scratch");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  CUcontext ctx = nullptr;
  Status st = current_context(&ctx);
  if (st != kOk) return st;
  if (!g_scratch_addr[device] || g_scratch_ctx[device] != ctx) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
      return fail(kCuda, std::string("cudaGetSymbolAddress(fixed scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[device] = ptr;
    g_scratch_ctx[device] = ctx;
  }
  *out = g_scratch_addr[device];
  return kOk;
}

// Makes `device` current and puts the caller's current device back on scope exit.
struct DeviceGuard {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceGuard(int device) {
    err = cudaGetDevice(&prev);
    if (err == cudaSuccess && prev != device) err = cudaSetDevice(device);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace
}  // namespace pwgpu

using namespace pwgpu;

extern "C" pwgpu_status pwgpu_apply_h_local_noalloc(pwgpu_handle* ph, int32_t spin, int32_t ik, const void* psi_dev,
                                                    int64_t ldpsi, int32_t nb, void* hpsi_dev, int64_t ldh,
                                                    void* stream) {
  int precision = 0;
  Handle* h = handle_state(ph, &precision);
  if (!h || !psi_dev || !hpsi_dev) return fail(kInvalid, "pwgpu_apply_h_local_noalloc: NULL argument");
  if (nb < 0) return fail(kInvalid, "pwgpu_apply_h_local_noalloc: nb must be non-negative");
  DeviceGuard guard(h->device);
  if (guard.err != cudaSuccess)
    return fail(kCuda, std::string("pwgpu_apply_h_local_noalloc: cudaSetDevice: ") + cudaGetErrorString(guard.err));
  void* scratch = nullptr;
  Status st = scratch_address(h->device, &scratch);
  if (st != kOk) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : h->stream;
  st = local_apply_on_scratch(*h, spin, ik, (const double2*)psi_dev, ldpsi, nb, (double2*)hpsi_dev, ldh, precision,
                              s, scratch, kNoAllocScratchBytes);
  if (st != kOk) {
    if (st == kInvalid)
      return fail(kInvalid, std::string("pwgpu_apply_h_local_noalloc: ") + pwgpu_last_error() +
                                " (fixed scratch is 32 MiB)");
    return st;
  }
  return kOk;
}
