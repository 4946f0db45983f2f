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
// cudaGetSymbolAddress and caches it; that first call should therefore come
// before any stream capture.  Every call shares the array and leaves the
// last call's intermediates in it; each call writes every scratch element
// it reads before reading it, so nothing has to start at zero.  Calls whose
// executions overlap on the GPU (other streams, other threads) race on the
// array and must be serialised by the caller.
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

// Device address of g_noalloc_scratch on `device` (looked up once per device
// with the device current).
Status scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return fail(kInvalid, "device ordinal out of range for the fixed scratch");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
      return fail(kCuda, std::string("cudaGetSymbolAddress(fixed scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[device] = ptr;
  }
  *out = g_scratch_addr[device];
  return kOk;
}

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
  PW_CUDA_TRY(cudaSetDevice(h->device));
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
