// Common device/host helpers for the pwgpu library: complex arithmetic on
// double2/float2, error plumbing, and the per-length FFT plan descriptor.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <atomic>
#include <string>

namespace pwgpu {

template <typename R> struct cvec;
template <> struct cvec<double> { using type = double2; };
template <> struct cvec<float> { using type = float2; };
template <typename R> using cplx = typename cvec<R>::type;

template <typename C> __host__ __device__ __forceinline__ C cmake(double re, double im) {
  C c; c.x = re; c.y = im; return c;
}
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  C c; c.x = a.x * b.x - a.y * b.y; c.y = a.x * b.y + a.y * b.x; return c;
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
  C c; c.x = a.x * b.x + a.y * b.y; c.y = a.y * b.x - a.x * b.y; return c;
}
// multiply by S*i where S = +1 or -1
template <int S, typename C> __host__ __device__ __forceinline__ C mul_si(C a) {
  C c;
  if (S > 0) { c.x = -a.y; c.y = a.x; } else { c.x = a.y; c.y = -a.x; }
  return c;
}

// Asynchronous global -> shared copy of one element of Bytes (4, 8 or 16)
// bytes (cp.async, no register staging); with valid false nothing is read
// and the destination is zero-filled.  Both addresses aligned to Bytes.
template <int Bytes>
__device__ __forceinline__ void cp_async_zfill(void* smem_dst, const void* gmem_src, bool valid) {
  static_assert(Bytes == 4 || Bytes == 8 || Bytes == 16, "cp.async copies 4, 8 or 16 bytes");
  const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
  const int src_bytes = valid ? Bytes : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(dst), "l"(gmem_src), "n"(Bytes),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's committed copy groups are pending
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Maximum number of radix stages per 1-D length (2,3,5-smooth lengths up to
// 1024 need at most 5 with radices 2,3,4,5,8,9).
constexpr int kMaxStages = 6;

// 1-D FFT plan for one length L = prod(radix[s]), radices in {2,3,4,5,8,9}.
// ns[s] = product of the radices of the stages before s (Stockham stride).
struct FftPlan {
  int L;
  int nstages;
  int radix[kMaxStages];
  int ns[kMaxStages];
  unsigned nsm[kMaxStages];  // ceil(2^32 / ns[s]) for division by ns (0 if ns == 1)
};

// Division magic for 0 <= j < 2^32 / d: j / d == __umulhi(j, magic(d)).
inline unsigned div_magic(int d) {
  return d <= 1 ? 0u : (unsigned)((((unsigned long long)1 << 32) + (unsigned long long)d - 1) / (unsigned long long)d);
}

// Status codes shared with include/pwgpu.h.
enum Status : int {
  kOk = 0,
  kInvalid = -1,
  kCuda = -2,
  kOom = -3,
  kNotConverged = -4,
  kTimeout = -5,
  kNotImplemented = -6,
  kState = -7,
};

struct Error {
  int code = kOk;
  std::string msg;
};

// Process-wide count of this library's kernel launches (read through
// pwgpu_kernel_launches); every launch site is followed by count_launch().
inline std::atomic<long long>& launch_counter() {
  static std::atomic<long long> c{0};
  return c;
}
inline void count_launch() { launch_counter().fetch_add(1, std::memory_order_relaxed); }

}  // namespace pwgpu

#define PW_CUDA_TRY(expr)                                                              \
  do {                                                                                 \
    cudaError_t _e = (expr);                                                           \
    if (_e != cudaSuccess) {                                                           \
      return ::pwgpu::fail(::pwgpu::kCuda, std::string(#expr ": ") + cudaGetErrorString(_e)); \
    }                                                                                  \
  } while (0)
