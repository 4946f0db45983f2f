// Scalar helpers of the dense FP64 kernels (eigh.cu, chol.cu): double is
// the real symmetric case, double2 the complex Hermitian one.
#pragma once

#include <cuda_runtime.h>

namespace pwgpu {
namespace dense {

__device__ __forceinline__ double cj(double x) { return x; }
__device__ __forceinline__ double2 cj(double2 x) { return make_double2(x.x, -x.y); }
__device__ __forceinline__ double mul(double a, double b) { return a * b; }
__device__ __forceinline__ double2 mul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 mul(double2 a, double b) { return make_double2(a.x * b, a.y * b); }
__device__ __forceinline__ double add(double a, double b) { return a + b; }
__device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double sub(double a, double b) { return a - b; }
__device__ __forceinline__ double2 sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double re(double x) { return x; }
__device__ __forceinline__ double re(double2 x) { return x.x; }
__device__ __forceinline__ double im(double) { return 0.0; }
__device__ __forceinline__ double im(double2 x) { return x.y; }
__device__ __forceinline__ double abs2(double x) { return x * x; }
__device__ __forceinline__ double abs2(double2 x) { return x.x * x.x + x.y * x.y; }
template <typename T> __device__ __forceinline__ T mk(double r, double i);
template <> __device__ __forceinline__ double mk<double>(double r, double) { return r; }
template <> __device__ __forceinline__ double2 mk<double2>(double r, double i) { return make_double2(r, i); }
__device__ __forceinline__ bool finite(double x) { return isfinite(x); }
__device__ __forceinline__ bool finite(double2 x) { return isfinite(x.x) && isfinite(x.y); }

__device__ __forceinline__ double shfl_down(double v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }
__device__ __forceinline__ double2 shfl_down(double2 v, int o) {
  return make_double2(__shfl_down_sync(0xffffffffu, v.x, o), __shfl_down_sync(0xffffffffu, v.y, o));
}
__device__ __forceinline__ double shfl(double v, int l) { return __shfl_sync(0xffffffffu, v, l); }
__device__ __forceinline__ double2 shfl(double2 v, int l) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, l), __shfl_sync(0xffffffffu, v.y, l));
}
// sum over the warp, result in every lane
template <typename T> __device__ __forceinline__ T warp_sum(T v) {
  for (int o = 16; o > 0; o >>= 1) v = add(v, shfl_down(v, o));
  return shfl(v, 0);
}

}  // namespace dense
}  // namespace pwgpu
