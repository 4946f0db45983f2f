// H|psi> for a block of bands: kinetic diagonal + local potential through
// sphere-pruned batched 3-D FFTs + Kleinman-Bylander nonlocal GEMMs.
//
// Replaces the dense per-k Hamiltonian of the reference
// (fill_hamiltonian_with_v_eff, scf/potentials.rs:163-190, plus
// NonlocalPotential::add_to_hamiltonian, potential/nonlocal.rs:432-450).
// The FFT form is exactly the dense form: with psi(r) and V(r) the
// unnormalised inverse transforms, (V psi)(G_i) = (1/N) FFT(V psi)[G_i]
// collects V(G) psi_j for every G == G_i - G_j on the wrapped grid, which
// is V_eff[miller_to_idx(m_i - m_j)] of the dense matrix.
//
// Pipeline per chunk of bands (intermediates sized to stay in L2):
//   K1 z-inverse on the Xp*Yp sphere columns, scattering psi(G)   -> A
//   K234, one kernel per z-plane of A (z-major) and group of bands, the plane
//        in shared memory: y-inverse of the Xp compact x-planes, x-inverse,
//        multiply by V(r), x-forward, y-forward keeping the Yp sphere rows
//   K5 z-forward, gather the sphere, scale 1/N, add T psi          A -> Hpsi
// then  P = B^H psi,  Q = D P (block diagonal),  Hpsi += B Q.
// Grids whose plane does not fit shared memory run the middle as three
// kernels over a second intermediate B (column-major A):
//   K2 y-inverse per compact x-plane                               A -> B
//   K3 x-inverse, multiply by V(r), x-forward (in place)           B
//   K4 y-forward, keep the Yp sphere rows                          B -> A
#include <cublas_v2.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <tuple>
#include <mutex>
#include <numeric>
#include <set>
#include <type_traits>
#include <vector>

#include "fft_smem.cuh"
#include "handle.hpp"

namespace pwgpu {

namespace {

constexpr int kThreads = 256;
constexpr int kTileElems = 2048;
constexpr int kMaxDynSmem = 2 * (kTileElems + 1024) * 16;  // worst case: two FP64 tiles

__device__ __forceinline__ int wrap_idx(int n, int d) { return n < 0 ? n + d : n; }

template <typename C> __device__ __forceinline__ C to_c(double2 v) { return cmake<C>(v.x, v.y); }

// Every FFT kernel runs on a (W, TY) thread block: threadIdx.x indexes the W
// interleaved lines of the tile, threadIdx.y strides along the lines.

// K1: scatter sphere coefficients of W columns and z-inverse-FFT them.
// ZM: A is z-major ([band][z][column]) for the fused middle kernel, else
// column-major ([band][column][z]).
template <typename R, bool ZM = false>
__global__ void __launch_bounds__(kThreads) k_zinv(const double2* __restrict__ psi, long ldpsi,
                                                  cplx<R>* __restrict__ A, const int* __restrict__ col_start,
                                                  const int* __restrict__ pt_ig, const int* __restrict__ pt_col,
                                                  const int* __restrict__ pt_z, int ncol, int d2, unsigned md2,
                                                  FftPlan pz, const cplx<R>* __restrict__ twz,
                                                  unsigned mw = 0) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x;
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* scr = buf + W * d2;
  const int c0 = blockIdx.x * W;
  const int b = blockIdx.y;
  const int nl = min(W, ncol - c0);
  const int tid = threadIdx.y * W + threadIdx.x;
  const int T = W * blockDim.y;
  for (int e = threadIdx.y; e < d2; e += blockDim.y) buf[e * W + threadIdx.x] = cmake<C>(0.0, 0.0);
  __syncthreads();
  const double2* ps = psi + (long)b * ldpsi;
  const int i0 = col_start[c0], i1 = col_start[c0 + nl];
  for (int i = i0 + tid; i < i1; i += T) buf[pt_z[i] * W + (pt_col[i] - c0)] = to_c<C>(ps[pt_ig[i]]);
  __syncthreads();
  const C* res = fft_lines<+1>(buf, scr, pz, W, twz);
  if constexpr (ZM) {
    C* out = A + (long)b * d2 * ncol + c0;
    for (int i = tid; i < W * d2; i += T) {
      const int e = fast_div(i, W, mw), c = i - e * W;
      if (c < nl) out[(long)e * ncol + c] = res[e * W + c];
    }
  } else {
    C* out = A + ((long)b * ncol + c0) * d2;
    for (int i = tid; i < nl * d2; i += T) {
      const int c = fast_div(i, d2, md2), e = i - c * d2;
      out[i] = res[e * W + c];
    }
  }
}

// K5: z-forward-FFT W columns, gather the sphere, Hpsi = buf/N + T psi.
template <typename R, bool ZM = false>
__global__ void __launch_bounds__(kThreads) k_zfwd(const cplx<R>* __restrict__ A, const double2* __restrict__ psi,
                                                  long ldpsi, double2* __restrict__ hpsi, long ldh,
                                                  const double* __restrict__ kin, double scale,
                                                  const int* __restrict__ col_start, const int* __restrict__ pt_ig,
                                                  const int* __restrict__ pt_col, const int* __restrict__ pt_z,
                                                  int ncol, int d2, unsigned md2, FftPlan pz,
                                                  const cplx<R>* __restrict__ twz, unsigned mw = 0) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x;
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* scr = buf + W * d2;
  const int c0 = blockIdx.x * W;
  const int b = blockIdx.y;
  const int nl = min(W, ncol - c0);
  const int tid = threadIdx.y * W + threadIdx.x;
  const int T = W * blockDim.y;
  // asynchronous copies, columns past the last one zero-filled
  if constexpr (ZM) {
    const C* in = A + (long)b * d2 * ncol + c0;
    for (int i = tid; i < W * d2; i += T) {
      const int e = fast_div(i, W, mw), c = i - e * W;
      cp_async_zfill<sizeof(C)>(&buf[e * W + c], c < nl ? (const void*)(in + (long)e * ncol + c) : (const void*)A,
                                c < nl);
    }
  } else {
    const C* in = A + ((long)b * ncol + c0) * d2;
    for (int i = tid; i < W * d2; i += T) {
      const int c = fast_div(i, d2, md2), e = i - c * d2;
      cp_async_zfill<sizeof(C)>(&buf[e * W + c], c < nl ? (const void*)(in + i) : (const void*)A, c < nl);
    }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  const C* res = fft_lines<-1>(buf, scr, pz, W, twz);
  const double2* ps = psi + (long)b * ldpsi;
  double2* hs = hpsi + (long)b * ldh;
  const int i0 = col_start[c0], i1 = col_start[c0 + nl];
  for (int i = i0 + tid; i < i1; i += T) {
    const int ig = pt_ig[i];
    const C v = res[pt_z[i] * W + (pt_col[i] - c0)];
    const double2 p = ps[ig];
    const double t = kin[ig];
    hs[ig] = make_double2((double)v.x * scale + t * p.x, (double)v.y * scale + t * p.y);
  }
}

// K2 (S=+1): rows q<Yp of A -> y-inverse -> all d1 rows of B.
// K4 (S=-1): all d1 rows of B -> y-forward -> rows q<Yp of A.
// A tile is one compact x-plane p and W consecutive z offsets.
template <typename R, int S>
__global__ void __launch_bounds__(kThreads) k_y(cplx<R>* __restrict__ A, cplx<R>* __restrict__ B, int Xp, int Yp,
                                               int m1, int d1, int d2, FftPlan py, const cplx<R>* __restrict__ twy) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x;
  const int w = threadIdx.x;
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* scr = buf + d1 * W;
  const int p = blockIdx.x;
  const int z0 = blockIdx.y * W;
  const int b = blockIdx.z;
  const bool live = w < d2 - z0;
  const long ncol = (long)Xp * Yp;
  C* a_base = A + ((long)b * ncol + (long)p * Yp) * d2 + z0 + w;
  C* b_base = B + (((long)b * Xp + p) * d1) * d2 + z0 + w;
  // rows copied asynchronously (all in flight at once), missing rows zero-filled
  if (S > 0) {
    // row y holds compact row q = y + m1 (y <= m1) or y - d1 + m1 (y >= d1 - m1), else zero
    for (int y = threadIdx.y; y < d1; y += blockDim.y) {
      const int q = y <= m1 ? y + m1 : (y >= d1 - m1 ? y - d1 + m1 : -1);
      const bool ok = live && q >= 0;
      cp_async_zfill<sizeof(C)>(&buf[y * W + w], ok ? (const void*)(a_base + (long)q * d2) : (const void*)A, ok);
    }
  } else {
    for (int y = threadIdx.y; y < d1; y += blockDim.y)
      cp_async_zfill<sizeof(C)>(&buf[y * W + w], live ? (const void*)(b_base + (long)y * d2) : (const void*)B, live);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  const C* res = fft_lines<S>(buf, scr, py, W, twy);
  if (!live) return;
  if (S > 0) {
    for (int y = threadIdx.y; y < d1; y += blockDim.y) b_base[(long)y * d2] = res[y * W + w];
  } else {
    for (int q = threadIdx.y; q < Yp; q += blockDim.y) a_base[(long)q * d2] = res[wrap_idx(q - m1, d1) * W + w];
  }
}

// K3: compact x rows of B -> x-inverse -> * V(r) -> x-forward -> compact rows.
// A tile is one y row and W consecutive z offsets.
template <typename R>
__global__ void __launch_bounds__(kThreads) k_xv(cplx<R>* __restrict__ B, const R* __restrict__ vr, int Xp, int m0,
                                                int d0, int d1, int d2, FftPlan px, const cplx<R>* __restrict__ twx) {
  using C = cplx<R>;
  // FP32 tiles also stage their V(r) rows in shared memory (xv_smem)
  constexpr bool kStageV = std::is_same<R, float>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x;
  const int w = threadIdx.x;
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* scr = buf + d0 * W;
  R* vt = reinterpret_cast<R*>(scr + d0 * W);
  const int y = blockIdx.x;
  const int z0 = blockIdx.y * W;
  const int b = blockIdx.z;
  const bool live = w < d2 - z0;
  const long plane = (long)d1 * d2;
  C* base = B + (long)b * Xp * plane + (long)y * d2 + z0 + w;
  const R* vb = vr + (long)y * d2 + z0 + w;
  // every row of the tile in flight at once: asynchronous copies, rows
  // outside the compact x range (and columns past d2) zero-filled
  for (int x = threadIdx.y; x < d0; x += blockDim.y) {
    const int q = x <= m0 ? x + m0 : (x >= d0 - m0 ? x - d0 + m0 : -1);
    const bool ok = live && q >= 0;
    cp_async_zfill<sizeof(C)>(&buf[x * W + w], ok ? (const void*)(base + (long)q * plane) : (const void*)B, ok);
  }
  cp_async_commit();
  if constexpr (kStageV) {
    for (int x = threadIdx.y; x < d0; x += blockDim.y)
      cp_async_zfill<sizeof(R)>(&vt[x * W + w], live ? (const void*)(vb + (long)x * plane) : (const void*)vr, live);
    cp_async_commit();
    cp_async_wait<1>();  // the tile; the V rows may still be arriving
  } else {
    cp_async_wait<0>();
  }
  __syncthreads();
  C* r1 = fft_lines<+1>(buf, scr, px, W, twx);
  if constexpr (kStageV) {
    cp_async_wait<0>();
    __syncthreads();
  }
  for (int x = threadIdx.y; x < d0; x += blockDim.y)
    if (live) r1[x * W + w] = r1[x * W + w] * (kStageV ? vt[x * W + w] : vb[(long)x * plane]);
  __syncthreads();
  const C* r2 = fft_lines<-1>(r1, r1 == buf ? scr : buf, px, W, twx);
  if (!live) return;
  for (int q = threadIdx.y; q < Xp; q += blockDim.y) base[(long)q * plane] = r2[wrap_idx(q - m0, d0) * W + w];
}

// K234: one z-plane of the z-major A (ncol = Xp*Yp compact columns) for a
// group of bands, the whole plane in shared memory: y-inverse of the Xp
// compact x-planes (Xp lines of length d1), expansion to all d0 x rows,
// x-inverse (d1 lines of length d0), multiplication by this plane of V(r),
// x-forward, compaction to the Xp x-planes, y-forward, and the Yp sphere rows
// written back in place.  Shared memory: the plane XB (d0 x d1, lines along
// x interleaved by y), its Stockham scratch XS (which also holds the y-lines
// YB/YS, Xp x d1 each, element y of line p at y*Xp + p) and the V(r) plane.
// The x transforms run inverse then forward on the same plan, so their
// result is back in XB whatever the stage count, and the y buffers in XS are
// free again.  Global traffic per band: the compact plane read and written
// once (contiguous), V(r) once per block.
template <typename R>
__global__ void __launch_bounds__(kThreads) k_yxy(cplx<R>* __restrict__ A, const R* __restrict__ vz, int nb, int bpc,
                                                 int Xp, int Yp, int m0, int m1, int d0, int d1, int d2,
                                                 unsigned mXp, unsigned mYp, unsigned md1, FftPlan px, FftPlan py,
                                                 const cplx<R>* __restrict__ twx, const cplx<R>* __restrict__ twy) {
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int z = blockIdx.x;
  const int plane = d0 * d1;
  const int ncol = Xp * Yp;
  const int ny = Xp * d1;
  C* XB = reinterpret_cast<C*>(smem_raw);
  C* XS = XB + plane;
  R* VP = reinterpret_cast<R*>(XS + plane);
  C* YB = XS;
  C* YS = XS + ny;
  const int tid = threadIdx.x, T = blockDim.x;
  for (int i = tid; i < plane; i += T) VP[i] = vz[(long)z * plane + i];
  const int b0 = blockIdx.y * bpc;
  const int b1 = min(nb, b0 + bpc);
  for (int b = b0; b < b1; ++b) {
    C* Ab = A + ((long)b * d2 + z) * ncol;
    // compact rows q < Yp into y = wrap(q - m1); the rows between stay zero
    for (int i = tid; i < ncol; i += T) {
      const int p = fast_div(i, Yp, mYp), q = i - p * Yp;
      const int y = q - m1 < 0 ? q - m1 + d1 : q - m1;
      YB[y * Xp + p] = Ab[i];
    }
    for (int i = tid; i < (d1 - Yp) * Xp; i += T) YB[(m1 + 1) * Xp + i] = cmake<C>(0.0, 0.0);
    __syncthreads();
    const C* yr = line_fft<+1>(YB, YS, py, Xp, mXp, twy);
    // expand: x row wrap(p - m0) <- compact plane p, the other x rows zero
    for (int i = tid; i < plane; i += T) {
      const int x = fast_div(i, d1, md1), y = i - x * d1;
      const int p = x <= m0 ? x + m0 : (x >= d0 - m0 ? x - d0 + m0 : -1);
      XB[i] = p >= 0 ? yr[y * Xp + p] : cmake<C>(0.0, 0.0);
    }
    __syncthreads();
    C* xr = line_fft<+1>(XB, XS, px, d1, md1, twx);
    for (int i = tid; i < plane; i += T) xr[i] = xr[i] * VP[i];
    __syncthreads();
    C* xf = line_fft<-1>(xr, xr == XB ? XS : XB, px, d1, md1, twx);  // == XB
    for (int i = tid; i < ny; i += T) {
      const int y = fast_div(i, Xp, mXp), p = i - y * Xp;
      const int x = p - m0 < 0 ? p - m0 + d0 : p - m0;
      YB[i] = xf[x * d1 + y];
    }
    __syncthreads();
    const C* yf = line_fft<-1>(YB, YS, py, Xp, mXp, twy);
    for (int i = tid; i < ncol; i += T) {
      const int p = fast_div(i, Yp, mYp), q = i - p * Yp;
      const int y = q - m1 < 0 ? q - m1 + d1 : q - m1;
      Ab[i] = yf[y * Xp + p];
    }
    __syncthreads();
  }
}

// The same pass with both axes of two-stage lengths known at compile time
// (x: X0 * X1, y: Y0 * Y1) and the data movement folded into the stages:
// the y-inverse's second stage scatters into the x layout, the x-inverse's
// first stage gathers the compact x-planes (other rows zero), the x-forward's
// first stage multiplies by V(r), its second stage keeps only the compact
// x-planes in the y layout.  Twiddles staged in shared memory.  Buffers:
// P0 (d0 x d1), P1 (d0 x d1), YB/YS inside P1 while the y-lines are live.
// Threads per block: one round of butterflies for the larger-radix stage of
// the x transforms (d1 lines x d0 / max(X0, X1) butterflies: 576 for
// 72 = 8 x 9), at least 512.  Every stage ends at a block barrier, so a
// stage that needs a second, mostly idle round costs nearly twice its work.
// Measured on the 72^3 grid (160-band block, FP32): 512 threads 0.49 ms,
// 576 0.465 ms, 672 (one round for both stages, registers capped at 40 for
// two blocks per SM) 0.473 ms.
template <int X0, int X1, int Y0, int Y1> constexpr int yxy_threads() {
  constexpr int b = Y0 * Y1 * (X0 < X1 ? X0 : X1);
  constexpr int t = (b + 31) / 32 * 32;
  return t < 512 ? 512 : (t > 1024 ? 1024 : t);
}
template <typename R, int X0, int X1, int Y0, int Y1>
__global__ void __launch_bounds__(yxy_threads<X0, X1, Y0, Y1>(), sizeof(R) == 4 ? 2 : 1) k_yxy_ct(cplx<R>* __restrict__ A, const R* __restrict__ vz, int nb,
                                                       int bpc, int Xp, int Yp, int m0, int m1, int d2, unsigned mXp,
                                                       unsigned mYp, unsigned md1, const cplx<R>* __restrict__ twx,
                                                       const cplx<R>* __restrict__ twy) {
  using C = cplx<R>;
  constexpr int d0 = X0 * X1, d1 = Y0 * Y1, plane = d0 * d1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int z = blockIdx.x;
  const int ncol = Xp * Yp;
  const int ny = Xp * d1;
  C* P0 = reinterpret_cast<C*>(smem_raw);
  C* P1 = P0 + plane;
  R* VP = reinterpret_cast<R*>(P1 + plane);
  C* TX = reinterpret_cast<C*>(VP + plane);  // d0 twiddles of x
  C* TY = TX + d0;                            // d1 twiddles of y
  C* YB = P1;
  C* YS = P1 + ny;
  const int tid = threadIdx.x, T = blockDim.x;
  for (int i = tid; i < plane; i += T) VP[i] = vz[(long)z * plane + i];
  for (int i = tid; i < d0; i += T) TX[i] = twx[i];
  for (int i = tid; i < d1; i += T) TY[i] = twy[i];
  const int b0 = blockIdx.y * bpc;
  const int b1 = min(nb, b0 + bpc);
  for (int b = b0; b < b1; ++b) {
    C* Ab = A + ((long)b * d2 + z) * ncol;
    __syncthreads();  // the previous band's readers of YB are done (and the staging above is visible)
    for (int i = tid; i < ncol; i += T) {
      const int p = fast_div(i, Yp, mYp), q = i - p * Yp;
      const int y = q - m1 < 0 ? q - m1 + d1 : q - m1;
      YB[y * Xp + p] = Ab[i];
    }
    for (int i = tid; i < (d1 - Yp) * Xp; i += T) YB[(m1 + 1) * Xp + i] = cmake<C>(0.0, 0.0);
    __syncthreads();
    // y-inverse: Xp lines (element y of line p at y*Xp + p); the result goes straight to the x
    // layout of P0 (element x of line y at x*d1 + y) at x = wrap(p - m0)
    line_fft2_f<+1, Y0, Y1>(Xp, mXp, TY, YS, [&](int e, int l) { return YB[e * Xp + l]; },
                            [&](int e, int l, C v) {
                              const int x = l - m0 < 0 ? l - m0 + d0 : l - m0;
                              P0[x * d1 + e] = v;
                            });
    // x-inverse: d1 lines; rows outside the compact x range are zero (never stored above)
    line_fft2_f<+1, X0, X1>(d1, md1, TX, P1,
                            [&](int e, int l) {
                              return (e <= m0 || e >= d0 - m0) ? P0[e * d1 + l] : cmake<C>(0.0, 0.0);
                            },
                            [&](int e, int l, C v) { P0[e * d1 + l] = v * VP[e * d1 + l]; });
    // x-forward; the second stage keeps the compact x-planes, in the y layout of YB
    line_fft2_f<-1, X0, X1>(d1, md1, TX, P1, [&](int e, int l) { return P0[e * d1 + l]; },
                            [&](int e, int l, C v) {
                              if (e <= m0 || e >= d0 - m0) {
                                const int p = e <= m0 ? e + m0 : e - d0 + m0;
                                P0[l * Xp + p] = v;
                              }
                            });
    // y-forward on the compact planes (now in P0 as y-lines), the sphere rows back to A
    line_fft2_f<-1, Y0, Y1>(Xp, mXp, TY, P1, [&](int e, int l) { return P0[e * Xp + l]; },
                            [&](int e, int l, C v) {
                              if (e <= m1 || e >= d1 - m1) {
                                const int q = e <= m1 ? e + m1 : e - d1 + m1;
                                Ab[l * Yp + q] = v;
                              }
                            });
  }
}

template <typename R> inline size_t yxy_ct_smem(int d0, int d1) {
  return 2 * (size_t)d0 * d1 * sizeof(cplx<R>) + (size_t)d0 * d1 * sizeof(R) + (size_t)(d0 + d1) * sizeof(cplx<R>);
}

// Shared memory of a k_yxy block: two d0 x d1 planes and the V(r) plane.
template <typename R> inline size_t yxy_smem(int d0, int d1) {
  return 2 * (size_t)d0 * d1 * sizeof(cplx<R>) + (size_t)d0 * d1 * sizeof(R);
}
constexpr size_t kFusedSmemMax = 227 * 1024;

// The fused middle kernel serves grids whose plane (two copies plus V(r))
// fits shared memory and whose y-lines (2 Xp d1) fit in one plane.
template <typename R> inline bool fused_ok(const GridMaps& g) {
  return yxy_smem<R>(g.d[0], g.d[1]) <= kFusedSmemMax && 2 * g.Xp <= g.d[0];
}

// Launch the compile-time form of the fused pass when the x and y lengths
// are one of the instantiated two-stage lengths (72, 40, 25, 24 on both
// axes); false otherwise (the caller runs the generic k_yxy).
template <typename R, int X0, int X1>
void launch_yxy_ct_n(const GridMaps& g, cplx<R>* A, const R* vz, int nb, int bpc, const cplx<R>* twx,
                     const cplx<R>* twy, cudaStream_t s) {
  k_yxy_ct<R, X0, X1, X0, X1><<<dim3(g.d[2], (nb + bpc - 1) / bpc), yxy_threads<X0, X1, X0, X1>(), yxy_ct_smem<R>(g.d[0], g.d[1]), s>>>(
      A, vz, nb, bpc, g.Xp, g.Yp, g.m[0], g.m[1], g.d[2], div_magic(g.Xp), div_magic(g.Yp), div_magic(g.d[1]), twx,
      twy);
  count_launch();
}
inline int two_stage_key(const FftPlan& p) { return p.nstages == 2 ? p.radix[0] * 16 + p.radix[1] : -1; }
template <typename R>
bool launch_yxy_ct(const GridMaps& g, cplx<R>* A, const R* vz, int nb, int bpc, const cplx<R>* twx,
                   const cplx<R>* twy, cudaStream_t s) {
  const int kx = two_stage_key(g.plan[0]);
  if (kx != two_stage_key(g.plan[1]) || yxy_ct_smem<R>(g.d[0], g.d[1]) > kFusedSmemMax) return false;
  switch (kx) {
    case 8 * 16 + 9: launch_yxy_ct_n<R, 8, 9>(g, A, vz, nb, bpc, twx, twy, s); return true;
    case 8 * 16 + 5: launch_yxy_ct_n<R, 8, 5>(g, A, vz, nb, bpc, twx, twy, s); return true;
    case 5 * 16 + 5: launch_yxy_ct_n<R, 5, 5>(g, A, vz, nb, bpc, twx, twy, s); return true;
    case 8 * 16 + 3: launch_yxy_ct_n<R, 8, 3>(g, A, vz, nb, bpc, twx, twy, s); return true;
    default: return false;
  }
}

// K1 and K5 of the fused pipeline with the z transform's two radix stages
// fixed at compile time (d2 = Z0 * Z1): the first stage of K1 reads the
// scattered sphere columns from shared memory and its second writes the
// z-major planes straight to global memory; K5's first stage reads the
// z-major planes straight from global memory and its second writes shared
// memory for the sphere gather.  One-dimensional blocks of kZThreads.
constexpr int kZThreads = 256;
template <typename R, int Z0, int Z1>
__global__ void __launch_bounds__(kZThreads) k_zinv_ct(const double2* __restrict__ psi, long ldpsi,
                                                      cplx<R>* __restrict__ A, const int* __restrict__ col_start,
                                                      const int* __restrict__ pt_ig, const int* __restrict__ pt_col,
                                                      const int* __restrict__ pt_z, int ncol, int W, unsigned mW,
                                                      const cplx<R>* __restrict__ twz) {
  using C = cplx<R>;
  constexpr int d2 = Z0 * Z1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* scr = buf + W * d2;
  const int c0 = blockIdx.x * W;
  const int b = blockIdx.y;
  const int nl = min(W, ncol - c0);
  const int tid = threadIdx.x, T = blockDim.x;
  for (int i = tid; i < W * d2; i += T) buf[i] = cmake<C>(0.0, 0.0);
  __syncthreads();
  const double2* ps = psi + (long)b * ldpsi;
  const int i0 = col_start[c0], i1 = col_start[c0 + nl];
  for (int i = i0 + tid; i < i1; i += T) buf[pt_z[i] * W + (pt_col[i] - c0)] = to_c<C>(ps[pt_ig[i]]);
  __syncthreads();
  C* out = A + (long)b * d2 * ncol + c0;
  line_fft2_f<+1, Z0, Z1>(W, mW, twz, scr, [&](int e, int l) { return buf[e * W + l]; },
                          [&](int e, int l, C v) {
                            if (l < nl) out[(long)e * ncol + l] = v;
                          });
}

template <typename R, int Z0, int Z1>
__global__ void __launch_bounds__(kZThreads) k_zfwd_ct(const cplx<R>* __restrict__ A, const double2* __restrict__ psi,
                                                      long ldpsi, double2* __restrict__ hpsi, long ldh,
                                                      const double* __restrict__ kin, double scale,
                                                      const int* __restrict__ col_start, const int* __restrict__ pt_ig,
                                                      const int* __restrict__ pt_col, const int* __restrict__ pt_z,
                                                      int ncol, int W, unsigned mW, const cplx<R>* __restrict__ twz) {
  using C = cplx<R>;
  constexpr int d2 = Z0 * Z1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  C* scr = buf + W * d2;
  const int c0 = blockIdx.x * W;
  const int b = blockIdx.y;
  const int nl = min(W, ncol - c0);
  const int tid = threadIdx.x, T = blockDim.x;
  const C* in = A + (long)b * d2 * ncol + c0;
  line_fft2_f<-1, Z0, Z1>(W, mW, twz, scr,
                          [&](int e, int l) { return l < nl ? in[(long)e * ncol + l] : cmake<C>(0.0, 0.0); },
                          [&](int e, int l, C v) { buf[e * W + l] = v; });
  const double2* ps = psi + (long)b * ldpsi;
  double2* hs = hpsi + (long)b * ldh;
  const int i0 = col_start[c0], i1 = col_start[c0 + nl];
  for (int i = i0 + tid; i < i1; i += T) {
    const int ig = pt_ig[i];
    const C v = buf[pt_z[i] * W + (pt_col[i] - c0)];
    const double2 p = ps[ig];
    const double t = kin[ig];
    hs[ig] = make_double2((double)v.x * scale + t * p.x, (double)v.y * scale + t * p.y);
  }
}

// The compile-time z pass for the two-stage z lengths (72, 40, 25, 24);
// false for others (the caller runs the generic kernels).
template <typename R> bool z_ct_ok(const GridMaps& g) {
  switch (two_stage_key(g.plan[2])) {
    case 8 * 16 + 9: case 8 * 16 + 5: case 5 * 16 + 5: case 8 * 16 + 3: return true;
    default: return false;
  }
}
template <typename R>
void launch_zinv_ct(const GridMaps& g, int W, const double2* psi, long ldpsi, cplx<R>* A, int nb, const cplx<R>* tw,
                    cudaStream_t s) {
  const dim3 grid((g.ncol + W - 1) / W, nb);
  const size_t smem = 2 * (size_t)W * g.d[2] * sizeof(cplx<R>);
  const unsigned mW = div_magic(W);
  switch (two_stage_key(g.plan[2])) {
    case 8 * 16 + 9:
      k_zinv_ct<R, 8, 9><<<grid, kZThreads, smem, s>>>(psi, ldpsi, A, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, W, mW, tw);
      break;
    case 8 * 16 + 5:
      k_zinv_ct<R, 8, 5><<<grid, kZThreads, smem, s>>>(psi, ldpsi, A, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, W, mW, tw);
      break;
    case 5 * 16 + 5:
      k_zinv_ct<R, 5, 5><<<grid, kZThreads, smem, s>>>(psi, ldpsi, A, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, W, mW, tw);
      break;
    default:
      k_zinv_ct<R, 8, 3><<<grid, kZThreads, smem, s>>>(psi, ldpsi, A, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, W, mW, tw);
      break;
  }
  count_launch();
}
template <typename R>
void launch_zfwd_ct(const GridMaps& g, int W, const cplx<R>* A, const double2* psi, long ldpsi, double2* hpsi, long ldh,
                    const double* kin, double scale, int nb, const cplx<R>* tw, cudaStream_t s) {
  const dim3 grid((g.ncol + W - 1) / W, nb);
  const size_t smem = 2 * (size_t)W * g.d[2] * sizeof(cplx<R>);
  const unsigned mW = div_magic(W);
  switch (two_stage_key(g.plan[2])) {
    case 8 * 16 + 9:
      k_zfwd_ct<R, 8, 9><<<grid, kZThreads, smem, s>>>(A, psi, ldpsi, hpsi, ldh, kin, scale, g.col_start, g.pt_ig,
                                                       g.pt_col, g.pt_z, g.ncol, W, mW, tw);
      break;
    case 8 * 16 + 5:
      k_zfwd_ct<R, 8, 5><<<grid, kZThreads, smem, s>>>(A, psi, ldpsi, hpsi, ldh, kin, scale, g.col_start, g.pt_ig,
                                                       g.pt_col, g.pt_z, g.ncol, W, mW, tw);
      break;
    case 5 * 16 + 5:
      k_zfwd_ct<R, 5, 5><<<grid, kZThreads, smem, s>>>(A, psi, ldpsi, hpsi, ldh, kin, scale, g.col_start, g.pt_ig,
                                                       g.pt_col, g.pt_z, g.ncol, W, mW, tw);
      break;
    default:
      k_zfwd_ct<R, 8, 3><<<grid, kZThreads, smem, s>>>(A, psi, ldpsi, hpsi, ldh, kin, scale, g.col_start, g.pt_ig,
                                                       g.pt_col, g.pt_z, g.ncol, W, mW, tw);
      break;
  }
  count_launch();
}

// V(r) [x][y][z] -> [z][x][y], FP64 and FP32
__global__ void k_zmajor(const double* __restrict__ vr, double* __restrict__ vz64, float* __restrict__ vz32, int d0,
                         int d1, int d2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long n = (long)d0 * d1 * d2;
  if (i >= n) return;
  const int z = (int)(i % d2);
  const long xy = i / d2;
  const long o = (long)z * d0 * d1 + xy;
  const double v = vr[i];
  vz64[o] = v;
  vz32[o] = (float)v;
}

// Shared memory of a k_xv tile: two W x d0 line buffers, plus the V(r) rows
// for FP32 tiles
template <typename R> inline size_t xv_smem(int W, int d0) {
  return 2 * (size_t)W * d0 * sizeof(cplx<R>) + (std::is_same<R, float>::value ? (size_t)W * d0 * sizeof(float) : 0);
}

// Density: for each band of the chunk, compact x rows of B -> x-inverse ->
// rho(x, y, z) += fw[b] |psi_b(r)|^2 (compute_density, scf/density.rs:59-97).
// One block per (y row, W z offsets) owns its rho tile, so no atomics.
__global__ void __launch_bounds__(kThreads) k_x_density(const double2* __restrict__ B, const double* __restrict__ fw,
                                                       int nb, double* __restrict__ rho, int Xp, int m0, int d0,
                                                       int d1, int d2, FftPlan px, const double2* __restrict__ twx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x;
  const int w = threadIdx.x;
  double2* buf = reinterpret_cast<double2*>(smem_raw);
  double2* scr = buf + d0 * W;
  const int y = blockIdx.x;
  const int z0 = blockIdx.y * W;
  const bool live = w < d2 - z0;
  const long plane = (long)d1 * d2;
  // each thread accumulates the rows x = threadIdx.y + k*blockDim.y it owns
  constexpr int kMaxRows = 16;
  double acc[kMaxRows];
#pragma unroll
  for (int k = 0; k < kMaxRows; ++k) acc[k] = 0.0;
  for (int b = 0; b < nb; ++b) {
    const double2* base = B + (long)b * Xp * plane + (long)y * d2 + z0 + w;
    for (int x = threadIdx.y; x < d0; x += blockDim.y) {
      const int q = x <= m0 ? x + m0 : (x >= d0 - m0 ? x - d0 + m0 : -1);
      const bool ok = live && q >= 0;
      cp_async_zfill<16>(&buf[x * W + w], ok ? (const void*)(base + (long)q * plane) : (const void*)B, ok);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    const double2* res = fft_lines<+1>(buf, scr, px, W, twx);
    const double f = fw[b];
#pragma unroll
    for (int k = 0; k < kMaxRows; ++k) {
      const int x = threadIdx.y + k * blockDim.y;
      if (x < d0) {
        const double2 v = res[x * W + w];
        acc[k] += f * (v.x * v.x + v.y * v.y);
      }
    }
    __syncthreads();
  }
  if (!live) return;
  double* rb = rho + (long)y * d2 + z0 + w;
#pragma unroll
  for (int k = 0; k < kMaxRows; ++k) {
    const int x = threadIdx.y + k * blockDim.y;
    if (x < d0) rb[(long)x * plane] += acc[k];
  }
}

// Full-grid line FFT along one axis, grid viewed as [outer][L][inner].
// inner == 1: a tile is W consecutive rows (contiguous lines, transposed
// into the interleaved layout); inner > 1: one outer index and W
// consecutive inner offsets.
template <int S>
__global__ void __launch_bounds__(kThreads) k_fft_axis(double2* __restrict__ g, int outer, int L, int inner,
                                                      unsigned mL, FftPlan p, const double2* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x;
  double2* buf = reinterpret_cast<double2*>(smem_raw);
  double2* scr = buf + W * L;
  const int tid = threadIdx.y * W + threadIdx.x;
  const int T = W * blockDim.y;
  if (inner == 1) {
    const int r0 = blockIdx.x * W;
    const int nl = min(W, outer - r0);
    double2* src = g + (long)r0 * L;
    for (int i = tid; i < W * L; i += T) {
      const int c = fast_div(i, L, mL), e = i - c * L;
      buf[e * W + c] = (c < nl) ? src[i] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const double2* res = fft_lines<S>(buf, scr, p, W, tw);
    for (int i = tid; i < nl * L; i += T) {
      const int c = fast_div(i, L, mL), e = i - c * L;
      src[i] = res[e * W + c];
    }
  } else {
    const int o = blockIdx.y;
    const int w = threadIdx.x;
    const int i0 = blockIdx.x * W;
    const bool live = w < inner - i0;
    double2* src = g + (long)o * L * inner + i0 + w;
    for (int l = threadIdx.y; l < L; l += blockDim.y)
      buf[l * W + w] = live ? src[(long)l * inner] : make_double2(0.0, 0.0);
    __syncthreads();
    const double2* res = fft_lines<S>(buf, scr, p, W, tw);
    if (!live) return;
    for (int l = threadIdx.y; l < L; l += blockDim.y) src[(long)l * inner] = res[l * W + w];
  }
}

// Q = D P with D block-diagonal over atoms (each block dense, row-major).
__global__ void k_apply_d(const double2* __restrict__ P, double2* __restrict__ Q, int n_ch, int nb,
                          const int* __restrict__ ch_atom, const int* __restrict__ atom_ch_start,
                          const int* __restrict__ d_off, const double* __restrict__ d_vals) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)n_ch * nb) return;
  const int c = (int)(t % n_ch);
  const int b = (int)(t / n_ch);
  const int a = ch_atom[c];
  const int s = atom_ch_start[a];
  const int nc = atom_ch_start[a + 1] - s;
  const double* drow = d_vals + d_off[a] + (long)(c - s) * nc;
  const double2* pcol = P + (long)b * n_ch + s;
  double re = 0.0, im = 0.0;
  for (int j = 0; j < nc; ++j) {
    const double dv = drow[j];
    re += dv * pcol[j].x;
    im += dv * pcol[j].y;
  }
  Q[(long)b * n_ch + c] = make_double2(re, im);
}

__global__ void k_real_to_r32(const double2* __restrict__ in, double* __restrict__ out64, float* __restrict__ out32,
                              long n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    out64[i] = in[i].x;
    out32[i] = (float)in[i].x;
  }
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------

bool make_plan(int L, FftPlan& p) {
  p.L = L;
  p.nstages = 0;
  int rem = L;
  std::vector<int> rad;
  while (rem % 8 == 0 && rem > 1) { rad.push_back(8); rem /= 8; }
  while (rem % 9 == 0) { rad.push_back(9); rem /= 9; }
  while (rem % 4 == 0) { rad.push_back(4); rem /= 4; }
  while (rem % 2 == 0) { rad.push_back(2); rem /= 2; }
  while (rem % 5 == 0) { rad.push_back(5); rem /= 5; }
  while (rem % 3 == 0) { rad.push_back(3); rem /= 3; }
  if (rem != 1 || (int)rad.size() > kMaxStages) return false;
  int ns = 1;
  for (size_t s = 0; s < rad.size(); ++s) {
    p.radix[s] = rad[s];
    p.ns[s] = ns;
    p.nsm[s] = div_magic(ns);
    ns *= rad[s];
  }
  p.nstages = (int)rad.size();
  return true;
}

// Tile width (lines per block): about kTileElems elements per tile.
int pick_w(const FftPlan& p, int cap) {
  return std::max(1, std::min(cap, kTileElems / std::max(1, p.L)));
}

// Balance W over n items: ceil(n / ceil(n / wmax)).
int balance_w(int n, int wmax) {
  if (n <= 0) return 1;
  const int chunks = (n + wmax - 1) / wmax;
  return (n + chunks - 1) / chunks;
}

// (W, TY) block for a tile of W lines: TY = kThreads / W rows of threads.
dim3 block_for(int W) { return dim3(W, std::max(1, kThreads / W), 1); }

// Odd tile width for tiles whose lines are filled by a transposing load
// (keeps the strided shared-memory stores at most 2-way bank conflicted).
int odd_w(int w) { return (w > 1 && (w % 2 == 0)) ? w - 1 : w; }

template <typename T> Status dalloc(T** p, size_t count) {
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) return fail(kOom, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return kOk;
}

// Opt every FFT kernel into the dynamic shared memory its largest tile needs
// (a per-device attribute: done once per device, under a lock, since handles
// may be created from several host threads).
Status configure_kernels() {
  static std::mutex mu;
  static std::set<int> done_devices;
  int dev = 0;
  PW_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (done_devices.count(dev)) return kOk;
  const int sm = kMaxDynSmem;
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  };
  set((const void*)k_zinv<double>); set((const void*)k_zinv<float>);
  set((const void*)k_zfwd<double>); set((const void*)k_zfwd<float>);
  set((const void*)k_y<double, 1>); set((const void*)k_y<double, -1>);
  set((const void*)k_y<float, 1>); set((const void*)k_y<float, -1>);
  set((const void*)k_xv<double>); set((const void*)k_xv<float>);
  set((const void*)k_fft_axis<1>); set((const void*)k_fft_axis<-1>);
  set((const void*)k_x_density);
  set((const void*)k_zinv<double, true>); set((const void*)k_zinv<float, true>);
  set((const void*)k_zinv_ct<double, 8, 9>); set((const void*)k_zinv_ct<float, 8, 9>);
  set((const void*)k_zinv_ct<double, 8, 5>); set((const void*)k_zinv_ct<float, 8, 5>);
  set((const void*)k_zinv_ct<double, 5, 5>); set((const void*)k_zinv_ct<float, 5, 5>);
  set((const void*)k_zinv_ct<double, 8, 3>); set((const void*)k_zinv_ct<float, 8, 3>);
  set((const void*)k_zfwd_ct<double, 8, 9>); set((const void*)k_zfwd_ct<float, 8, 9>);
  set((const void*)k_zfwd_ct<double, 8, 5>); set((const void*)k_zfwd_ct<float, 8, 5>);
  set((const void*)k_zfwd_ct<double, 5, 5>); set((const void*)k_zfwd_ct<float, 5, 5>);
  set((const void*)k_zfwd_ct<double, 8, 3>); set((const void*)k_zfwd_ct<float, 8, 3>);
  set((const void*)k_zfwd<double, true>); set((const void*)k_zfwd<float, true>);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_yxy<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFusedSmemMax);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)k_yxy<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFusedSmemMax);
  auto set_big = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFusedSmemMax);
  };
  set_big((const void*)k_yxy_ct<double, 8, 9, 8, 9>); set_big((const void*)k_yxy_ct<float, 8, 9, 8, 9>);
  set_big((const void*)k_yxy_ct<double, 8, 5, 8, 5>); set_big((const void*)k_yxy_ct<float, 8, 5, 8, 5>);
  set_big((const void*)k_yxy_ct<double, 5, 5, 5, 5>); set_big((const void*)k_yxy_ct<float, 5, 5, 5, 5>);
  set_big((const void*)k_yxy_ct<double, 8, 3, 8, 3>); set_big((const void*)k_yxy_ct<float, 8, 3, 8, 3>);
  if (e != cudaSuccess) return fail(kCuda, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  done_devices.insert(dev);
  return kOk;
}

}  // namespace

// FP32 tile widths by measurement.  For each axis the candidate widths W
// that fit the shared memory of an FP64 tile (2 W L 16 bytes <= kMaxDynSmem)
// -- and, on the x axis, the density kernel's 16 rows per thread -- are timed
// on this grid with the FP32 kernel of the axis (z-inverse, y-inverse, x pass)
// over the handle's scratch, the fastest kept.  The kernels compute each line
// the same way whatever the tile holds, so the choice changes speed only.
// FP64 tiles keep the heuristic widths (twice the bytes per tile: wider ones
// cost resident blocks).  Results are cached per device and grid shape (a
// server builds a handle per job); a failed timing keeps the heuristic.
static Status autotune_tiles(Handle& h) {
  GridMaps& g = h.g;
  const int d0 = g.d[0], d1 = g.d[1], d2 = g.d[2];
  int dev = 0;
  PW_CUDA_TRY(cudaGetDevice(&dev));
  struct Key {
    int dev, d0, d1, d2, Xp, Yp, ncol;
    bool operator<(const Key& o) const {
      return std::tie(dev, d0, d1, d2, Xp, Yp, ncol) < std::tie(o.dev, o.d0, o.d1, o.d2, o.Xp, o.Yp, o.ncol);
    }
  };
  static std::mutex mu;
  static std::map<Key, std::array<int, 3>> cache;
  const Key key{dev, d0, d1, d2, g.Xp, g.Yp, g.ncol};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      g.wx32 = it->second[0];
      g.wy32 = it->second[1];
      g.wz32 = it->second[2];
      return kOk;
    }
  }
  // FP32 launches carry 2 chunk bands (the scratch is sized for FP64
  // chunks); the z kernel reads its psi rows from tmp_grid (N entries)
  const int nb = 2 * h.chunk;
  const int nb_in = (int)std::max<long>(1, std::min<long>(nb, g.N / std::max(1, h.n_pw)));
  float2* A = reinterpret_cast<float2*>(h.work_a);
  float2* B = reinterpret_cast<float2*>(h.work_b);
  const double2* psi = h.tmp_grid;                               // nb x n_pw <= N entries
  const float* vr = reinterpret_cast<const float*>(h.tmp_grid);  // N entries
  const cudaStream_t s = h.stream;
  cudaEvent_t e0, e1;
  PW_CUDA_TRY(cudaEventCreate(&e0));
  PW_CUDA_TRY(cudaEventCreate(&e1));
  auto fits = [&](int W, int L) { return W >= 1 && W <= kThreads && 2L * W * L * 16 <= kMaxDynSmem; };
  auto best = [&](const std::vector<int>& cands, int L, int fallback, auto launch) -> int {
    int arg = fallback;
    float tbest = 1e30f;
    for (int W : cands) {
      if (!fits(W, L)) continue;
      launch(W);  // warm-up
      cudaEventRecord(e0, s);
      for (int r = 0; r < 5; ++r) launch(W);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) return fallback;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (cudaGetLastError() != cudaSuccess) return fallback;
      if (ms < tbest) {
        tbest = ms;
        arg = W;
      }
    }
    return arg;
  };
  const std::vector<int> even = {8, 12, 16, 18, 20, 24, 28, 32, 36, 40, 48};
  const std::vector<int> odd = {7, 9, 11, 15, 17, 21, 25, 31, 33, 41, 63};
  std::vector<int> cx;
  for (int W : even)
    if (d0 <= 16 * (kThreads / W)) cx.push_back(W);
  // the z width is measured on the kernel the pipeline will run: the
  // compile-time z pass (one-dimensional blocks, so wider tiles fit) when
  // the z length has one, else the generic kernel
  const bool zct = z_ct_ok<float>(g);
  std::vector<int> zc = odd;
  if (zct) zc.push_back(81);
  const int wz = best(zc, d2, g.wz, [&](int W) {
    if (zct) {
      launch_zinv_ct<float>(g, W, psi, h.n_pw, A, nb_in, g.tw32[2], s);
    } else {
      k_zinv<float><<<dim3((g.ncol + W - 1) / W, nb_in), block_for(W), 2 * (size_t)W * d2 * sizeof(float2), s>>>(
          psi, h.n_pw, A, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, d2, div_magic(d2), g.plan[2], g.tw32[2]);
    }
  });
  const int wy = best(even, d1, g.wy, [&](int W) {
    k_y<float, +1><<<dim3(g.Xp, (d2 + W - 1) / W, nb), block_for(W), 2 * (size_t)W * d1 * sizeof(float2), s>>>(
        A, B, g.Xp, g.Yp, g.m[1], d1, d2, g.plan[1], g.tw32[1]);
  });
  const int wx = best(cx, d0, g.wx, [&](int W) {
    k_xv<float><<<dim3(d1, (d2 + W - 1) / W, nb), block_for(W), xv_smem<float>(W, d0), s>>>(
        B, vr, g.Xp, g.m[0], d0, d1, d2, g.plan[0], g.tw32[0]);
  });
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  PW_CUDA_TRY(cudaStreamSynchronize(s));
  PW_CUDA_TRY(cudaGetLastError());
  if (h.trace)
    std::fprintf(stderr, "pwgpu FP32 tiles %dx%dx%d: x %d y %d z %d (heuristic %d %d %d)\n", d0, d1, d2, wx, wy, wz,
                 g.wx, g.wy, g.wz);
  g.wx32 = wx;
  g.wy32 = wy;
  g.wz32 = wz;
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = {wx, wy, wz};
  return kOk;
}

Status build_grid_maps(Handle& h, const int* miller) {
  GridMaps& g = h.g;
  for (int a = 0; a < 3; ++a) {
    if (!make_plan(g.d[a], g.plan[a]))
      return fail(kNotImplemented, "FFT length " + std::to_string(g.d[a]) + " is not 2,3,5-smooth (or too long)");
  }
  g.N = (long)g.d[0] * g.d[1] * g.d[2];
  int m[3] = {0, 0, 0};
  for (int i = 0; i < h.n_pw; ++i)
    for (int a = 0; a < 3; ++a) m[a] = std::max(m[a], std::abs(miller[3 * i + a]));
  for (int a = 0; a < 3; ++a) {
    if (2 * m[a] + 1 > g.d[a])
      return fail(kInvalid, "FFT grid dimension " + std::to_string(g.d[a]) + " on axis " + std::to_string(a) +
                                " is smaller than 2*max|n|+1 = " + std::to_string(2 * m[a] + 1) +
                                "; sphere points would alias");
    g.m[a] = m[a];
  }
  g.Xp = 2 * m[0] + 1;
  g.Yp = 2 * m[1] + 1;
  g.ncol = g.Xp * g.Yp;
  // sort points by column, stable in basis order
  std::vector<int> col(h.n_pw), order(h.n_pw), zi(h.n_pw), gf(h.n_pw);
  for (int i = 0; i < h.n_pw; ++i) {
    const int n0 = miller[3 * i], n1 = miller[3 * i + 1], n2 = miller[3 * i + 2];
    col[i] = (n0 + m[0]) * g.Yp + (n1 + m[1]);
    zi[i] = n2 < 0 ? n2 + g.d[2] : n2;
    const int x = n0 < 0 ? n0 + g.d[0] : n0, y = n1 < 0 ? n1 + g.d[1] : n1;
    gf[i] = (x * g.d[1] + y) * g.d[2] + zi[i];
  }
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return col[a] < col[b]; });
  std::vector<int> cs(g.ncol + 1, 0), pig(h.n_pw), pcol(h.n_pw), pz(h.n_pw);
  for (int s = 0; s < h.n_pw; ++s) {
    const int i = order[s];
    pig[s] = i;
    pcol[s] = col[i];
    pz[s] = zi[i];
    cs[col[i] + 1]++;
  }
  for (int c = 0; c < g.ncol; ++c) cs[c + 1] += cs[c];
  Status st;
  if ((st = dalloc(&g.col_start, g.ncol + 1)) != kOk) return st;
  if ((st = dalloc(&g.pt_ig, h.n_pw)) != kOk) return st;
  if ((st = dalloc(&g.pt_col, h.n_pw)) != kOk) return st;
  if ((st = dalloc(&g.pt_z, h.n_pw)) != kOk) return st;
  if ((st = dalloc(&g.g_to_fft, h.n_pw)) != kOk) return st;
  PW_CUDA_TRY(cudaMemcpy(g.col_start, cs.data(), cs.size() * sizeof(int), cudaMemcpyHostToDevice));
  PW_CUDA_TRY(cudaMemcpy(g.pt_ig, pig.data(), h.n_pw * sizeof(int), cudaMemcpyHostToDevice));
  PW_CUDA_TRY(cudaMemcpy(g.pt_col, pcol.data(), h.n_pw * sizeof(int), cudaMemcpyHostToDevice));
  PW_CUDA_TRY(cudaMemcpy(g.pt_z, pz.data(), h.n_pw * sizeof(int), cudaMemcpyHostToDevice));
  PW_CUDA_TRY(cudaMemcpy(g.g_to_fft, gf.data(), h.n_pw * sizeof(int), cudaMemcpyHostToDevice));
  // twiddle tables tw[m] = exp(-2 pi i m / L) in extended precision
  for (int a = 0; a < 3; ++a) {
    const int L = g.d[a];
    std::vector<double2> t64(L);
    std::vector<float2> t32(L);
    for (int k = 0; k < L; ++k) {
      const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)L;
      t64[k] = make_double2((double)cosl(ang), (double)sinl(ang));
      t32[k] = make_float2((float)t64[k].x, (float)t64[k].y);
    }
    if ((st = dalloc(&g.tw64[a], L)) != kOk) return st;
    if ((st = dalloc(&g.tw32[a], L)) != kOk) return st;
    PW_CUDA_TRY(cudaMemcpy(g.tw64[a], t64.data(), L * sizeof(double2), cudaMemcpyHostToDevice));
    PW_CUDA_TRY(cudaMemcpy(g.tw32[a], t32.data(), L * sizeof(float2), cudaMemcpyHostToDevice));
  }
  g.wz = odd_w(balance_w(g.ncol, pick_w(g.plan[2], 64)));
  g.wy = balance_w(g.d[2], pick_w(g.plan[1], 32));
  g.wx = balance_w(g.d[2], pick_w(g.plan[0], 32));
  g.wx32 = g.wx;
  g.wy32 = g.wy;
  g.wz32 = g.wz;
  if (Status st0 = configure_kernels(); st0 != kOk) return st0;
  // band chunk: keep A + B of one chunk within ~48 MB (FP64) of L2
  const double per_band = 16.0 * ((double)g.ncol * g.d[2] + (double)g.Xp * g.d[1] * g.d[2]);
  h.chunk = std::max(1, std::min(64, (int)(48.0e6 / per_band)));
  if ((st = dalloc((double2**)&h.work_a, (size_t)h.chunk * g.ncol * g.d[2])) != kOk) return st;
  if ((st = dalloc((double2**)&h.work_b, (size_t)h.chunk * g.Xp * g.d[1] * g.d[2])) != kOk) return st;
  if ((st = dalloc(&h.tmp_grid, (size_t)g.N)) != kOk) return st;
  return autotune_tiles(h);
}

Status ensure_nl_capacity(Handle& h, int nb) {
  if (nb <= h.nl_cap) return kOk;
  if (h.nl_p) cudaFree(h.nl_p);
  if (h.nl_q) cudaFree(h.nl_q);
  h.nl_p = h.nl_q = nullptr;
  Status st;
  if ((st = dalloc(&h.nl_p, (size_t)std::max(1, h.n_ch) * nb)) != kOk) return st;
  if ((st = dalloc(&h.nl_q, (size_t)std::max(1, h.n_ch) * nb)) != kOk) return st;
  h.nl_cap = nb;
  return kOk;
}

Status fft3d_full(Handle& h, double2* data, int sign, cudaStream_t stream) {
  GridMaps& g = h.g;
  const int d0 = g.d[0], d1 = g.d[1], d2 = g.d[2];
  struct Ax { int outer, L, inner, a; };
  const Ax axes[3] = {{d0 * d1, d2, 1, 2}, {d0, d1, d2, 1}, {1, d0, d1 * d2, 0}};
  for (const Ax& ax : axes) {
    const FftPlan& p = g.plan[ax.a];
    if (p.nstages == 0) continue;
    int W;
    dim3 grid;
    if (ax.inner == 1) {
      W = odd_w(balance_w(ax.outer, pick_w(p, 64)));
      grid = dim3((ax.outer + W - 1) / W, 1, 1);
    } else {
      W = balance_w(ax.inner, pick_w(p, 64));
      grid = dim3((ax.inner + W - 1) / W, ax.outer, 1);
    }
    const size_t sm = 2 * (size_t)W * ax.L * sizeof(double2);
    const dim3 blk = block_for(W);
    const unsigned mL = div_magic(ax.L);
    if (sign < 0)
      k_fft_axis<-1><<<grid, blk, sm, stream>>>(data, ax.outer, ax.L, ax.inner, mL, p, g.tw64[ax.a]);
    else
      k_fft_axis<+1><<<grid, blk, sm, stream>>>(data, ax.outer, ax.L, ax.inner, mL, p, g.tw64[ax.a]);
    count_launch();
  }
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

Status set_veff_from_g(Handle& h, int spin, const double2* veff_g_dev, cudaStream_t stream) {
  const long N = h.g.N;
  PW_CUDA_TRY(cudaMemcpyAsync(h.tmp_grid, veff_g_dev, N * sizeof(double2), cudaMemcpyDeviceToDevice, stream));
  Status st = fft3d_full(h, h.tmp_grid, +1, stream);
  if (st != kOk) return st;
  k_real_to_r32<<<(unsigned)((N + 255) / 256), 256, 0, stream>>>(h.tmp_grid, h.veff_r[spin], h.veff_r32[spin], N); count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return veff_zmajor(h, spin, stream);
}

Status veff_zmajor(Handle& h, int spin, cudaStream_t stream) {
  const long N = h.g.N;
  k_zmajor<<<(unsigned)((N + 255) / 256), 256, 0, stream>>>(h.veff_r[spin], h.veff_rz[spin], h.veff_rz32[spin], h.g.d[0],
                                                            h.g.d[1], h.g.d[2]);
  count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// Records an event after each launch when profiling (stage timings).
void mark(StageTimer* t, int stage, cudaStream_t s) {
  if (!t) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, s);
  t->events.push_back(e);
  t->stage.push_back(stage);
}

Status apply_d_blocks(Handle& h, int nb, cudaStream_t s) {
  const long tot = (long)h.n_ch * nb;
  k_apply_d<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(h.nl_p, h.nl_q, h.n_ch, nb, h.ch_atom, h.atom_ch_start,
                                                          h.d_off, h.d_vals);
  count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

template <typename R>
static Status local_chunk(Handle& h, int spin, int ik, const double2* psi, long ldpsi, int nb, double2* hpsi,
                          long ldh, cudaStream_t s, StageTimer* tm) {
  using C = cplx<R>;
  GridMaps& g = h.g;
  const int d0 = g.d[0], d1 = g.d[1], d2 = g.d[2];
  // FP32 tiles use the measured widths, FP64 ones the heuristic widths
  const bool f32 = std::is_same<R, float>::value;
  const int wx = f32 ? g.wx32 : g.wx, wy = f32 ? g.wy32 : g.wy, wz = f32 ? g.wz32 : g.wz;
  C* A = reinterpret_cast<C*>(h.work_a);
  C* B = reinterpret_cast<C*>(h.work_b);
  const C* tw0 = std::is_same<R, double>::value ? (const C*)g.tw64[0] : (const C*)g.tw32[0];
  const C* tw1 = std::is_same<R, double>::value ? (const C*)g.tw64[1] : (const C*)g.tw32[1];
  const C* tw2 = std::is_same<R, double>::value ? (const C*)g.tw64[2] : (const C*)g.tw32[2];
  const R* vr = std::is_same<R, double>::value ? (const R*)h.veff_r[spin] : (const R*)h.veff_r32[spin];
  const double scale = 1.0 / (double)g.N;
  if (fused_ok<R>(g)) {
    // K1 (z-major A), K234 fused per z-plane, K5
    const R* vz = std::is_same<R, double>::value ? (const R*)h.veff_rz[spin] : (const R*)h.veff_rz32[spin];
    if (z_ct_ok<R>(g)) {
      launch_zinv_ct<R>(g, wz, psi, ldpsi, A, nb, tw2, s);
    } else {
      k_zinv<R, true><<<dim3((g.ncol + wz - 1) / wz, nb), block_for(wz), 2 * (size_t)wz * d2 * sizeof(C), s>>>(
          psi, ldpsi, A, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, d2, div_magic(d2), g.plan[2], tw2,
          div_magic(wz)); count_launch();
    }
    mark(tm, 0, s);
    const int groups = std::max(1, std::min(nb, (2 * 148 + d2 - 1) / d2));
    const int bpc = (nb + groups - 1) / groups;
    if (!launch_yxy_ct<R>(g, A, vz, nb, bpc, tw0, tw1, s)) {
      k_yxy<R><<<dim3(d2, (nb + bpc - 1) / bpc), kThreads, yxy_smem<R>(d0, d1), s>>>(
          A, vz, nb, bpc, g.Xp, g.Yp, g.m[0], g.m[1], d0, d1, d2, div_magic(g.Xp), div_magic(g.Yp), div_magic(d1),
          g.plan[0], g.plan[1], tw0, tw1); count_launch();
    }
    mark(tm, 2, s);
    if (z_ct_ok<R>(g)) {
      launch_zfwd_ct<R>(g, wz, A, psi, ldpsi, hpsi, ldh, h.kp[ik].kinetic, scale, nb, tw2, s);
    } else {
      k_zfwd<R, true><<<dim3((g.ncol + wz - 1) / wz, nb), block_for(wz), 2 * (size_t)wz * d2 * sizeof(C), s>>>(
          A, psi, ldpsi, hpsi, ldh, h.kp[ik].kinetic, scale, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, d2,
          div_magic(d2), g.plan[2], tw2, div_magic(wz)); count_launch();
    }
    mark(tm, 4, s);
    PW_CUDA_TRY(cudaGetLastError());
    return kOk;
  }
  {
    dim3 grid((g.ncol + wz - 1) / wz, nb);
    k_zinv<R><<<grid, block_for(wz), 2 * (size_t)wz * d2 * sizeof(C), s>>>(
        psi, ldpsi, A, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, d2, div_magic(d2), g.plan[2], tw2); count_launch();
    mark(tm, 0, s);
  }
  {
    dim3 grid(g.Xp, (d2 + wy - 1) / wy, nb);
    k_y<R, +1><<<grid, block_for(wy), 2 * (size_t)wy * d1 * sizeof(C), s>>>(A, B, g.Xp, g.Yp, g.m[1], d1, d2,
                                                                              g.plan[1], tw1); count_launch();
    mark(tm, 1, s);
  }
  {
    dim3 grid(d1, (d2 + wx - 1) / wx, nb);
    k_xv<R><<<grid, block_for(wx), xv_smem<R>(wx, d0), s>>>(B, vr, g.Xp, g.m[0], d0, d1, d2,
                                                                           g.plan[0], tw0); count_launch();
    mark(tm, 2, s);
  }
  {
    dim3 grid(g.Xp, (d2 + wy - 1) / wy, nb);
    k_y<R, -1><<<grid, block_for(wy), 2 * (size_t)wy * d1 * sizeof(C), s>>>(A, B, g.Xp, g.Yp, g.m[1], d1, d2,
                                                                              g.plan[1], tw1); count_launch();
    mark(tm, 3, s);
  }
  {
    dim3 grid((g.ncol + wz - 1) / wz, nb);
    k_zfwd<R><<<grid, block_for(wz), 2 * (size_t)wz * d2 * sizeof(C), s>>>(
        A, psi, ldpsi, hpsi, ldh, h.kp[ik].kinetic, scale, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, d2,
        div_magic(d2), g.plan[2], tw2); count_launch();
    mark(tm, 4, s);
  }
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// The five local kernels on explicit scratch A / B (used by the
// allocation-free entry point; the handle's own buffers are not touched).
template <typename R>
static void local_chunk_on(Handle& h, int spin, int ik, const double2* psi, long ldpsi, int nb, double2* hpsi,
                           long ldh, cudaStream_t s, cplx<R>* A, cplx<R>* B) {
  using C = cplx<R>;
  GridMaps& g = h.g;
  const int d0 = g.d[0], d1 = g.d[1], d2 = g.d[2];
  // FP32 tiles use the measured widths, FP64 ones the heuristic widths
  const bool f32 = std::is_same<R, float>::value;
  const int wx = f32 ? g.wx32 : g.wx, wy = f32 ? g.wy32 : g.wy, wz = f32 ? g.wz32 : g.wz;
  const bool dbl = std::is_same<R, double>::value;
  const C* tw0 = dbl ? (const C*)g.tw64[0] : (const C*)g.tw32[0];
  const C* tw1 = dbl ? (const C*)g.tw64[1] : (const C*)g.tw32[1];
  const C* tw2 = dbl ? (const C*)g.tw64[2] : (const C*)g.tw32[2];
  const R* vr = dbl ? (const R*)h.veff_r[spin] : (const R*)h.veff_r32[spin];
  k_zinv<R><<<dim3((g.ncol + wz - 1) / wz, nb), block_for(wz), 2 * (size_t)wz * d2 * sizeof(C), s>>>(
      psi, ldpsi, A, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, d2, div_magic(d2), g.plan[2], tw2); count_launch();
  k_y<R, +1><<<dim3(g.Xp, (d2 + wy - 1) / wy, nb), block_for(wy), 2 * (size_t)wy * d1 * sizeof(C), s>>>(
      A, B, g.Xp, g.Yp, g.m[1], d1, d2, g.plan[1], tw1); count_launch();
  k_xv<R><<<dim3(d1, (d2 + wx - 1) / wx, nb), block_for(wx), xv_smem<R>(wx, d0), s>>>(
      B, vr, g.Xp, g.m[0], d0, d1, d2, g.plan[0], tw0); count_launch();
  k_y<R, -1><<<dim3(g.Xp, (d2 + wy - 1) / wy, nb), block_for(wy), 2 * (size_t)wy * d1 * sizeof(C), s>>>(
      A, B, g.Xp, g.Yp, g.m[1], d1, d2, g.plan[1], tw1); count_launch();
  k_zfwd<R><<<dim3((g.ncol + wz - 1) / wz, nb), block_for(wz), 2 * (size_t)wz * d2 * sizeof(C), s>>>(
      A, psi, ldpsi, hpsi, ldh, h.kp[ik].kinetic, 1.0 / (double)g.N, g.col_start, g.pt_ig, g.pt_col, g.pt_z,
      g.ncol, d2, div_magic(d2), g.plan[2], tw2); count_launch();
}

Status local_apply_on_scratch(Handle& h, int spin, int ik, const double2* psi, long ldpsi, int nb, double2* hpsi,
                              long ldh, int precision, cudaStream_t s, void* scratch, size_t scratch_bytes) {
  if (ik < 0 || ik >= h.n_k) return fail(kInvalid, "k-point index out of range");
  if (spin < 0 || spin >= h.nspin) return fail(kInvalid, "spin index out of range");
  if (ldpsi < h.n_pw || ldh < h.n_pw) return fail(kInvalid, "leading dimension smaller than n_pw");
  if (nb <= 0) return kOk;
  GridMaps& g = h.g;
  const size_t cb = precision == 0 ? sizeof(double2) : sizeof(float2);
  const size_t a_elems = (size_t)g.ncol * g.d[2];
  const size_t b_elems = (size_t)g.Xp * g.d[1] * g.d[2];
  const size_t per_band = (a_elems + b_elems) * cb;
  // 256 bytes of margin for aligning B behind A
  const int chunk = scratch_bytes > 256 ? (int)std::min<size_t>(64, (scratch_bytes - 256) / per_band) : 0;
  if (chunk < 1)
    return fail(kInvalid, "grid too large for the fixed scratch: one band needs " + std::to_string(per_band) +
                              " bytes, the scratch holds " + std::to_string(scratch_bytes));
  unsigned char* base = static_cast<unsigned char*>(scratch);
  const size_t a_bytes = ((a_elems * chunk * cb) + 255) / 256 * 256;
  for (int c0 = 0; c0 < nb; c0 += chunk) {
    const int cnt = std::min(chunk, nb - c0);
    if (precision == 0)
      local_chunk_on<double>(h, spin, ik, psi + (long)c0 * ldpsi, ldpsi, cnt, hpsi + (long)c0 * ldh, ldh, s,
                             reinterpret_cast<double2*>(base), reinterpret_cast<double2*>(base + a_bytes));
    else
      local_chunk_on<float>(h, spin, ik, psi + (long)c0 * ldpsi, ldpsi, cnt, hpsi + (long)c0 * ldh, ldh, s,
                            reinterpret_cast<float2*>(base), reinterpret_cast<float2*>(base + a_bytes));
  }
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

Status density_accumulate(Handle& h, const double2* psi, long ldpsi, int nb, const double* fw_dev, double* rho,
                          cudaStream_t s) {
  GridMaps& g = h.g;
  const int d0 = g.d[0], d1 = g.d[1], d2 = g.d[2];
  double2* A = reinterpret_cast<double2*>(h.work_a);
  double2* B = reinterpret_cast<double2*>(h.work_b);
  if ((d0 + (kThreads / g.wx) - 1) / (kThreads / g.wx) > 16) return fail(kNotImplemented, "density: x tile too tall");
  for (int c0 = 0; c0 < nb; c0 += h.chunk) {
    const int cnt = std::min(h.chunk, nb - c0);
    {
      dim3 grid((g.ncol + g.wz - 1) / g.wz, cnt);
      k_zinv<double><<<grid, block_for(g.wz), 2 * (size_t)g.wz * d2 * sizeof(double2), s>>>(
          psi + (long)c0 * ldpsi, ldpsi, A, g.col_start, g.pt_ig, g.pt_col, g.pt_z, g.ncol, d2, div_magic(d2),
          g.plan[2], g.tw64[2]); count_launch();
    }
    {
      dim3 grid(g.Xp, (d2 + g.wy - 1) / g.wy, cnt);
      k_y<double, +1><<<grid, block_for(g.wy), 2 * (size_t)g.wy * d1 * sizeof(double2), s>>>(
          A, B, g.Xp, g.Yp, g.m[1], d1, d2, g.plan[1], g.tw64[1]); count_launch();
    }
    {
      dim3 grid(d1, (d2 + g.wx - 1) / g.wx, 1);
      k_x_density<<<grid, block_for(g.wx), 2 * (size_t)g.wx * d0 * sizeof(double2), s>>>(
          B, fw_dev + c0, cnt, rho, g.Xp, g.m[0], d0, d1, d2, g.plan[0], g.tw64[0]); count_launch();
    }
  }
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

Status apply_local_device(Handle& h, int spin, int ik, const double2* psi, long ldpsi, int nb, double2* hpsi,
                          long ldh, int precision, cudaStream_t s, StageTimer* tm) {
  // the work buffers are sized for h.chunk FP64 bands; FP32 fits twice as many
  const int chunk = precision == 0 ? h.chunk : 2 * h.chunk;
  for (int c0 = 0; c0 < nb; c0 += chunk) {
    const int cnt = std::min(chunk, nb - c0);
    Status st;
    if (precision == 0)
      st = local_chunk<double>(h, spin, ik, psi + (long)c0 * ldpsi, ldpsi, cnt, hpsi + (long)c0 * ldh, ldh, s, tm);
    else
      st = local_chunk<float>(h, spin, ik, psi + (long)c0 * ldpsi, ldpsi, cnt, hpsi + (long)c0 * ldh, ldh, s, tm);
    if (st != kOk) return st;
  }
  return kOk;
}

Status nonlocal_pq(Handle& h, int ik, const double2* psi, long ldpsi, int nb, cudaStream_t s, StageTimer* tm) {
  if (h.n_ch <= 0 || nb <= 0) return kOk;
  Status st;
  if ((st = ensure_nl_capacity(h, nb)) != kOk) return st;
  cublasSetStream(h.blas, s);
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  const cuDoubleComplex* Bm = reinterpret_cast<const cuDoubleComplex*>(h.kp[ik].b);
  cublasStatus_t cs = cublasZgemm(h.blas, CUBLAS_OP_C, CUBLAS_OP_N, h.n_ch, nb, h.n_pw, &one, Bm, h.n_pw,
                                  reinterpret_cast<const cuDoubleComplex*>(psi), (int)ldpsi, &zero,
                                  reinterpret_cast<cuDoubleComplex*>(h.nl_p), h.n_ch);
  if (cs != CUBLAS_STATUS_SUCCESS) return fail(kCuda, "cublasZgemm (B^H psi) failed");
  mark(tm, 5, s);
  const long tot = (long)h.n_ch * nb;
  k_apply_d<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(h.nl_p, h.nl_q, h.n_ch, nb, h.ch_atom, h.atom_ch_start,
                                                          h.d_off, h.d_vals); count_launch();
  mark(tm, 6, s);
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

Status apply_h_device(Handle& h, int spin, int ik, const double2* psi, long ldpsi, int nb, double2* hpsi, long ldh,
                      int precision, cudaStream_t s, StageTimer* tm) {
  if (ik < 0 || ik >= h.n_k) return fail(kInvalid, "apply_h: k-point index out of range");
  if (spin < 0 || spin >= h.nspin) return fail(kInvalid, "apply_h: spin index out of range");
  if (nb <= 0) return kOk;
  if (ldpsi < h.n_pw || ldh < h.n_pw) return fail(kInvalid, "apply_h: leading dimension smaller than n_pw");
  Status st;
  mark(tm, -1, s);
  if ((st = apply_local_device(h, spin, ik, psi, ldpsi, nb, hpsi, ldh, precision, s, tm)) != kOk) return st;
  if (h.n_ch > 0 && precision == 1 && nl_mixed_eligible(h)) {
    if ((st = nonlocal_mixed(h, ik, psi, ldpsi, nb, hpsi, ldh, s, tm)) != kOk) return st;
  } else if (h.n_ch > 0) {
    if ((st = nonlocal_pq(h, ik, psi, ldpsi, nb, s, tm)) != kOk) return st;
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
    const cuDoubleComplex* Bm = reinterpret_cast<const cuDoubleComplex*>(h.kp[ik].b);
    cublasStatus_t cs = cublasZgemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_N, h.n_pw, nb, h.n_ch, &one, Bm, h.n_pw,
                     reinterpret_cast<const cuDoubleComplex*>(h.nl_q), h.n_ch, &one,
                     reinterpret_cast<cuDoubleComplex*>(hpsi), (int)ldh);
    if (cs != CUBLAS_STATUS_SUCCESS) return fail(kCuda, "cublasZgemm (B Q) failed");
    mark(tm, 7, s);
    PW_CUDA_TRY(cudaGetLastError());
  }
  return kOk;
}

}  // namespace pwgpu
