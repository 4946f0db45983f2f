// In-shared-memory batched 1-D FFTs for 2,3,5-smooth lengths.
//
// A thread block holds a tile of `nlines` lines of length L in shared
// memory, plus a scratch tile of the same size.  Each Stockham stage
// (radix R in {2,3,4,5,8}, stride Ns) reads one tile and writes the other
// in auto-sorted order, one butterfly per thread at a time, so only R
// complex values live in registers.  Twiddles come from
// a per-length table tw[m] = exp(-2*pi*i*m/L), m < L, computed on the host
// in extended precision; the inverse uses the conjugate.  Both directions
// are unnormalised, matching the reference's FFT3D (fft.rs:19-114).
#pragma once

#include "pw_common.cuh"

namespace pwgpu {

// cos/sin constants of the small DFT kernels (exact values written out).
#define PW_SQRT1_2 0.70710678118654752440
#define PW_SIN60 0.86602540378443864676
#define PW_C1_5 0.30901699437494742410   // cos(2pi/5)
#define PW_S1_5 0.95105651629515357212   // sin(2pi/5)
#define PW_C2_5 (-0.80901699437494742410)  // cos(4pi/5)
#define PW_S2_5 0.58778525229247312917   // sin(4pi/5)

template <int S, typename C> __device__ __forceinline__ void dft2(C* v) {
  C a = v[0] + v[1], b = v[0] - v[1];
  v[0] = a; v[1] = b;
}

template <int S, typename C> __device__ __forceinline__ void dft4(C& u0, C& u1, C& u2, C& u3) {
  C s02 = u0 + u2, d02 = u0 - u2, s13 = u1 + u3, d13 = mul_si<S>(u1 - u3);
  u0 = s02 + s13; u2 = s02 - s13; u1 = d02 + d13; u3 = d02 - d13;
}

template <int S, typename C> __device__ __forceinline__ void dft3(C* v) {
  using R = decltype(v[0].x);
  C s = v[1] + v[2];
  C d = mul_si<S>(v[1] - v[2]) * (R)PW_SIN60;
  C m = v[0] - s * (R)0.5;
  v[0] = v[0] + s;
  v[1] = m + d;
  v[2] = m - d;
}

template <int S, typename C> __device__ __forceinline__ void dft5(C* v) {
  using R = decltype(v[0].x);
  C a1 = v[1] + v[4], b1 = v[1] - v[4], a2 = v[2] + v[3], b2 = v[2] - v[3];
  C x0 = v[0];
  C r1 = x0 + a1 * (R)PW_C1_5 + a2 * (R)PW_C2_5;
  C r2 = x0 + a1 * (R)PW_C2_5 + a2 * (R)PW_C1_5;
  C i1 = mul_si<S>(b1 * (R)PW_S1_5 + b2 * (R)PW_S2_5);
  C i2 = mul_si<S>(b1 * (R)PW_S2_5 - b2 * (R)PW_S1_5);
  v[0] = x0 + a1 + a2;
  v[1] = r1 + i1;
  v[4] = r1 - i1;
  v[2] = r2 + i2;
  v[3] = r2 - i2;
}

template <int S, typename C> __device__ __forceinline__ void dft8(C* v) {
  using R = decltype(v[0].x);
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<S>(e0, e1, e2, e3);
  dft4<S>(o0, o1, o2, o3);
  // twiddles w8^q, w8 = exp(S*2*pi*i/8)
  C t1, t3;
  t1.x = (R)PW_SQRT1_2 * (o1.x - S * o1.y);
  t1.y = (R)PW_SQRT1_2 * (o1.y + S * o1.x);
  C t2 = mul_si<S>(o2);
  t3.x = (R)PW_SQRT1_2 * (-o3.x - S * o3.y);
  t3.y = (R)PW_SQRT1_2 * (-o3.y + S * o3.x);
  v[0] = e0 + o0; v[4] = e0 - o0;
  v[1] = e1 + t1; v[5] = e1 - t1;
  v[2] = e2 + t2; v[6] = e2 - t2;
  v[3] = e3 + t3; v[7] = e3 - t3;
}

template <int R_, int S, typename C> __device__ __forceinline__ void dft(C* v) {
  if constexpr (R_ == 2) dft2<S>(v);
  else if constexpr (R_ == 3) dft3<S>(v);
  else if constexpr (R_ == 4) dft4<S>(v[0], v[1], v[2], v[3]);
  else if constexpr (R_ == 5) dft5<S>(v);
  else dft8<S>(v);
}

// Maps a tile line index to its base offset in shared memory and gives the
// element stride along the line.
struct LineMap {
  int lmul;     // base offset = line * lmul
  int estride;  // stride between consecutive elements of a line
};

// One Stockham stage over all lines of the tile, src -> dst (both tiles of
// the same shape).  Each thread takes butterflies tid, tid+T, ... and holds
// only the R values of the current one in registers.
template <int R_, int S, typename C>
__device__ __forceinline__ void fft_stage(const C* __restrict__ src, C* __restrict__ dst, int L, int Ns, int nlines,
                                          LineMap lm, const C* __restrict__ tw) {
  const int LR = L / R_;
  const int nbf = nlines * LR;
  const int twstep = L / (Ns * R_);
  for (int bf = threadIdx.x; bf < nbf; bf += blockDim.x) {
    const int line = bf / LR;
    const int j = bf - line * LR;
    const int k = j % Ns;
    const int base = line * lm.lmul;
    C v[R_];
#pragma unroll
    for (int r = 0; r < R_; ++r) {
      C x = src[base + (j + r * LR) * lm.estride];
      if (r > 0) {
        const C w = tw[k * r * twstep];
        x = (S < 0) ? cmul(x, w) : cmulc(x, w);
      }
      v[r] = x;
    }
    dft<R_, S>(v);
    const int ob = base + ((j / Ns) * Ns * R_ + k) * lm.estride;
    const int os = Ns * lm.estride;
#pragma unroll
    for (int q = 0; q < R_; ++q) dst[ob + q * os] = v[q];
  }
  __syncthreads();
}

// Full 1-D transform of every line of the tile (S = -1 forward, +1 inverse).
// The data starts in `a`; `b` is scratch of the same size.  Returns the
// buffer that holds the result (a or b, by the parity of the stage count).
template <int S, typename C>
__device__ __forceinline__ C* fft_lines(C* a, C* b, const FftPlan& p, int nlines, LineMap lm,
                                        const C* __restrict__ tw) {
  C* src = a;
  C* dst = b;
  for (int s = 0; s < p.nstages; ++s) {
    switch (p.radix[s]) {
      case 2: fft_stage<2, S>(src, dst, p.L, p.ns[s], nlines, lm, tw); break;
      case 3: fft_stage<3, S>(src, dst, p.L, p.ns[s], nlines, lm, tw); break;
      case 4: fft_stage<4, S>(src, dst, p.L, p.ns[s], nlines, lm, tw); break;
      case 5: fft_stage<5, S>(src, dst, p.L, p.ns[s], nlines, lm, tw); break;
      default: fft_stage<8, S>(src, dst, p.L, p.ns[s], nlines, lm, tw); break;
    }
    C* t = src; src = dst; dst = t;
  }
  return src;
}

}  // namespace pwgpu
