// In-shared-memory batched 1-D FFTs for 2,3,5-smooth lengths.
//
// A thread block holds a tile of W interleaved lines of length L in shared
// memory, plus a scratch tile of the same size.  Each Stockham stage
// (radix R in {2,3,4,5,8,9}, stride Ns) reads one tile and writes the other
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

#define PW_C1_9 0.76604444311897803520    // cos(2pi/9)
#define PW_S1_9 0.64278760968653932632    // sin(2pi/9)
#define PW_C2_9 0.17364817766693034885    // cos(4pi/9)
#define PW_S2_9 0.98480775301220805936    // sin(4pi/9)
#define PW_C4_9 (-0.93969262078590838405) // cos(8pi/9)
#define PW_S4_9 0.34202014332566873304    // sin(8pi/9)

// 9-point DFT as 3 x 3: inner DFT3 over n1 (stride 3), twiddle w9^(n2*k1),
// outer DFT3 over n2; X[k1 + 3 k2].
template <int S, typename C> __device__ __forceinline__ void dft9(C* v) {
  using R = decltype(v[0].x);
  C y[3][3];
#pragma unroll
  for (int n2 = 0; n2 < 3; ++n2) {
    C t[3] = {v[n2], v[n2 + 3], v[n2 + 6]};
    dft3<S>(t);
    y[n2][0] = t[0]; y[n2][1] = t[1]; y[n2][2] = t[2];
  }
  // w9^m = cos(2 pi m/9) + S i sin(2 pi m/9), m in {1, 2, 4}
  const C w1 = cmake<C>(PW_C1_9, S * PW_S1_9);
  const C w2 = cmake<C>(PW_C2_9, S * PW_S2_9);
  const C w4 = cmake<C>(PW_C4_9, S * PW_S4_9);
  y[1][1] = cmul(y[1][1], w1);
  y[1][2] = cmul(y[1][2], w2);
  y[2][1] = cmul(y[2][1], w2);
  y[2][2] = cmul(y[2][2], w4);
  (void)sizeof(R);
#pragma unroll
  for (int k1 = 0; k1 < 3; ++k1) {
    C t[3] = {y[0][k1], y[1][k1], y[2][k1]};
    dft3<S>(t);
    v[k1] = t[0]; v[k1 + 3] = t[1]; v[k1 + 6] = t[2];
  }
}

template <int R_, int S, typename C> __device__ __forceinline__ void dft(C* v) {
  if constexpr (R_ == 2) dft2<S>(v);
  else if constexpr (R_ == 3) dft3<S>(v);
  else if constexpr (R_ == 4) dft4<S>(v[0], v[1], v[2], v[3]);
  else if constexpr (R_ == 5) dft5<S>(v);
  else if constexpr (R_ == 9) dft9<S>(v);
  else dft8<S>(v);
}

// Exact j / d for 0 <= j, j*d < 2^32 with m = ceil(2^32 / d) (d >= 2).
__device__ __forceinline__ int fast_div(int j, int d, unsigned m) {
  return d == 1 ? j : (int)__umulhi((unsigned)j, m);
}

// One Stockham stage, src -> dst.  Tile layout: element e of line l sits at
// e*W + l (lines interleaved, W = blockDim.x); threadIdx.x is the line and
// threadIdx.y strides the L/R butterflies, so a warp reads and writes
// adjacent shared-memory words and shares one twiddle.
template <int R_, int S, typename C>
__device__ __forceinline__ void fft_stage(const C* __restrict__ src, C* __restrict__ dst, int L, int Ns,
                                          unsigned nsm, int W, const C* __restrict__ tw) {
  const int LR = L / R_;
  const int twstep = L / (Ns * R_);
  const int line = threadIdx.x;
  for (int j = threadIdx.y; j < LR; j += blockDim.y) {
    const int jq = fast_div(j, Ns, nsm);
    const int k = j - jq * Ns;
    C v[R_];
#pragma unroll
    for (int r = 0; r < R_; ++r) {
      C x = src[(j + r * LR) * W + line];
      if (r > 0 && Ns > 1) {
        const C w = tw[k * r * twstep];
        x = (S < 0) ? cmul(x, w) : cmulc(x, w);
      }
      v[r] = x;
    }
    dft<R_, S>(v);
    const int ob = (jq * Ns * R_ + k) * W + line;
    const int os = Ns * W;
#pragma unroll
    for (int q = 0; q < R_; ++q) dst[ob + q * os] = v[q];
  }
  __syncthreads();
}

// The same stage with the radix, the stride Ns and the length known at
// compile time: constant index arithmetic and twiddle steps.
template <int R_, int Ns, int L, int S, typename C>
__device__ __forceinline__ void fft_stage_ct(const C* __restrict__ src, C* __restrict__ dst, int W,
                                             const C* __restrict__ tw) {
  constexpr int LR = L / R_;
  constexpr int twstep = L / (Ns * R_);
  const int line = threadIdx.x;
  for (int j = threadIdx.y; j < LR; j += blockDim.y) {
    const int jq = j / Ns;
    const int k = j - jq * Ns;
    C v[R_];
#pragma unroll
    for (int r = 0; r < R_; ++r) {
      C x = src[(j + r * LR) * W + line];
      if (r > 0 && Ns > 1) {
        const C w = tw[k * r * twstep];
        x = (S < 0) ? cmul(x, w) : cmulc(x, w);
      }
      v[r] = x;
    }
    dft<R_, S>(v);
    const int ob = (jq * Ns * R_ + k) * W + line;
#pragma unroll
    for (int q = 0; q < R_; ++q) dst[ob + q * Ns * W] = v[q];
  }
  __syncthreads();
}

// Two-stage lengths R0 * R1 (plan order: radix R0 first, stride 1; then R1,
// stride R0); the result ends in `a`.
template <int S, int R0, int R1, typename C>
__device__ __forceinline__ C* fft_lines_2(C* a, C* b, int W, const C* __restrict__ tw) {
  fft_stage_ct<R0, 1, R0 * R1, S>(a, b, W, tw);
  fft_stage_ct<R1, R0, R0 * R1, S>(b, a, W, tw);
  return a;
}

// Full 1-D transform of the W interleaved lines of a tile (S = -1 forward,
// +1 inverse).  The data starts in `a`; `b` is scratch of the same size.
// Returns the buffer holding the result (by the parity of the stage count).
// Common two-stage lengths take a compile-time path; the rest the plan's.
template <int S, typename C>
__device__ __forceinline__ C* fft_lines(C* a, C* b, const FftPlan& p, int W, const C* __restrict__ tw) {
  if (p.nstages == 2) {
    switch (p.radix[0] * 16 + p.radix[1]) {
      case 8 * 16 + 9: return fft_lines_2<S, 8, 9>(a, b, W, tw);   // 72
      case 8 * 16 + 5: return fft_lines_2<S, 8, 5>(a, b, W, tw);   // 40
      case 8 * 16 + 8: return fft_lines_2<S, 8, 8>(a, b, W, tw);   // 64
      case 8 * 16 + 4: return fft_lines_2<S, 8, 4>(a, b, W, tw);   // 32
      case 8 * 16 + 3: return fft_lines_2<S, 8, 3>(a, b, W, tw);   // 24
      case 8 * 16 + 2: return fft_lines_2<S, 8, 2>(a, b, W, tw);   // 16
      case 9 * 16 + 9: return fft_lines_2<S, 9, 9>(a, b, W, tw);   // 81
      case 9 * 16 + 5: return fft_lines_2<S, 9, 5>(a, b, W, tw);   // 45
      case 9 * 16 + 4: return fft_lines_2<S, 9, 4>(a, b, W, tw);   // 36
      case 9 * 16 + 3: return fft_lines_2<S, 9, 3>(a, b, W, tw);   // 27
      case 9 * 16 + 2: return fft_lines_2<S, 9, 2>(a, b, W, tw);   // 18
      case 5 * 16 + 5: return fft_lines_2<S, 5, 5>(a, b, W, tw);   // 25
      case 4 * 16 + 5: return fft_lines_2<S, 4, 5>(a, b, W, tw);   // 20
      default: break;
    }
  }
  C* src = a;
  C* dst = b;
  // Unrolled over the stage slots so every plan field is read at a fixed
  // parameter-bank offset (a runtime index would go through the slow
  // indexed-constant path), and if-chains instead of a jump table.
#pragma unroll
  for (int s = 0; s < kMaxStages; ++s) {
    if (s < p.nstages) {
      const int Ns = p.ns[s];
      const unsigned m = p.nsm[s];
      const int R = p.radix[s];
      if (R == 8) fft_stage<8, S>(src, dst, p.L, Ns, m, W, tw);
      else if (R == 9) fft_stage<9, S>(src, dst, p.L, Ns, m, W, tw);
      else if (R == 4) fft_stage<4, S>(src, dst, p.L, Ns, m, W, tw);
      else if (R == 5) fft_stage<5, S>(src, dst, p.L, Ns, m, W, tw);
      else if (R == 3) fft_stage<3, S>(src, dst, p.L, Ns, m, W, tw);
      else fft_stage<2, S>(src, dst, p.L, Ns, m, W, tw);
      C* t = src; src = dst; dst = t;
    }
  }
  return src;
}

// ---------------------------------------------------------------------------
// The same transforms for a tile of nl interleaved lines on a 1-D thread
// block (element e of line l at e*nl + l), any nl: butterfly t of a stage is
// line t mod nl, position t / nl, so consecutive threads touch consecutive
// words.  nlm = div_magic(nl).
// ---------------------------------------------------------------------------

template <int R_, int Ns, int L, int S, typename C>
__device__ __forceinline__ void stage_nl_ct(const C* __restrict__ src, C* __restrict__ dst, int nl, unsigned nlm,
                                            const C* __restrict__ tw) {
  constexpr int LR = L / R_;
  constexpr int twstep = L / (Ns * R_);
  for (int t = threadIdx.x; t < nl * LR; t += blockDim.x) {
    const int j = fast_div(t, nl, nlm);
    const int l = t - j * nl;
    const int jq = j / Ns;
    const int k = j - jq * Ns;
    C v[R_];
#pragma unroll
    for (int r = 0; r < R_; ++r) {
      C x = src[(j + r * LR) * nl + l];
      if (r > 0 && Ns > 1) {
        const C w = tw[k * r * twstep];
        x = (S < 0) ? cmul(x, w) : cmulc(x, w);
      }
      v[r] = x;
    }
    dft<R_, S>(v);
    const int ob = (jq * Ns * R_ + k) * nl + l;
#pragma unroll
    for (int q = 0; q < R_; ++q) dst[ob + q * Ns * nl] = v[q];
  }
  __syncthreads();
}

template <int R_, int S, typename C>
__device__ __forceinline__ void stage_nl(const C* __restrict__ src, C* __restrict__ dst, int L, int Ns, unsigned nsm,
                                         int nl, unsigned nlm, const C* __restrict__ tw) {
  const int LR = L / R_;
  const int twstep = L / (Ns * R_);
  for (int t = threadIdx.x; t < nl * LR; t += blockDim.x) {
    const int j = fast_div(t, nl, nlm);
    const int l = t - j * nl;
    const int jq = fast_div(j, Ns, nsm);
    const int k = j - jq * Ns;
    C v[R_];
#pragma unroll
    for (int r = 0; r < R_; ++r) {
      C x = src[(j + r * LR) * nl + l];
      if (r > 0 && Ns > 1) {
        const C w = tw[k * r * twstep];
        x = (S < 0) ? cmul(x, w) : cmulc(x, w);
      }
      v[r] = x;
    }
    dft<R_, S>(v);
    const int ob = (jq * Ns * R_ + k) * nl + l;
#pragma unroll
    for (int q = 0; q < R_; ++q) dst[ob + q * Ns * nl] = v[q];
  }
  __syncthreads();
}

template <int S, int R0, int R1, typename C>
__device__ __forceinline__ C* line_fft_2(C* a, C* b, int nl, unsigned nlm, const C* __restrict__ tw) {
  stage_nl_ct<R0, 1, R0 * R1, S>(a, b, nl, nlm, tw);
  stage_nl_ct<R1, R0, R0 * R1, S>(b, a, nl, nlm, tw);
  return a;
}

// Full 1-D transform of the nl interleaved lines of a tile; the result is in
// `a` for an even number of stages and in `b` for an odd number.
template <int S, typename C>
__device__ __forceinline__ C* line_fft(C* a, C* b, const FftPlan& p, int nl, unsigned nlm, const C* __restrict__ tw) {
  if (p.nstages == 2) {
    switch (p.radix[0] * 16 + p.radix[1]) {
      case 8 * 16 + 9: return line_fft_2<S, 8, 9>(a, b, nl, nlm, tw);   // 72
      case 8 * 16 + 5: return line_fft_2<S, 8, 5>(a, b, nl, nlm, tw);   // 40
      case 8 * 16 + 8: return line_fft_2<S, 8, 8>(a, b, nl, nlm, tw);   // 64
      case 8 * 16 + 4: return line_fft_2<S, 8, 4>(a, b, nl, nlm, tw);   // 32
      case 8 * 16 + 3: return line_fft_2<S, 8, 3>(a, b, nl, nlm, tw);   // 24
      case 9 * 16 + 5: return line_fft_2<S, 9, 5>(a, b, nl, nlm, tw);   // 45
      case 9 * 16 + 4: return line_fft_2<S, 9, 4>(a, b, nl, nlm, tw);   // 36
      case 5 * 16 + 5: return line_fft_2<S, 5, 5>(a, b, nl, nlm, tw);   // 25
      default: break;
    }
  }
  C* src = a;
  C* dst = b;
#pragma unroll
  for (int s = 0; s < kMaxStages; ++s) {
    if (s < p.nstages) {
      const int Ns = p.ns[s];
      const unsigned m = p.nsm[s];
      const int R = p.radix[s];
      if (R == 8) stage_nl<8, S>(src, dst, p.L, Ns, m, nl, nlm, tw);
      else if (R == 9) stage_nl<9, S>(src, dst, p.L, Ns, m, nl, nlm, tw);
      else if (R == 4) stage_nl<4, S>(src, dst, p.L, Ns, m, nl, nlm, tw);
      else if (R == 5) stage_nl<5, S>(src, dst, p.L, Ns, m, nl, nlm, tw);
      else if (R == 3) stage_nl<3, S>(src, dst, p.L, Ns, m, nl, nlm, tw);
      else stage_nl<2, S>(src, dst, p.L, Ns, m, nl, nlm, tw);
      C* t = src; src = dst; dst = t;
    }
  }
  return src;
}

// Stage with caller-supplied element access: ld(e, l) returns element e of
// line l of the input, st(e, l, v) stores element e of line l of the output,
// so the first and last stages of a transform can gather, scale or scatter
// on the way (no separate passes).
template <int R_, int Ns, int L, int S, typename C, typename Ld, typename St>
__device__ __forceinline__ void stage_f(int nl, unsigned nlm, const C* __restrict__ tw, Ld ld, St st) {
  constexpr int LR = L / R_;
  constexpr int twstep = L / (Ns * R_);
  for (int t = threadIdx.x; t < nl * LR; t += blockDim.x) {
    const int j = fast_div(t, nl, nlm);
    const int l = t - j * nl;
    const int jq = j / Ns;
    const int k = j - jq * Ns;
    C v[R_];
#pragma unroll
    for (int r = 0; r < R_; ++r) {
      C x = ld(j + r * LR, l);
      if (r > 0 && Ns > 1) {
        const C w = tw[k * r * twstep];
        x = (S < 0) ? cmul(x, w) : cmulc(x, w);
      }
      v[r] = x;
    }
    dft<R_, S>(v);
    const int ob = jq * Ns * R_ + k;
#pragma unroll
    for (int q = 0; q < R_; ++q) st(ob + q * Ns, l, v[q]);
  }
  __syncthreads();
}

// Two-stage transform of length R0 * R1 over nl lines: stage one reads
// through ld and writes tmp (interleaved), stage two reads tmp and writes
// through st.
template <int S, int R0, int R1, typename C, typename Ld, typename St>
__device__ __forceinline__ void line_fft2_f(int nl, unsigned nlm, const C* __restrict__ tw, C* __restrict__ tmp, Ld ld,
                                            St st) {
  stage_f<R0, 1, R0 * R1, S>(nl, nlm, tw, ld, [&](int e, int l, C v) { tmp[e * nl + l] = v; });
  stage_f<R1, R0, R0 * R1, S>(nl, nlm, tw, [&](int e, int l) { return tmp[e * nl + l]; }, st);
}

}  // namespace pwgpu
