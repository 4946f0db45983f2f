// Kleinman-Bylander term of the mixed form as 3xBF16 tensor-core products.
//
// H_NL psi = B D B^H psi (potential/nonlocal.rs:432-450) is two complex
// GEMMs.  Each is written as one real GEMM through the embedding
//   P = B^H psi:   [B_r, B_i] (n_ch x 2 n_pw) * [[psi_r, psi_i], [psi_i, -psi_r]]  -> [P_r, P_i]
//   Y = B Q:       [B_r, B_i] (n_pw x 2 n_ch) * [[Q_r, Q_i], [-Q_i, Q_r]]          -> [Y_r, Y_i]
// and every real operand x is split x = hi + lo with hi = bf16(x),
// lo = bf16(x - hi).  The three products hi*hi + hi*lo + lo*hi (lo*lo is
// dropped, ~2^-16 relative) are summed by one GEMM whose K runs over the
// concatenation [A_hi | A_hi | A_lo] x [B_hi ; B_lo ; B_hi], accumulated in
// FP32 on the tensor cores.  The first GEMM (K = 6 n_pw, small M x N) is cut
// into split-K slices through the GEMM's batch index; the slice partials
// are summed in FP64 by the epilogue kernel that also forms complex P.  The
// projector operands are constant per k-point and are split once.
//
// Gamma-real handles hold their bands and projectors as packed real vectors
// (B_r, n_pw x n_ch); their two products are real from the start:
//   P = B_r^T u = hi(B_r^T) [u_hi | u_lo] + lo(B_r^T) u_hi
//   Y = B_r Q   = hi(B_r) [Q_hi | Q_lo] + lo(B_r) Q_hi
// each operand stored once as hi and once as lo (two GEMM calls a product).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "gemm_bf16.hpp"
#include "handle.hpp"

namespace pwgpu {

namespace {

inline long round_up(long x, long m) { return (x + m - 1) / m * m; }

__device__ __forceinline__ void split_bf16(double v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  const float f = (float)v;
  hi = __float2bfloat16_rn(f);
  lo = __float2bfloat16_rn(f - __bfloat162float(hi));
}

// A1[c][k], c < m1pad, k < k1pad: row c = [hi | hi | lo] of [B_r(:,c), B_i(:,c)]
__global__ void k_build_a1(const double2* __restrict__ b, int n_pw, int n_ch, long k1pad, int m1pad,
                           __nv_bfloat16* __restrict__ a1) {
  const long total = (long)m1pad * k1pad;
  const long seg_len = 2L * n_pw;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const long c = t / k1pad, k = t - c * k1pad;
    __nv_bfloat16 out = __float2bfloat16_rn(0.0f);
    if (c < n_ch && k < 3 * seg_len) {
      const int seg = (int)(k / seg_len);
      const long r = k - seg * seg_len;
      const double2 z = b[(r < n_pw ? r : r - n_pw) + c * (long)n_pw];
      __nv_bfloat16 hi, lo;
      split_bf16(r < n_pw ? z.x : z.y, hi, lo);
      out = seg < 2 ? hi : lo;
    }
    a1[t] = out;
  }
}

// A2[G][k], G < m2pad, k < k2pad: row G = [hi | hi | lo] of [B_r(G,:), B_i(G,:)]
__global__ void k_build_a2(const double2* __restrict__ b, int n_pw, int n_ch, long k2pad, long m2pad,
                           __nv_bfloat16* __restrict__ a2) {
  const long total = m2pad * k2pad;
  const long seg_len = 2L * n_ch;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const long g = t / k2pad, k = t - g * k2pad;
    __nv_bfloat16 out = __float2bfloat16_rn(0.0f);
    if (g < n_pw && k < 3 * seg_len) {
      const int seg = (int)(k / seg_len);
      const long r = k - seg * seg_len;
      const double2 z = b[g + (r < n_ch ? r : r - n_ch) * (long)n_pw];
      __nv_bfloat16 hi, lo;
      split_bf16(r < n_ch ? z.x : z.y, hi, lo);
      out = seg < 2 ? hi : lo;
    }
    a2[t] = out;
  }
}

// B1[j][k], j < 2 nb, k < k1pad: column j = [hi | lo | hi] of
// [psi_r; psi_i] (j < nb) or [psi_i; -psi_r] (j >= nb), band j mod nb,
// zero beyond 6 n_pw.  One thread per element (i, band): it reads psi once
// and writes its twelve entries (three segments of both columns, real and
// imaginary halves); rounding is symmetric, so the split of -psi_r is the
// negated split of psi_r.
__global__ void k_split_psi(const double2* __restrict__ psi, long ldpsi, int n_pw, int nb, long k1pad,
                            __nv_bfloat16* __restrict__ b1) {
  const int band = blockIdx.y;
  const long seg = 2L * n_pw;
  const long pad = k1pad - 3 * seg;
  __nv_bfloat16* c0 = b1 + (long)band * k1pad;
  __nv_bfloat16* c1 = b1 + (long)(nb + band) * k1pad;
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_pw; i += (long)gridDim.x * blockDim.x) {
    const double2 z = psi[band * ldpsi + i];
    __nv_bfloat16 hx, lx, hy, ly;
    split_bf16(z.x, hx, lx);
    split_bf16(z.y, hy, ly);
#pragma unroll
    for (int sg = 0; sg < 3; ++sg) {
      const long b = sg * seg + i;
      const bool lo = sg == 1;
      c0[b] = lo ? lx : hx;
      c0[b + n_pw] = lo ? ly : hy;
      c1[b] = lo ? ly : hy;
      c1[b + n_pw] = __hneg(lo ? lx : hx);
    }
    for (long q = i; q < pad; q += n_pw) {
      c0[3 * seg + q] = zero;
      c1[3 * seg + q] = zero;
    }
  }
}

// B2[j][k], j < 2 nb, k < k2pad: column j = [hi | lo | hi] of
// [Q_r; -Q_i] (j < nb) or [Q_i; Q_r] (j >= nb).  One grid row per column.
__global__ void k_split_q(const double2* __restrict__ q, int n_ch, int nb, long k2pad, __nv_bfloat16* __restrict__ b2) {
  const int j = blockIdx.y;
  const int part = j >= nb;
  const long band = part ? j - nb : j;
  const long seg_len = 2L * n_ch;
  const double2* col = q + band * n_ch;
  __nv_bfloat16* out = b2 + (long)j * k2pad;
  for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < k2pad; k += (long)gridDim.x * blockDim.x) {
    __nv_bfloat16 o = __float2bfloat16_rn(0.0f);
    if (k < 3 * seg_len) {
      const int seg = k >= 2 * seg_len ? 2 : (k >= seg_len ? 1 : 0);
      const long r = k - seg * seg_len;
      const double2 z = col[r < n_ch ? r : r - n_ch];
      const double v = part == 0 ? (r < n_ch ? z.x : -z.y) : (r < n_ch ? z.y : z.x);
      __nv_bfloat16 hi, lo;
      split_bf16(v, hi, lo);
      o = seg == 1 ? lo : hi;
    }
    out[k] = o;
  }
}

// P[c + b n_ch] = sum over slices of (D1[c, b], D1[c, nb + b])
__global__ void k_sum_p(const float* __restrict__ d1, int m1pad, int nb, int slices, long slice_stride, int n_ch,
                        double2* __restrict__ p) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)n_ch * nb) return;
  const int c = (int)(t % n_ch);
  const int b = (int)(t / n_ch);
  double re = 0.0, im = 0.0;
  for (int s = 0; s < slices; ++s) {
    const float* d = d1 + s * slice_stride;
    re += d[c + (long)b * m1pad];
    im += d[c + (long)(nb + b) * m1pad];
  }
  p[t] = make_double2(re, im);
}

// hpsi[G, b] += (D2[G, b], D2[G, nb + b])
__global__ void k_add_nl(const float* __restrict__ d2, long m2pad, int n_pw, int nb, double2* __restrict__ hpsi,
                         long ldh) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)n_pw * nb) return;
  const long g = t % n_pw;
  const long b = t / n_pw;
  double2 h = hpsi[g + b * ldh];
  h.x += d2[g + b * m2pad];
  h.y += d2[g + (nb + b) * m2pad];
  hpsi[g + b * ldh] = h;
}

// Real forms for Gamma-real handles (b: packed B_r, n x n_ch column-major).
// Each operand is stored once as hi and once as lo (no duplicated hi), and a
// product is two GEMM calls: hi x [x_hi | x_lo] and lo x x_hi, the three
// partial results summed in FP64 by the epilogue.
// A[r][k] (r < rows_pad, k < kpad) = hi or lo of B_r(k, r) (transposed: T) or
// B_r(r, k) (not transposed), zero outside; one flat index per element.
template <bool Trans>
__global__ void k_build_hilo_real(const double* __restrict__ b, int n, int n_ch, long rows_pad, long kpad,
                                  __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo) {
  // one grid row per output row r, threads along k (coalesced for the transposed form, whose source
  // column r is contiguous; the other form reads row r of B_r with stride n)
  const long rows = Trans ? n_ch : n, kk = Trans ? n : n_ch;
  for (long r = blockIdx.y; r < rows_pad; r += gridDim.y) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < kpad; k += (long)gridDim.x * blockDim.x) {
      __nv_bfloat16 h = __float2bfloat16_rn(0.0f), l = h;
      if (r < rows && k < kk) split_bf16(Trans ? b[k + r * (long)n] : b[r + k * (long)n], h, l);
      hi[r * kpad + k] = h;
      lo[r * kpad + k] = l;
    }
  }
}

// Columns of X (rows x nc, ld ldx) split into out[j] = hi(X(:, j)) and
// out[nc + j] = lo(X(:, j)), each column kpad long (zero-padded); one grid
// row per column j.
__global__ void k_split_hilo_cols(const double* __restrict__ x, long ldx, int rows, int nc, long kpad,
                                  __nv_bfloat16* __restrict__ out) {
  const int j = blockIdx.y;
  const double* col = x + (long)j * ldx;
  __nv_bfloat16* oh = out + (long)j * kpad;
  __nv_bfloat16* ol = out + (long)(nc + j) * kpad;
  for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < kpad; k += (long)gridDim.x * blockDim.x) {
    __nv_bfloat16 h = __float2bfloat16_rn(0.0f), l = h;
    if (k < rows) split_bf16(col[k], h, l);
    oh[k] = h;
    ol[k] = l;
  }
}

// P[c + b n_ch] = sum over slices of (hi x [u_hi | u_lo]) + (lo x u_hi):
// D1 holds per slice an m1pad x 2nb block, D3 per slice an m1pad x nb block
__global__ void k_sum_p_real(const float* __restrict__ d1, const float* __restrict__ d3, int m1pad, int nb, int slices,
                             long stride1, long stride3, int n_ch, double* __restrict__ p) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)n_ch * nb) return;
  const int c = (int)(t % n_ch);
  const int b = (int)(t / n_ch);
  double acc = 0.0;
  for (int s = 0; s < slices; ++s) {
    acc += (double)d1[s * stride1 + c + (long)b * m1pad] + (double)d1[s * stride1 + c + (long)(nb + b) * m1pad];
    acc += d3[s * stride3 + c + (long)b * m1pad];
  }
  p[t] = acc;
}

// hu[G, b] += D2[G, b] + D2[G, nb + b] + D4[G, b]
__global__ void k_add_nl_real(const float* __restrict__ d2, const float* __restrict__ d4, long m2pad, int n, int nb,
                              double* __restrict__ hu, long ldh) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)n * nb) return;
  const long g = t % n;
  const long b = t / n;
  hu[g + b * ldh] += ((double)d2[g + b * m2pad] + (double)d2[g + (nb + b) * m2pad]) + (double)d4[g + b * m2pad];
}

inline unsigned grid_for(long n) { return (unsigned)std::min<long>(148L * 16, std::max<long>(1, (n + 255) / 256)); }

}  // namespace

// Per-k split projector operands and per-call buffers of the mixed form.
struct NlMixed {
  long k1pad = 0, k2pad = 0, m2pad = 0;
  int m1pad = 0;
  std::vector<__nv_bfloat16*> a1, a2;  // per k
  __nv_bfloat16 *b1 = nullptr, *b2 = nullptr;
  float *d1 = nullptr, *d2 = nullptr;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  int nb_cap = 0, slices_cap = 0;
};

static void release_one(NlMixed*& m) {
  if (!m) return;
  for (auto p : m->a1) if (p) cudaFree(p);
  for (auto p : m->a2) if (p) cudaFree(p);
  if (m->b1) cudaFree(m->b1);
  if (m->b2) cudaFree(m->b2);
  if (m->d1) cudaFree(m->d1);
  if (m->d2) cudaFree(m->d2);
  if (m->ws) cudaFree(m->ws);
  delete m;
  m = nullptr;
}

void release_nl_mixed(Handle& h) {
  release_one(h.nlm);
  release_one(h.nlm_real);
}

// Below a few hundred channels and a few thousand plane waves the projector
// products are a handful of 128x128 tiles: the split/cast kernels and
// launches of the 3xBF16 form then cost more than one FP64 ZGEMM (measured on
// the 8-atom cells: 64-144 channels, 1,045-3,791 plane waves).
bool nl_mixed_eligible(const Handle& h) { return h.n_ch >= 256 && h.n_pw >= 4096; }

static Status nl_alloc(void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) return fail(kOom, std::string("cudaMalloc (mixed projectors): ") + cudaGetErrorString(e));
  return kOk;
}

// Split-K slices of the first product: up to `target` 128x128 tiles in
// flight, and the per-call operand buffers for n2 right-hand columns.
static int pick_slices(const NlMixed& m, int n2, long target) {
  const long tiles = ((m.m1pad + 127) / 128) * ((n2 + 127) / 128);
  int slices = 1;
  while (slices < 32 && tiles * slices * 2 <= target && m.k1pad / (slices * 2) >= 2048) slices *= 2;
  return slices;
}

// Tiles in flight for the Gamma-real products: a third of the SMs, so that
// the concurrent solves of a batch (each with its own handle and stream)
// keep running beside them; each tile holds an SM's shared memory.
constexpr long kRealTileTarget = 48;

static Status ensure_call_buffers(NlMixed& m, int n2, int slices) {
  if (n2 <= m.nb_cap && slices <= m.slices_cap) return kOk;
  const int cap = std::max(n2, m.nb_cap);
  const int scap = std::max(slices, m.slices_cap);
  if (m.b1) cudaFree(m.b1);
  if (m.b2) cudaFree(m.b2);
  if (m.d1) cudaFree(m.d1);
  if (m.d2) cudaFree(m.d2);
  if (m.ws) cudaFree(m.ws);
  m.b1 = m.b2 = nullptr;
  m.d1 = m.d2 = nullptr;
  m.ws = nullptr;
  m.nb_cap = m.slices_cap = 0;
  Status st;
  if ((st = nl_alloc((void**)&m.b1, (size_t)cap * m.k1pad * 2)) != kOk) return st;
  if ((st = nl_alloc((void**)&m.b2, (size_t)cap * m.k2pad * 2)) != kOk) return st;
  if ((st = nl_alloc((void**)&m.d1, (size_t)m.m1pad * cap * scap * 4)) != kOk) return st;
  if ((st = nl_alloc((void**)&m.d2, (size_t)m.m2pad * cap * 4)) != kOk) return st;
  size_t ws = gemm_bf16_workspace((int)m.m2pad, cap, (int)m.k2pad, 1);
  for (int sl = 1; sl <= scap; sl *= 2) ws = std::max(ws, gemm_bf16_workspace(m.m1pad, cap, (int)(m.k1pad / sl), sl));
  if ((st = nl_alloc(&m.ws, ws)) != kOk) return st;
  m.ws_bytes = ws;
  m.nb_cap = cap;
  m.slices_cap = scap;
  return kOk;
}

Status nonlocal_mixed_real(Handle& h, const double* u, long ldu, int nb, double* hu, long ldh, cudaStream_t s) {
  if (!h.gam.on) return fail(kState, "nonlocal_mixed_real: not a Gamma-real handle");
  if (h.n_ch <= 0 || nb <= 0) return kOk;
  const int n = h.n_pw;
  if (!h.nlm_real) {
    // a1 = {hi, lo} of B_r^T (n_ch x n), a2 = {hi, lo} of B_r (n x n_ch)
    h.nlm_real = new NlMixed();
    h.nlm_real->a1.assign(2, nullptr);
    h.nlm_real->a2.assign(2, nullptr);
    h.nlm_real->k1pad = round_up(n, 64L * 32);
    h.nlm_real->k2pad = round_up(h.n_ch, 64);
    h.nlm_real->m1pad = (int)round_up(h.n_ch, 8);
    h.nlm_real->m2pad = round_up(n, 8);
  }
  NlMixed& m = *h.nlm_real;
  Status st;
  if (!m.a1[0]) {
    for (int q = 0; q < 2; ++q) {
      if ((st = nl_alloc((void**)&m.a1[q], (size_t)m.m1pad * m.k1pad * 2)) != kOk) return st;
      if ((st = nl_alloc((void**)&m.a2[q], (size_t)m.m2pad * m.k2pad * 2)) != kOk) return st;
    }
    k_build_hilo_real<true><<<dim3((unsigned)std::min<long>(32, (m.k1pad + 255) / 256),
                                   (unsigned)std::min<long>(m.m1pad, 65535)), 256, 0, s>>>(
        h.gam.b_real, n, h.n_ch, m.m1pad, m.k1pad, m.a1[0], m.a1[1]);
    count_launch();
    k_build_hilo_real<false><<<dim3((unsigned)std::min<long>(32, (m.k2pad + 255) / 256),
                                    (unsigned)std::min<long>(m.m2pad, 65535)), 256, 0, s>>>(
        h.gam.b_real, n, h.n_ch, m.m2pad, m.k2pad, m.a2[0], m.a2[1]);
    count_launch();
  }
  // operand columns: [x_hi | x_lo] (2 nb); D1 / D2: hi x [x_hi | x_lo], D3 / D4: lo x x_hi (after D1 / D2)
  const int slices = pick_slices(m, 2 * nb, kRealTileTarget);
  const long ks = m.k1pad / slices;
  if ((st = ensure_call_buffers(m, 3 * nb, slices)) != kOk) return st;
  if ((st = ensure_gamma_pq(h, nb)) != kOk) return st;
  k_split_hilo_cols<<<dim3((unsigned)std::min<long>(64, (m.k1pad + 255) / 256), nb), 256, 0, s>>>(u, ldu, n, nb,
                                                                                                  m.k1pad, m.b1);
  count_launch();
  const long stride1 = (long)m.m1pad * 2 * nb, stride3 = (long)m.m1pad * nb;
  float* d3 = m.d1 + stride1 * slices;
  if ((st = gemm_bf16_tn_f32(m.a1[0], m.k1pad, ks, m.b1, m.k1pad, ks, m.d1, m.m1pad, stride1, m.m1pad, 2 * nb,
                             (int)ks, slices, m.ws, m.ws_bytes, s)) != kOk)
    return st;
  if ((st = gemm_bf16_tn_f32(m.a1[1], m.k1pad, ks, m.b1, m.k1pad, ks, d3, m.m1pad, stride3, m.m1pad, nb, (int)ks,
                             slices, m.ws, m.ws_bytes, s)) != kOk)
    return st;
  k_sum_p_real<<<(unsigned)(((long)h.n_ch * nb + 255) / 256), 256, 0, s>>>(m.d1, d3, m.m1pad, nb, slices, stride1,
                                                                           stride3, h.n_ch, h.gam_p);
  count_launch();
  if ((st = apply_d_real(h, nb, s)) != kOk) return st;
  k_split_hilo_cols<<<dim3((unsigned)std::min<long>(64, (m.k2pad + 255) / 256), nb), 256, 0, s>>>(
      h.gam_q, h.n_ch, h.n_ch, nb, m.k2pad, m.b2);
  count_launch();
  float* d4 = m.d2 + m.m2pad * 2 * nb;
  if ((st = gemm_bf16_tn_f32(m.a2[0], m.k2pad, 0, m.b2, m.k2pad, 0, m.d2, m.m2pad, 0, (int)m.m2pad, 2 * nb,
                             (int)m.k2pad, 1, m.ws, m.ws_bytes, s)) != kOk)
    return st;
  if ((st = gemm_bf16_tn_f32(m.a2[1], m.k2pad, 0, m.b2, m.k2pad, 0, d4, m.m2pad, 0, (int)m.m2pad, nb, (int)m.k2pad,
                             1, m.ws, m.ws_bytes, s)) != kOk)
    return st;
  k_add_nl_real<<<(unsigned)(((long)n * nb + 255) / 256), 256, 0, s>>>(m.d2, d4, m.m2pad, n, nb, hu, ldh);
  count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

Status nonlocal_mixed(Handle& h, int ik, const double2* psi, long ldpsi, int nb, double2* hpsi, long ldh,
                      cudaStream_t s, StageTimer* tm) {
  if (!h.nlm) {
    h.nlm = new NlMixed();
    h.nlm->a1.assign(h.n_k, nullptr);
    h.nlm->a2.assign(h.n_k, nullptr);
    h.nlm->k1pad = round_up(6L * h.n_pw, 64L * 32);
    h.nlm->k2pad = round_up(6L * h.n_ch, 64);
    h.nlm->m1pad = (int)round_up(h.n_ch, 8);
    h.nlm->m2pad = round_up(h.n_pw, 8);
  }
  NlMixed& m = *h.nlm;
  Status st;
  if (!m.a1[ik]) {
    if ((st = nl_alloc((void**)&m.a1[ik], (size_t)m.m1pad * m.k1pad * 2)) != kOk) return st;
    if ((st = nl_alloc((void**)&m.a2[ik], (size_t)m.m2pad * m.k2pad * 2)) != kOk) return st;
    k_build_a1<<<grid_for((long)m.m1pad * m.k1pad), 256, 0, s>>>(h.kp[ik].b, h.n_pw, h.n_ch, m.k1pad, m.m1pad,
                                                                m.a1[ik]);
    count_launch();
    k_build_a2<<<grid_for(m.m2pad * m.k2pad), 256, 0, s>>>(h.kp[ik].b, h.n_pw, h.n_ch, m.k2pad, m.m2pad, m.a2[ik]);
    count_launch();
  }
  // split-K slices of the first product: about two waves of 128x128 tiles
  const long tiles = ((m.m1pad + 127) / 128) * ((2L * nb + 127) / 128);
  int slices = 1;
  while (slices < 32 && tiles * slices < 2 * 148 && m.k1pad / (slices * 2) >= 2048) slices *= 2;
  const long ks = m.k1pad / slices;
  if (nb > m.nb_cap || slices > m.slices_cap) {
    const int cap = std::max(nb, m.nb_cap);
    const int scap = std::max(slices, m.slices_cap);
    if (m.b1) cudaFree(m.b1);
    if (m.b2) cudaFree(m.b2);
    if (m.d1) cudaFree(m.d1);
    if (m.d2) cudaFree(m.d2);
    if (m.ws) cudaFree(m.ws);
    m.b1 = m.b2 = nullptr;
    m.d1 = m.d2 = nullptr;
    m.ws = nullptr;
    if ((st = nl_alloc((void**)&m.b1, (size_t)2 * cap * m.k1pad * 2)) != kOk) return st;
    if ((st = nl_alloc((void**)&m.b2, (size_t)2 * cap * m.k2pad * 2)) != kOk) return st;
    if ((st = nl_alloc((void**)&m.d1, (size_t)m.m1pad * 2 * cap * scap * 4)) != kOk) return st;
    if ((st = nl_alloc((void**)&m.d2, (size_t)m.m2pad * 2 * cap * 4)) != kOk) return st;
    size_t ws = std::max(gemm_bf16_workspace(m.m1pad, 2 * cap, (int)(m.k1pad / scap), scap),
                         gemm_bf16_workspace((int)m.m2pad, 2 * cap, (int)m.k2pad, 1));
    for (int sl = 1; sl <= scap; sl *= 2)
      ws = std::max(ws, gemm_bf16_workspace(m.m1pad, 2 * cap, (int)(m.k1pad / sl), sl));
    if ((st = nl_alloc(&m.ws, ws)) != kOk) return st;
    m.ws_bytes = ws;
    m.nb_cap = cap;
    m.slices_cap = scap;
  }
  if ((st = ensure_nl_capacity(h, nb)) != kOk) return st;
  const int n2 = 2 * nb;
  k_split_psi<<<dim3((unsigned)std::min<long>(64, (h.n_pw + 255) / 256), nb), 256, 0, s>>>(psi, ldpsi, h.n_pw, nb,
                                                                                          m.k1pad, m.b1);
  count_launch();
  const long slice_stride = (long)m.m1pad * n2;
  if ((st = gemm_bf16_tn_f32(m.a1[ik], m.k1pad, ks, m.b1, m.k1pad, ks, m.d1, m.m1pad, slice_stride, m.m1pad, n2,
                             (int)ks, slices, m.ws, m.ws_bytes, s)) != kOk)
    return st;
  k_sum_p<<<(unsigned)(((long)h.n_ch * nb + 255) / 256), 256, 0, s>>>(m.d1, m.m1pad, nb, slices, slice_stride, h.n_ch,
                                                                       h.nl_p);
  count_launch();
  mark(tm, 5, s);
  if ((st = apply_d_blocks(h, nb, s)) != kOk) return st;
  mark(tm, 6, s);
  k_split_q<<<dim3((unsigned)std::min<long>(64, (m.k2pad + 255) / 256), n2), 256, 0, s>>>(h.nl_q, h.n_ch, nb,
                                                                                        m.k2pad, m.b2);
  count_launch();
  if ((st = gemm_bf16_tn_f32(m.a2[ik], m.k2pad, 0, m.b2, m.k2pad, 0, m.d2, m.m2pad, 0, (int)m.m2pad, n2,
                             (int)m.k2pad, 1, m.ws, m.ws_bytes, s)) != kOk)
    return st;
  k_add_nl<<<(unsigned)(((long)h.n_pw * nb + 255) / 256), 256, 0, s>>>(m.d2, m.m2pad, h.n_pw, nb, hpsi, ldh);
  count_launch();
  mark(tm, 7, s);
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

}  // namespace pwgpu
