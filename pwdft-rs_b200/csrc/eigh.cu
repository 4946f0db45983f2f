// Dense Hermitian / real symmetric eigensolver of the Rayleigh-Ritz step, one
// thread-block cluster per problem.
//
// Replaces the dense self_adjoint_eigen of the reference's per-k solve
// (pwdft-core/src/eigensolver/dense.rs:50-98, faer 0.24) where the
// matrix-free eigensolver needs it: the lowest nev eigenpairs of the
// m x m subspace matrix of each LOBPCG step (m <= 544).  One kernel does
// the whole solve on C = 1..16 CTAs of one cluster:
//
//  1. Householder reduction to real symmetric tridiagonal form, unblocked
//     (the zhetd2 recurrence: v, tau from the column below the diagonal,
//     p = tau A v, w = p - tau/2 (p^H v) v, A -= v w^H + w v^H).  The matrix
//     stays in shared memory for the whole reduction: column j lives in CTA
//     (j mod C), so the product A v needs no cross-CTA reduction (each CTA
//     owns whole columns of a Hermitian matrix = whole rows of A v).  Per
//     step the owner of column k broadcasts v into every CTA's shared
//     memory (distributed shared memory stores), one cluster barrier, every
//     CTA broadcasts its entries of p, a second barrier, every CTA updates
//     its own columns.  v stays in column k for the back-transform.
//  2. Eigenvalues of the tridiagonal T by multisection: one warp per
//     eigenvalue index, 32 Sturm counts per round (the three-term
//     recurrence of det(T - x I) with power-of-two rescaling; a zero term
//     takes the sign that counts it, as the zero pivot of the LDL^T count
//     does), until the interval is a few ulps wide.
//  3. Eigenvectors of T by inverse iteration, one thread per eigenvalue:
//     Gaussian elimination of T - lambda I with partial pivoting (a zero
//     pivot is replaced by eps ||T||), then two solves from a seeded start
//     vector.  Vectors whose eigenvalues lie within 1e-5 ||T|| of each
//     other are orthonormalised group by group (modified Gram-Schmidt,
//     twice), one warp per group; elsewhere inverse iteration leaves them
//     orthogonal to eps ||T|| / gap.
//  4. Back-transform x = H(0) ... H(m-2) z, one warp per eigenvector, the
//     vector in registers and the reflectors read from the owning CTAs'
//     shared memory.
//
// Every loop is bounded and every thread reaches the same sequence of
// cluster barriers.  Status: 0 ok, 1 a non-finite eigenvalue or vector.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <set>
#include <string>

#include "handle.hpp"
#include "dense_ops.cuh"
#include "linalg.hpp"

namespace cg = cooperative_groups;

// Phase timestamps for development builds (-DPWGPU_EIGH_PHASES): thread 0 of
// CTA 0 records %globaltimer at each phase boundary into eigh_phase_ns[].
#ifdef PWGPU_EIGH_PHASES
__device__ unsigned long long eigh_phase_ns[8];
__device__ long long eigh_sub_cycles[8];
#define EIGH_SUB_DECL long long sub_last_ = clock64(), sub_acc_[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#define EIGH_SUB(n)                                                             \
  do {                                                                          \
    if (rank == 0 && tid == 0) {                                                \
      const long long t_ = clock64();                                           \
      sub_acc_[n] += t_ - sub_last_;                                            \
      sub_last_ = t_;                                                           \
    }                                                                           \
  } while (0)
#define EIGH_SUB_STORE                                                          \
  do {                                                                          \
    if (rank == 0 && tid == 0)                                                  \
      for (int n_ = 0; n_ < 8; ++n_) eigh_sub_cycles[n_] = sub_acc_[n_];        \
  } while (0)
#define EIGH_MARK(n)                                                            \
  do {                                                                          \
    if (rank == 0 && tid == 0) {                                                \
      unsigned long long t_;                                                    \
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_));                    \
      eigh_phase_ns[n] = t_;                                                    \
    }                                                                           \
  } while (0)
#else
#define EIGH_MARK(n) \
  do {               \
  } while (0)
#define EIGH_SUB_DECL
#define EIGH_SUB(n) \
  do {              \
  } while (0)
#define EIGH_SUB_STORE \
  do {                 \
  } while (0)
#endif

namespace pwgpu {

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kRegRows = 17;               // rows per lane in the back-transform
constexpr int kMaxM = 32 * kRegRows;       // 544
constexpr int kMaxCluster = 16;
constexpr int kBisectRounds = 48;
constexpr double kEps = 1.1102230246251565e-16;  // 2^-53
constexpr size_t kSmemLimit = 227 * 1024;

using namespace dense;

// The two halves of a cluster barrier (release on arrival, acquire on the
// wait); every thread of every CTA arrives once, then waits, per phase.
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }

// Shared-memory layout of one CTA (identical on host and device).
struct Layout {
  size_t a, v, p, s, sc, d, e2, tau, eig, grp, red, hh, total;
};
__host__ __device__ inline size_t align16(size_t x) { return (x + 15) / 16 * 16; }
__host__ __device__ inline Layout layout(int m, int C, int tsz) {
  Layout L;
  const int ncl = (m + C - 1) / C;
  size_t o = 0;
  const size_t stage = (size_t)8 * ((m + 31) & ~31);  // 8 staged reflectors of the back-transform
  L.a = o;   o = align16(o + ((size_t)ncl * m > stage ? (size_t)ncl * m : stage) * tsz);  // owned columns
  L.v = o;   o = align16(o + 2 * (size_t)m * tsz);    // Householder vector, double-buffered
  L.p = o;   o = align16(o + (size_t)m * tsz);        // p = tau A v, all entries
  L.s = o;   o = align16(o + 2 * kMaxCluster * (size_t)tsz);  // per-CTA partials of p^H v
  L.sc = o;  o = align16(o + 2 * 4 * sizeof(double)); // tau (re, im), d_k, e_k per parity
  L.d = o;   o = align16(o + (size_t)m * sizeof(double));
  L.e2 = o;  o = align16(o + (size_t)m * sizeof(double));
  L.tau = o; o = align16(o + 2 * (size_t)m * tsz);  // tau of every step, then w of the current step
  L.eig = o; o = align16(o + (size_t)m * sizeof(double));
  L.grp = o; o = align16(o + (size_t)(m + 1) * sizeof(int));
  L.red = o; o = align16(o + 2 * kWarps * (size_t)tsz);
  L.hh = o;  o = align16(o + 8 * sizeof(double));
  L.total = o;
  return L;
}

// Number of eigenvalues of the tridiagonal (d, e2 = e^2 >= 1e-40, scaled to
// ||T|| <= 1) below x: sign changes of the three-term sequence of
// det(T - x I).  A zero term counts as a sign change (the zero pivot of the
// LDL^T count is taken as negative) and cannot repeat, since e2 > 0; with
// ||T|| <= 1 a term grows by at most 3x a step, so the power-of-two
// rescaling is checked once every eight steps.  The value chain is one
// fused multiply-add per step; d and e2 are read eight at a time.
__device__ __forceinline__ int sturm_count(const double* __restrict__ d, const double* __restrict__ e2, int m,
                                           double x) {
  double pp = 1.0, p = d[0] - x;
  bool sp = p <= 0.0;  // sign of the previous term as counted (a zero counts as negative after a positive)
  int cnt = sp;
  int i = 1;
  for (; i + 8 <= m; i += 8) {
    double dd[8], ee[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      dd[u] = d[i + u] - x;
      ee[u] = e2[i + u - 1];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const double pn = fma(dd[u], p, -ee[u] * pp);
      const bool sn = pn == 0.0 ? !sp : pn < 0.0;
      cnt += sn != sp;
      sp = sn;
      pp = p;
      p = pn;
    }
    const double ap = fmax(fabs(p), fabs(pp));
    if (ap > 0x1p+400) {
      p *= 0x1p-400;
      pp *= 0x1p-400;
    } else if (ap < 0x1p-400) {
      p *= 0x1p+400;
      pp *= 0x1p+400;
    }
  }
  for (; i < m; ++i) {
    const double pn = fma(d[i] - x, p, -e2[i - 1] * pp);
    const bool sn = pn == 0.0 ? !sp : pn < 0.0;
    cnt += sn != sp;
    sp = sn;
    pp = p;
    p = pn;
  }
  return cnt;
}

// Offset (in doubles) of the Gram blocks in the work buffer: after the 7 m nev
// doubles of phase 3, rounded up to 32 bytes so that complex entries are aligned.
__host__ __device__ inline size_t gram_offset(int m, int nev) { return ((size_t)7 * m * nev + 3) / 4 * 4; }
// Offset of the reflectors copied out of shared memory (m x m, complex size): after the Gram blocks.
__host__ __device__ inline size_t vglob_offset(int m, int nev) {
  return gram_offset(m, nev) + (size_t)128 * ((m + 3) / 4 + 1);
}

// Seeded start vector entry in [-1, 1).
__device__ __forceinline__ double start_entry(int i, int j) {
  uint64_t x = 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1) + 0xD1B54A32D192ED03ull * (uint64_t)(j + 7);
  x ^= x >> 31;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  x ^= x >> 33;
  return (double)(x >> 11) * 0x1p-52 - 1.0;
}

template <typename T> __device__ __forceinline__ T shfl_xor(T v, int o);
template <> __device__ __forceinline__ double shfl_xor<double>(double v, int o) {
  return __shfl_xor_sync(0xffffffffu, v, o);
}
template <> __device__ __forceinline__ double2 shfl_xor<double2>(double2 v, int o) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 1)
    k_eigh_cluster(const T* __restrict__ A, long lda, int m, int nev, double* __restrict__ w_out, T* __restrict__ Z,
                   long ldz, double* __restrict__ work, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem[];
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const Layout L = layout(m, C, (int)sizeof(T));
  T* a_loc = reinterpret_cast<T*>(smem + L.a);
  T* vbuf = reinterpret_cast<T*>(smem + L.v);
  T* pbuf = reinterpret_cast<T*>(smem + L.p);
  T* sbuf = reinterpret_cast<T*>(smem + L.s);
  double* scal = reinterpret_cast<double*>(smem + L.sc);
  double* dv = reinterpret_cast<double*>(smem + L.d);
  double* e2v = reinterpret_cast<double*>(smem + L.e2);
  T* tauv = reinterpret_cast<T*>(smem + L.tau);
  double* eig = reinterpret_cast<double*>(smem + L.eig);
  int* grp = reinterpret_cast<int*>(smem + L.grp);
  T* red = reinterpret_cast<T*>(smem + L.red);
  double* hh = reinterpret_cast<double*>(smem + L.hh);
  __shared__ double ev_off[kMaxM];  // off-diagonal e_k (the signed beta of each step)
  __shared__ double tnorm_s;
  __shared__ int bad;
  __shared__ int ngrp;
  const int nown = (m - rank + C - 1) / C;  // columns rank, rank + C, ... below m
  const int lgC = __ffs(C) - 1;              // C is a power of two
  T* wbuf = tauv + m;                        // w = p + alpha v of the current step

  EIGH_MARK(0);
  if (tid == 0) bad = 0;
  for (int s = 0; s < nown; ++s) {
    const T* src = A + (long)(rank + s * C) * lda;
    for (int i = tid; i < m; i += kThreads) a_loc[(size_t)s * m + i] = src[i];
  }
  cluster.sync();  // every CTA has started and loaded its columns
  EIGH_MARK(1);

  // ---- 1. Householder tridiagonalisation ----
  // Exchanges are pulled, never pushed.  The reflector of a step goes
  // through L2: its owner writes it to the reflector store in global memory
  // (which the back-transform reads anyway) and the other CTAs read it from
  // there, because fifteen CTAs pulling one CTA's shared memory measured
  // ~5 us a step at m = 540 against well under 1 us from L2.  The entries of
  // p (spread over all CTAs) and the step's scalars are remote shared-memory
  // loads; remote stores are several times slower than either.
  // Reflector of column kk, by all threads of its owner: v into the column
  // (leading 1) and into the store, (tau, d_kk, e_kk) into the owner's scal
  // of parity kk & 1.
  T* vglob_w = reinterpret_cast<T*>(work + vglob_offset(m, nev));
  __shared__ double s2_part[kWarps];  // per-warp partial sums of |col[i]|^2, rows >= kk + 2
  // have_parts: s2_part already holds the partials (summed while the column was updated)
  auto house = [&](int kk, bool have_parts) {
    T* col = a_loc + (size_t)(kk >> lgC) * m;
    if (warp == 0) {
      double s2 = 0.0;
      if (have_parts) {
        s2 = lane < kWarps ? s2_part[lane] : 0.0;
      } else {
        for (int i = kk + 2 + lane; i < m; i += 32) s2 += abs2(col[i]);
      }
      s2 = warp_sum(s2);
      if (lane == 0) {
        const T alpha = col[kk + 1];
        const double ar = re(alpha), ai = im(alpha);
        double tr = 0.0, ti = 0.0, beta = ar, sr = 0.0, si = 0.0;
        if (s2 > 0.0 || ai != 0.0) {
          const double nrm = sqrt(ar * ar + ai * ai + s2);
          beta = ar >= 0.0 ? -nrm : nrm;
          const double ib = 1.0 / beta;
          tr = (beta - ar) * ib;
          ti = -ai * ib;
          const double dr = ar - beta, di = ai, iden = 1.0 / (dr * dr + di * di);  // scale = 1 / (alpha - beta)
          sr = dr * iden;
          si = -di * iden;
        }
        double* sc2 = scal + 4 * (kk & 1);
        sc2[0] = tr;
        sc2[1] = ti;
        sc2[2] = re(col[kk]);
        sc2[3] = beta;
        hh[0] = sr;
        hh[1] = si;
      }
    }
    __syncthreads();
    const double* sc2 = scal + 4 * (kk & 1);
    const bool rf = sc2[0] != 0.0 || sc2[1] != 0.0;
    const T scale = mk<T>(hh[0], hh[1]);
    T* vg = vglob_w + (size_t)kk * m;
    for (int i = kk + 1 + tid; i < m; i += kThreads) {
      const T x = i == kk + 1 ? mk<T>(1.0, 0.0) : (rf ? mul(col[i], scale) : mk<T>(0.0, 0.0));
      col[i] = x;
      vg[i] = x;
    }
  };

  // B1 of a step is split: the owner of the next column arrives as soon as
  // its reflector is out and updates its other columns afterwards, so that
  // update is off the path the other CTAs wait on; the rest arrive after
  // their update.  B2 is a full cluster barrier.
  if (m > 1 && rank == 0) house(0, false);
  cluster_arrive();
  EIGH_SUB_DECL
  for (int k = 0; k < m - 1; ++k) {
    const int par = k & 1;
    const int owner = k & (C - 1);
    EIGH_SUB(0);
    cluster_wait();  // B1: the reflector of column k is in the store and its owner's scal
    EIGH_SUB(1);
    // pull v (rows k+1 .. m-1) and the step's scalars from the owner
    const T* vb;
    if (owner == rank) {
      vb = a_loc + (size_t)(k >> lgC) * m;
    } else {
      const T* src = vglob_w + (size_t)k * m;  // written before B1 by the owner; read past L1
      for (int i = k + 1 + tid; i < m; i += kThreads) vbuf[i] = __ldcg(src + i);
      if (tid < 4) scal[4 * par + tid] = cluster.map_shared_rank(scal, owner)[4 * par + tid];
      vb = vbuf;
      __syncthreads();
    }
    const double* sc = scal + 4 * par;
    const T tau = mk<T>(sc[0], sc[1]);
    const bool refl = sc[0] != 0.0 || sc[1] != 0.0;
    if (tid == 0) {
      dv[k] = sc[2];
      ev_off[k] = sc[3];
      tauv[k] = tau;
    }
    const int s0 = k + 1 > rank ? (k + 1 - rank + C - 1) >> lgC : 0;  // first owned slot with column > k
    const int na = nown - s0;
    const bool look = k + 1 < m - 1 && rank == ((k + 1) & (C - 1));  // this CTA reflects column k + 1 next
    // R lanes per owned column (a power of two dividing 32)
    int R = 32;
    while (R > 1 && na * R > kThreads) R >>= 1;
    const int r = lane & (R - 1);
    const int gpw = 32 / R;  // column groups per warp
    if (refl) {
      // p_j = tau sum_i conj(A[i, j]) v_i for owned j > k, R lanes per column; partials of p^H v
      T part = mk<T>(0.0, 0.0);
      for (int gb = warp * gpw; gb < na; gb += kWarps * gpw) {
        const int g = gb + lane / R;
        const bool act = g < na;
        const int sl = s0 + (act ? g : 0);
        const T* col = a_loc + (size_t)sl * m;
        T acc0 = mk<T>(0.0, 0.0), acc1 = mk<T>(0.0, 0.0), acc2 = mk<T>(0.0, 0.0), acc3 = mk<T>(0.0, 0.0);
        if (act) {
          int i = k + 1 + r;
          for (; i + 3 * R < m; i += 4 * R) {
            acc0 = add(acc0, mul(cj(col[i]), vb[i]));
            acc1 = add(acc1, mul(cj(col[i + R]), vb[i + R]));
            acc2 = add(acc2, mul(cj(col[i + 2 * R]), vb[i + 2 * R]));
            acc3 = add(acc3, mul(cj(col[i + 3 * R]), vb[i + 3 * R]));
          }
          for (; i < m; i += R) acc0 = add(acc0, mul(cj(col[i]), vb[i]));
        }
        T acc = add(add(acc0, acc1), add(acc2, acc3));
        for (int o = R / 2; o > 0; o >>= 1) acc = add(acc, shfl_xor(acc, o));
        if (act && r == 0) {
          const int j = rank + (sl << lgC);
          const T pj = mul(tau, acc);
          pbuf[j] = pj;
          part = add(part, mul(cj(pj), vb[j]));
        }
      }
      EIGH_SUB(2);
      part = warp_sum(part);
      if (lane == 0) red[warp] = part;
      __syncthreads();
      if (warp == 0) {
        const T tot = warp_sum(lane < kWarps ? red[lane] : mk<T>(0.0, 0.0));
        if (lane == 0) sbuf[kMaxCluster * par + rank] = tot;
      }
      EIGH_SUB(3);
      cluster.sync();  // B2: every CTA's entries of p and partial of p^H v are in place
      EIGH_SUB(4);
      // pull the other partials, then w = p + alpha v over rows k+1 .. m-1 into pbuf (entries of p
      // owned elsewhere pulled on the way)
      if (tid < C && tid != rank)
        sbuf[kMaxCluster * par + tid] = cluster.map_shared_rank(sbuf, tid)[kMaxCluster * par + tid];
      __syncthreads();
      T ssum = mk<T>(0.0, 0.0);
      for (int q = 0; q < C; ++q) ssum = add(ssum, sbuf[kMaxCluster * par + q]);
      const T alpha = mul(mul(tau, ssum), -0.5);
      for (int i = k + 1 + tid; i < m; i += kThreads) {
        const int q = i & (C - 1);
        const T pi = q == rank ? pbuf[i] : cluster.map_shared_rank(pbuf, q)[i];
        wbuf[i] = add(pi, mul(alpha, vb[i]));
      }
      __syncthreads();
      EIGH_SUB(5);
      if (look) {
        // column k + 1 first, so that its reflector is ready early
        // (with the norm its reflector needs summed on the way)
        T* col = a_loc + (size_t)((k + 1) >> lgC) * m;
        const T cwj = cj(wbuf[k + 1]), cvj = cj(vb[k + 1]);
        double s2 = 0.0;
        for (int i = k + 1 + tid; i < m; i += kThreads) {
          const T x = sub(col[i], add(mul(vb[i], cwj), mul(wbuf[i], cvj)));
          col[i] = x;
          if (i >= k + 3) s2 += abs2(x);
        }
        s2 = warp_sum(s2);
        if (lane == 0) s2_part[warp] = s2;
        __syncthreads();
        house(k + 1, true);
        cluster_arrive();
      }
      EIGH_SUB(6);
      for (int gb = warp * gpw; gb < na; gb += kWarps * gpw) {
        const int g = gb + lane / R;
        if (g >= na) continue;
        const int sl = s0 + g;
        const int j = rank + (sl << lgC);
        if (look && j == k + 1) continue;
        T* col = a_loc + (size_t)sl * m;
        const T cwj = cj(wbuf[j]), cvj = cj(vb[j]);
#pragma unroll 4
        for (int i = k + 1 + r; i < m; i += R) col[i] = sub(col[i], add(mul(vb[i], cwj), mul(wbuf[i], cvj)));
      }
    } else if (look) {
      house(k + 1, false);
      cluster_arrive();
    }
    __syncthreads();
    if (!look) cluster_arrive();
    EIGH_SUB(7);
  }
  cluster_wait();  // completes the last arrival
  EIGH_SUB_STORE;
  // the reflector store complete (column k holds v_k on rows k+1 .. m-1, zero above), for the back-transform
  for (int sl = 0; sl < nown; ++sl) {
    const int k = rank + sl * C;
    const T* col = a_loc + (size_t)sl * m;
    for (int i = tid; i < m; i += kThreads) vglob_w[(size_t)k * m + i] = i > k ? col[i] : mk<T>(0.0, 0.0);
  }
  // last diagonal entry
  if (rank == (m - 1) % C && tid == 0) dv[m - 1] = re(a_loc[(size_t)((m - 1) / C) * m + (m - 1)]);
  if (tid == 0) ev_off[m - 1] = 0.0;
  cluster.sync();
  if (rank != (m - 1) % C && tid == 0) dv[m - 1] = re(cluster.map_shared_rank(a_loc, (m - 1) % C)[(size_t)((m - 1) / C) * m + (m - 1)]);
  cluster.sync();
  EIGH_MARK(2);

  // ---- 2. eigenvalues by multisection on T / ||T|| ----
  if (warp == 0) {
    double gl = INFINITY, gu = -INFINITY;
    for (int i = lane; i < m; i += 32) {
      const double rr = (i > 0 ? fabs(ev_off[i - 1]) : 0.0) + fabs(ev_off[i]);
      gl = fmin(gl, dv[i] - rr);
      gu = fmax(gu, dv[i] + rr);
    }
    for (int o = 16; o > 0; o >>= 1) {
      gl = fmin(gl, __shfl_xor_sync(0xffffffffu, gl, o));
      gu = fmax(gu, __shfl_xor_sync(0xffffffffu, gu, o));
    }
    if (lane == 0) {
      const double tn = fmax(fabs(gl), fabs(gu));
      tnorm_s = tn > 0.0 && isfinite(tn) ? tn : 1.0;
      if (!isfinite(tn)) bad = 1;
    }
  }
  __syncthreads();
  const double tnorm = tnorm_s, itn = 1.0 / tnorm;
  for (int i = tid; i < m; i += kThreads) {
    dv[i] *= itn;
    ev_off[i] *= itn;
    // an off-diagonal below 1e-20 ||T|| counts as 1e-20 in the Sturm sequence, so a zero term never
    // propagates (a perturbation far below rounding)
    e2v[i] = fmax(ev_off[i] * ev_off[i], 1e-40);
  }
  __syncthreads();
  {
    const double glo = -1.0 - 4.0 * kEps * m, ghi = 1.0 + 4.0 * kEps * m;  // the scaled Gershgorin interval
    const int tt = C * kThreads;
    int P = 32;  // points per eigenvalue and round
    while (P > 1 && (long)nev * P > tt) P >>= 1;
    const int pr = lane & (P - 1), seg = lane & ~(P - 1);
    const int ng = tt / P;
    for (int jb = (rank * kThreads + warp * 32) / P; jb < nev; jb += ng) {
      const int j = jb + lane / P;
      const bool act = j < nev;
      double lo = glo, hi = ghi;
      for (int round = 0; round < kBisectRounds; ++round) {
        const bool done = !act || hi - lo <= 2.0 * kEps * fmax(fabs(lo), fabs(hi)) + kEps;
        if (__all_sync(0xffffffffu, done)) break;
        const double x = lo + (hi - lo) * (double)(pr + 1) / (double)(P + 1);
        const int cnt = sturm_count(dv, e2v, m, x);
        const unsigned bits = (__ballot_sync(0xffffffffu, act && cnt > j) >> seg) & (P == 32 ? 0xffffffffu : ((1u << P) - 1u));
        const int l = bits ? __ffs(bits) - 1 : P;
        const double xhi = __shfl_sync(0xffffffffu, x, seg + (l < P ? l : P - 1));
        const double xlo = __shfl_sync(0xffffffffu, x, seg + (l > 0 ? l - 1 : 0));
        if (!done) {
          const double nlo = l > 0 ? xlo : lo;
          const double nhi = l < P ? xhi : hi;
          if (!(nhi < hi) && !(nlo > lo)) {
            hi = lo = 0.5 * (lo + hi);  // no representable progress
          } else {
            lo = nlo;
            hi = nhi;
          }
        }
      }
      if (act && pr == 0) {
        const double lam = 0.5 * (lo + hi);
        for (int q = 0; q < C; ++q) cluster.map_shared_rank(eig, q)[j] = lam;
        w_out[j] = lam * tnorm;
        if (!isfinite(lam)) bad = 1;
      }
    }
  }
  cluster.sync();
  EIGH_MARK(3);

  // ---- 3. inverse iteration on T / ||T||, one thread per eigenvalue ----
  // work: per row i and eigenvalue j (index i * nev + j) the U row {1/u0, u1, u2, rhs} as double4 and the
  // row operation {l, swapped} as double2; then the vectors, column j at zt + j * m
  {
    double4* U4 = reinterpret_cast<double4*>(work);
    double2* F2 = reinterpret_cast<double2*>(work + (size_t)4 * m * nev);
    double* zt = work + (size_t)6 * m * nev;
    const double piv_min = kEps;
    const int nj = (nev + C - 1) / C;
    for (int jj = tid; jj < nj; jj += kThreads) {
      const int j = rank * nj + jj;
      if (j >= nev) break;
      const double lam = eig[j];
      // factorisation, the start vector carried as right-hand side
      double a = dv[0] - lam, b = m > 1 ? ev_off[0] : 0.0, cur = start_entry(0, j);
      for (int i = 0; i < m - 1; ++i) {
        const size_t o = (size_t)i * nev + j;
        const double c = ev_off[i];
        const double dn = dv[i + 1] - lam, en = i + 1 < m - 1 ? ev_off[i + 1] : 0.0;
        const double nxt = start_entry(i + 1, j);
        if (fabs(a) >= fabs(c)) {
          if (fabs(a) < piv_min) a = a < 0.0 ? -piv_min : piv_min;
          const double ia = 1.0 / a, l = c * ia;
          U4[o] = make_double4(ia, b, 0.0, cur);
          F2[o] = make_double2(l, 0.0);
          const double ncur = nxt - l * cur;
          a = dn - l * b;
          b = en;
          cur = ncur;
        } else {
          const double ic = 1.0 / c, l = a * ic;
          U4[o] = make_double4(ic, dn, en, nxt);
          F2[o] = make_double2(l, 1.0);
          const double ncur = cur - l * nxt;
          a = b - l * dn;
          b = -l * en;
          cur = ncur;
        }
      }
      if (fabs(a) < piv_min) a = a < 0.0 ? -piv_min : piv_min;
      U4[(size_t)(m - 1) * nev + j] = make_double4(1.0 / a, 0.0, 0.0, cur);
      double scale = 1.0;
      for (int it = 0; it < 2; ++it) {
        if (it > 0) {
          // the stored row operations on the normalised vector
          double c0 = U4[j].w * scale;
          int i = 0;
          for (; i + 8 <= m - 1; i += 8) {
            double2 f[8];
            double nx[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              f[q] = F2[(size_t)(i + q) * nev + j];
              nx[q] = U4[(size_t)(i + q + 1) * nev + j].w * scale;
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              double out;
              if (f[q].y == 0.0) {
                out = c0;
                c0 = nx[q] - f[q].x * c0;
              } else {
                out = nx[q];
                c0 = c0 - f[q].x * nx[q];
              }
              reinterpret_cast<double*>(&U4[(size_t)(i + q) * nev + j])[3] = out;
            }
          }
          for (; i < m - 1; ++i) {
            const double2 f = F2[(size_t)i * nev + j];
            const double nx = U4[(size_t)(i + 1) * nev + j].w * scale;
            double out;
            if (f.y == 0.0) {
              out = c0;
              c0 = nx - f.x * c0;
            } else {
              out = nx;
              c0 = c0 - f.x * nx;
            }
            reinterpret_cast<double*>(&U4[(size_t)i * nev + j])[3] = out;
          }
          reinterpret_cast<double*>(&U4[(size_t)(m - 1) * nev + j])[3] = c0;
        }
        // back-substitution, eight rows per batch of loads
        double y1 = 0.0, y2 = 0.0, nrm2 = 0.0;
        int i = m - 1;
        for (; i >= 7; i -= 8) {
          double4 u[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) u[q] = U4[(size_t)(i - q) * nev + j];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const double yi = (u[q].w - u[q].y * y1 - u[q].z * y2) * u[q].x;
            reinterpret_cast<double*>(&U4[(size_t)(i - q) * nev + j])[3] = yi;
            nrm2 += yi * yi;
            y2 = y1;
            y1 = yi;
          }
        }
        for (; i >= 0; --i) {
          const double4 u = U4[(size_t)i * nev + j];
          const double yi = (u.w - u.y * y1 - u.z * y2) * u.x;
          reinterpret_cast<double*>(&U4[(size_t)i * nev + j])[3] = yi;
          nrm2 += yi * yi;
          y2 = y1;
          y1 = yi;
        }
        const bool okn = nrm2 > 0.0 && isfinite(nrm2);
        scale = okn ? 1.0 / sqrt(nrm2) : 0.0;
        if (!okn) bad = 1;
      }
      double* zj = zt + (size_t)j * m;
      for (int i = 0; i < m; ++i) zj[i] = U4[(size_t)i * nev + j].w * scale;
    }
  }
  __threadfence();
  cluster.sync();
  EIGH_MARK(4);

  const int gw = rank * kWarps + warp, nw = C * kWarps;
  // ---- 3b. groups of close eigenvalues: modified Gram-Schmidt, twice ----
  {
    double* zt = work + (size_t)6 * m * nev;
    if (tid == 0) {
      const double gtol = 1e-5;  // in units of ||T||
      int n = 0;
      int start = 0;
      for (int j = 1; j <= nev; ++j) {
        if (j == nev || eig[j] - eig[j - 1] > gtol) {
          if (j - start > 1) {
            grp[2 * n] = start;
            grp[2 * n + 1] = j;
            ++n;
          }
          start = j;
        }
      }
      ngrp = n;
    }
    __syncthreads();
    for (int g = gw; g < ngrp; g += nw) {
      const int g0 = grp[2 * g], g1 = grp[2 * g + 1];
      for (int j = g0; j < g1; ++j) {
        double* zj = zt + (size_t)j * m;
        for (int pass = 0; pass < 2; ++pass) {
          for (int i = g0; i < j; ++i) {
            const double* zi = zt + (size_t)i * m;
            double dot = 0.0;
            for (int rr = lane; rr < m; rr += 32) dot += zi[rr] * zj[rr];
            dot = warp_sum(dot);
            for (int rr = lane; rr < m; rr += 32) zj[rr] -= dot * zi[rr];
            __syncwarp();
          }
        }
        double n2 = 0.0;
        for (int rr = lane; rr < m; rr += 32) n2 += zj[rr] * zj[rr];
        n2 = warp_sum(n2);
        const double scn = n2 > 0.0 ? 1.0 / sqrt(n2) : 0.0;
        if (!(n2 > 0.0) && lane == 0) bad = 1;
        for (int rr = lane; rr < m; rr += 32) zj[rr] *= scn;
        __syncwarp();
      }
    }
  }
  // ---- 4a. Gram blocks of the reflectors: G[b][q][p] = v_kq^H v_kp, kq = m-2-BR*b-q, p < q ----
  constexpr int BR = sizeof(T) == sizeof(double) ? 8 : 4;  // reflectors per round of the back-transform
  constexpr int NPAIR = BR * (BR - 1) / 2;
  const int nblk = (m - 1 + BR - 1) / BR;
  T* gram = reinterpret_cast<T*>(work + gram_offset(m, nev));
  const T* vglob = reinterpret_cast<const T*>(work + vglob_offset(m, nev));
  for (int t = gw; t < nblk * NPAIR; t += nw) {
    const int b = t / NPAIR;
    int pq = t % NPAIR, q = 1;
    while (pq >= q) {
      pq -= q;
      ++q;
    }
    const int p = pq;  // 0 <= p < q < BR
    const int k0 = m - 2 - BR * b;
    const int kq = k0 - q, kp = k0 - p;
    T acc = mk<T>(0.0, 0.0);
    if (kq >= 0) {
      const T* vq = vglob + (size_t)kq * m;
      const T* vp = vglob + (size_t)kp * m;
      for (int i = kp + 1 + lane; i < m; i += 32) acc = add(acc, mul(cj(vq[i]), vp[i]));
    }
    acc = warp_sum(acc);
    if (lane == 0) gram[(size_t)b * 64 + q * 8 + p] = acc;
  }
  __threadfence();
  cluster.sync();
  EIGH_MARK(5);

  // ---- 4. back-transform x = H(0) ... H(m-2) z, one warp per vector, BR reflectors per round ----
  // Each round the CTA stages the round's reflectors (from global memory, where they are L2-resident)
  // and their Gram block into shared memory; every warp then applies them to its vector in registers.
  // The staged rows have stride mp (m rounded up to 32) and start zeroed, so rows outside a
  // reflector's support contribute exact zeros and the inner loops carry no predicates; row slots
  // wholly below the round's first row, or past m, are skipped (warp-uniform tests).
  {
    const double* zt = work + (size_t)6 * m * nev;
    const int mp = (m + 31) & ~31;
    const int nt = mp >> 5;
    T* sv = a_loc;  // BR x mp staged reflectors (the matrix columns are no longer needed)
    __shared__ T sgram[64];
    __shared__ T stau[8];
    const int waves = (nev + nw - 1) / nw;
    for (int wv = 0; wv < waves; ++wv) {
      const int j = gw + wv * nw;
      const bool live = j < nev;  // a warp without a vector still helps to stage
      // each wave starts from zeroed staging rows (the previous wave's last rounds filled low rows)
      __syncthreads();
      for (int e = tid; e < BR * mp; e += kThreads) sv[e] = mk<T>(0.0, 0.0);
      T z[kRegRows];
#pragma unroll
      for (int t = 0; t < kRegRows; ++t) {
        const int i = lane + 32 * t;
        z[t] = mk<T>(live && i < m ? zt[(size_t)j * m + i] : 0.0, 0.0);
      }
      for (int b = 0; b < nblk; ++b) {
        const int k0 = m - 2 - BR * b;
        const int lo = k0 - BR + 2 > 0 ? k0 - BR + 2 : 0;  // first row any reflector of the round touches
        __syncthreads();  // the previous round's readers are done
        for (int q = 0; q < BR; ++q) {
          const int kq = k0 - q;
          if (kq < 0) break;
          const T* src = vglob + (size_t)kq * m;
          for (int i = lo + tid; i < m; i += kThreads) sv[q * mp + i] = src[i];
        }
        if (tid < 64) sgram[tid] = gram[(size_t)b * 64 + tid];
        if (tid < BR) stau[tid] = k0 - tid >= 0 ? tauv[k0 - tid] : mk<T>(0.0, 0.0);
        __syncthreads();
        if (!live) continue;
        const int t0 = lo >> 5;
        T sq[BR];
#pragma unroll
        for (int q = 0; q < BR; ++q) sq[q] = mk<T>(0.0, 0.0);
#pragma unroll
        for (int t = 0; t < kRegRows; ++t) {
          if (t < t0 || t >= nt) continue;
          const int i = lane + 32 * t;
#pragma unroll
          for (int q = 0; q < BR; ++q) sq[q] = add(sq[q], mul(cj(sv[q * mp + i]), z[t]));
        }
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
          for (int q = 0; q < BR; ++q) sq[q] = add(sq[q], shfl_xor(sq[q], o));
        }
        T f[BR];
#pragma unroll
        for (int q = 0; q < BR; ++q) {
          T sv_q = sq[q];
#pragma unroll
          for (int p = 0; p < q; ++p) sv_q = sub(sv_q, mul(f[p], sgram[q * 8 + p]));
          f[q] = mul(stau[q], sv_q);
        }
#pragma unroll
        for (int t = 0; t < kRegRows; ++t) {
          if (t < t0 || t >= nt) continue;
          const int i = lane + 32 * t;
          T zz = z[t];
#pragma unroll
          for (int q = 0; q < BR; ++q) zz = sub(zz, mul(sv[q * mp + i], f[q]));
          z[t] = zz;
        }
      }
      if (live) {
        bool ok = true;
#pragma unroll
        for (int t = 0; t < kRegRows; ++t) {
          const int i = lane + 32 * t;
          if (i < m) {
            Z[(size_t)j * ldz + i] = z[t];
            ok = ok && finite(z[t]);
          }
        }
        if (!ok) bad = 1;
      }
    }
  }
  __syncthreads();
  EIGH_MARK(6);
  if (tid == 0 && bad) atomicExch(status, 1);
  cluster.sync();  // no CTA leaves while another may still read its shared memory
}

// The smallest cluster whose CTAs hold the matrix in shared memory (0: none).
int min_cluster(int m, int tsz) {
  for (int C = 1; C <= kMaxCluster; C *= 2)
    if (layout(m, C, tsz).total + 2 * kMaxM * sizeof(double) <= kSmemLimit) return C;
  return 0;
}

// The cluster size to use: measured on B200, a 16-CTA cluster is fastest
// for every m > 64 (at m = 135 / 180 / 270 the solve takes 0.43 / 0.53 /
// 0.74 of its time on the smallest cluster that fits, mostly through the
// back-transform, bisection and inverse iteration that spread over the
// CTAs) and within a few percent at m = 360; 8 CTAs below, and never more
// CTAs than columns.
int pick_cluster(int m, int tsz) {
  const int c0 = min_cluster(m, tsz);
  if (c0 == 0) return 0;
  int want = m > 64 ? 16 : 8;
  while (want > m) want /= 2;
  return std::max(c0, want);
}

// The shared-memory and cluster-size opt-ins are per-device attributes: set
// once per device, under a lock (solves on several host threads reach here).
template <typename T> Status set_attributes() {
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  PW_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(dev)) return kOk;
  auto kern = k_eigh_cluster<T>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kSmemLimit - 2 * kMaxM * sizeof(double)));
  if (err == cudaSuccess) err = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (err != cudaSuccess) return fail(kCuda, std::string("eigh_cluster attributes: ") + cudaGetErrorString(err));
  done.insert(dev);
  return kOk;
}

template <typename T> cudaLaunchConfig_t launch_config(int m, int C, cudaLaunchAttribute* attr, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(kThreads, 1, 1);
  cfg.dynamicSmemBytes = layout(m, C, (int)sizeof(T)).total;
  cfg.stream = s;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// Whether a cluster of C CTAs with this kernel's shared memory can be
// resident on the current device (checked once per cluster size).
template <typename T> bool cluster_fits(int m, int C) {
  static std::mutex mu;
  static int cache[2][kMaxCluster + 1] = {};  // [real, complex][C]: 0 unknown, 1 fits, 2 does not
  const int slot = sizeof(T) == sizeof(double) ? 0 : 1;
  std::lock_guard<std::mutex> lock(mu);
  // the largest m that uses a cluster size has the most shared memory: probe at that size
  int& c = cache[slot][C];
  if (c == 0) {
    if (set_attributes<T>() != kOk) return false;
    int mm = 1;  // the largest m a cluster of C CTAs can hold: the most shared memory
    for (int t = 1; t <= kMaxM; ++t)
      if (layout(t, C, (int)sizeof(T)).total + 2 * kMaxM * sizeof(double) <= kSmemLimit) mm = t;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = launch_config<T>(mm, C, attr, nullptr);
    int n = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&n, k_eigh_cluster<T>, &cfg);
    c = (e == cudaSuccess && n > 0) ? 1 : 2;
    if (e != cudaSuccess) cudaGetLastError();
  }
  return c == 1;
}

// The preferred cluster size, halved while such a cluster cannot be
// resident on this device (0 when none can).
template <typename T> int choose_cluster(int m) {
  if (m < 1 || m > kMaxM) return 0;
  const int c0 = min_cluster(m, (int)sizeof(T));
  if (c0 == 0) return 0;
  int C = pick_cluster(m, (int)sizeof(T));
  while (C > c0 && !cluster_fits<T>(m, C)) C /= 2;
  return cluster_fits<T>(m, C) ? C : 0;
}

template <typename T>
Status launch_eigh(const T* A, long lda, int m, int nev, double* w, T* Z, long ldz, double* work, int* status,
                   cudaStream_t s) {
  const int C = choose_cluster<T>(m);
  if (C == 0) return fail(kInvalid, "eigh_cluster: matrix too large for the cluster eigensolver");
  Status r = set_attributes<T>();
  if (r != kOk) return r;
  auto kern = k_eigh_cluster<T>;
  PW_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), s));
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config<T>(m, C, attr, s);
  cudaError_t e = cudaLaunchKernelEx(&cfg, kern, A, lda, m, nev, w, Z, ldz, work, status);
  count_launch();
  if (e != cudaSuccess) return fail(kCuda, std::string("eigh_cluster launch: ") + cudaGetErrorString(e));
  return kOk;
}


}  // namespace

size_t eigh_cluster_work_doubles(int m, int nev) {
  // U rows, row operations and vectors (7 m nev), then the reflectors' Gram blocks (64 complex per block of 8)
  return vglob_offset(m, std::max(nev, 1)) + (size_t)2 * m * m;
}

bool eigh_cluster_supported(int m, bool complex_matrix) {
  return eigh_cluster_size(m, complex_matrix) > 0;
}

int eigh_cluster_size(int m, bool complex_matrix) {
  return complex_matrix ? choose_cluster<double2>(m) : choose_cluster<double>(m);
}

Status eigh_cluster(const double* A, long lda, int m, int nev, double* w, double* Z, long ldz, double* work,
                    int* status, cudaStream_t s) {
  return launch_eigh<double>(A, lda, m, nev, w, Z, ldz, work, status, s);
}

Status eigh_cluster(const double2* A, long lda, int m, int nev, double* w, double2* Z, long ldz, double* work,
                    int* status, cudaStream_t s) {
  return launch_eigh<double2>(A, lda, m, nev, w, Z, ldz, work, status, s);
}

}  // namespace pwgpu
