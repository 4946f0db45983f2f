// Cholesky factorisation with the inverse factor, G = R^H R and Ri = R^-1,
// for the Cholesky-QR orthonormalisation of the eigensolver's blocks (the
// reference orthonormalises through faer's dense factorisations in
// eigensolver/dense.rs:183-260; here one cluster launch does both the
// factor and its inverse).
//
// Design: one thread-block cluster of up to 16 CTAs, G and Ri in global
// memory (they are a few hundred KB and stay in L2), blocked right-looking
// over B x B tiles (B = 32 real, 16 complex).  Step k of nblk:
//   A(k)  the diagonal tile is factored by one warp with the columns in
//         registers (lane j holds column j of G_kk, then row j of its
//         inverse Z_kk = R_kk^-1, built column by column as the factor
//         proceeds: Z_jc = (delta_jc - sum_{l<c} Z_jl R_lc) / R_cc);
//   B(k)  panel tiles R_kj = Z_kk^H G_kj (j > k) and the inverse's column
//         block Z_ik = -S_ik Z_kk (i < k) from the running sums S;
//   C(k)  trailing tiles G_ij -= R_ki^H R_kj (k < i <= j) and the running
//         sums S_ij += Z_ik R_kj (i <= k < j, stored in Ri's tile (i, j)),
//         while CTA 0 updates the next diagonal tile and factors it (A(k+1)).
// Two cluster barriers per step.  The sums follow from Z R = I read column
// block by column block: Z_ik R_kk = -sum_{i<=l<k} Z_il R_lk.
//
// Pivots: info = 1 + the first row whose pivot is not positive (or not a
// number), as LAPACK's potrf counts; every CTA then leaves at the same step.

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <string>

#include "dense_ops.cuh"
#include "handle.hpp"
#include "linalg.hpp"

namespace pwgpu {

namespace {

namespace cg = cooperative_groups;
using namespace dense;

constexpr int kCholThreads = 256;
constexpr int kCholMaxCluster = 16;

template <typename T> struct TileB;
template <> struct TileB<double> { static constexpr int value = 32; };
template <> struct TileB<double2> { static constexpr int value = 16; };

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ double2 ldcg(const double2* p) { return __ldcg(p); }
__device__ __forceinline__ double zero_of(double) { return 0.0; }
__device__ __forceinline__ double2 zero_of(double2) { return make_double2(0.0, 0.0); }

// Tile (ti, tj) of the q x q column-major matrix M into shared memory s
// (column-major, leading dimension B + 1), zero outside the matrix.
template <typename T>
__device__ __forceinline__ void load_tile(const T* M, int q, int ti, int tj, T* s) {
  constexpr int B = TileB<T>::value, LD = B + 1;
  for (int e = threadIdx.x; e < B * B; e += kCholThreads) {
    const int r = e % B, c = e / B;
    const int gr = ti * B + r, gc = tj * B + c;
    s[r + c * LD] = (gr < q && gc < q) ? ldcg(M + gr + (long)gc * q) : zero_of(T());
  }
}

// Output mapping of a tile product: thread t owns column t / RT and rows
// t % RT + RT u, u < UR.
template <typename T> struct TileMap {
  static constexpr int B = TileB<T>::value;
  static constexpr int UR = B * B / kCholThreads;
  static constexpr int RT = B / UR;
};

template <typename T>
__device__ __forceinline__ void load_owned(const T* M, int q, int ti, int tj, T (&acc)[TileMap<T>::UR]) {
  constexpr int B = TileMap<T>::B, UR = TileMap<T>::UR, RT = TileMap<T>::RT;
  const int c = threadIdx.x / RT, r0 = threadIdx.x % RT;
#pragma unroll
  for (int u = 0; u < UR; ++u) {
    const int gr = ti * B + r0 + RT * u, gc = tj * B + c;
    acc[u] = (gr < q && gc < q) ? ldcg(M + gr + (long)gc * q) : zero_of(T());
  }
}

template <typename T>
__device__ __forceinline__ void store_owned(T* M, int q, int ti, int tj, const T (&acc)[TileMap<T>::UR]) {
  constexpr int B = TileMap<T>::B, UR = TileMap<T>::UR, RT = TileMap<T>::RT;
  const int c = threadIdx.x / RT, r0 = threadIdx.x % RT;
#pragma unroll
  for (int u = 0; u < UR; ++u) {
    const int gr = ti * B + r0 + RT * u, gc = tj * B + c;
    if (gr < q && gc < q) M[gr + (long)gc * q] = acc[u];
  }
}

// acc (+/-)= op(A) B over one tile, A and B in shared memory; op(A) = A,
// or A^H when HA (A(r, l) read as conj(A(l, r))).
template <typename T, bool HA, bool SUB>
__device__ __forceinline__ void tile_mma(const T* sA, const T* sB, T (&acc)[TileMap<T>::UR]) {
  constexpr int B = TileMap<T>::B, UR = TileMap<T>::UR, RT = TileMap<T>::RT, LD = B + 1;
  const int c = threadIdx.x / RT, r0 = threadIdx.x % RT;
#pragma unroll 8
  for (int l = 0; l < B; ++l) {
    const T b = sB[l + c * LD];
#pragma unroll
    for (int u = 0; u < UR; ++u) {
      const int r = r0 + RT * u;
      const T a = HA ? cj(sA[l + r * LD]) : sA[r + l * LD];
      acc[u] = SUB ? sub(acc[u], mul(a, b)) : add(acc[u], mul(a, b));
    }
  }
}

// Factor the diagonal tile kd held in shared memory sD (column-major,
// leading dimension B + 1, upper triangle valid) with warp 0: writes
// Z_kk = R_kk^-1 into Ri's tile (kd, kd) (zero below the diagonal), R's
// diagonal into rdiag, and on a failed pivot *info and *flag.  Rows and
// columns beyond q are treated as the identity.  Lane j keeps column j in
// registers; each finished row of R goes back into sD (row c of the tile),
// from where the other lanes read it as broadcasts.
template <typename T>
__device__ void factor_diag(T* sD, int q, int kd, T* Ri, double* rdiag, int* info, int* flag) {
  constexpr int B = TileB<T>::value, LD = B + 1;
  if (threadIdx.x >= 32) return;
  const int j = threadIdx.x;
  const int gj = kd * B + j;
  T a[B];  // column j of the tile, then of R_kk
  T z[B];  // row j of Z_kk
#pragma unroll
  for (int i = 0; i < B; ++i) {
    a[i] = gj < q ? (i <= j ? sD[i + j * LD] : zero_of(T())) : mk<T>(i == j ? 1.0 : 0.0, 0.0);
    z[i] = zero_of(T());
  }
  __syncwarp();
  int bad = -1;
  double rjj = 1.0;  // R_jj, taken at step j (a[] is indexed by compile-time constants only)
#pragma unroll
  for (int c = 0; c < B; ++c) {
    double d = re(shfl(a[c], c));
    if (!(d > 0.0)) {
      if (bad < 0) bad = c;
      d = 1.0;  // carry on with a harmless pivot; the result is discarded
    }
    const double rc = sqrt(d), ir = 1.0 / rc;
    if (j >= c) a[c] = mul(a[c], ir);  // row c of R (lane c: R_cc = rc)
    if (j == c) rjj = rc;
    sD[c + j * LD] = j >= c ? a[c] : zero_of(T());
    __syncwarp();
    // trailing rows first: the next pivot depends on them.  Every lane
    // updates every row (entries below the diagonal of column j hold finite
    // values that are never read), which keeps a[] in registers
#pragma unroll
    for (int i = c + 1; i < B; ++i) a[i] = sub(a[i], mul(cj(sD[c + i * LD]), a[c]));  // R_ci R_cj
    // Z_jc = (delta_jc - sum_{l<c} Z_jl R_lc) / R_cc, four partial sums
    T s0 = zero_of(T()), s1 = zero_of(T()), s2 = zero_of(T()), s3 = zero_of(T());
#pragma unroll
    for (int l = 0; l < c; ++l) {
      const T t = mul(z[l], sD[l + c * LD]);
      if ((l & 3) == 0) s0 = add(s0, t);
      else if ((l & 3) == 1) s1 = add(s1, t);
      else if ((l & 3) == 2) s2 = add(s2, t);
      else s3 = add(s3, t);
    }
    z[c] = mul(sub(mk<T>(j == c ? 1.0 : 0.0, 0.0), add(add(s0, s1), add(s2, s3))), ir);
  }
  // Z row j into Ri (lanes write consecutive rows of each column)
#pragma unroll
  for (int c = 0; c < B; ++c) {
    const int gc = kd * B + c;
    if (gj < q && gc < q) Ri[gj + (long)gc * q] = z[c];
  }
  if (gj < q && rdiag) rdiag[gj] = rjj;
  if (bad >= 0 && kd * B + bad < q && j == 0) {
    *info = kd * B + bad + 1;
    *flag = 1;
  }
}

// One tile product of a phase: C (+/-)= op(A) B with op(A) = A^H when ha;
// C starts from zero unless init.
template <typename T> struct TileTask {
  const T* A;
  int ai, aj;
  const T* Bm;
  int bi, bj;
  T* Cm;
  int ci, cj;
  bool ha, sub, init;
};

// A tile in registers (the load_tile mapping: element e = tid + 256 u).
template <typename T>
__device__ __forceinline__ void fetch_regs(const T* M, int q, int ti, int tj, T (&r)[TileMap<T>::UR]) {
  constexpr int B = TileB<T>::value, UR = TileMap<T>::UR;
#pragma unroll
  for (int u = 0; u < UR; ++u) {
    const int e = threadIdx.x + kCholThreads * u;
    const int gr = ti * B + e % B, gc = tj * B + e / B;
    r[u] = (gr < q && gc < q) ? ldcg(M + gr + (long)gc * q) : zero_of(T());
  }
}
template <typename T> __device__ __forceinline__ void regs_to_smem(const T (&r)[TileMap<T>::UR], T* s) {
  constexpr int B = TileB<T>::value, UR = TileMap<T>::UR, LD = B + 1;
#pragma unroll
  for (int u = 0; u < UR; ++u) {
    const int e = threadIdx.x + kCholThreads * u;
    s[e % B + (e / B) * LD] = r[u];
  }
}

template <typename T>
__device__ __forceinline__ void run_mma(const T* sA, const T* sB, bool ha, bool sub, T (&acc)[TileMap<T>::UR]) {
  if (ha) {
    if (sub) tile_mma<T, true, true>(sA, sB, acc);
    else tile_mma<T, true, false>(sA, sB, acc);
  } else {
    if (sub) tile_mma<T, false, true>(sA, sB, acc);
    else tile_mma<T, false, false>(sA, sB, acc);
  }
}

// Run tasks t = first, first + stride, ... < n of a phase, the operand
// tiles and the starting C of the next task loaded into registers while the
// current one computes.  fixedA / fixedB: an operand already in shared
// memory (the task's A or B pointer is then ignored).
template <typename T, typename Decode>
__device__ __forceinline__ void run_tasks(int first, int stride, int n, int q, Decode decode, T* sA, T* sB,
                                          const T* fixedA, const T* fixedB) {
  constexpr int UR = TileMap<T>::UR;
  if (first >= n) return;
  T ra[UR], rb[UR], rc[UR];
  TileTask<T> cur = decode(first);
  auto fetch = [&](const TileTask<T>& tk) {
    if (!fixedA) fetch_regs<T>(tk.A, q, tk.ai, tk.aj, ra);
    if (!fixedB) fetch_regs<T>(tk.Bm, q, tk.bi, tk.bj, rb);
    if (tk.init) {
      load_owned<T>(tk.Cm, q, tk.ci, tk.cj, rc);
    } else {
#pragma unroll
      for (int u = 0; u < UR; ++u) rc[u] = zero_of(T());
    }
  };
  fetch(cur);
  for (int t = first; t < n; t += stride) {
    if (!fixedA) regs_to_smem<T>(ra, sA);
    if (!fixedB) regs_to_smem<T>(rb, sB);
    T acc[UR];
#pragma unroll
    for (int u = 0; u < UR; ++u) acc[u] = rc[u];
    __syncthreads();
    TileTask<T> nxt = cur;
    if (t + stride < n) {
      nxt = decode(t + stride);
      fetch(nxt);  // in flight during the product
    }
    run_mma<T>(fixedA ? fixedA : sA, fixedB ? fixedB : sB, cur.ha, cur.sub, acc);
    store_owned<T>(cur.Cm, q, cur.ci, cur.cj, acc);
    __syncthreads();
    cur = nxt;
  }
}

template <typename T>
__global__ void __launch_bounds__(kCholThreads, 1) k_chol_inv(T* __restrict__ G, int q, T* __restrict__ Ri,
                                                             double* __restrict__ rdiag, int* __restrict__ info) {
  constexpr int B = TileB<T>::value, LD = B + 1, UR = TileMap<T>::UR;
  __shared__ T sA[B * LD];
  __shared__ T sB[B * LD];
  __shared__ T sZ[B * LD];
  __shared__ int flag;
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int nblk = (q + B - 1) / B;
  const int nlower = nblk * (nblk - 1) / 2;

  if (threadIdx.x == 0) flag = 0;
  // tiles strictly below the diagonal of Ri are zero
  for (int t = rank; t < nlower; t += C) {
    int i = 1, rem = t;  // t-th tile of the list (1,0), (2,0), (2,1), (3,0), ...
    while (rem >= i) {
      rem -= i;
      ++i;
    }
    T z[UR];
#pragma unroll
    for (int u = 0; u < UR; ++u) z[u] = zero_of(T());
    store_owned<T>(Ri, q, i, rem, z);
  }
  if (rank == 0) {
    load_tile<T>(G, q, 0, 0, sA);
    __syncthreads();
    factor_diag<T>(sA, q, 0, Ri, rdiag, info, &flag);
  }
  cluster.sync();

  for (int k = 0; k < nblk; ++k) {
    if (*cluster.map_shared_rank(&flag, 0) != 0) break;  // same value in every CTA: all leave here
    // ---- B(k): panel R_kj = Z_kk^H G_kj (j > k); inverse column block Z_ik = -S_ik Z_kk (i < k) ----
    const int npanel = nblk - 1 - k;
    if (rank < nblk - 1) {
      load_tile<T>(Ri, q, k, k, sZ);  // Z_kk (visible to all threads after the first barrier below)
      // panel tasks: A = Z_kk (fixed, conjugate-transposed), B = G_kj (fetched into sB)
      auto panel = [&](int t) {
        TileTask<T> tk{};
        const int j = k + 1 + t;
        tk.Bm = G; tk.bi = k; tk.bj = j;
        tk.Cm = G; tk.ci = k; tk.cj = j;
        tk.ha = true; tk.sub = false; tk.init = false;
        return tk;
      };
      run_tasks<T>(rank, C, npanel, q, panel, sA, sB, sZ, nullptr);
      // inverse tasks: A = S_ik (fetched into sA), B = Z_kk (fixed)
      auto zcol = [&](int t) {
        TileTask<T> tk{};
        tk.A = Ri; tk.ai = t; tk.aj = k;
        tk.Cm = Ri; tk.ci = t; tk.cj = k;
        tk.ha = false; tk.sub = true; tk.init = false;
        return tk;
      };
      // continue the rank's round-robin where the panel list left off
      const int first = ((rank - npanel) % C + C) % C;
      run_tasks<T>(first, C, k, q, zcol, sA, sB, nullptr, sZ);
    }
    if (k == nblk - 1) break;
    cluster.sync();
    // ---- C(k): trailing update and running sums; CTA 0 takes the next diagonal tile ----
    const int m = nblk - 1 - k;           // trailing block rows / columns
    const int n_trail = m * (m + 1) / 2;  // tiles (i, j), k < i <= j
    const int n_tasks = n_trail - 1 + (k + 1) * m;
    if (rank == 0) {
      T acc[UR];
      load_owned<T>(G, q, k + 1, k + 1, acc);
      load_tile<T>(G, q, k, k + 1, sA);
      __syncthreads();
      tile_mma<T, true, true>(sA, sA, acc);
      __syncthreads();
      {
        constexpr int RT = TileMap<T>::RT;
        const int c = threadIdx.x / RT, r0 = threadIdx.x % RT;
#pragma unroll
        for (int u = 0; u < UR; ++u) sB[r0 + RT * u + c * LD] = acc[u];
      }
      __syncthreads();
      factor_diag<T>(sB, q, k + 1, Ri, rdiag, info, &flag);
      __syncthreads();
    }
    const int workers = C > 1 ? C - 1 : 1;
    const int wid = C > 1 ? rank - 1 : 0;
    if (wid >= 0) {
      auto ctask = [&](int t) {
        TileTask<T> tk{};
        if (t < n_trail - 1) {
          // trailing tile number t + 1 of the list (k+1,k+1), (k+1,k+2), (k+2,k+2), (k+1,k+3), ...
          int jj = 0, rem = t + 1;
          while (rem > jj) {
            rem -= jj + 1;
            ++jj;
          }
          const int i = k + 1 + rem, j = k + 1 + jj;
          tk.A = G; tk.ai = k; tk.aj = i;
          tk.Bm = G; tk.bi = k; tk.bj = j;
          tk.Cm = G; tk.ci = i; tk.cj = j;
          tk.ha = true; tk.sub = true; tk.init = true;
        } else {
          const int u2 = t - (n_trail - 1);
          const int i = u2 % (k + 1), j = k + 1 + u2 / (k + 1);
          tk.A = Ri; tk.ai = i; tk.aj = k;
          tk.Bm = G; tk.bi = k; tk.bj = j;
          tk.Cm = Ri; tk.ci = i; tk.cj = j;
          tk.ha = false; tk.sub = false; tk.init = i != k;
        }
        return tk;
      };
      run_tasks<T>(wid, workers, n_tasks, q, ctask, sA, sB, nullptr, nullptr);
    }
    cluster.sync();
  }
  cluster.sync();  // CTA 0's flag may still be read by the others
}

int pick_chol_cluster(int q, int tile) {
  const int nblk = (q + tile - 1) / tile;
  if (nblk >= 6) return 16;
  if (nblk >= 4) return 8;
  if (nblk >= 3) return 4;
  if (nblk >= 2) return 2;
  return 1;
}

// The cluster-size opt-in is a per-device attribute: set once per device,
// under a lock (solves on several host threads reach here).
template <typename T> Status chol_attributes() {
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  PW_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(dev)) return kOk;
  cudaError_t err = cudaFuncSetAttribute(k_chol_inv<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (err != cudaSuccess) return fail(kCuda, std::string("chol_inv attributes: ") + cudaGetErrorString(err));
  done.insert(dev);
  return kOk;
}

// Whether a cluster of C CTAs of the kernel can be resident (checked once
// per size); a smaller cluster is used otherwise.
template <typename T> bool chol_cluster_fits(int C) {
  static std::mutex mu;
  static int cache[kCholMaxCluster + 1] = {};
  std::lock_guard<std::mutex> lock(mu);
  int& c = cache[C];
  if (c == 0) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(kCholThreads, 1, 1);
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&n, k_chol_inv<T>, &cfg);
    c = (e == cudaSuccess && n > 0) ? 1 : 2;
    if (e != cudaSuccess) cudaGetLastError();
  }
  return c == 1;
}

template <typename T> Status launch_chol(T* G, int q, T* Ri, double* rdiag, int* info, cudaStream_t s) {
  if (q < 1) return fail(kInvalid, "chol_inv: q must be positive");
  Status r = chol_attributes<T>();
  if (r != kOk) return r;
  int C = pick_chol_cluster(q, TileB<T>::value);
  while (C > 1 && !chol_cluster_fits<T>(C)) C /= 2;
  PW_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int), s));
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  cfg.gridDim = dim3(C, 1, 1);
  cfg.blockDim = dim3(kCholThreads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_chol_inv<T>, G, q, Ri, rdiag, info);
  count_launch();
  if (e != cudaSuccess) return fail(kCuda, std::string("chol_inv launch: ") + cudaGetErrorString(e));
  return kOk;
}

}  // namespace

Status chol_inv(double* G, int q, double* Ri, double* rdiag, int* info, cudaStream_t s) {
  return launch_chol<double>(G, q, Ri, rdiag, info, s);
}

Status chol_inv(double2* G, int q, double2* Ri, double* rdiag, int* info, cudaStream_t s) {
  return launch_chol<double2>(G, q, Ri, rdiag, info, s);
}

int chol_inv_cluster_size(int q, bool complex_matrix) {
  return pick_chol_cluster(q, complex_matrix ? TileB<double2>::value : TileB<double>::value);
}

}  // namespace pwgpu
