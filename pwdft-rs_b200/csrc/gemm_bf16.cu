// BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05.mma,
// accumulators in TMEM, operands staged by TMA), built from CUTLASS's sm100
// collective templates: one CTA per 128x128 tile (1x1 cluster, so no
// cluster-multicast loads), warp-specialised TMA producer / MMA / epilogue.
//
//   D[l] (M x N, column-major, ldd) = A[l] (M x K, row-major, lda) * B[l] (K x N, column-major, ldb)
//
// for l = 0..L-1 with element strides strideA/B/D between batches.  The
// 3xBF16 projector products use the batch index as split-K slices whose
// FP32 partials are summed by the caller's epilogue kernel.
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <string>

#include "cutlass/cutlass.h"
#include "cute/tensor.hpp"
#include "cutlass/epilogue/collective/collective_builder.hpp"
#include "cutlass/gemm/collective/collective_builder.hpp"
#include "cutlass/gemm/device/gemm_universal_adapter.h"
#include "cutlass/gemm/dispatch_policy.hpp"
#include "cutlass/gemm/kernel/gemm_universal.hpp"

#include "gemm_bf16.hpp"
#include "handle.hpp"

namespace pwgpu {

namespace {

using namespace cute;

using ElementA = cutlass::bfloat16_t;
using ElementB = cutlass::bfloat16_t;
using ElementD = float;
using ElementAcc = float;
using LayoutA = cutlass::layout::RowMajor;
using LayoutB = cutlass::layout::ColumnMajor;
using LayoutD = cutlass::layout::ColumnMajor;
constexpr int kAlignA = 8;
constexpr int kAlignB = 8;
constexpr int kAlignD = 4;

using MmaTileShape = Shape<_128, _128, _64>;
using ClusterShape = Shape<_1, _1, _1>;

using CollectiveEpilogue = typename cutlass::epilogue::collective::CollectiveBuilder<
    cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, MmaTileShape, ClusterShape,
    cutlass::epilogue::collective::EpilogueTileAuto, ElementAcc, ElementAcc, ElementD, LayoutD, kAlignD, ElementD,
    LayoutD, kAlignD, cutlass::epilogue::TmaWarpSpecialized1Sm>::CollectiveOp;

using CollectiveMainloop = typename cutlass::gemm::collective::CollectiveBuilder<
    cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, ElementA, LayoutA, kAlignA, ElementB, LayoutB, kAlignB,
    ElementAcc, MmaTileShape, ClusterShape,
    cutlass::gemm::collective::StageCountAutoCarveout<static_cast<int>(
        sizeof(typename CollectiveEpilogue::SharedStorage))>,
    cutlass::gemm::KernelTmaWarpSpecialized1SmSm100>::CollectiveOp;

using GemmKernel = cutlass::gemm::kernel::GemmUniversal<Shape<int, int, int, int>, CollectiveMainloop,
                                                        CollectiveEpilogue, void>;
using Gemm = cutlass::gemm::device::GemmUniversalAdapter<GemmKernel>;

using StrideA = typename GemmKernel::StrideA;
using StrideB = typename GemmKernel::StrideB;
using StrideC = typename GemmKernel::StrideC;
using StrideD = typename GemmKernel::StrideD;

typename Gemm::Arguments make_args(const void* A, long lda, long sa, const void* B, long ldb, long sb, float* D,
                                   long ldd, long sd, int M, int N, int K, int L) {
  StrideA stA{};
  cute::get<0>(stA) = lda;
  cute::get<2>(stA) = sa;
  StrideB stB{};
  cute::get<0>(stB) = ldb;
  cute::get<2>(stB) = sb;
  StrideD stD{};
  cute::get<1>(stD) = ldd;
  cute::get<2>(stD) = sd;
  StrideC stC = stD;
  typename Gemm::Arguments args{cutlass::gemm::GemmUniversalMode::kGemm,
                                {M, N, K, L},
                                {reinterpret_cast<const ElementA*>(A), stA, reinterpret_cast<const ElementB*>(B), stB},
                                {{1.0f, 0.0f}, D, stC, D, stD}};
  return args;
}

}  // namespace

size_t gemm_bf16_workspace(int M, int N, int K, int L) {
  auto args = make_args(nullptr, K, 0, nullptr, K, 0, nullptr, M, 0, M, N, K, L);
  return Gemm::get_workspace_size(args);
}

Status gemm_bf16_tn_f32(const void* A, long lda, long strideA, const void* B, long ldb, long strideB, float* D,
                        long ldd, long strideD, int M, int N, int K, int L, void* workspace, size_t ws_bytes,
                        cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0 || L <= 0) return kOk;
  if ((lda % kAlignA) || (ldb % kAlignB) || (ldd % kAlignD) || (strideA % kAlignA) || (strideB % kAlignB) ||
      (strideD % kAlignD))
    return fail(kInvalid, "gemm_bf16: leading dimensions / batch strides not 16-byte aligned");
  auto args = make_args(A, lda, strideA, B, ldb, strideB, D, ldd, strideD, M, N, K, L);
  if (Gemm::can_implement(args) != cutlass::Status::kSuccess) return fail(kInvalid, "gemm_bf16: cannot implement");
  if (Gemm::get_workspace_size(args) > ws_bytes) return fail(kInvalid, "gemm_bf16: workspace too small");
  // The kernel's shared-memory limit is set once per device and the kernel is
  // launched through the adapter's static run() (a plain launch for a 1x1x1
  // cluster).  The adapter's initialize() sets the attribute on every call;
  // made by the host threads of four concurrent Si64 solves around every
  // projector product, that driver call held the batch at 4.2 solves/s
  // against 4.7-4.8 without it (B200).
  {
    static std::mutex mu;
    static std::set<int> done;
    int dev = 0;
    PW_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (!done.count(dev)) {
      const int smem = (int)GemmKernel::SharedStorageSize;
      if (smem >= (48 << 10)) {
        cudaError_t e = cudaFuncSetAttribute(cutlass::device_kernel<GemmKernel>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return fail(kCuda, std::string("gemm_bf16: ") + cudaGetErrorString(e));
      }
      done.insert(dev);
    }
  }
  if (GemmKernel::initialize_workspace(args, workspace, s) != cutlass::Status::kSuccess)
    return fail(kCuda, "gemm_bf16: workspace initialisation failed");
  typename GemmKernel::Params params = GemmKernel::to_underlying_arguments(args, workspace);
  if (Gemm::run(params, s) != cutlass::Status::kSuccess) return fail(kCuda, "gemm_bf16: run failed");
  count_launch();
  PW_CUDA_TRY(cudaGetLastError());
  return kOk;
}

}  // namespace pwgpu
