// BF16 tensor-core GEMM with FP32 accumulation and output (gemm_bf16.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

#include "pw_common.cuh"

namespace pwgpu {

// D[l] = A[l] * B[l] for l < L: A M x K row-major (lda), B K x N column-major
// (ldb), D M x N column-major FP32 (ldd); batch strides in elements.  All
// leading dimensions and batch strides must be 16-byte multiples.
Status gemm_bf16_tn_f32(const void* A, long lda, long strideA, const void* B, long ldb, long strideB, float* D,
                        long ldd, long strideD, int M, int N, int K, int L, void* workspace, size_t ws_bytes,
                        cudaStream_t s);
size_t gemm_bf16_workspace(int M, int N, int K, int L);

}  // namespace pwgpu
