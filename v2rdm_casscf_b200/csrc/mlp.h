// Launchers of the learned warm start's MLP kernels (mlp.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace v2g {

// C[M x N] = op(A)[M x K] op(B)[K x N] (+ bias) (ReLU) (C += when accumulate),
// row-major with leading dimensions; FP32 arithmetic, deterministic.
void mlp_gemm(int M, int N, int K, const float* A, int lda, bool transA, const float* B, int ldb, bool transB,
              const float* bias, bool relu, bool accumulate, float* C, int ldc, cudaStream_t s);
// the same with BF16 B (the weights)
void mlp_gemm_bf16(int M, int N, int K, const float* A, int lda, bool transA, const __nv_bfloat16* B, int ldb,
                   bool transB, const float* bias, bool relu, bool accumulate, float* C, int ldc, cudaStream_t s);
// dy[i] = 0 where y[i] <= 0
void mlp_relu_back(int64_t n, const float* y, float* dy, cudaStream_t s);
// db[n] = sum over rows of dy[m, n]
void mlp_col_sum(int M, int N, const float* dy, float* db, cudaStream_t s);
// d = 2 (out - t) scale; partial[block] = sum (out - t)^2 (mlp_mse_blocks() blocks)
int mlp_mse_blocks();
void mlp_mse(int64_t n, const float* out, const float* t, float scale, float* d, double* partial, cudaStream_t s);
// one Adam step (step >= 1) on w with gradient g, moments m and v; w16 = bf16(w)
void mlp_adam(int64_t n, float* w, const float* g, float* m, float* v, __nv_bfloat16* w16, float lr, int step,
              cudaStream_t s);
void mlp_to_bf16(int64_t n, const float* w, __nv_bfloat16* w16, cudaStream_t s);

}  // namespace v2g
