// Kernels of the learned warm start's pair-wise MLP: FP32 arithmetic with
// BF16 weights for inference and training (FP32 master weights, Adam).
//
// Every dense layer is C = op(A) op(B) (+ bias) (ReLU) on row-major FP32 /
// BF16 matrices, tiled 64 x 64 x 16 with 256 threads and a 4 x 4 block of C
// per thread; the weight gradient dW = dY^T X (a reduction over all rows) is
// the same kernel with op(A) transposed, so every sum runs in a fixed order
// (no atomics) and training is deterministic.
#include <cuda_bf16.h>

#include "kernels.cuh"
#include "mlp.h"

namespace v2g {

namespace {

constexpr int kT = 64, kK = 16;

template <class TB>
__device__ __forceinline__ float to_f(TB v);
template <>
__device__ __forceinline__ float to_f<float>(float v) {
    return v;
}
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) {
    return __bfloat162float(v);
}

// C[M x N] = op(A)[M x K] op(B)[K x N] (+ bias[n]) (ReLU), or C += ... when
// accumulate; op(A)(m, k) = transA ? A[k * lda + m] : A[m * lda + k], same for B.
template <class TB>
__global__ void __launch_bounds__(256) mlp_gemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                       bool transA, const TB* __restrict__ B, int ldb, bool transB,
                                                       const float* __restrict__ bias, int relu, int accumulate,
                                                       float* __restrict__ C, int ldc) {
    __shared__ float As[kK][kT + 1];
    __shared__ float Bs[kK][kT + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * kT, n0 = blockIdx.x * kT;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += kK) {
        for (int i = threadIdx.x; i < kT * kK; i += 256) {
            const int mm = transA ? i % kT : i / kK, kk = transA ? i / kT : i % kK;
            const int m = m0 + mm, k = k0 + kk;
            float v = 0.f;
            if (m < M && k < K) v = transA ? A[(int64_t)k * lda + m] : A[(int64_t)m * lda + k];
            As[kk][mm] = v;
            const int nn = transB ? i / kK : i % kT, kb = transB ? i % kK : i / kT;
            const int n = n0 + nn, kq = k0 + kb;
            float w = 0.f;
            if (n < N && kq < K) w = to_f<TB>(transB ? B[(int64_t)n * ldb + kq] : B[(int64_t)kq * ldb + n]);
            Bs[kb][nn] = w;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kK; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int m = m0 + ty + 16 * i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int n = n0 + tx + 16 * j;
            if (n >= N) continue;
            float v = acc[i][j];
            if (bias) v += bias[n];
            if (relu) v = fmaxf(v, 0.f);
            float* c = C + (int64_t)m * ldc + n;
            *c = accumulate ? *c + v : v;
        }
    }
}

// dY <- dY * (Y > 0) (ReLU backward; Y is the layer's output after the ReLU)
__global__ void relu_back_kernel(int64_t n, const float* __restrict__ y, float* __restrict__ dy) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!(y[i] > 0.f)) dy[i] = 0.f;
}

// column sums db[n] = sum_m dY[m, n] (fixed order: one thread per column)
__global__ void col_sum_kernel(int M, int N, const float* __restrict__ dy, float* __restrict__ db) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int m = 0; m < M; m++) s += dy[(int64_t)m * N + n];
    db[n] = s;
}

// mean squared error: d = (out - t) * scale, per-block partial sums of d^2 / scale
__global__ void mse_kernel(int64_t n, const float* __restrict__ out, const float* __restrict__ t, float scale,
                           float* __restrict__ d, double* __restrict__ partial) {
    __shared__ double sh[256];
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float e = out[i] - t[i];
        d[i] = 2.f * e * scale;
        s += (double)e * e;
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// Adam (Kingma and Ba 2015) on the FP32 master weights, then the BF16 copy
__global__ void adam_kernel(int64_t n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, __nv_bfloat16* __restrict__ w16, float lr, float b1, float b2,
                            float c1, float c2, float eps) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        w16[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void to_bf16_kernel(int64_t n, const float* __restrict__ w, __nv_bfloat16* __restrict__ w16) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        w16[i] = __float2bfloat16_rn(w[i]);
}

inline int grid1(int64_t n) {
    int64_t g = (n + 255) / 256;
    return (int)(g < 1 ? 1 : (g > 148 * 8 ? 148 * 8 : g));
}

}  // namespace

void mlp_gemm(int M, int N, int K, const float* A, int lda, bool transA, const float* B, int ldb, bool transB,
              const float* bias, bool relu, bool accumulate, float* C, int ldc, cudaStream_t s) {
    dim3 grid((N + kT - 1) / kT, (M + kT - 1) / kT);
    mlp_gemm_kernel<float><<<grid, 256, 0, s>>>(M, N, K, A, lda, transA, B, ldb, transB, bias, relu, accumulate, C,
                                                ldc);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void mlp_gemm_bf16(int M, int N, int K, const float* A, int lda, bool transA, const __nv_bfloat16* B, int ldb,
                   bool transB, const float* bias, bool relu, bool accumulate, float* C, int ldc, cudaStream_t s) {
    dim3 grid((N + kT - 1) / kT, (M + kT - 1) / kT);
    mlp_gemm_kernel<__nv_bfloat16><<<grid, 256, 0, s>>>(M, N, K, A, lda, transA, B, ldb, transB, bias, relu,
                                                        accumulate, C, ldc);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void mlp_relu_back(int64_t n, const float* y, float* dy, cudaStream_t s) {
    relu_back_kernel<<<grid1(n), 256, 0, s>>>(n, y, dy);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void mlp_col_sum(int M, int N, const float* dy, float* db, cudaStream_t s) {
    col_sum_kernel<<<(N + 127) / 128, 128, 0, s>>>(M, N, dy, db);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

int mlp_mse_blocks() { return 148; }

void mlp_mse(int64_t n, const float* out, const float* t, float scale, float* d, double* partial, cudaStream_t s) {
    mse_kernel<<<mlp_mse_blocks(), 256, 0, s>>>(n, out, t, scale, d, partial);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void mlp_adam(int64_t n, float* w, const float* g, float* m, float* v, __nv_bfloat16* w16, float lr, int step,
              cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    adam_kernel<<<grid1(n), 256, 0, s>>>(n, w, g, m, v, w16, lr, b1, b2, c1, c2, 1e-8f);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void mlp_to_bf16(int64_t n, const float* w, __nv_bfloat16* w16, cudaStream_t s) {
    to_bf16_kernel<<<grid1(n), 256, 0, s>>>(n, w, w16);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

}  // namespace v2g
