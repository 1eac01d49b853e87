// PSD-cone projection of Update_xz (v2rdm_solver.cc:3216-3289) in FP64.
//
// For every primal block the reference symmetrises U = mu x + A^T y - c,
// diagonalises it (Matrix::diagonalize) and rebuilds x = V+ (L+/mu) V+^T and
// z = -V- L- V-^T.  Here:
//   * blocks with n <= 64 are diagonalised by a parallel cyclic Jacobi method
//     in shared memory, one CTA per block, and x and z are rebuilt in the same
//     kernel;
//   * larger blocks use a two-sided block Jacobi method on a workspace padded
//     to a multiple of 64: each round pairs 32-wide column blocks, solves the
//     64 x 64 pair problems with the same shared-memory Jacobi, and rotates the
//     workspace W and the eigenvector matrix V tile by tile.  The eigenvectors
//     of the previous outer iteration seed the next one (W = V^T U V), so a
//     warm solve needs one or two sweeps.  x = V diag(max(L,0)/mu) V^T and
//     z = mu x - U come from one batched GEMM.
// Jacobi's rotations need no ordering of eigenvalues and are robust for the
// clustered and exactly degenerate spectra these blocks have.
#include <cfloat>

#include "kernels.cuh"

namespace v2g {

namespace {

constexpr int kJ = 64;        // largest matrix the shared-memory Jacobi handles
constexpr int kLd = kJ + 1;   // padded leading dimension (bank spread)
constexpr int kJThreads = 256;

// Circle-method round robin on Ne players, round r in [0, Ne-2], pair k.
__device__ __forceinline__ void rr_pair(int Ne, int r, int k, int& p, int& q) {
    if (k == 0) {
        p = Ne - 1;
        q = r;
    } else {
        p = (r + k) % (Ne - 1);
        q = (r - k + Ne - 1) % (Ne - 1);
    }
    if (p > q) {
        int t = p;
        p = q;
        q = t;
    }
}

__device__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += red[i];
        red[32] = s;
    }
    __syncthreads();
    return red[32];
}

// Parallel cyclic Jacobi on the symmetric N x N matrix A (shared memory,
// leading dimension kLd).  On return A is diagonal to tol_rel (relative
// Frobenius off-diagonal norm) and V holds the eigenvectors as columns.
__device__ void jacobi_smem(double* A, double* V, int N, int max_sweeps, double tol_rel) {
    __shared__ double rc[kJ / 2], rs[kJ / 2];
    __shared__ int rp[kJ / 2], rq[kJ / 2];
    __shared__ double red[33];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int Ne = N + (N & 1);
    const int npairs = Ne / 2;
    for (int i = tid; i < N * N; i += nt) V[(i / N) * kLd + (i % N)] = (i / N == i % N) ? 1.0 : 0.0;
    __syncthreads();
    if (N < 2) return;
    for (int sweep = 0; sweep < max_sweeps; sweep++) {
        double off = 0.0, tot = 0.0;
        for (int i = tid; i < N * N; i += nt) {
            const double a = A[(i / N) * kLd + (i % N)];
            tot += a * a;
            if (i / N != i % N) off += a * a;
        }
        off = block_sum(off, red);
        tot = block_sum(tot, red);
        if (!(off > tol_rel * tol_rel * tot)) break;
        for (int r = 0; r < Ne - 1; r++) {
            for (int k = tid; k < npairs; k += nt) {
                int p, q;
                rr_pair(Ne, r, k, p, q);
                double c = 1.0, s = 0.0;
                if (q < N) {
                    const double apq = A[p * kLd + q];
                    const double app = A[p * kLd + p], aqq = A[q * kLd + q];
                    if (fabs(apq) > 1e-18 * (fabs(app) + fabs(aqq)) && apq != 0.0) {
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        s = t * c;
                    }
                }
                rc[k] = c;
                rs[k] = s;
                rp[k] = p;
                rq[k] = q;
            }
            __syncthreads();
            // A <- J^T A  (rows p, q)
            for (int idx = tid; idx < npairs * N; idx += nt) {
                const int k = idx / N, j = idx % N;
                const double s = rs[k];
                if (s == 0.0) continue;
                const double c = rc[k];
                const int p = rp[k], q = rq[k];
                const double apj = A[p * kLd + j], aqj = A[q * kLd + j];
                A[p * kLd + j] = c * apj - s * aqj;
                A[q * kLd + j] = s * apj + c * aqj;
            }
            __syncthreads();
            // A <- A J, V <- V J  (columns p, q)
            for (int idx = tid; idx < npairs * N; idx += nt) {
                const int k = idx / N, i = idx % N;
                const double s = rs[k];
                if (s == 0.0) continue;
                const double c = rc[k];
                const int p = rp[k], q = rq[k];
                const double aip = A[i * kLd + p], aiq = A[i * kLd + q];
                A[i * kLd + p] = c * aip - s * aiq;
                A[i * kLd + q] = s * aip + c * aiq;
                const double vip = V[i * kLd + p], viq = V[i * kLd + q];
                V[i * kLd + p] = c * vip - s * viq;
                V[i * kLd + q] = s * vip + c * viq;
            }
            __syncthreads();
        }
    }
}

constexpr double kJacobiTol = 1e-15;
constexpr int kJacobiSweeps = 40;

__global__ void __launch_bounds__(kJThreads) small_project_kernel(const BlockTask* __restrict__ tasks, int B,
                                                                  const double* __restrict__ aty,
                                                                  const double* __restrict__ c, double* x, double* z,
                                                                  const double* __restrict__ mu,
                                                                  const int* __restrict__ mask) {
    extern __shared__ double sm[];
    double* A = sm;
    double* V = sm + kJ * kLd;
    const BlockTask t = tasks[blockIdx.x];
    const int b = t.inst;
    if (mask && !mask[b]) return;
    const int N = t.n;
    const double m = mu[b];
    for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
        const int p = i / N, q = i % N;
        const int64_t e1 = (t.xoff + (int64_t)p * N + q) * B + b;
        const int64_t e2 = (t.xoff + (int64_t)q * N + p) * B + b;
        const double t1 = (aty[e1] - c[e1]) + m * x[e1];
        const double t2 = (aty[e2] - c[e2]) + m * x[e2];
        A[p * kLd + q] = 0.5 * (t1 + t2);
    }
    __syncthreads();
    jacobi_smem(A, V, N, kJacobiSweeps, kJacobiTol);
    __syncthreads();
    for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
        const int p = i / N, q = i % N;
        double sx = 0.0, sz = 0.0;
        for (int j = 0; j < N; j++) {
            const double lam = A[j * kLd + j];
            if (lam > 0.0)
                sx += (V[p * kLd + j] * lam / m) * V[q * kLd + j];
            else if (lam < 0.0)
                sz += (-V[p * kLd + j] * lam) * V[q * kLd + j];
        }
        const int64_t e = (t.xoff + (int64_t)p * N + q) * B + b;
        x[e] = sx;
        z[e] = sz;
    }
}

// ---- large blocks ----------------------------------------------------------

__global__ void form_u_kernel(const BlockTask* __restrict__ tasks, int B, const double* __restrict__ aty,
                              const double* __restrict__ c, const double* __restrict__ x,
                              const double* __restrict__ mu, const int* __restrict__ mask, double* __restrict__ Uw) {
    const BlockTask t = tasks[blockIdx.y];
    const int p = blockIdx.x;
    if (p >= t.np) return;
    const int b = t.inst;
    if (mask && !mask[b]) return;
    const int N = t.n;
    const double m = mu[b];
    double* row = Uw + t.woff + (int64_t)p * t.np;
    for (int q = threadIdx.x; q < t.np; q += blockDim.x) {
        double v = 0.0;
        if (p < N && q < N) {
            const int64_t e1 = (t.xoff + (int64_t)p * N + q) * B + b;
            const int64_t e2 = (t.xoff + (int64_t)q * N + p) * B + b;
            const double t1 = (aty[e1] - c[e1]) + m * x[e1];
            const double t2 = (aty[e2] - c[e2]) + m * x[e2];
            v = 0.5 * (t1 + t2);
        }
        row[q] = v;
    }
}

__global__ void cold_start_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ Uw,
                                  double* __restrict__ Ww, double* __restrict__ Vw, const int* __restrict__ bmask) {
    const BlockTask t = tasks[blockIdx.y];
    const int p = blockIdx.x;
    if (p >= t.np || (bmask && !bmask[blockIdx.y])) return;
    const int64_t o = t.woff + (int64_t)p * t.np;
    for (int q = threadIdx.x; q < t.np; q += blockDim.x) {
        Ww[o + q] = Uw[o + q];
        Vw[o + q] = (p == q) ? 1.0 : 0.0;
    }
}

// C = op(A) diag(d) op(B) on 64 x 64 tiles; 256 threads, 4 x 4 outputs each.
__global__ void __launch_bounds__(256) gemm_kernel(const BlockTask* __restrict__ tasks,
                                                   const GemmTile* __restrict__ tiles, const double* __restrict__ A,
                                                   int transA, const double* __restrict__ Bm, int transB,
                                                   const double* __restrict__ dvec, double* __restrict__ C,
                                                   const int* __restrict__ bmask) {
    constexpr int BK = 16;
    __shared__ double As[BK][64 + 1];
    __shared__ double Bs[BK][64 + 1];
    const GemmTile tl = tiles[blockIdx.x];
    if (bmask && !bmask[tl.task]) return;
    const BlockTask t = tasks[tl.task];
    const int np = t.np;
    const double* a = A + t.woff;
    const double* bb = Bm + t.woff;
    const double* d = dvec ? dvec + t.doff : nullptr;  // one weight vector (np) per block
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int i0 = tl.ti * 64, j0 = tl.tj * 64;
    double acc[4][4] = {};
    for (int k0 = 0; k0 < np; k0 += BK) {
        for (int l = threadIdx.x; l < BK * 64; l += 256) {
            int kk, ii;
            if (transA) {
                kk = l / 64;
                ii = l % 64;
                As[kk][ii] = a[(int64_t)(k0 + kk) * np + i0 + ii];
            } else {
                ii = l / BK;
                kk = l % BK;
                As[kk][ii] = a[(int64_t)(i0 + ii) * np + k0 + kk];
            }
        }
        for (int l = threadIdx.x; l < BK * 64; l += 256) {
            int kk, jj;
            if (transB) {
                jj = l / BK;
                kk = l % BK;
                Bs[kk][jj] = bb[(int64_t)(j0 + jj) * np + k0 + kk];
            } else {
                kk = l / 64;
                jj = l % 64;
                Bs[kk][jj] = bb[(int64_t)(k0 + kk) * np + j0 + jj];
            }
        }
        __syncthreads();
        if (d) {
            for (int l = threadIdx.x; l < BK * 64; l += 256) As[l / 64][l % 64] *= d[k0 + l / 64];
            __syncthreads();
        }
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            double av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) av[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) bv[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] += av[i] * bv[j];
        }
        __syncthreads();
    }
    double* cc = C + t.woff;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) cc[(int64_t)(i0 + ty + 16 * i) * np + j0 + tx + 16 * j] = acc[i][j];
}

// Global index of local row a (0..63) of pair (I, J): first 32 rows are column
// block I, the next 32 are block J.
__device__ __forceinline__ int pair_idx(int I, int J, int a) { return a < 32 ? I * 32 + a : J * 32 + (a - 32); }

__global__ void __launch_bounds__(kJThreads) bj_solve_kernel(const BlockTask* __restrict__ tasks,
                                                             const PairTask* __restrict__ pt, int round, double* Ww,
                                                             double* __restrict__ Qbuf, const int* __restrict__ bmask) {
    extern __shared__ double sm[];
    double* S = sm;
    double* Q = sm + kJ * kLd;
    const PairTask pk = pt[blockIdx.x];
    if (bmask && !bmask[pk.task]) return;
    const BlockTask t = tasks[pk.task];
    int I, J;
    rr_pair(t.nb, round % (t.nb - 1), pk.k, I, J);
    const double* w = Ww + t.woff;
    for (int l = threadIdx.x; l < 64 * 64; l += blockDim.x) {
        const int a = l / 64, bq = l % 64;
        S[a * kLd + bq] = w[(int64_t)pair_idx(I, J, a) * t.np + pair_idx(I, J, bq)];
    }
    __syncthreads();
    jacobi_smem(S, Q, 64, kJacobiSweeps, kJacobiTol);
    __syncthreads();
    double* qo = Qbuf + t.qoff + (int64_t)pk.k * 4096;
    for (int l = threadIdx.x; l < 64 * 64; l += blockDim.x) qo[l] = Q[(l / 64) * kLd + (l % 64)];
}

// out(64x64, smem ld kLd) = opL(L) * M * R, where L and R are 64x64 row-major
// in global memory; used for W tile = Q1^T T Q2 and V tile = T Q.
__device__ void tile_rotate(double* T, double* Qs, const double* Q1g, const double* Q2g, bool left) {
    // T <- T * Q2
    for (int l = threadIdx.x; l < 4096; l += blockDim.x) Qs[(l / 64) * kLd + l % 64] = Q2g[l];
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[4][4] = {};
    for (int k = 0; k < 64; k++) {
        double av[4], bv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) av[i] = T[(ty + 16 * i) * kLd + k];
#pragma unroll
        for (int j = 0; j < 4; j++) bv[j] = Qs[k * kLd + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] += av[i] * bv[j];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) T[(ty + 16 * i) * kLd + tx + 16 * j] = acc[i][j];
    if (!left) {
        __syncthreads();
        return;
    }
    // T <- Q1^T * T
    __syncthreads();
    for (int l = threadIdx.x; l < 4096; l += blockDim.x) Qs[(l / 64) * kLd + l % 64] = Q1g[l];
    __syncthreads();
    double acc2[4][4] = {};
    for (int k = 0; k < 64; k++) {
        double av[4], bv[4];
#pragma unroll
        for (int i = 0; i < 4; i++) av[i] = Qs[k * kLd + ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; j++) bv[j] = T[k * kLd + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc2[i][j] += av[i] * bv[j];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) T[(ty + 16 * i) * kLd + tx + 16 * j] = acc2[i][j];
    __syncthreads();
}

__global__ void __launch_bounds__(256) bj_update_w_kernel(const BlockTask* __restrict__ tasks,
                                                          const WTileTask* __restrict__ wt, int round, double* Ww,
                                                          const double* __restrict__ Qbuf,
                                                          const int* __restrict__ bmask) {
    extern __shared__ double sm[];
    double* T = sm;
    double* Qs = sm + kJ * kLd;
    const WTileTask w = wt[blockIdx.x];
    if (bmask && !bmask[w.task]) return;
    const BlockTask t = tasks[w.task];
    const int r = round % (t.nb - 1);
    int I1, J1, I2, J2;
    rr_pair(t.nb, r, w.k1, I1, J1);
    rr_pair(t.nb, r, w.k2, I2, J2);
    double* base = Ww + t.woff;
    for (int l = threadIdx.x; l < 4096; l += blockDim.x) {
        const int a = l / 64, bq = l % 64;
        T[a * kLd + bq] = base[(int64_t)pair_idx(I1, J1, a) * t.np + pair_idx(I2, J2, bq)];
    }
    __syncthreads();
    tile_rotate(T, Qs, Qbuf + t.qoff + (int64_t)w.k1 * 4096, Qbuf + t.qoff + (int64_t)w.k2 * 4096, true);
    for (int l = threadIdx.x; l < 4096; l += blockDim.x) {
        const int a = l / 64, bq = l % 64;
        base[(int64_t)pair_idx(I1, J1, a) * t.np + pair_idx(I2, J2, bq)] = T[a * kLd + bq];
    }
}

__global__ void __launch_bounds__(256) bj_update_v_kernel(const BlockTask* __restrict__ tasks,
                                                          const VTileTask* __restrict__ vt, int round, double* Vw,
                                                          const double* __restrict__ Qbuf,
                                                          const int* __restrict__ bmask) {
    extern __shared__ double sm[];
    double* T = sm;
    double* Qs = sm + kJ * kLd;
    const VTileTask v = vt[blockIdx.x];
    if (bmask && !bmask[v.task]) return;
    const BlockTask t = tasks[v.task];
    int I, J;
    rr_pair(t.nb, round % (t.nb - 1), v.k, I, J);
    double* base = Vw + t.woff;
    const int r0 = v.chunk * 64;
    for (int l = threadIdx.x; l < 4096; l += blockDim.x) {
        const int a = l / 64, bq = l % 64;
        T[a * kLd + bq] = base[(int64_t)(r0 + a) * t.np + pair_idx(I, J, bq)];
    }
    __syncthreads();
    tile_rotate(T, Qs, nullptr, Qbuf + t.qoff + (int64_t)v.k * 4096, false);
    for (int l = threadIdx.x; l < 4096; l += blockDim.x) {
        const int a = l / 64, bq = l % 64;
        base[(int64_t)(r0 + a) * t.np + pair_idx(I, J, bq)] = T[a * kLd + bq];
    }
}

__global__ void bj_check_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ Ww, double tol,
                                int* __restrict__ bmask) {
    __shared__ double red[33];
    if (!bmask[blockIdx.x]) return;
    const BlockTask t = tasks[blockIdx.x];
    const double* w = Ww + t.woff;
    double off = 0.0, tot = 0.0;
    const int64_t nn = (int64_t)t.np * t.np;
    for (int64_t i = threadIdx.x; i < nn; i += blockDim.x) {
        const double a = w[i];
        tot += a * a;
        if (i / t.np != i % t.np) off += a * a;
    }
    off = block_sum(off, red);
    tot = block_sum(tot, red);
    if (threadIdx.x == 0 && !(off > tol * tol * tot)) bmask[blockIdx.x] = 0;
}

__global__ void count_open_kernel(int n, const int* __restrict__ bmask, int* out) {
    int c = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) c += bmask[i] != 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    __shared__ int s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) tot += s[i];
        *out = tot;
    }
}

__global__ void pos_weights_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ Ww,
                                   const double* __restrict__ mu, double* __restrict__ dw) {
    const BlockTask t = tasks[blockIdx.x];
    const double m = mu[t.inst];
    double* d = dw + t.doff;
    for (int j = threadIdx.x; j < t.np; j += blockDim.x) {
        const double lam = Ww[t.woff + (int64_t)j * t.np + j];
        d[j] = (lam > 0.0) ? lam / m : 0.0;
    }
}

__global__ void write_xz_kernel(const BlockTask* __restrict__ tasks, int B, const double* __restrict__ Xw,
                                const double* __restrict__ Uw, const double* __restrict__ mu,
                                const int* __restrict__ mask, double* __restrict__ x, double* __restrict__ z) {
    const BlockTask t = tasks[blockIdx.y];
    const int p = blockIdx.x;
    if (p >= t.n) return;
    const int b = t.inst;
    if (mask && !mask[b]) return;
    const double m = mu[b];
    for (int q = threadIdx.x; q < t.n; q += blockDim.x) {
        const int64_t w = t.woff + (int64_t)p * t.np + q;
        const int64_t e = (t.xoff + (int64_t)p * t.n + q) * B + b;
        const double xv = Xw[w];
        x[e] = xv;
        z[e] = m * xv - Uw[w];
    }
}

constexpr size_t kJacobiSmem = 2 * kJ * kLd * sizeof(double);

void set_smem_attrs() {
    static bool done = false;
    if (done) return;
    cudaFuncSetAttribute(small_project_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJacobiSmem);
    cudaFuncSetAttribute(bj_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJacobiSmem);
    cudaFuncSetAttribute(bj_update_w_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJacobiSmem);
    cudaFuncSetAttribute(bj_update_v_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJacobiSmem);
    done = true;
}

}  // namespace

void launch_small_project(const BlockTask* tasks, int ntasks, int B, const double* aty, const double* c, double* x,
                          double* z, const double* mu, const int* mask, cudaStream_t s) {
    if (ntasks == 0) return;
    set_smem_attrs();
    small_project_kernel<<<ntasks, kJThreads, kJacobiSmem, s>>>(tasks, B, aty, c, x, z, mu, mask);
}

void launch_form_u(const BlockTask* tasks, int ntasks, int max_np, int B, const double* aty, const double* c,
                      const double* x, const double* mu, const int* mask, double* Uw, cudaStream_t s) {
    if (ntasks == 0) return;
    form_u_kernel<<<dim3(max_np, ntasks), 128, 0, s>>>(tasks, B, aty, c, x, mu, mask, Uw);
}

void launch_cold_start(const BlockTask* tasks, int ntasks, int max_np, const double* Uw, double* Ww, double* Vw,
                          const int* bmask, cudaStream_t s) {
    if (ntasks == 0) return;
    cold_start_kernel<<<dim3(max_np, ntasks), 128, 0, s>>>(tasks, Uw, Ww, Vw, bmask);
}

void launch_gemm(const BlockTask* tasks, const GemmTile* tiles, int ntiles, const double* A, bool transA,
                 const double* Bm, bool transB, const double* dvec, double* C, const int* bmask, cudaStream_t s) {
    if (ntiles == 0) return;
    gemm_kernel<<<ntiles, 256, 0, s>>>(tasks, tiles, A, transA, Bm, transB, dvec, C, bmask);
}

void launch_bj_solve(const BlockTask* tasks, const PairTask* pt, int npt, int round, double* Ww, double* Qbuf,
                     const int* bmask, cudaStream_t s) {
    if (npt == 0) return;
    set_smem_attrs();
    bj_solve_kernel<<<npt, kJThreads, kJacobiSmem, s>>>(tasks, pt, round, Ww, Qbuf, bmask);
}

void launch_bj_update_w(const BlockTask* tasks, const WTileTask* wt, int nwt, int round, double* Ww,
                        const double* Qbuf, const int* bmask, cudaStream_t s) {
    if (nwt == 0) return;
    set_smem_attrs();
    bj_update_w_kernel<<<nwt, 256, kJacobiSmem, s>>>(tasks, wt, round, Ww, Qbuf, bmask);
}

void launch_bj_update_v(const BlockTask* tasks, const VTileTask* vt, int nvt, int round, double* Vw,
                        const double* Qbuf, const int* bmask, cudaStream_t s) {
    if (nvt == 0) return;
    set_smem_attrs();
    bj_update_v_kernel<<<nvt, 256, kJacobiSmem, s>>>(tasks, vt, round, Vw, Qbuf, bmask);
}

void launch_bj_check(const BlockTask* tasks, int ntasks, const double* Ww, double tol, int* bmask, int* n_open,
                     cudaStream_t s) {
    if (ntasks == 0) return;
    bj_check_kernel<<<ntasks, 256, 0, s>>>(tasks, Ww, tol, bmask);
    count_open_kernel<<<1, 1024, 0, s>>>(ntasks, bmask, n_open);
}

void launch_pos_weights(const BlockTask* tasks, int ntasks, const double* Ww, const double* mu, double* dw,
                        cudaStream_t s) {
    if (ntasks == 0) return;
    pos_weights_kernel<<<ntasks, 128, 0, s>>>(tasks, Ww, mu, dw);
}

void launch_write_xz(const BlockTask* tasks, int ntasks, int max_n, int B, const double* Xw, const double* Uw,
                        const double* mu, const int* mask, double* x, double* z, cudaStream_t s) {
    if (ntasks == 0) return;
    write_xz_kernel<<<dim3(max_n, ntasks), 128, 0, s>>>(tasks, B, Xw, Uw, mu, mask, x, z);
}

}  // namespace v2g
