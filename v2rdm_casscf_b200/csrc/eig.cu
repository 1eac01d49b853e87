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
#include <cooperative_groups.h>

#include <cfloat>

#include <mutex>
#include <vector>

#include "kernels.cuh"

namespace v2g {

namespace {

constexpr int kJ = 64;        // largest matrix the shared-memory Jacobi handles
constexpr int kLd = kJ + 1;   // padded leading dimension (bank spread)
// threads of the shared-memory Jacobi CTAs: a round's passes over the 2 x 2
// blocks and the columns of V spread over 16 warps (9 % faster projections on
// H10 than 8 warps; same arithmetic)
constexpr int kJThreads = 512;

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
// leading dimension kLd), round-robin ordering.  A pair (p,q) is rotated when
// |a_pq| > rot_eps * sqrt(|a_pp a_qq|) (tested squared) and above an absolute floor of
// 1e-17 ||A||_F; the method stops when a sweep would rotate no pair (the
// classical threshold criterion, which a relative off-norm test near the
// rounding floor would never reach) or after max_sweeps.  That test runs on
// all pairs at once before each sweep, so the rotation-free last sweep of the
// textbook loop costs one pass over A instead of N - 1 synchronised rounds
// (the result is the same: a sweep that starts with no pair above the
// thresholds changes nothing).  On return V holds the eigenvectors as columns
// and diag(A) the eigenvalues.
// With init_v = false, V already holds an orthogonal matrix (the previous
// eigenvectors of a warm start) and the rotations accumulate onto it.
__device__ void jacobi_smem(double* A, double* V, int N, int max_sweeps, double rot_eps, bool init_v = true,
                            double abs_tol = 0.0) {
    __shared__ double rc[kJ / 2], rs[kJ / 2];
    __shared__ int rp[kJ / 2], rq[kJ / 2];
    __shared__ double red[33];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int Ne = N + (N & 1);
    const int npairs = Ne / 2;
    if (init_v)
        for (int i = tid; i < N * N; i += nt) V[(i / N) * kLd + (i % N)] = (i / N == i % N) ? 1.0 : 0.0;
    __syncthreads();
    if (N < 2) return;
    double tot = 0.0;
    for (int i = tid; i < N * N; i += nt) {
        const double a = A[(i / N) * kLd + (i % N)];
        tot += a * a;
    }
    const double floor_abs = fmax(1e-17 * sqrt(block_sum(tot, red)), abs_tol);
    for (int sweep = 0; sweep < max_sweeps; sweep++) {
        int any = 0;
        for (int i = tid; i < N * N && !any; i += nt) {
            const int p = i / N, q = i % N;
            if (p >= q) continue;
            const double apq = fabs(A[p * kLd + q]);
            any = apq > floor_abs && apq > rot_eps * sqrt(fabs(A[p * kLd + p]) * fabs(A[q * kLd + q]));
        }
        if (!__syncthreads_or(any)) break;
        for (int r = 0; r < Ne - 1; r++) {
            for (int k = tid; k < npairs; k += nt) {
                int p, q;
                rr_pair(Ne, r, k, p, q);
                double c = 1.0, s = 0.0;
                if (q < N) {
                    const double apq = A[p * kLd + q];
                    const double app = A[p * kLd + p], aqq = A[q * kLd + q];
                    if (fabs(apq) > floor_abs && apq * apq > rot_eps * rot_eps * fabs(app * aqq)) {
                        // the angle to FP32 accuracy (an inexact angle leaves a
                        // residual of ~1e-7 |a_pq| that the next sweep removes);
                        // c, s exactly orthogonal in FP64 for that angle
                        const float tau = (float)((aqq - app) / 2.0) / (float)apq;
                        const float tf = copysignf(1.0f, tau) / (fabsf(tau) + sqrtf(fmaf(tau, tau, 1.0f)));
                        const double t = (double)tf;
                        c = rsqrt(1.0 + t * t);
                        s = t * c;
                    }
                }
                rc[k] = c;
                rs[k] = s;
                rp[k] = p;
                rq[k] = q;
            }
            __syncthreads();
            // A <- J^T A J in one pass: the round's pairs are disjoint, so A splits
            // into 2 x 2 blocks (pair a rows, pair b columns) that transform
            // independently, in place (a pair with the padding index of odd N has
            // s = 0 and a single row / column)
            for (int idx = tid; idx < npairs * npairs; idx += nt) {
                const int a = idx / npairs, bb = idx % npairs;
                const double sa = rs[a], sb = rs[bb];
                if (sa == 0.0 && sb == 0.0) continue;
                const double ca = rc[a], cb = rc[bb];
                const int pa = rp[a], qa = rq[a], pb = rp[bb], qb = rq[bb];
                const bool qa_ok = qa < N, qb_ok = qb < N;
                const double x00 = A[pa * kLd + pb];
                const double x01 = qb_ok ? A[pa * kLd + qb] : 0.0;
                const double x10 = qa_ok ? A[qa * kLd + pb] : 0.0;
                const double x11 = (qa_ok && qb_ok) ? A[qa * kLd + qb] : 0.0;
                // rows: J^T
                const double y00 = ca * x00 - sa * x10, y01 = ca * x01 - sa * x11;
                const double y10 = sa * x00 + ca * x10, y11 = sa * x01 + ca * x11;
                // columns: J
                A[pa * kLd + pb] = cb * y00 - sb * y01;
                if (qb_ok) A[pa * kLd + qb] = sb * y00 + cb * y01;
                if (qa_ok) A[qa * kLd + pb] = cb * y10 - sb * y11;
                if (qa_ok && qb_ok) A[qa * kLd + qb] = sb * y10 + cb * y11;
            }
            // V <- V J  (columns p, q; V is not read by the pass above)
            for (int idx = tid; idx < npairs * N; idx += nt) {
                const int k = idx / N, i = idx % N;
                const double s = rs[k];
                if (s == 0.0) continue;
                const double c = rc[k];
                const int p = rp[k], q = rq[k];
                const double vip = V[i * kLd + p], viq = V[i * kLd + q];
                V[i * kLd + p] = c * vip - s * viq;
                V[i * kLd + q] = s * vip + c * viq;
            }
            __syncthreads();
        }
    }
}

constexpr double kJacobiRotEps = 1e-15;
constexpr int kJacobiSweeps = 20;
constexpr int kPairSweeps = 1;

// vsave (optional): the block's eigenvectors, n x n at t.woff, kept across
// outer iterations.  With warm set, the Jacobi starts from them: A <- V^T U V
// (nearly diagonal once the iteration settles, so one to three sweeps
// converge it instead of ~10 from the identity) and the rotations accumulate
// onto V.  Without warm the Jacobi starts from V = I; vsave is written either way.
__global__ void __launch_bounds__(kJThreads) small_project_kernel(const BlockTask* __restrict__ tasks, int B,
                                                                  const double* __restrict__ aty,
                                                                  const double* __restrict__ c, double* x, double* z,
                                                                  const double* __restrict__ mu,
                                                                  const int* __restrict__ mask,
                                                                  double* __restrict__ vsave, int warm,
                                                                  const double* __restrict__ stol) {
    extern __shared__ double sm[];
    double* A = sm;
    double* V = sm + kJ * kLd;
    double* T = sm + 2 * kJ * kLd;  // only with vsave (the launch then has room for it)
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
    const bool use_warm = vsave && warm;
    if (use_warm) {
        const double* vs = vsave + t.woff;
        for (int i = threadIdx.x; i < N * N; i += blockDim.x) V[(i / N) * kLd + (i % N)] = vs[i];
        __syncthreads();
        // T = A V, then A = V^T T (symmetrised)
        for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
            const int p = i / N, q = i % N;
            double acc = 0.0;
            for (int k = 0; k < N; k++) acc += A[p * kLd + k] * V[k * kLd + q];
            T[p * kLd + q] = acc;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
            const int p = i / N, q = i % N;
            double acc = 0.0;
            for (int k = 0; k < N; k++) acc += V[k * kLd + p] * T[k * kLd + q];
            A[p * kLd + q] = acc;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
            const int p = i / N, q = i % N;
            if (p < q) {
                const double v = 0.5 * (A[p * kLd + q] + A[q * kLd + p]);
                A[p * kLd + q] = v;
                A[q * kLd + p] = v;
            }
        }
    }
    __syncthreads();
    // with stol, off-diagonal entries below the instance's share of the
    // adaptive tolerance are left (x and z stay PSD; the residual is bounded)
    jacobi_smem(A, V, N, kJacobiSweeps, kJacobiRotEps, !use_warm, stol ? stol[b] : 0.0);
    __syncthreads();
    if (vsave) {
        double* vs = vsave + t.woff;
        for (int i = threadIdx.x; i < N * N; i += blockDim.x) vs[i] = V[(i / N) * kLd + (i % N)];
    }
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

// C = op(A) diag(d) op(B) on 64 x 64 tiles of the padded workspaces.
// S x S threads per tile (S = 64 / R), each holding an R x R block of C in
// registers (rows ty + S i, columns tx + S j).  R = 8 (64 threads): 16
// shared-memory loads feed 64 FMAs, which matches the FP64 FMA rate to the
// shared-memory bandwidth; the launch for large grids.  R = 4 (256 threads):
// four times the warps per tile and a quarter of the serial FMA chain per
// thread, for grids too small to fill the GPU (one instance's few blocks),
// where the kernel is latency-bound.  The K loop is double buffered through
// registers; every C entry is one FMA chain in k order in both forms.
constexpr int kGemmBK = 16;
constexpr int kGemmLd = 64 + 1;

template <int NT>
__device__ __forceinline__ void gemm_load_chunk(const double* __restrict__ a, const double* __restrict__ bb, int np,
                                                int i0, int j0, int k0, bool transA, bool transB,
                                                double ra[1024 / NT], double rb[1024 / NT]) {
    // 1024 elements per operand chunk, 1024 / NT per thread
#pragma unroll
    for (int u = 0; u < 1024 / NT; u++) {
        const int l = threadIdx.x + NT * u;
        if (transA) {
            const int kk = l >> 6, ii = l & 63;
            ra[u] = a[(int64_t)(k0 + kk) * np + i0 + ii];
        } else {
            const int ii = l >> 4, kk = l & 15;
            ra[u] = a[(int64_t)(i0 + ii) * np + k0 + kk];
        }
        if (transB) {
            const int jj = l >> 4, kk = l & 15;
            rb[u] = bb[(int64_t)(j0 + jj) * np + k0 + kk];
        } else {
            const int kk = l >> 6, jj = l & 63;
            rb[u] = bb[(int64_t)(k0 + kk) * np + j0 + jj];
        }
    }
}

template <int NT>
__device__ __forceinline__ void gemm_store_chunk(double (*As)[kGemmLd], double (*Bs)[kGemmLd], bool transA,
                                                 bool transB, const double ra[1024 / NT], const double rb[1024 / NT],
                                                 const double* __restrict__ d, int k0) {
#pragma unroll
    for (int u = 0; u < 1024 / NT; u++) {
        const int l = threadIdx.x + NT * u;
        int kk, ii, jj;
        if (transA) {
            kk = l >> 6;
            ii = l & 63;
        } else {
            ii = l >> 4;
            kk = l & 15;
        }
        As[kk][ii] = d ? ra[u] * d[k0 + kk] : ra[u];
        if (transB) {
            jj = l >> 4;
            kk = l & 15;
        } else {
            kk = l >> 6;
            jj = l & 63;
        }
        Bs[kk][jj] = rb[u];
    }
}

template <int R>
__global__ void __launch_bounds__((64 / R) * (64 / R)) gemm_kernel(const BlockTask* __restrict__ tasks,
                                                                   const GemmTile* __restrict__ tiles,
                                                                   const double* __restrict__ A, int transA,
                                                                   const double* __restrict__ Bm, int transB,
                                                                   const double* __restrict__ dvec,
                                                                   double* __restrict__ C,
                                                                   const int* __restrict__ bmask) {
    constexpr int S = 64 / R, NT = S * S, U = 1024 / NT;
    __shared__ double As[2][kGemmBK][kGemmLd];
    __shared__ double Bs[2][kGemmBK][kGemmLd];
    const GemmTile tl = tiles[blockIdx.x];
    if (bmask && !bmask[tl.task]) return;
    const BlockTask t = tasks[tl.task];
    const int np = t.np;
    const double* a = A + t.woff;
    const double* bb = Bm + t.woff;
    const double* d = dvec ? dvec + t.doff : nullptr;
    const int tx = threadIdx.x % S, ty = threadIdx.x / S;
    const int i0 = tl.ti * 64, j0 = tl.tj * 64;
    double acc[R][R];
#pragma unroll
    for (int i = 0; i < R; i++)
#pragma unroll
        for (int j = 0; j < R; j++) acc[i][j] = 0.0;
    double ra[U], rb[U];
    gemm_load_chunk<NT>(a, bb, np, i0, j0, 0, transA, transB, ra, rb);
    gemm_store_chunk<NT>(As[0], Bs[0], transA, transB, ra, rb, d, 0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < np; k0 += kGemmBK) {
        const bool more = k0 + kGemmBK < np;
        if (more) gemm_load_chunk<NT>(a, bb, np, i0, j0, k0 + kGemmBK, transA, transB, ra, rb);
#pragma unroll
        for (int kk = 0; kk < kGemmBK; kk++) {
            double av[R], bv[R];
#pragma unroll
            for (int i = 0; i < R; i++) av[i] = As[buf][kk][ty + S * i];
#pragma unroll
            for (int j = 0; j < R; j++) bv[j] = Bs[buf][kk][tx + S * j];
#pragma unroll
            for (int i = 0; i < R; i++)
#pragma unroll
                for (int j = 0; j < R; j++) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
        if (more) {
            gemm_store_chunk<NT>(As[buf ^ 1], Bs[buf ^ 1], transA, transB, ra, rb, d, k0 + kGemmBK);
            __syncthreads();
            buf ^= 1;
        }
    }
    double* cc = C + t.woff;
#pragma unroll
    for (int i = 0; i < R; i++)
#pragma unroll
        for (int j = 0; j < R; j++) cc[(int64_t)(i0 + ty + S * i) * np + j0 + tx + S * j] = acc[i][j];
}

// Split-K form for the smallest grids (one instance's few blocks): a cluster
// of kSplitK CTAs per 64 x 64 tile, CTA r of the cluster summing k in
// [r np / kSplitK, (r + 1) np / kSplitK) as gemm_kernel<4> does; the partial
// tiles meet in rank 0's registers through distributed shared memory, added
// in rank order (a fixed order: no atomics, no second launch).  kSplitK times
// the CTAs of gemm_kernel<4>, each with a quarter of the FMA chain.
constexpr int kSplitK = 4;
__global__ void __cluster_dims__(kSplitK, 1, 1) __launch_bounds__(256)
    gemm_splitk_kernel(const BlockTask* __restrict__ tasks, const GemmTile* __restrict__ tiles,
                       const double* __restrict__ A, int transA, const double* __restrict__ Bm, int transB,
                       const double* __restrict__ dvec, double* __restrict__ C, const int* __restrict__ bmask) {
    namespace cg = cooperative_groups;
    constexpr int R = 4, S = 16, NT = 256, U = 1024 / NT;
    // the two operand buffers, and after the K loop the CTA's partial tile
    // (64 rows of kGemmLd: the same 4,160 doubles)
    __shared__ double sm[2 * 2 * kGemmBK * kGemmLd];
    auto As = reinterpret_cast<double (*)[kGemmBK][kGemmLd]>(sm);
    auto Bs = reinterpret_cast<double (*)[kGemmBK][kGemmLd]>(sm + 2 * kGemmBK * kGemmLd);
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const GemmTile tl = tiles[blockIdx.x / kSplitK];
    if (bmask && !bmask[tl.task]) return;  // every CTA of the cluster: the same tile
    const BlockTask t = tasks[tl.task];
    const int np = t.np;
    const double* a = A + t.woff;
    const double* bb = Bm + t.woff;
    const double* d = dvec ? dvec + t.doff : nullptr;
    const int tx = threadIdx.x % S, ty = threadIdx.x / S;
    const int i0 = tl.ti * 64, j0 = tl.tj * 64;
    const int kq = np / kSplitK, kb = rank * kq, ke = kb + kq;  // np is a multiple of 64
    double acc[R][R];
#pragma unroll
    for (int i = 0; i < R; i++)
#pragma unroll
        for (int j = 0; j < R; j++) acc[i][j] = 0.0;
    double ra[U], rb[U];
    gemm_load_chunk<NT>(a, bb, np, i0, j0, kb, transA, transB, ra, rb);
    gemm_store_chunk<NT>(As[0], Bs[0], transA, transB, ra, rb, d, kb);
    __syncthreads();
    int buf = 0;
    for (int k0 = kb; k0 < ke; k0 += kGemmBK) {
        const bool more = k0 + kGemmBK < ke;
        if (more) gemm_load_chunk<NT>(a, bb, np, i0, j0, k0 + kGemmBK, transA, transB, ra, rb);
#pragma unroll
        for (int kk = 0; kk < kGemmBK; kk++) {
            double av[R], bv[R];
#pragma unroll
            for (int i = 0; i < R; i++) av[i] = As[buf][kk][ty + S * i];
#pragma unroll
            for (int j = 0; j < R; j++) bv[j] = Bs[buf][kk][tx + S * j];
#pragma unroll
            for (int i = 0; i < R; i++)
#pragma unroll
                for (int j = 0; j < R; j++) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
        if (more) {
            gemm_store_chunk<NT>(As[buf ^ 1], Bs[buf ^ 1], transA, transB, ra, rb, d, k0 + kGemmBK);
            __syncthreads();
            buf ^= 1;
        }
    }
    __syncthreads();  // the operand buffers become the partial tile
#pragma unroll
    for (int i = 0; i < R; i++)
#pragma unroll
        for (int j = 0; j < R; j++) sm[(ty + S * i) * kGemmLd + tx + S * j] = acc[i][j];
    cl.sync();
    if (rank == 0) {
        double* cc = C + t.woff;
#pragma unroll
        for (int i = 0; i < R; i++)
#pragma unroll
            for (int j = 0; j < R; j++) {
                const int o = (ty + S * i) * kGemmLd + tx + S * j;
                double v = 0.0;
                for (int r = 0; r < kSplitK; r++) v += cl.map_shared_rank(sm, r)[o];
                cc[(int64_t)(i0 + ty + S * i) * np + j0 + tx + S * j] = v;
            }
    }
    cl.sync();  // the partial tiles stay alive until rank 0 has read them
}

// Global index of local row a (0..63) of pair (I, J): first 32 rows are column
// block I, the next 32 are block J.
__device__ __forceinline__ int pair_idx(int I, int J, int a) { return a < 32 ? I * 32 + a : J * 32 + (a - 32); }

__global__ void __launch_bounds__(kJThreads) bj_solve_kernel(const BlockTask* __restrict__ tasks,
                                                             const PairTask* __restrict__ pt, int round, double* Ww,
                                                             double* __restrict__ Qbuf, const int* __restrict__ bmask,
                                                             const double* __restrict__ pthr,
                                                             int* __restrict__ qskip) {
    extern __shared__ double sm[];
    __shared__ double red[33];
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
    // a pair problem already diagonal to the block's share of its tolerance
    // is left alone: its rotation is the identity and the updates skip it
    const int64_t qi = (t.qoff >> 12) + pk.k;
    double off = 0.0;
    for (int l = threadIdx.x; l < 64 * 64; l += blockDim.x)
        if (l / 64 != l % 64) {
            const double v = S[(l / 64) * kLd + (l % 64)];
            off += v * v;
        }
    off = block_sum(off, red);
    if (off <= pthr[pk.task]) {
        if (threadIdx.x == 0) qskip[qi] = 1;
        return;
    }
    if (threadIdx.x == 0) qskip[qi] = 0;
    // the outer block-Jacobi sweeps iterate anyway: a few inner sweeps suffice
    jacobi_smem(S, Q, 64, kPairSweeps, kJacobiRotEps);
    __syncthreads();
    double* qo = Qbuf + t.qoff + (int64_t)pk.k * 4096;
    for (int l = threadIdx.x; l < 64 * 64; l += blockDim.x) qo[l] = Q[(l / 64) * kLd + (l % 64)];
}

// T (64x64, smem ld kLd) <- Q1^T T Q2, where Q1 and Q2 are 64x64 row-major
// in global memory and either may be null (identity); used for W tile =
// Q1^T T Q2 and V tile = T Q.
__device__ void tile_rotate(double* T, double* Qs, const double* Q1g, const double* Q2g) {
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    if (Q2g) {
        // T <- T * Q2
        for (int l = threadIdx.x; l < 4096; l += blockDim.x) Qs[(l / 64) * kLd + l % 64] = Q2g[l];
        __syncthreads();
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
        __syncthreads();
    }
    if (!Q1g) return;
    // T <- Q1^T * T
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

// W tiles first (blockIdx.x < nwt), then V tiles: one launch per round.
__global__ void __launch_bounds__(256) bj_update_wv_kernel(const BlockTask* __restrict__ tasks,
                                                           const WTileTask* __restrict__ wt, int nwt,
                                                           const VTileTask* __restrict__ vt, int round,
                                                           double* Ww, double* Vw, const double* __restrict__ Qbuf,
                                                           const int* __restrict__ bmask,
                                                           const int* __restrict__ qskip) {
    extern __shared__ double sm[];
    double* T = sm;
    double* Qs = sm + kJ * kLd;
    if ((int)blockIdx.x < nwt) {
        const WTileTask w = wt[blockIdx.x];
        if (bmask && !bmask[w.task]) return;
        const BlockTask t = tasks[w.task];
        const bool s1 = qskip[(t.qoff >> 12) + w.k1] != 0, s2 = qskip[(t.qoff >> 12) + w.k2] != 0;
        if (s1 && s2) return;
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
        tile_rotate(T, Qs, s1 ? nullptr : Qbuf + t.qoff + (int64_t)w.k1 * 4096,
                    s2 ? nullptr : Qbuf + t.qoff + (int64_t)w.k2 * 4096);
        for (int l = threadIdx.x; l < 4096; l += blockDim.x) {
            const int a = l / 64, bq = l % 64;
            base[(int64_t)pair_idx(I1, J1, a) * t.np + pair_idx(I2, J2, bq)] = T[a * kLd + bq];
        }
        return;
    }
    const VTileTask v = vt[blockIdx.x - nwt];
    if (bmask && !bmask[v.task]) return;
    const BlockTask t = tasks[v.task];
    if (qskip[(t.qoff >> 12) + v.k]) return;
    int I, J;
    rr_pair(t.nb, round % (t.nb - 1), v.k, I, J);
    double* base = Vw + t.woff;
    const int r0 = v.chunk * 64;
    for (int l = threadIdx.x; l < 4096; l += blockDim.x) {
        const int a = l / 64, bq = l % 64;
        T[a * kLd + bq] = base[(int64_t)(r0 + a) * t.np + pair_idx(I, J, bq)];
    }
    __syncthreads();
    tile_rotate(T, Qs, nullptr, Qbuf + t.qoff + (int64_t)v.k * 4096);
    for (int l = threadIdx.x; l < 4096; l += blockDim.x) {
        const int a = l / 64, bq = l % 64;
        base[(int64_t)(r0 + a) * t.np + pair_idx(I, J, bq)] = T[a * kLd + bq];
    }
}

// Convergence test of the block Jacobi, in two deterministic passes:
// per padded row the off-diagonal and total squared sums, then per block.
__global__ void bj_rowsum_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ Ww,
                                 const int* __restrict__ bmask, double* __restrict__ rowsum) {
    __shared__ double red[33];
    const int task = blockIdx.y;
    if (!bmask[task]) return;
    const BlockTask t = tasks[task];
    const int p = blockIdx.x;
    if (p >= t.np) return;
    const double* w = Ww + t.woff + (int64_t)p * t.np;
    double off = 0.0, tot = 0.0;
    for (int q = threadIdx.x; q < t.np; q += blockDim.x) {
        const double a = w[q];
        tot += a * a;
        if (q != p) off += a * a;
    }
    off = block_sum(off, red);
    tot = block_sum(tot, red);
    if (threadIdx.x == 0) {
        rowsum[2 * (t.doff + p)] = off;
        rowsum[2 * (t.doff + p) + 1] = tot;
    }
}

__global__ void bj_check_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ rowsum,
                                const double* __restrict__ tols, const double* __restrict__ abs_tols,
                                const int* __restrict__ max_sweeps, int sweeps_done, int* __restrict__ bmask,
                                double* __restrict__ pthr) {
    __shared__ double red[33];
    if (!bmask[blockIdx.x]) return;
    if (max_sweeps && sweeps_done >= max_sweeps[blockIdx.x]) {
        if (threadIdx.x == 0) bmask[blockIdx.x] = 0;
        return;
    }
    const double tol = tols[blockIdx.x];
    const double atol = abs_tols ? abs_tols[blockIdx.x] : 0.0;
    const BlockTask t = tasks[blockIdx.x];
    double off = 0.0, tot = 0.0;
    for (int p = threadIdx.x; p < t.np; p += blockDim.x) {
        off += rowsum[2 * (t.doff + p)];
        tot += rowsum[2 * (t.doff + p) + 1];
    }
    off = block_sum(off, red);
    tot = block_sum(tot, red);
    const double lim = fmax(tol * tol * tot, atol * atol);
    if (threadIdx.x == 0) {
        if (!(off > lim)) bmask[blockIdx.x] = 0;
        // per pair problem: the block's limit shared over the nb (nb - 1) / 2
        // pair problems of a sweep
        pthr[blockIdx.x] = lim / (0.5 * (double)t.nb * (double)(t.nb - 1));
    }
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

// dx = max(lam, 0) / mu and dz = max(-lam, 0), zero on padding
__global__ void pos_weights_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ lam,
                                   const double* __restrict__ mu, const int* __restrict__ bmask,
                                   double* __restrict__ dx, double* __restrict__ dz) {
    if (bmask && !bmask[blockIdx.x]) return;
    const BlockTask t = tasks[blockIdx.x];
    const double m = mu[t.inst];
    for (int j = threadIdx.x; j < t.np; j += blockDim.x) {
        const double l = lam[t.doff + j];
        const bool real = j < t.n;
        dx[t.doff + j] = (real && l > 0.0) ? l / m : 0.0;
        dz[t.doff + j] = (real && l < 0.0) ? -l : 0.0;
    }
}

// lam = diag(W) for blocks diagonalised by Jacobi
__global__ void lam_from_diag_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ Ww,
                                     const int* __restrict__ bmask, double* __restrict__ lam) {
    if (bmask && !bmask[blockIdx.x]) return;
    const BlockTask t = tasks[blockIdx.x];
    for (int j = threadIdx.x; j < t.np; j += blockDim.x) lam[t.doff + j] = Ww[t.woff + (int64_t)j * t.np + j];
}

// ---- Ogita-Aishima refinement of the previous eigenvectors -------------------
//
// With S = V^T U V and G = V^T V (R = I - G), the refined eigenvalues are
// lam_i = s_ii / g_ii and the correction V <- V (I + E) has
//   E_ij = (s_ij - lam_j g_ij) / (lam_j - lam_i)   (i != j),   E_ii = (1 - g_ii) / 2,
// which removes the off-diagonal part of S to first order and restores
// orthogonality (Ogita and Aishima, Japan J. Indust. Appl. Math. 35 (2018)
// 1007-1035, Algorithm 1).  A pair whose coupling is negligible gets the
// orthogonality term only; a pair with |E_ij| > kHard (nearly degenerate and
// strongly coupled, where the first-order step is invalid) marks its block
// for the Jacobi fallback.  emax[block] = max |E_ij| decides convergence:
// the error left after the update is of order emax^2.

constexpr double kHard = 0.1;
constexpr double kFroMax = 0.2;

__global__ void oa_lambda_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ S,
                                 const double* __restrict__ G, const int* __restrict__ bmask,
                                 double* __restrict__ lam, double* __restrict__ scale, int* __restrict__ restart) {
    __shared__ double red[33];
    __shared__ int bad;
    if (bmask && !bmask[blockIdx.x]) return;
    const BlockTask t = tasks[blockIdx.x];
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    double mx = 0.0;
    for (int i = threadIdx.x; i < t.np; i += blockDim.x) {
        const int64_t d = t.woff + (int64_t)i * t.np + i;
        const double l = (i < t.n) ? S[d] / G[d] : 0.0;
        lam[t.doff + i] = l;
        mx = fmax(mx, fabs(l));
        // eigenvectors drifted far from orthonormal, or values broke down
        // (the refinement itself corrects deviations of order ||E||^2; only a
        // large drift means a step went wrong)
        if (i < t.n && (!isfinite(l) || !(fabs(G[d] - 1.0) <= 0.25))) bad = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0 && bad) restart[blockIdx.x] = 1;
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, red[w]);
        scale[blockIdx.x] = m;
    }
}

// One pass per row: partner[i] = the j most strongly coupled to i among the
// pairs the first-order step cannot handle (|num| > kHard |gap|, not
// negligible), ranked by |num| / |gap| with ties to the smaller j; -1 if none.
// Mutual partners form a matching that the update rotates exactly.
__global__ void oa_pairs_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ S,
                                const double* __restrict__ G, const double* __restrict__ lam,
                                const double* __restrict__ scale, const int* __restrict__ bmask,
                                int* __restrict__ partner, int* __restrict__ hard,
                                unsigned long long* __restrict__ gdev, int* __restrict__ restart) {
    __shared__ double sr[256];
    __shared__ int sj[256];
    __shared__ double sg[256];
    const int task = blockIdx.y;
    if (bmask && !bmask[task]) return;
    const BlockTask t = tasks[task];
    const int i = blockIdx.x;
    if (i >= t.np) return;
    double best = -1.0;
    int bj = -1;
    double gd = 0.0;  // max_j |G_ij - delta_ij| of this row: how far V is from orthonormal
    if (i < t.n) {
        const double negligible = 1e-15 * scale[task];
        const double li = lam[t.doff + i];
        for (int j = threadIdx.x; j < t.n; j += blockDim.x) {
            const int64_t w = t.woff + (int64_t)i * t.np + j;
            gd = fmax(gd, fabs(G[w] - (j == i ? 1.0 : 0.0)));
            if (j == i) continue;
            const double lj = lam[t.doff + j];
            const double num = fabs(S[w] - lj * G[w]);
            const double gap = fabs(lj - li);
            if (num > negligible && !(num <= kHard * gap)) {
                const double ratio = gap > 0.0 ? num / gap : DBL_MAX;
                if (ratio > best) {
                    best = ratio;
                    bj = j;
                }
            }
        }
    }
    sr[threadIdx.x] = best;
    sj[threadIdx.x] = bj;
    sg[threadIdx.x] = gd;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sg[threadIdx.x] = fmax(sg[threadIdx.x], sg[threadIdx.x + w]);
            const double r2 = sr[threadIdx.x + w];
            const int j2 = sj[threadIdx.x + w];
            if (r2 > sr[threadIdx.x] || (r2 == sr[threadIdx.x] && j2 >= 0 && (sj[threadIdx.x] < 0 || j2 < sj[threadIdx.x]))) {
                sr[threadIdx.x] = r2;
                sj[threadIdx.x] = j2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partner[t.doff + i] = sj[0];
        if (gdev && sg[0] > 0.0) atomicMax(gdev + task, (unsigned long long)__double_as_longlong(sg[0]));
        // eigenvectors far from orthonormal: the block restarts cold
        if (!(sg[0] <= 0.25)) restart[task] = 1;
    }
}

// M = I + E.  Isolated strongly coupled pairs (partner of each other) get
// the exact Jacobi rotation of their 2 x 2 problem instead of the first-order
// step; the next sweep sees them decoupled.
__global__ void oa_update_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ S,
                                 const double* __restrict__ G, const double* __restrict__ lam,
                                 const double* __restrict__ scale, const int* __restrict__ partner,
                                 const int* __restrict__ bmask, double* __restrict__ M,
                                 unsigned long long* __restrict__ emax, int* __restrict__ hard,
                                 double* __restrict__ erow) {
    __shared__ double red[33];
    const int task = blockIdx.y;
    if (bmask && !bmask[task]) return;
    const BlockTask t = tasks[task];
    const int i = blockIdx.x;
    if (i >= t.np) return;
    const double negligible = 1e-15 * scale[task];
    const double li = lam[t.doff + i];
    const int pi = (i < t.n) ? partner[t.doff + i] : -1;
    double emx = 0.0, esq = 0.0;
    int hd = 0;  // hard flags now come from oa_fro_kernel only
    // exact rotation of a mutual pair (i, pi); a row whose strongest partner
    // is taken waits for a later sweep (its hard pairs get E = 0 now)
    double rc = 1.0, rs = 0.0, pend = 0.0;
    bool rot = false, pending = false;
    if (pi >= 0 && partner[t.doff + pi] == i) {
        const int p = i < pi ? i : pi, q = i < pi ? pi : i;
        const double app = lam[t.doff + p], aqq = lam[t.doff + q];
        const int64_t wpq = t.woff + (int64_t)p * t.np + q;
        const double apq = S[wpq] - aqq * G[wpq];
        const double tau = (aqq - app) / (2.0 * apq);
        const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        rc = 1.0 / sqrt(1.0 + tt * tt);
        rs = tt * rc;
        rot = true;
        emx = fabs(rs);
    } else if (pi >= 0) {
        pending = true;
        const int64_t w = t.woff + (int64_t)i * t.np + pi;
        pend = fabs(S[w] - lam[t.doff + pi] * G[w]);
    }
    for (int j = threadIdx.x; j < t.np; j += blockDim.x) {
        const int64_t w = t.woff + (int64_t)i * t.np + j;
        double m;
        if (i >= t.n || j >= t.n) {
            m = (i == j) ? 1.0 : 0.0;
        } else if (i == j) {
            // the norm correction (1 - g_ii) / 2 applies to rotated columns too
            m = (rot ? rc : 1.0) + 0.5 * (1.0 - G[w]);
        } else if (rot && j == pi) {
            // J_pp = c, J_pq = s, J_qp = -s, J_qq = c with p < q, plus the
            // orthogonality term of the pair (first order, like every pair)
            m = ((i < j) ? rs : -rs) - 0.5 * G[w];
        } else {
            const double lj = lam[t.doff + j];
            const double num = S[w] - lj * G[w];
            const double gap = lj - li;
            double e;
            if (fabs(num) <= negligible) {
                e = -0.5 * G[w];
            } else if (!(fabs(num) <= kHard * fabs(gap))) {
                // strongly coupled: rotated in this or a later sweep; only the
                // orthogonality term now (Ogita-Aishima's rule for clustered
                // pairs), so that V stays orthonormal inside clusters
                e = -0.5 * G[w];
                pending = true;
                pend = fmax(pend, fabs(num));
            } else {
                e = num / gap;
            }
            emx = fmax(emx, fabs(e));
            esq += e * e;
            m = e;
        }
        M[w] = m;
    }
    esq = block_sum(esq, red);
    if (threadIdx.x == 0) erow[t.doff + i] = esq;
    // a pair left for a later sweep leaves a residual of its coupling; expressed
    // on the emax scale (residual ~ emax^2 scale) so the block's tolerance
    // decides whether another sweep is needed
    if (pending) emx = fmax(emx, scale[task] > 0.0 ? sqrt(pend / scale[task]) : 1.0);
    for (int o = 16; o > 0; o >>= 1) {
        emx = fmax(emx, __shfl_down_sync(0xffffffffu, emx, o));
        hd |= __shfl_down_sync(0xffffffffu, hd, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (emx > 0.0) atomicMax(emax + task, (unsigned long long)__double_as_longlong(emx));
        if (hd) atomicOr(hard + task, 1);
    }
}

// After an analysis: upd = ref & !hard (apply V <- V M), jac |= ref & hard,
// ref = upd & (emax > tol) (another sweep needed); counts ref into n_ref.
__global__ void oa_fro_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ erow,
                              const int* __restrict__ bmask, int* __restrict__ hard) {
    __shared__ double red[33];
    if (bmask && !bmask[blockIdx.x]) return;
    const BlockTask t = tasks[blockIdx.x];
    double s = 0.0;
    for (int i = threadIdx.x; i < t.n; i += blockDim.x) s += erow[t.doff + i];
    s = block_sum(s, red);
    // a first-order step is only trusted while ||E||_F stays small
    if (threadIdx.x == 0 && !(s <= kFroMax * kFroMax)) hard[blockIdx.x] = 1;
}

__global__ void oa_masks_kernel(int ntasks, const unsigned long long* __restrict__ emax,
                                const int* __restrict__ hard, const double* __restrict__ tols,
                                const double* __restrict__ abs_tols, const double* __restrict__ scale,
                                int* __restrict__ ref,
                                int* __restrict__ upd, int* __restrict__ jac, int* __restrict__ n_ref) {
    int cnt = 0;
    for (int t = threadIdx.x; t < ntasks; t += blockDim.x) {
        const int r = ref[t];
        const int h = hard[t];
        upd[t] = r && !h;
        if (r && h) jac[t] = 1;
        const double e = __longlong_as_double((long long)emax[t]);
        // residual after the update ~ emax^2 * scale: stop when that is below the
        // absolute tolerance, or when emax is below the relative one
        double lim = tols[t];
        if (abs_tols && scale[t] > 0.0) lim = fmax(lim, sqrt(abs_tols[t] / scale[t]));
        const int again = r && !h && (e > lim);
        ref[t] = again;
        cnt += again;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    __shared__ int s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += s[w];
        *n_ref = tot;
    }
}

// M = I + (I - G) / 2 on the n x n part (identity on the padding): V M is one
// Newton-Schulz step towards the orthonormal polar factor of V (G = V^T V);
// it squares the distance from orthonormal.
__global__ void ortho_step_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ G,
                                  const int* __restrict__ bmask, double* __restrict__ M) {
    if (bmask && !bmask[blockIdx.y]) return;
    const BlockTask t = tasks[blockIdx.y];
    const int p = blockIdx.x;
    if (p >= t.np) return;
    for (int q = threadIdx.x; q < t.np; q += blockDim.x) {
        const int64_t w = t.woff + (int64_t)p * t.np + q;
        const double id = (p == q) ? 1.0 : 0.0;
        M[w] = (p < t.n && q < t.n) ? id + 0.5 * (id - G[w]) : id;
    }
}

// C <- upper triangle of C mirrored to the lower one (tile granularity: the
// GEMM computed tiles ti <= tj only)
__global__ void mirror_kernel(const BlockTask* __restrict__ tasks, double* __restrict__ C,
                              const int* __restrict__ bmask) {
    if (bmask && !bmask[blockIdx.y]) return;
    const BlockTask t = tasks[blockIdx.y];
    const int p = blockIdx.x;
    if (p >= t.np) return;
    double* c = C + t.woff;
    // row p, columns q < 64 * (p / 64): lower tiles
    const int qend = (p / 64) * 64;
    for (int q = threadIdx.x; q < qend; q += blockDim.x) c[(int64_t)p * t.np + q] = c[(int64_t)q * t.np + p];
}

__global__ void block_mask_kernel(const BlockTask* __restrict__ tasks, int ntasks, const int* __restrict__ mask,
                                  int* __restrict__ bmask) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntasks; t += gridDim.x * blockDim.x)
        bmask[t] = mask[tasks[t].inst] != 0;
}

__global__ void uncap_kernel(int n, const int* __restrict__ sel, int* __restrict__ max_sweeps) {
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (sel[i]) max_sweeps[i] = 1 << 20;
}

__global__ void merge_mask_kernel(int n, const int* __restrict__ src, int* __restrict__ dst) {
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (src[i]) dst[i] = 1;
}

__global__ void copy_blocks_kernel(const BlockTask* __restrict__ tasks, const double* __restrict__ src,
                                   double* __restrict__ dst, const int* __restrict__ bmask) {
    if (bmask && !bmask[blockIdx.y]) return;
    const BlockTask t = tasks[blockIdx.y];
    const int p = blockIdx.x;
    if (p >= t.np) return;
    const int64_t o = t.woff + (int64_t)p * t.np;
    for (int q = threadIdx.x; q < t.np; q += blockDim.x) dst[o + q] = src[o + q];
}

__global__ void count_kernel(int n, const int* __restrict__ mask, int* out) {
    int c = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) c += mask[i] != 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    __shared__ int s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += s[w];
        *out = tot;
    }
}

__global__ void write_xz_kernel(const BlockTask* __restrict__ tasks, int B, const double* __restrict__ Xw,
                                const double* __restrict__ Zw, const int* __restrict__ mask, double* __restrict__ x,
                                double* __restrict__ z) {
    const BlockTask t = tasks[blockIdx.y];
    const int p = blockIdx.x;
    if (p >= t.n) return;
    const int b = t.inst;
    if (mask && !mask[b]) return;
    for (int q = threadIdx.x; q < t.n; q += blockDim.x) {
        const int64_t w = t.woff + (int64_t)p * t.np + q;
        const int64_t e = (t.xoff + (int64_t)p * t.n + q) * B + b;
        x[e] = Xw[w];
        z[e] = Zw[w];
    }
}

constexpr size_t kJacobiSmem = 2 * kJ * kLd * sizeof(double);
constexpr size_t kJacobiWarmSmem = 3 * kJ * kLd * sizeof(double);  // + the T of a warm start

// The 66,560 B of dynamic shared memory of the Jacobi kernels need an opt-in
// per kernel and per device.  Each device is set up once; a failed attempt is
// retried on the next launch, whose own error then reaches the caller.
void set_smem_attrs() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return;
    static std::mutex mu;
    static std::vector<char> done;
    std::lock_guard<std::mutex> lk(mu);
    if ((size_t)dev < done.size() && done[dev]) return;
    bool ok = cudaFuncSetAttribute(small_project_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kJacobiWarmSmem) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(bj_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kJacobiSmem) == cudaSuccess;
    ok = ok && cudaFuncSetAttribute(bj_update_wv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kJacobiSmem) == cudaSuccess;
    if (!ok) return;
    if ((size_t)dev >= done.size()) done.resize(dev + 1, 0);
    done[dev] = 1;
}

}  // namespace

void launch_small_project(const BlockTask* tasks, int ntasks, int B, const double* aty, const double* c, double* x,
                          double* z, const double* mu, const int* mask, cudaStream_t s, double* vsave, bool warm,
                          const double* stol) {
    if (ntasks == 0) return;
    set_smem_attrs();
    small_project_kernel<<<ntasks, kJThreads, vsave ? kJacobiWarmSmem : kJacobiSmem, s>>>(
        tasks, B, aty, c, x, z, mu, mask, vsave, warm ? 1 : 0, stol);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_form_u(const BlockTask* tasks, int ntasks, int max_np, int B, const double* aty, const double* c,
                      const double* x, const double* mu, const int* mask, double* Uw, cudaStream_t s) {
    if (ntasks == 0) return;
    form_u_kernel<<<dim3(max_np, ntasks), 128, 0, s>>>(tasks, B, aty, c, x, mu, mask, Uw);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_cold_start(const BlockTask* tasks, int ntasks, int max_np, const double* Uw, double* Ww, double* Vw,
                          const int* bmask, cudaStream_t s) {
    if (ntasks == 0) return;
    cold_start_kernel<<<dim3(max_np, ntasks), 128, 0, s>>>(tasks, Uw, Ww, Vw, bmask);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_gemm(const BlockTask* tasks, const GemmTile* tiles, int ntiles, const double* A, bool transA,
                 const double* Bm, bool transB, const double* dvec, double* C, const int* bmask, cudaStream_t s) {
    if (ntiles == 0) return;
    // below two tiles per SM (148 SMs) the 256-thread form hides the latency
    // the 64-thread form cannot; below half a tile per SM, the split-K
    // clusters also spread each tile's K over four CTAs
    if (ntiles * kSplitK <= 2 * 148)
        gemm_splitk_kernel<<<ntiles * kSplitK, 256, 0, s>>>(tasks, tiles, A, transA, Bm, transB, dvec, C, bmask);
    else if (ntiles < 2 * 148)
        gemm_kernel<4><<<ntiles, 256, 0, s>>>(tasks, tiles, A, transA, Bm, transB, dvec, C, bmask);
    else
        gemm_kernel<8><<<ntiles, 64, 0, s>>>(tasks, tiles, A, transA, Bm, transB, dvec, C, bmask);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_bj_solve(const BlockTask* tasks, const PairTask* pt, int npt, int round, double* Ww, double* Qbuf,
                     const int* bmask, const double* pthr, int* qskip, cudaStream_t s) {
    if (npt == 0) return;
    set_smem_attrs();
    bj_solve_kernel<<<npt, kJThreads, kJacobiSmem, s>>>(tasks, pt, round, Ww, Qbuf, bmask, pthr, qskip);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_bj_update_wv(const BlockTask* tasks, const WTileTask* wt, int nwt, const VTileTask* vt, int nvt, int round,
                         double* Ww, double* Vw, const double* Qbuf, const int* bmask, const int* qskip,
                         cudaStream_t s) {
    if (nwt + nvt == 0) return;
    set_smem_attrs();
    bj_update_wv_kernel<<<nwt + nvt, 256, kJacobiSmem, s>>>(tasks, wt, nwt, vt, round, Ww, Vw, Qbuf, bmask, qskip);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_bj_check(const BlockTask* tasks, int ntasks, int max_np, const double* Ww, const double* tol,
                     const double* abs_tol, const int* max_sweeps, int sweeps_done, double* rowsum, int* bmask,
                     double* pthr, int* n_open, cudaStream_t s) {
    if (ntasks == 0) return;
    bj_rowsum_kernel<<<dim3(max_np, ntasks), 128, 0, s>>>(tasks, Ww, bmask, rowsum);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    bj_check_kernel<<<ntasks, 256, 0, s>>>(tasks, rowsum, tol, abs_tol, max_sweeps, sweeps_done, bmask, pthr);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    count_open_kernel<<<1, 1024, 0, s>>>(ntasks, bmask, n_open);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_pos_weights(const BlockTask* tasks, int ntasks, const double* lam, const double* mu, const int* bmask,
                        double* dx, double* dz, cudaStream_t s) {
    if (ntasks == 0) return;
    pos_weights_kernel<<<ntasks, 128, 0, s>>>(tasks, lam, mu, bmask, dx, dz);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_lam_from_diag(const BlockTask* tasks, int ntasks, const double* Ww, const int* bmask, double* lam,
                          cudaStream_t s) {
    if (ntasks == 0) return;
    lam_from_diag_kernel<<<ntasks, 128, 0, s>>>(tasks, Ww, bmask, lam);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_oa_analyze(const BlockTask* tasks, int ntasks, int max_np, const double* S, const double* G,
                       const int* bmask, double* lam, double* scale, int* partner, double* M,
                       unsigned long long* emax, int* hard, double* erow, int* restart, unsigned long long* gdev,
                       cudaStream_t s) {
    if (ntasks == 0) return;
    oa_lambda_kernel<<<ntasks, 256, 0, s>>>(tasks, S, G, bmask, lam, scale, restart);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    oa_pairs_kernel<<<dim3(max_np, ntasks), 256, 0, s>>>(tasks, S, G, lam, scale, bmask, partner, hard, gdev,
                                                          restart);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    oa_update_kernel<<<dim3(max_np, ntasks), 256, 0, s>>>(tasks, S, G, lam, scale, partner, bmask, M, emax,
                                                           hard, erow);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    oa_fro_kernel<<<ntasks, 256, 0, s>>>(tasks, erow, bmask, hard);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_oa_masks(int ntasks, const unsigned long long* emax, const int* hard, const double* tol,
                     const double* abs_tol, const double* scale, int* ref, int* upd, int* jac, int* n_ref,
                     cudaStream_t s) {
    if (ntasks == 0) return;
    oa_masks_kernel<<<1, 1024, 0, s>>>(ntasks, emax, hard, tol, abs_tol, scale, ref, upd, jac, n_ref);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_copy_blocks(const BlockTask* tasks, int ntasks, int max_np, const double* src, double* dst,
                        const int* bmask, cudaStream_t s) {
    if (ntasks == 0) return;
    copy_blocks_kernel<<<dim3(max_np, ntasks), 128, 0, s>>>(tasks, src, dst, bmask);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_mirror(const BlockTask* tasks, int ntasks, int max_np, double* C, const int* bmask, cudaStream_t s) {
    if (ntasks == 0) return;
    mirror_kernel<<<dim3(max_np, ntasks), 128, 0, s>>>(tasks, C, bmask);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_ortho_step(const BlockTask* tasks, int ntasks, int max_np, const double* G, const int* bmask, double* M,
                       cudaStream_t s) {
    if (ntasks == 0) return;
    ortho_step_kernel<<<dim3(max_np, ntasks), 128, 0, s>>>(tasks, G, bmask, M);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_block_mask(const BlockTask* tasks, int ntasks, const int* mask, int* bmask, cudaStream_t s) {
    if (ntasks == 0) return;
    block_mask_kernel<<<(ntasks + 255) / 256, 256, 0, s>>>(tasks, ntasks, mask, bmask);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_uncap(int n, const int* sel, int* max_sweeps, cudaStream_t s) {
    if (n == 0) return;
    uncap_kernel<<<1, 1024, 0, s>>>(n, sel, max_sweeps);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_merge_mask(int n, const int* src, int* dst, cudaStream_t s) {
    if (n == 0) return;
    merge_mask_kernel<<<1, 1024, 0, s>>>(n, src, dst);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_count(int n, const int* mask, int* out, cudaStream_t s) {
    count_kernel<<<1, 1024, 0, s>>>(n, mask, out);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_write_xz(const BlockTask* tasks, int ntasks, int max_n, int B, const double* Xw, const double* Zw,
                     const int* mask, double* x, double* z, cudaStream_t s) {
    if (ntasks == 0) return;
    write_xz_kernel<<<dim3(max_n, ntasks), 128, 0, s>>>(tasks, B, Xw, Zw, mask, x, z);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

}  // namespace v2g
