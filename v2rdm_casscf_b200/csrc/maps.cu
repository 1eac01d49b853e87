// Constraint maps, CG vector kernels and per-instance reductions (FP64).
//
// The maps A and A^T are applied as gathers over bucketed-ELL tables shared
// by all instances of a group (see kernels.cuh for the layouts).  A^T is
// the transpose of A's table, so every primal element sums its contributing
// constraints itself: no atomics, deterministic order, and the two maps are
// exact adjoints.  These kernels are HBM-bound; their algorithmic traffic per
// application is 8 * (dimx + nconstraints) bytes per instance.
#include <map>
#include <mutex>

#include "kernels.cuh"

namespace v2g {

std::atomic<long> g_kernel_launches{0};

namespace {

constexpr int kThreads = 256;

inline int grid_for(int64_t work, int threads = kThreads) {
    int64_t g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > 148 * 64) g = 148 * 64;
    return (int)g;
}

constexpr int kRedBlocks = 148 * 4;
constexpr int kSpmvBlocks = 148 * 64;

// Thread mapping shared by the map and vector kernels that also reduce: the
// rows are cut into passes of T/B rows; pass k goes to block k % G, where
// thread t handles instance t % B of row t / B.  A thread therefore always
// serves the same instance (per-instance partial sums come out in a fixed
// order) and the rows in flight at any moment form one contiguous window,
// which keeps the gathers of neighbouring rows in L2.
struct Chunk {
    int64_t first, stride, nrows;
    int b, rsub, rows_per_pass;
    bool live;
};
__device__ __forceinline__ Chunk chunk_of(int64_t nrows, int B) {
    Chunk c;
    c.rows_per_pass = blockDim.x / B;
    const int lanes = c.rows_per_pass * B;
    c.b = threadIdx.x % B;
    c.rsub = threadIdx.x / B;
    c.live = threadIdx.x < lanes;
    c.first = (int64_t)blockIdx.x * c.rows_per_pass + c.rsub;
    c.stride = (int64_t)gridDim.x * c.rows_per_pass;
    c.nrows = nrows;
    return c;
}

// Per-instance sum over the CTA of v, where thread t holds instance t % B;
// the sum for instance b is returned to thread b < B (0 elsewhere), in a fixed
// order.  When B divides 32 the lanes of one instance sit at stride B in every
// warp: shuffles fold them, then thread b adds the warps' sums; otherwise
// thread b walks its rows.  The CTA synchronises on entry and on exit, so
// the shared scratch can be reused right away.
__device__ __forceinline__ double cta_instance_sum(double v, int B) {
    __shared__ double sh[kThreads];
    double s = 0.0;
    __syncthreads();
    if ((32 % B) == 0) {
        for (int o = 16; o >= B; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane < B) sh[warp * B + lane] = v;
        __syncthreads();
        if ((int)threadIdx.x < B)
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w * B + threadIdx.x];
    } else {
        sh[threadIdx.x] = v;
        __syncthreads();
        if ((int)threadIdx.x < B) {
            const int rows_per_pass = blockDim.x / B;
            for (int k = 0; k < rows_per_pass; k++) s += sh[threadIdx.x + k * B];
        }
    }
    __syncthreads();
    return s;
}

// Per-instance block partial of v, written to partial[slot * B + b] (slot is
// the block's index among the partial sums, not always blockIdx.x).
__device__ __forceinline__ void block_partial(double v, int B, double* __restrict__ partial, int64_t slot) {
    const double s = cta_instance_sum(v, B);
    if ((int)threadIdx.x < B) partial[slot * B + threadIdx.x] = s;
}

// Per-row epilogue shared by the map kernels.
struct Epi {
    const double* sub;
    const double* coef;
    const double* add;
    const double* dotv;
    double* out;
};
// COH: the vectors are written by other CTAs of the same (persistent) launch,
// so they are loaded through L2 (ld.global.cg), never from a stale L1 line.
template <bool STREAM = false, bool COH = false>
__device__ __forceinline__ double epilogue(const Epi& e, int64_t r, int B, int b, double s) {
    const int64_t t = r * B + b;
    if (e.sub) s -= e.sub[r];
    if (e.coef) s *= e.coef[b];
    if (e.add) s += e.add[t];
    if (STREAM)
        __stcs(e.out + t, s);  // written once, not read again by this launch
    else
        e.out[t] = s;
    if (!e.dotv) return 0.0;
    return (COH ? __ldcg(e.dotv + t) : e.dotv[t]) * s;
}

// Bucketed-ELL part.  One lane per row (slot index i of its bucket) and a
// chunk of up to CH consecutive instances per thread: the table loads of a
// warp are 32 consecutive slots (coalesced), and every thread keeps
// W x (instances) independent gathers in flight.  The instances of a chunk are
// adjacent in memory ([col * B + b0 .. b0 + cnt)), loaded as double2 when B is
// even.  Per instance the entries are summed in slot order, so the result does
// not depend on the chunking.  CH = 4 (80 registers, three CTAs per SM) was
// the fastest of 2, 4 and 8 at n = 12..20 with 8..20 instances (B200); single
// instances use CH = 2 (64 registers).
constexpr int kSlotBatch = 4;  // slots whose gathers are issued together

struct Blocks {
    int start[kMaxBuckets + 1];  // first row tile of each bucket
    int nchunk;                  // instance chunks per row tile
};

template <int W, bool VEC, int CH, bool STREAM, bool PK, bool COH>
__device__ __forceinline__ void ell_rows(const DevMap& M, int bi, int64_t tile0, int64_t ntile, int B, int b0,
                                         int cnt, unsigned act, const double* __restrict__ in, const Epi& e,
                                         const double* sbook, double (&dot)[CH]) {
    constexpr int KB = W < kSlotBatch ? W : kSlotBatch;
    const int64_t ns = M.nslots[bi];
    const int32_t* rows = M.rows + M.row_off[bi];
    const int32_t* cols = M.cols + M.ent_off[bi];
    const double* vals = PK ? nullptr : M.vals + M.ent_off[bi];
    for (int64_t i = tile0 * kThreads + threadIdx.x; i < ns; i += ntile * kThreads) {
        double acc[CH];
#pragma unroll
        for (int j = 0; j < CH; j++) acc[j] = 0.0;
#pragma unroll
        for (int k0 = 0; k0 < W; k0 += KB) {
            int c[KB];
            double v[KB];
#pragma unroll
            for (int k = 0; k < KB; k++) {
                const int32_t wd = STREAM ? __ldcs(cols + (int64_t)(k0 + k) * ns + i)
                                          : __ldg(cols + (int64_t)(k0 + k) * ns + i);
                if (PK) {
                    c[k] = wd < 0 ? -1 : (wd & ((1 << kCodeShift) - 1));
                    v[k] = sbook[wd < 0 ? 0 : (wd >> kCodeShift)];
                } else {
                    c[k] = wd;
                    v[k] = STREAM ? __ldcs(vals + (int64_t)(k0 + k) * ns + i)
                                  : __ldg(vals + (int64_t)(k0 + k) * ns + i);
                }
            }
#pragma unroll
            for (int k = 0; k < KB; k++) {
                if (c[k] < 0) continue;
                const double* g = in + (int64_t)c[k] * B + b0;
                if (VEC) {
#pragma unroll
                    for (int j = 0; j < CH; j += 2)
                        if (j < cnt) {
                            const double2 q = COH ? __ldcg(reinterpret_cast<const double2*>(g + j))
                                                  : __ldg(reinterpret_cast<const double2*>(g + j));
                            acc[j] += v[k] * q.x;
                            acc[j + 1] += v[k] * q.y;
                        }
                } else {
#pragma unroll
                    for (int j = 0; j < CH; j++)
                        if (j < cnt) acc[j] += v[k] * (COH ? __ldcg(g + j) : __ldg(g + j));
                }
            }
        }
        const int64_t r = STREAM ? __ldcs(rows + i) : rows[i];
#pragma unroll
        for (int j = 0; j < CH; j++)
            if (j < cnt && ((act >> j) & 1u)) dot[j] += epilogue<STREAM, COH>(e, r, B, b0 + j, acc[j]);
    }
}

// Instances [b0, b0 + cnt) of chunk ch: balanced, and in pairs when B is even
// (so that double2 loads stay 16-byte aligned).
__device__ __forceinline__ void chunk_range(int B, int nchunk, int ch, int& b0, int& cnt) {
    if ((B & 1) == 0) {
        const int P = B / 2;
        b0 = 2 * (int)(((int64_t)ch * P) / nchunk);
        cnt = 2 * (int)(((int64_t)(ch + 1) * P) / nchunk) - b0;
    } else {
        b0 = (int)(((int64_t)ch * B) / nchunk);
        cnt = (int)(((int64_t)(ch + 1) * B) / nchunk) - b0;
    }
}

// Long rows: one CTA per row; thread t sums entries k = t / B, t / B + T / B,
// ... for instance t % B, then a fixed-order reduction per instance.  Run by
// the CTAs of ell_kernel past its row tiles (one launch per map).
template <bool COH>
__device__ __forceinline__ void long_row(const DevMap& M, int B, const double* __restrict__ in, const Epi& e,
                                         const int* __restrict__ mask, double* __restrict__ partial,
                                         int partial_base, int lr) {
    __shared__ double shl[kThreads];
    const int lanes = blockDim.x / B;
    const int b = threadIdx.x % B;
    const int l = threadIdx.x / B;
    const int r = M.long_rows[lr];
    const int k0 = M.long_ptr[lr], k1 = M.long_ptr[lr + 1];
    double s = 0.0;
    if (threadIdx.x < lanes * B)
        for (int k = k0 + l; k < k1; k += lanes) {
            const double* g = in + (int64_t)M.long_col[k] * B + b;
            s += M.long_val[k] * (COH ? __ldcg(g) : *g);
        }
    shl[threadIdx.x] = s;
    __syncthreads();
    double acc = 0.0;
    if (threadIdx.x < B) {
        double t = 0.0;
        for (int q = 0; q < lanes; q++) t += shl[threadIdx.x + q * B];
        if (!(mask && !mask[threadIdx.x])) acc = epilogue<false, COH>(e, r, B, threadIdx.x, t);
    }
    __syncthreads();
    if (partial) block_partial(threadIdx.x < B ? acc : 0.0, B, partial, (int64_t)partial_base + lr);
    if (COH) __syncthreads();  // the shared partials are reused by the CTA's next unit
}

// One row tile of an ELL bucket of width code wv (= 2 width + (B even)).
template <int CH, bool STREAM, bool PK, bool COH>
__device__ __forceinline__ void ell_tile(int wv, const DevMap& M, int bi, int64_t t0, int64_t nt, int B, int b0,
                                         int cnt, unsigned act, const double* __restrict__ in, const Epi& e,
                                         const double* sbook, double (&dot)[CH]) {
#define V2G_ELL(W, V) ell_rows<W, V, CH, STREAM, PK, COH>(M, bi, t0, nt, B, b0, cnt, act, in, e, sbook, dot)
    switch (wv) {
        case 2: V2G_ELL(1, false); break;
        case 3: V2G_ELL(1, true); break;
        case 4: V2G_ELL(2, false); break;
        case 5: V2G_ELL(2, true); break;
        case 8: V2G_ELL(4, false); break;
        case 9: V2G_ELL(4, true); break;
        case 16: V2G_ELL(8, false); break;
        case 17: V2G_ELL(8, true); break;
        case 32: V2G_ELL(16, false); break;
        case 33: V2G_ELL(16, true); break;
        case 64: V2G_ELL(32, false); break;
        default: V2G_ELL(32, true); break;
    }
#undef V2G_ELL
}

// Work unit `blk` of one map application: a row tile of an ELL bucket times
// an instance chunk (per-instance partial sums of the optional dot into
// partial[tile * B + b]), or, past the tiles, one long row (its partial at
// slot ntiles + row).  ell_kernel runs one unit per CTA; the persistent CG
// kernel walks the units of a map with its whole grid (COH loads).
template <int CH, bool STREAM, bool COH>
__device__ __forceinline__ void ell_unit(const DevMap& M, const Blocks& bl, int B, const double* __restrict__ in,
                                         const Epi& e, const int* mask, double* __restrict__ partial,
                                         const double* sbook, int blk) {
    const int ntiles = bl.start[M.nb];
    if (blk >= ntiles * bl.nchunk) {
        long_row<COH>(M, B, in, e, mask, partial, ntiles, blk - ntiles * bl.nchunk);
        return;
    }
    const int tile = blk / bl.nchunk;
    const int ch = blk % bl.nchunk;
    int bi = 0;
    while (bi + 1 < M.nb && tile >= bl.start[bi + 1]) bi++;
    int b0, cnt;
    chunk_range(B, bl.nchunk, ch, b0, cnt);
    unsigned act = 0;
    for (int j = 0; j < cnt; j++)
        if (!mask || mask[b0 + j]) act |= 1u << j;
    double dot[CH];
#pragma unroll
    for (int j = 0; j < CH; j++) dot[j] = 0.0;
    if (act) {
        const int64_t t0 = tile - bl.start[bi], nt = bl.start[bi + 1] - bl.start[bi];
        const int wv = M.width[bi] * 2 + ((B & 1) == 0 ? 1 : 0);
        if (M.book)
            ell_tile<CH, STREAM, true, COH>(wv, M, bi, t0, nt, B, b0, cnt, act, in, e, sbook, dot);
        else
            ell_tile<CH, STREAM, false, COH>(wv, M, bi, t0, nt, B, b0, cnt, act, in, e, sbook, dot);
    }
    if (!partial) return;
    // per-instance block sums in a fixed order: warp shuffles, then warps
    __shared__ double sh[kThreads / 32][CH];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < CH; j++) {
        double v = dot[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[warp][j] = v;
    }
    __syncthreads();
    if ((int)threadIdx.x < cnt) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; w++) t += sh[w][threadIdx.x];
        partial[(int64_t)tile * B + b0 + threadIdx.x] = t;
    }
    if (COH) __syncthreads();  // sh is reused by the CTA's next unit
}

template <int CH, bool STREAM>
__global__ void __launch_bounds__(kThreads) ell_kernel(DevMap M, Blocks bl, int B, const double* __restrict__ in,
                                                       Epi e, const int* __restrict__ mask,
                                                       double* __restrict__ partial) {
    // the coefficient book of a packed table, in shared memory
    __shared__ double sbook[kBookSize];
    if (M.book) {
        if (threadIdx.x < kBookSize) sbook[threadIdx.x] = M.book[threadIdx.x];
        __syncthreads();
    }
    ell_unit<CH, STREAM, false>(M, bl, B, in, e, mask, partial, sbook, blockIdx.x);
}

// Stage 1: block g reduces a contiguous chunk of elements for every instance;
// thread t handles instance t % B on element rows t / B, t / B + T/B, ...
__global__ void reduce_stage1(int mode, int64_t n, int B, const double* __restrict__ u, const double* __restrict__ v,
                              const double* __restrict__ w, const double* __restrict__ row,
                              double* __restrict__ partial) {
    const int rows_per_pass = blockDim.x / B;
    const int lanes = rows_per_pass * B;
    const int b = threadIdx.x % B;
    const int rsub = threadIdx.x / B;
    double acc = 0.0;
    if (threadIdx.x < lanes) {
        const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
        const int64_t e0 = blockIdx.x * chunk;
        const int64_t e1 = (e0 + chunk < n) ? e0 + chunk : n;
        for (int64_t e = e0 + rsub; e < e1; e += rows_per_pass) {
            const int64_t i = e * B + b;
            double term;
            switch (mode) {
                case RED_DOT: term = u[i] * v[i]; break;
                case RED_ED: {
                    double d = (u[i] + v[i]) - w[i];
                    term = d * d;
                    break;
                }
                case RED_EP: {
                    double d = u[i] - row[e];
                    term = d * d;
                    break;
                }
                default: term = u[i] * row[e]; break;
            }
            acc += term;
        }
    }
    const double s = cta_instance_sum(acc, B);
    if ((int)threadIdx.x < B) partial[(int64_t)blockIdx.x * B + threadIdx.x] = s;
}

// Stage 2: one block per instance sums its nblk partials with a fixed tree
// (deterministic), instead of one thread walking a long dependent chain.
__global__ void reduce_stage2(int nblk, int B, const double* __restrict__ partial, double* __restrict__ out) {
    __shared__ double sh[kThreads];
    const int b = blockIdx.x;
    double s = 0.0;
    for (int k = threadIdx.x; k < nblk; k += blockDim.x) s += partial[(int64_t)k * B + b];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[b] = sh[0];
}

// out[e * B + b] = row ? row[e] : 0 for instances with mask[b] set
__global__ void set_rows_kernel(int64_t n, int B, const double* __restrict__ row, double* __restrict__ out,
                                const int* __restrict__ mask) {
    const int64_t total = n * B;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t % B);
        if (mask && !mask[b]) continue;
        out[t] = row ? row[t / B] : 0.0;
    }
}

__global__ void c_minus_z_kernel(int64_t n, int B, const double* __restrict__ c, double* __restrict__ z,
                                 const int* __restrict__ mask) {
    const int64_t total = n * B;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t % B);
        if (mask && !mask[b]) continue;
        z[t] = -z[t] + c[t];
    }
}

__global__ void cg_extrapolate_kernel(int64_t n, int B, double* __restrict__ y, double* __restrict__ yprev,
                                      const int* __restrict__ mode) {
    const int64_t total = n * B;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int m = mode[(int)(t % B)];
        if (m == 0) continue;
        const double v = y[t];
        if (m == 2) y[t] = v + (v - yprev[t]);
        yprev[t] = v;
    }
}

// ---- Anderson acceleration (kernels.cuh) ----

__global__ void aa_save_kernel(int64_t nx, int B, const double* __restrict__ x, const double* __restrict__ z,
                               double* __restrict__ w, const int* __restrict__ mode) {
    const int64_t half = nx * B, total = 2 * half;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        if (!mode[(int)(t % B)]) continue;
        w[t] = (t < half) ? x[t] : z[t - half];
    }
}

// Rows e of the state are walked with the chunk mapping of the reducing
// kernels, so each thread keeps one instance and its 2 m dot products come
// out in a fixed order.
template <int MAXM>
__global__ void __launch_bounds__(kThreads) aa_update_kernel(
    int64_t nx, int B, int m, const double* __restrict__ x, const double* __restrict__ z,
    const double* __restrict__ w, double* __restrict__ fprev, double* __restrict__ gprev, double* __restrict__ dF,
    double* __restrict__ dG, const int* __restrict__ mode, const int* __restrict__ slot,
    double* __restrict__ partial) {
    const int64_t nrows = 2 * nx, half = nx * B;
    const size_t col = (size_t)nrows * B;
    const Chunk ch = chunk_of(nrows, B);
    // acc[2 j] = dF_slot.dF_j, acc[2 j + 1] = dF_j.f; f.f in ff (one spare
    // entry keeps every unrolled index of the output loop in bounds)
    double acc[2 * MAXM + 1];
#pragma unroll
    for (int k = 0; k < 2 * MAXM + 1; k++) acc[k] = 0.0;
    double ff = 0.0;
    if (ch.live) {
        const int b = ch.b;
        const int md = mode[b];
        const int s = slot[b];
        if (md) {
            for (int64_t e = ch.first; e < ch.nrows; e += ch.stride) {
                const int64_t t = e * B + b;
                const double g = (e < nx) ? x[t] : z[t - half];
                const double f = g - w[t];
                if (md == 2) {
                    const double df = f - fprev[t];
                    dF[(size_t)s * col + t] = df;
                    dG[(size_t)s * col + t] = g - gprev[t];
#pragma unroll
                    for (int j = 0; j < MAXM; j++) {
                        if (j < m) {
                            const double dj = (j == s) ? df : dF[(size_t)j * col + t];
                            acc[2 * j] += df * dj;
                            acc[2 * j + 1] += dj * f;
                        }
                    }
                }
                ff += f * f;
                fprev[t] = f;
                gprev[t] = g;
            }
        }
    }
    // partial[(k * gridDim.x + block) * B + b] for k <= 2 m
#pragma unroll
    for (int k = 0; k < 2 * MAXM + 1; k++) {
        if (k <= 2 * m) {
            const double sum = cta_instance_sum((k == 2 * m) ? ff : acc[k], B);
            if ((int)threadIdx.x < B) partial[((int64_t)k * gridDim.x + blockIdx.x) * B + threadIdx.x] = sum;
        }
    }
}

// out[k * B + b] = sum over blocks of partial[(k * nblk + block) * B + b], one
// CTA per (k, b), fixed tree order
__global__ void reduce_stage2_multi(int nblk, int B, const double* __restrict__ partial, double* __restrict__ out) {
    __shared__ double sh[kThreads];
    const int k = blockIdx.x / B, b = blockIdx.x % B;
    const double* p = partial + (int64_t)k * nblk * B;
    double s = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) s += p[(int64_t)i * B + b];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

template <int MAXM>
__global__ void aa_mix_kernel(int64_t nx, int B, int m, double* __restrict__ x, double* __restrict__ z,
                              const double* __restrict__ dG, const double* __restrict__ gamma,
                              const int* __restrict__ mix) {
    const int64_t half = nx * B, total = 2 * half;
    const size_t col = (size_t)total;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t % B);
        if (!mix[b]) continue;
        double v = (t < half) ? x[t] : z[t - half];
#pragma unroll
        for (int j = 0; j < MAXM; j++) {
            if (j < m) {
                const double gj = gamma[b * m + j];
                if (gj != 0.0) v -= gj * dG[(size_t)j * col + t];
            }
        }
        if (t < half)
            x[t] = v;
        else
            z[t - half] = v;
    }
}

__global__ void cg_init_kernel(int64_t n, int B, const double* __restrict__ rhs, const double* __restrict__ Ap,
                               double* __restrict__ r, double* __restrict__ p, const CgScalars* __restrict__ cs) {
    const int64_t total = n * B;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t % B);
        if (!cs[b].active) continue;
        const double v = rhs[t] - Ap[t];
        r[t] = v;
        p[t] = v;
    }
}

__global__ void cg_set_rr_kernel(int B, CgScalars* cs, const double* rr, int* n_active) {
    int cnt = 0;
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        if (cs[b].active) {
            cs[b].rr = rr[b];
            cs[b].rrmin = rr[b];
            cnt++;
        }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if (threadIdx.x == 0) *n_active = cnt;
}

__global__ void cg_alpha_kernel(int B, CgScalars* cs, const double* pap) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B || !cs[b].active) return;
    cs[b].pap = pap[b];
    if (!(pap[b] > 0.0)) {
        // p has no component outside the null space of A^T (or r = 0): no step
        cs[b].alpha = 0.0;
        cs[b].active = 0;
        cs[b].stalled = 1;
        return;
    }
    cs[b].alpha = cs[b].rr / pap[b];
}

// y += alpha p ; r -= alpha Ap ; partial[., b] of r.r (cg_solver.cc:159-165)
__global__ void cg_update_yr_kernel(int64_t n, int B, double* __restrict__ y, double* __restrict__ r,
                                    const double* __restrict__ p, const double* __restrict__ Ap,
                                    const CgScalars* __restrict__ cs, double* __restrict__ partial) {
    const Chunk ch = chunk_of(n, B);
    double acc = 0.0;
    if (ch.live) {
        const int b = ch.b;
        const bool act = cs[b].active;
        const double a = cs[b].alpha;
        for (int64_t e = ch.first; e < ch.nrows; e += ch.stride) {
            const int64_t t = e * B + b;
            double rv = r[t];
            if (act) {
                y[t] += a * p[t];
                rv += -a * Ap[t];
                r[t] = rv;
            }
            acc += rv * rv;
        }
    }
    block_partial(acc, B, partial, blockIdx.x);
}

// y += alpha p ; r -= alpha Ap with alpha = r.r / p.Ap computed by every
// thread from the instance's scalars (no separate alpha launch; p.Ap <= 0
// takes no step and the beta kernel stops the instance); partial[., b] of
// r.r.  Block 0 clears the active-instance counter that the beta kernel
// fills.
__global__ void cg_step_yr_kernel(int64_t n, int B, double* __restrict__ y, double* __restrict__ r,
                                  const double* __restrict__ p, const double* __restrict__ Ap,
                                  const CgScalars* __restrict__ cs, const double* __restrict__ pap,
                                  double* __restrict__ partial, int* __restrict__ n_active) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_active = 0;
    const Chunk ch = chunk_of(n, B);
    double acc = 0.0;
    if (ch.live) {
        const int b = ch.b;
        const double pp = pap[b];
        const bool act = cs[b].active && pp > 0.0;
        const double a = act ? cs[b].rr / pp : 0.0;
        for (int64_t e = ch.first; e < ch.nrows; e += ch.stride) {
            const int64_t t = e * B + b;
            double rv = r[t];
            if (act) {
                y[t] += a * p[t];
                rv += -a * Ap[t];
                r[t] = rv;
            }
            acc += rv * rv;
        }
    }
    block_partial(acc, B, partial, blockIdx.x);
}

// The scalars of cg_solver.cc:159-177 after a step with p.Ap = pap and the new
// r.r = rn: alpha, the ||r|| < tol test, beta and the iteration count, the
// stops on p.Ap <= 0 and on residual growth (kCgGrowth).
__device__ __forceinline__ void cg_scalar_step(CgScalars& c, double pap, double rn) {
    c.do_p = 0;
    if (!c.active) return;
    c.pap = pap;
    if (!(c.pap > 0.0)) {
        // p has no component outside the null space of A^T (or r = 0): no step
        c.alpha = 0.0;
        c.active = 0;
        c.stalled = 1;
        return;
    }
    c.alpha = c.rr / c.pap;
    c.rrnew = rn;
    if (!(sqrt(rn) < c.tol)) {
        if (rn > kCgGrowth * c.rrmin) {
            // diverging on the null space of A^T: keep the current y (kernels.cuh)
            c.active = 0;
            c.stalled = 1;
        } else {
            c.beta = rn / c.rr;
            c.rr = rn;
            c.rrmin = fmin(c.rrmin, rn);
            c.do_p = 1;
            c.iter += 1;
            if (c.iter >= c.maxiter) c.active = 0;
        }
    } else {
        c.active = 0;
    }
    if (!isfinite(rn)) c.active = 0;
}

// One block per instance: r.r from the step kernel's partials (fixed tree),
// then the scalars of cg_solver.cc:159-177: alpha, the ||r|| < tol test,
// beta and the iteration count, the stops on p.Ap <= 0 and on residual
// growth (kCgGrowth); counts the instances still iterating into n_active.
__global__ void cg_beta_reduce_kernel(int nblk, int B, const double* __restrict__ partial,
                                      const double* __restrict__ pap, CgScalars* cs, int* n_active) {
    __shared__ double sh[kThreads];
    const int b = blockIdx.x;
    double s = 0.0;
    for (int k = threadIdx.x; k < nblk; k += blockDim.x) s += partial[(int64_t)k * B + b];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    CgScalars c = cs[b];
    cg_scalar_step(c, pap[b], sh[0]);
    cs[b] = c;
    if (c.active) atomicAdd(n_active, 1);
}

// One warp: per instance, test ||r|| < tol (cg_solver.cc:167-171), else beta
// and iteration count; counts the instances still iterating.
__global__ void cg_beta_kernel(int B, CgScalars* cs, const double* rrnew, int* n_active) {
    int cnt = 0;
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        CgScalars c = cs[b];
        c.do_p = 0;
        if (c.active) {
            const double rn = rrnew[b];
            const double nrm = sqrt(rn);
            c.rrnew = rn;
            if (!(nrm < c.tol)) {
                if (rn > kCgGrowth * c.rrmin) {
                    // diverging on the null space of A^T: keep the current y (kernels.cuh)
                    c.active = 0;
                    c.stalled = 1;
                } else {
                    c.beta = rn / c.rr;
                    c.rr = rn;
                    c.rrmin = fmin(c.rrmin, rn);
                    c.do_p = 1;
                    c.iter += 1;
                    if (c.iter >= c.maxiter) c.active = 0;
                }
            } else {
                c.active = 0;
            }
            if (!isfinite(rn)) c.active = 0;
        }
        cnt += c.active;
        cs[b] = c;
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if (threadIdx.x == 0) *n_active = cnt;
}

__global__ void cg_update_p_kernel(int64_t n, int B, double* __restrict__ p, const double* __restrict__ r,
                                   const CgScalars* __restrict__ cs) {
    const int64_t total = n * B;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(t % B);
        if (!cs[b].do_p) continue;
        p[t] = cs[b].beta * p[t] + r[t];
    }
}

// ---- persistent CG for small groups ------------------------------------------
//
// One cooperative launch runs a whole CG solve (cg_solver.cc:141-177) for a
// group of at most kLoopMaxB instances: per iteration four phases over the
// whole grid (A^T p; A (A^T p) with the per-unit partials of p.Ap; y += alpha
// p and r -= alpha Ap with per-CTA partials of r.r; p = beta p + r),
// separated by grid barriers.  Every CTA sums the partials itself in the same
// fixed order, so every CTA holds the same scalars and takes the same
// decision to continue; no CTA waits for a value only another CTA computes.
// Vectors written inside the launch are read through L2 (ld.global.cg).
// Each barrier wait is bounded: a wait that runs out sets *err and the CTA
// leaves the kernel; the others then run out at their next wait.

constexpr long kGridWaitPolls = 1L << 25;  // about a second of polling (short sleeps)
constexpr int kLoopCtasPerSm = 3;

struct CgLoopArgs {
    DevMap A, AT;
    Blocks blA, blAT;  // unit layouts of the two maps for ell_unit<CH, false>
    int B;
    int64_t nc;
    double *y, *r, *p, *atp, *ap;
    CgScalars* cs;
    double* part_dot;  // (A's row tiles + long rows) x B
    double* part_rr;   // grid x B
    unsigned int* bar;
    int* err;
    int* n_active;
    int* iters;
    int cap;
};

// Arrive at barrier number target / gridDim.x of the launch and wait for all
// CTAs; false when the wait ran out.
__device__ __forceinline__ bool grid_wait(unsigned int* bar, unsigned int target, int* err) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        // release: the CTA's writes (ordered before this by the barrier above)
        // become visible to every CTA that acquires the counter
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
        unsigned int v = 0;
        for (long n = 0;; n++) {
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
            if (v >= target) break;
            if (n >= kGridWaitPolls) {
                atomicExch(err, 1);
                ok = 0;
                break;
            }
            if (n > 64) __nanosleep(32);
        }
    }
    __syncthreads();
    return ok != 0;
}

// out[b] = sum over k < n of part[k * B + b] for every instance b < B, the
// same fixed order in every CTA (strided per thread, warp shuffles, warps).
__device__ __forceinline__ void loop_reduce(const double* part, int n, int B, double* out) {
    __shared__ double wsum[kThreads / 32][kLoopMaxB];
    double acc[kLoopMaxB];
#pragma unroll
    for (int b = 0; b < kLoopMaxB; b++) acc[b] = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x)
#pragma unroll
        for (int b = 0; b < kLoopMaxB; b++)
            if (b < B) acc[b] += __ldcg(part + (int64_t)k * B + b);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int b = 0; b < kLoopMaxB; b++) {
        double v = acc[b];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) wsum[warp][b] = v;
    }
    __syncthreads();
    if ((int)threadIdx.x < B) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; w++) t += wsum[w][threadIdx.x];
        out[threadIdx.x] = t;
    }
    __syncthreads();
}

template <int CH>
__global__ void __launch_bounds__(kThreads, kLoopCtasPerSm) cg_loop_kernel(const CgLoopArgs L) {
    __shared__ double bookA[kBookSize], bookAT[kBookSize];
    __shared__ CgScalars sc[kLoopMaxB];
    __shared__ int sact[kLoopMaxB];
    __shared__ double spap[kLoopMaxB], srn[kLoopMaxB];
    __shared__ int s_any;
    const int B = L.B;
    if (threadIdx.x < kBookSize) {
        if (L.A.book) bookA[threadIdx.x] = L.A.book[threadIdx.x];
        if (L.AT.book) bookAT[threadIdx.x] = L.AT.book[threadIdx.x];
    }
    if ((int)threadIdx.x < B) {
        sc[threadIdx.x] = L.cs[threadIdx.x];
        sact[threadIdx.x] = sc[threadIdx.x].active;
    }
    __syncthreads();
    const unsigned int G = gridDim.x;
    unsigned int target = 0;
    const int unitsAT = L.blAT.start[L.AT.nb] * L.blAT.nchunk + L.AT.nlong;
    const int unitsA = L.blA.start[L.A.nb] * L.blA.nchunk + L.A.nlong;
    const int slotsA = L.blA.start[L.A.nb] + L.A.nlong;  // partial slots of the A map
    const Epi eAT{nullptr, nullptr, nullptr, nullptr, L.atp};
    const Epi eA{nullptr, nullptr, nullptr, L.p, L.ap};
    int it = 0;
    while (true) {
        if (threadIdx.x == 0) {
            int a = 0;
            for (int b = 0; b < B; b++) a |= sact[b];
            s_any = a;
        }
        __syncthreads();
        if (!s_any || it >= L.cap) break;
        // A^T p
        for (int u = blockIdx.x; u < unitsAT; u += G)
            ell_unit<CH, false, true>(L.AT, L.blAT, B, L.p, eAT, sact, nullptr, bookAT, u);
        target += G;
        if (!grid_wait(L.bar, target, L.err)) return;
        // Ap = A (A^T p) and the partials of p.Ap
        for (int u = blockIdx.x; u < unitsA; u += G)
            ell_unit<CH, false, true>(L.A, L.blA, B, L.atp, eA, sact, L.part_dot, bookA, u);
        target += G;
        if (!grid_wait(L.bar, target, L.err)) return;
        loop_reduce(L.part_dot, slotsA, B, spap);
        // y += alpha p, r -= alpha Ap (cg_solver.cc:159-165), partials of r.r
        {
            const int rpp = kThreads / B, lanes = rpp * B;
            const int b = threadIdx.x % B, rsub = threadIdx.x / B;
            double acc = 0.0;
            if ((int)threadIdx.x < lanes) {
                const double pp = spap[b];
                const bool act = sc[b].active && pp > 0.0;
                const double a = act ? sc[b].rr / pp : 0.0;
                for (int64_t e = (int64_t)blockIdx.x * rpp + rsub; e < L.nc; e += (int64_t)G * rpp) {
                    const int64_t t = e * B + b;
                    double rv = __ldcg(L.r + t);
                    if (act) {
                        L.y[t] = __ldcg(L.y + t) + a * __ldcg(L.p + t);
                        rv += -a * __ldcg(L.ap + t);
                        L.r[t] = rv;
                    }
                    acc += rv * rv;
                }
            }
            block_partial(acc, B, L.part_rr, blockIdx.x);
        }
        target += G;
        if (!grid_wait(L.bar, target, L.err)) return;
        loop_reduce(L.part_rr, (int)G, B, srn);
        if ((int)threadIdx.x < B) {
            cg_scalar_step(sc[threadIdx.x], spap[threadIdx.x], srn[threadIdx.x]);
            sact[threadIdx.x] = sc[threadIdx.x].active;
        }
        __syncthreads();
        // p = beta p + r where the instance continues (cg_solver.cc:173-176)
        for (int64_t t = (int64_t)blockIdx.x * kThreads + threadIdx.x; t < L.nc * B; t += (int64_t)G * kThreads) {
            const int b = (int)(t % B);
            if (!sc[b].do_p) continue;
            L.p[t] = sc[b].beta * __ldcg(L.p + t) + __ldcg(L.r + t);
        }
        it++;
        target += G;
        if (!grid_wait(L.bar, target, L.err)) return;
    }
    if (blockIdx.x == 0) {
        if ((int)threadIdx.x < B) L.cs[threadIdx.x] = sc[threadIdx.x];
        if (threadIdx.x == 0) {
            int cnt = 0;
            for (int b = 0; b < B; b++) cnt += sact[b];
            *L.n_active = cnt;
            *L.iters = it;
        }
    }
}

}  // namespace

static int spmv_grid(int64_t nrows, int B) {
    // enough blocks to fill the GPU; rows per block >= rows per pass
    const int64_t rows_per_pass = kThreads / B;
    int64_t g = (nrows + rows_per_pass - 1) / rows_per_pass;
    if (g > kSpmvBlocks) g = kSpmvBlocks;
    return (int)(g < 1 ? 1 : g);
}

// Row tiles (kThreads slots each) per ELL bucket, proportional to its slots,
// at most kSpmvBlocks tiles in all; every tile runs once per instance chunk.
const char* map_variant_name(int v) {
    static const char* names[kMapVariants] = {"2 instances/thread", "4 instances/thread",
                                              "4 instances/thread, streamed", "8 instances/thread, streamed"};
    return (v >= 0 && v < kMapVariants) ? names[v] : "built-in rule";
}

static int map_variant(const DevMap& M, int B) {
    if (M.variant >= 0 && M.variant < kMapVariants) return M.variant;
    return B <= 2 ? 0 : (B < 8 ? 1 : 2);
}

static Blocks map_blocks(const DevMap& M, int B) {
    Blocks bl{};
    const int var = map_variant(M, B);
    const int ch = var == 0 ? 2 : (var == 3 ? 8 : 4);
    bl.nchunk = (B + ch - 1) / ch;
    int64_t tot = 0;
    for (int i = 0; i < M.nb; i++) tot += (M.nslots[i] + kThreads - 1) / kThreads;
    const double scale = tot > kSpmvBlocks ? (double)kSpmvBlocks / (double)tot : 1.0;
    int acc = 0;
    for (int i = 0; i < M.nb; i++) {
        bl.start[i] = acc;
        int64_t g = (int64_t)(((M.nslots[i] + kThreads - 1) / kThreads) * scale);
        if (g < 1) g = 1;
        acc += (int)g;
    }
    bl.start[M.nb] = acc;
    return bl;
}

static int run_map(const DevMap& M, int B, const double* in, double* out, const double* sub, const double* coef,
                   const double* add, const int* mask, const double* dotv, double* partial, cudaStream_t s) {
    Epi e{sub, coef, add, dotv, out};
    const Blocks bl = map_blocks(M, B);
    if (M.nb > 0 || M.nlong > 0) {
        // one launch: the row tiles of the ELL buckets (times the instance
        // chunks), then one CTA per long row.  Variants: with 8 or more
        // instances the table loads and the output stores are streamed past
        // L1/L2 (cache-streaming hints), leaving the caches to the gathered
        // input (7 % faster at n = 17..20 on B200, slower for single
        // instances); the autotuner of each layout group picks per map
        const int g = bl.start[M.nb] * bl.nchunk + M.nlong;
        switch (map_variant(M, B)) {
            case 0: ell_kernel<2, false><<<g, kThreads, 0, s>>>(M, bl, B, in, e, mask, partial); break;
            case 1: ell_kernel<4, false><<<g, kThreads, 0, s>>>(M, bl, B, in, e, mask, partial); break;
            case 2: ell_kernel<4, true><<<g, kThreads, 0, s>>>(M, bl, B, in, e, mask, partial); break;
            default: ell_kernel<8, true><<<g, kThreads, 0, s>>>(M, bl, B, in, e, mask, partial); break;
        }
        g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    }
    return bl.start[M.nb] + M.nlong;  // partial blocks written
}

void launch_spmv(const DevMap& A, int B, const double* in, double* out, const double* sub, const double* coef,
                 const double* add, const int* mask, cudaStream_t s) {
    run_map(A, B, in, out, sub, coef, add, mask, nullptr, nullptr, s);
}

int64_t reduce_partial_size(int B) { return (int64_t)kSpmvBlocks * B; }

void launch_spmv_dot(const DevMap& A, int B, const double* in, double* out, const double* dotv, const int* mask,
                     double* partial, double* dot_out, cudaStream_t s) {
    const int g = run_map(A, B, in, out, nullptr, nullptr, nullptr, mask, dotv, partial, s);
    reduce_stage2<<<B, kThreads, 0, s>>>(g, B, partial, dot_out);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_reduce(ReduceMode mode, int64_t n, int B, const double* u, const double* v, const double* w,
                   const double* row, double* partial, double* out, cudaStream_t s) {
    reduce_stage1<<<kRedBlocks, kThreads, 0, s>>>((int)mode, n, B, u, v, w, row, partial);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    reduce_stage2<<<B, kThreads, 0, s>>>(kRedBlocks, B, partial, out);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_set_rows(int64_t n, int B, const double* row, double* out, const int* mask, cudaStream_t s) {
    set_rows_kernel<<<grid_for(n * B), kThreads, 0, s>>>(n, B, row, out, mask);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_aa_save(int64_t nx, int B, const double* x, const double* z, double* w, const int* mode, cudaStream_t s) {
    aa_save_kernel<<<grid_for(2 * nx * B), kThreads, 0, s>>>(nx, B, x, z, w, mode);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

int64_t aa_partial_size(int64_t nx, int B, int m) { return (int64_t)(2 * m + 1) * spmv_grid(2 * nx, B) * B; }

void launch_aa_update(int64_t nx, int B, int m, const double* x, const double* z, const double* w, double* fprev,
                      double* gprev, double* dF, double* dG, const int* mode, const int* slot, double* partial,
                      double* dots, cudaStream_t s) {
    const int g = spmv_grid(2 * nx, B);
    if (m <= 4)
        aa_update_kernel<4><<<g, kThreads, 0, s>>>(nx, B, m, x, z, w, fprev, gprev, dF, dG, mode, slot, partial);
    else if (m <= 8)
        aa_update_kernel<8><<<g, kThreads, 0, s>>>(nx, B, m, x, z, w, fprev, gprev, dF, dG, mode, slot, partial);
    else
        aa_update_kernel<kAndersonMax><<<g, kThreads, 0, s>>>(nx, B, m, x, z, w, fprev, gprev, dF, dG, mode, slot,
                                                               partial);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    reduce_stage2_multi<<<(2 * m + 1) * B, kThreads, 0, s>>>(g, B, partial, dots);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_aa_mix(int64_t nx, int B, int m, double* x, double* z, const double* dG, const double* gamma,
                   const int* mix, cudaStream_t s) {
    const int g = grid_for(2 * nx * B);
    if (m <= 4)
        aa_mix_kernel<4><<<g, kThreads, 0, s>>>(nx, B, m, x, z, dG, gamma, mix);
    else if (m <= 8)
        aa_mix_kernel<8><<<g, kThreads, 0, s>>>(nx, B, m, x, z, dG, gamma, mix);
    else
        aa_mix_kernel<kAndersonMax><<<g, kThreads, 0, s>>>(nx, B, m, x, z, dG, gamma, mix);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_cg_extrapolate(int64_t n, int B, double* y, double* yprev, const int* mode, cudaStream_t s) {
    cg_extrapolate_kernel<<<grid_for(n * B), kThreads, 0, s>>>(n, B, y, yprev, mode);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_c_minus_z(int64_t n, int B, const double* c, double* z, const int* mask, cudaStream_t s) {
    c_minus_z_kernel<<<grid_for(n * B), kThreads, 0, s>>>(n, B, c, z, mask);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

void launch_cg_init(int64_t n, int B, const double* rhs, const double* Ap, double* r, double* p, const CgScalars* cs,
                    cudaStream_t s) {
    cg_init_kernel<<<grid_for(n * B), kThreads, 0, s>>>(n, B, rhs, Ap, r, p, cs);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}
void launch_cg_set_rr(int B, CgScalars* cs, const double* rr, int* n_active, cudaStream_t s) {
    cg_set_rr_kernel<<<1, 32, 0, s>>>(B, cs, rr, n_active);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}
void launch_cg_alpha(int B, CgScalars* cs, const double* pap, cudaStream_t s) {
    cg_alpha_kernel<<<(B + 127) / 128, 128, 0, s>>>(B, cs, pap);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}
void launch_cg_update_yr(int64_t n, int B, double* y, double* r, const double* p, const double* Ap,
                         const CgScalars* cs, double* partial, double* rr_out, cudaStream_t s) {
    const int g = spmv_grid(n, B);
    cg_update_yr_kernel<<<g, kThreads, 0, s>>>(n, B, y, r, p, Ap, cs, partial);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    reduce_stage2<<<B, kThreads, 0, s>>>(g, B, partial, rr_out);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}
void launch_cg_step(int64_t n, int B, double* y, double* r, const double* p, const double* Ap, CgScalars* cs,
                    const double* pap, double* partial, int* n_active, cudaStream_t s) {
    const int g = spmv_grid(n, B);
    cg_step_yr_kernel<<<g, kThreads, 0, s>>>(n, B, y, r, p, Ap, cs, pap, partial, n_active);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    cg_beta_reduce_kernel<<<B, kThreads, 0, s>>>(g, B, partial, pap, cs, n_active);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}
void launch_cg_beta(int B, CgScalars* cs, const double* rrnew, int* n_active, cudaStream_t s) {
    cg_beta_kernel<<<1, 32, 0, s>>>(B, cs, rrnew, n_active);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}
// Condition of the device-side CG loop (the body of a WHILE node in the
// group's CUDA graph): another iteration while an instance still iterates,
// and never more than `cap` iterations in all.
__global__ void cg_while_kernel(cudaGraphConditionalHandle h, const int* __restrict__ n_active, int* count,
                                int cap) {
    const int c = *count + 1;
    *count = c;
    cudaGraphSetConditional(h, (*n_active > 0 && c < cap) ? 1u : 0u);
}
void launch_cg_while(cudaGraphConditionalHandle h, const int* n_active, int* count, int cap, cudaStream_t s) {
    cg_while_kernel<<<1, 1, 0, s>>>(h, n_active, count, cap);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}
void launch_cg_update_p(int64_t n, int B, double* p, const double* r, const CgScalars* cs, cudaStream_t s) {
    cg_update_p_kernel<<<grid_for(n * B), kThreads, 0, s>>>(n, B, p, r, cs);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

int cg_loop_grid(int device) {
    static std::mutex mu;
    static std::map<int, int> grid;
    std::lock_guard<std::mutex> lk(mu);
    auto it = grid.find(device);
    if (it != grid.end()) return it->second;
    int sms = 0, coop = 0, occ1 = 0, occ2 = 0, occ4 = 0;
    int g = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) == cudaSuccess && coop &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, cg_loop_kernel<1>, kThreads, 0) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, cg_loop_kernel<2>, kThreads, 0) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ4, cg_loop_kernel<4>, kThreads, 0) == cudaSuccess) {
        // three CTAs per SM (the launch bound of every form): the phases are
        // latency-bound gathers that want the warps
        const int per_sm = std::min(kLoopCtasPerSm, std::min(occ1, std::min(occ2, occ4)));
        if (per_sm >= 1) g = sms * per_sm;
    }
    cudaGetLastError();
    grid[device] = g;
    return g;
}

bool cg_loop_fits(int64_t nc, int B) { return B >= 1 && B <= kLoopMaxB && nc * B <= kLoopMaxElems; }

cudaError_t launch_cg_loop(const DevMap& A, const DevMap& AT, int B, int64_t nc, double* y, double* r, double* p,
                           double* atp, double* ap, CgScalars* cs, double* part_dot, double* part_rr,
                           unsigned int* bar, int* err, int* n_active, int* iters, int cap, int grid,
                           cudaStream_t s) {
    CgLoopArgs L;
    // one instance per thread for a single instance (fewer registers); the
    // unit layout is the 2-instance one, which has one chunk for B <= 2
    const int ch = B == 1 ? 1 : (B <= 2 ? 2 : 4);
    L.A = A;
    L.AT = AT;
    L.A.variant = L.AT.variant = (ch <= 2 ? 0 : 1);
    L.blA = map_blocks(L.A, B);
    L.blAT = map_blocks(L.AT, B);
    L.B = B;
    L.nc = nc;
    L.y = y;
    L.r = r;
    L.p = p;
    L.atp = atp;
    L.ap = ap;
    L.cs = cs;
    L.part_dot = part_dot;
    L.part_rr = part_rr;
    L.bar = bar;
    L.err = err;
    L.n_active = n_active;
    L.iters = iters;
    L.cap = cap;
    void* args[] = {&L};
    const void* fn = ch == 1 ? (const void*)cg_loop_kernel<1>
                             : (ch == 2 ? (const void*)cg_loop_kernel<2> : (const void*)cg_loop_kernel<4>);
    const cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, 0, s);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
    return e;
}

}  // namespace v2g
