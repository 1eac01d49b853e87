// Batched 3xTF32 GEMM on the fifth-generation tensor cores (tcgen05), for the
// mixed-precision projection of the large PSD blocks.
//
// C = op(A) diag(d) op(B) on the padded np x np FP64 workspaces of the block
// tasks (the same operands as gemm_kernel in eig.cu), computed to FP32
// accuracy: every FP64 input is rounded to FP32 and split into a TF32 high
// part and a TF32 low part (the residual), and the product is
// A_hi B_hi + A_hi B_lo + A_lo B_hi accumulated in FP32 (the "3xTF32" split;
// the dropped A_lo B_lo term and the splits' rounding are ~2^-22 relative).
//
// Two kernels per product:
//   * tc_split_kernel writes each operand once as TF32 (hi, lo) tiles in the
//     exact byte order the MMA reads from shared memory: K-major, no swizzle,
//     8-row x 16-byte core matrices, one 128-row x 32-K tile (16 KB) per (row
//     block, K chunk), hi then lo.  The transposes of op() and the diagonal
//     scaling happen here (coalesced FP64 reads through shared memory).
//   * tc_gemm_kernel computes a 128 x 128 tile of C with its accumulator in
//     tensor memory (128 columns).  A three-stage shared-memory ring is fed by
//     one producer thread with bulk copies (cp.async.bulk, 32 KB per operand
//     per stage, completion counted on the stage's mbarrier); one thread
//     issues the chunk's 12 tcgen05.mma (4 K steps of 8, three products) and
//     commits them to the stage's "empty" mbarrier; the four warps read the
//     accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile
//     rows) and store FP64.
// Every mbarrier wait is bounded; a wait that runs out sets g_tc_status, and
// the CTA then drains what it issued (bounded) and frees its tensor memory.
#include <cstdint>
#include <mutex>
#include <vector>

#include "kernels.cuh"

namespace v2g {

namespace {

constexpr int kTcM = 128;                        // rows of a C tile (MMA M)
constexpr int kTcN = 128;                        // columns of a C tile (MMA N)
constexpr int kTcK = 32;                         // K per pipeline stage
constexpr int kTcThreads = 128;                  // four warps: TMEM lanes 0..127
constexpr int kStages = 3;
constexpr int kTile = kTcM * kTcK * 4;           // one TF32 tile, 128 rows x 32 K (16 KB)
constexpr int kOperand = 2 * kTile;              // hi and lo of one operand (32 KB)
constexpr int kStage = 2 * kOperand;             // A and B (64 KB)
constexpr int kTcSmem = kStages * kStage + 256;  // + barriers and the TMEM address
constexpr long long kWaitLimit = 1ll << 26;      // polls of an mbarrier before giving up

// 0 = fine; 1 = an mbarrier wait ran out (the result of that launch is invalid)
__device__ int g_tc_status;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// element offset (4-byte units) of (row r, k) inside a 128 x 32 K-major tile:
// core matrices adjacent in K are 128 B apart (the descriptor's leading byte
// offset), 8-row groups 1024 B apart (its stride byte offset)
__device__ __forceinline__ int core_off(int r, int k) { return (r >> 3) * 256 + (k >> 2) * 32 + (r & 7) * 4 + (k & 3); }

// shared-memory matrix descriptor: start address, LBO 128 B, SBO 1024 B,
// descriptor version 1 (sm_100), no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           (1ull << 46);
}

// instruction descriptor of kind::tf32: D F32, A and B TF32, both K-major,
// N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                            ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ uint32_t to_tf32(float f) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
    return r;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long i = 0; i < kWaitLimit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// bulk copy global -> shared, completion counted on bar (16-byte aligned, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// 32 consecutive accumulator columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// One CTA per (task, 128-row block): the operand X(r, k) = rowmajor ?
// S[r * np + k] : S[k * np + r] (times d[k] when given), rows past np zero,
// written as TF32 hi / lo tiles: out + task.toff + (rb * nk + kc) * 2 * 4096,
// hi then lo, each in core-matrix order.
__global__ void __launch_bounds__(256) tc_split_kernel(const BlockTask* __restrict__ tasks,
                                                       const TcSplit* __restrict__ units,
                                                       const double* __restrict__ S, bool rowmajor,
                                                       const double* __restrict__ dvec, uint32_t* __restrict__ out,
                                                       const int* __restrict__ bmask) {
    __shared__ double tile[kTcM][kTcK + 1];
    const TcSplit u = units[blockIdx.x];
    if (bmask && !bmask[u.task]) return;
    const BlockTask t = tasks[u.task];
    const int np = t.np, nk = np / kTcK;
    const double* src = S + t.woff;
    const double* d = dvec ? dvec + t.doff : nullptr;
    // one K chunk per CTA on a 2-D grid (blockIdx.y); all chunks on a 1-D grid
    const int kc0 = gridDim.y > 1 ? (int)blockIdx.y : 0;
    const int kc1 = gridDim.y > 1 ? (int)blockIdx.y + 1 : nk;
    for (int kc = kc0; kc < kc1 && kc < nk; kc++) {
        const int k0 = kc * kTcK;
        if (rowmajor) {
            // a warp reads 32 consecutive K of one row
            for (int it = threadIdx.x; it < kTcM * kTcK; it += 256) {
                const int r = it / kTcK, k = it % kTcK;
                const int row = u.rb * kTcM + r;
                double v = 0.0;
                if (row < np) v = src[(int64_t)row * np + k0 + k];
                if (d) v *= d[k0 + k];
                tile[r][k] = v;
            }
        } else {
            // a warp reads 32 consecutive rows of one K
            for (int it = threadIdx.x; it < kTcM * kTcK; it += 256) {
                const int r = it % kTcM, k = it / kTcM;
                const int row = u.rb * kTcM + r;
                double v = 0.0;
                if (row < np) v = src[(int64_t)(k0 + k) * np + row];
                if (d) v *= d[k0 + k];
                tile[r][k] = v;
            }
        }
        __syncthreads();
        uint32_t* hi = out + t.toff + ((int64_t)u.rb * nk + kc) * 2 * (kTile / 4);
        uint32_t* lo = hi + kTile / 4;
        for (int o = threadIdx.x; o < kTcM * kTcK; o += 256) {
            // o = core_off(r, k)
            const int rg = o >> 8, k4 = (o >> 5) & 7, r8 = (o >> 2) & 7, kk = o & 3;
            const int r = rg * 8 + r8, k = k4 * 4 + kk;
            const float f = (float)tile[r][k];
            const uint32_t h = to_tf32(f);
            hi[o] = h;
            lo[o] = to_tf32(f - __uint_as_float(h));
        }
        __syncthreads();
    }
}

// C tile (ti, tj) of 128 x 128 from the split operands: A rows 128 ti.., B
// rows (the output columns) 128 tj..; rows and columns past np are not written.
__global__ void __launch_bounds__(kTcThreads) tc_gemm_kernel(const BlockTask* __restrict__ tasks,
                                                             const GemmTile* __restrict__ tiles,
                                                             const uint32_t* __restrict__ wa,
                                                             const uint32_t* __restrict__ wb, double* __restrict__ C,
                                                             const int* __restrict__ bmask) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const GemmTile tl = tiles[blockIdx.x];
    if (bmask && !bmask[tl.task]) return;
    const BlockTask t = tasks[tl.task];
    const int np = t.np, nk = np / kTcK;
    const int m0 = tl.ti * kTcM, n0 = tl.tj * kTcN;
    const unsigned char* ga = reinterpret_cast<const unsigned char*>(wa + t.toff) + (int64_t)tl.ti * nk * kOperand;
    const unsigned char* gb = reinterpret_cast<const unsigned char*>(wb + t.toff) + (int64_t)tl.tj * nk * kOperand;
    double* c = C + t.woff;

    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * kStage);  // full[3], empty[3], done
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kStages * kStage + 128);
    const uint32_t sbase = smem_addr(smem);
    auto full = [&](int s) { return smem_addr(&bars[s]); };
    auto empty = [&](int s) { return smem_addr(&bars[kStages + s]); };
    const uint32_t done = smem_addr(&bars[2 * kStages]);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0) {
        // 128 TMEM columns hold the 128 x 128 FP32 accumulator
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(kTcN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    // producer (thread 0) and MMA issuer (thread 32); their outcome reaches
    // every thread through the done barrier and the block vote below
    int role_ok = 1;
    if (threadIdx.x == 0) {
        for (int kc = 0; kc < nk; kc++) {
            const int s = kc % kStages, u = kc / kStages;
            if (u > 0 && !mbar_wait(empty(s), (uint32_t)((u - 1) & 1))) {
                role_ok = 0;
                break;
            }
            mbar_expect_tx(full(s), (uint32_t)kStage);
            bulk_g2s(sbase + s * kStage, ga + (int64_t)kc * kOperand, kOperand, full(s));
            bulk_g2s(sbase + s * kStage + kOperand, gb + (int64_t)kc * kOperand, kOperand, full(s));
        }
    } else if (threadIdx.x == 32) {
        int kc = 0;
        for (; kc < nk; kc++) {
            const int s = kc % kStages, u = kc / kStages;
            if (!mbar_wait(full(s), (uint32_t)(u & 1))) {
                role_ok = 0;
                break;
            }
            tc_fence_after();
            const uint32_t st = sbase + s * kStage;
            const uint32_t ahi = st, alo = st + kTile, bhi = st + kOperand, blo = st + kOperand + kTile;
#pragma unroll
            for (int ks = 0; ks < kTcK / 8; ks++) {
                const uint32_t o = ks * 256;  // two 128-byte core matrices per K step of 8
                mma_tf32(tmem, smem_desc(ahi + o), smem_desc(bhi + o), (kc > 0 || ks > 0) ? 1u : 0u);
                mma_tf32(tmem, smem_desc(ahi + o), smem_desc(blo + o), 1u);
                mma_tf32(tmem, smem_desc(alo + o), smem_desc(bhi + o), 1u);
            }
            mma_commit(empty(s));
        }
        // the last commit covers every MMA issued; a stopped issuer still
        // signals done once its issued MMAs have completed
        mma_commit(done);
    }
    // everyone: the accumulator is complete (or the issuer stopped)
    bool ok = mbar_wait(done, 0u);
    ok = __syncthreads_and(ok && role_ok) != 0;
    if (!ok) {
        if (threadIdx.x == 0) atomicExch(&g_tc_status, 1);
        // bulk copies still in flight complete on the full barriers: wait
        // (bounded) for the ones the producer issued before freeing the CTA
        if (threadIdx.x == 0)
            for (int s = 0; s < kStages && s < nk; s++) {
                const int last = ((nk - 1 - s) / kStages) * kStages + s;  // last chunk on stage s
                mbar_wait(full(s), (uint32_t)((last / kStages) & 1));
            }
    }
    tc_fence_after();
    if (ok) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int h = 0; h < kTcN / 32; h++) {
            float v[32];
            tmem_ld32(taddr + h * 32, v);
            const int col0 = n0 + h * 32;
            if (row < np && col0 < np) {
                double* o = c + (int64_t)row * np + col0;
#pragma unroll
                for (int j = 0; j < 32; j += 2) *reinterpret_cast<double2*>(o + j) = make_double2((double)v[j], (double)v[j + 1]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcN) : "memory");
}

void set_tc_smem_attr() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return;
    static std::mutex mu;
    static std::vector<char> done;
    std::lock_guard<std::mutex> lk(mu);
    if ((size_t)dev < done.size() && done[dev]) return;
    if (cudaFuncSetAttribute(tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem) != cudaSuccess)
        return;
    if ((size_t)dev >= done.size()) done.resize(dev + 1, 0);
    done[dev] = 1;
}

}  // namespace

int64_t tc_split_words(int np) { return (int64_t)((np + kTcM - 1) / kTcM) * kTcM * np * 2; }

void launch_tc_gemm(const TcPlan& p, bool sym, const double* A, bool transA, const double* Bm, bool transB,
                    const double* dvec, double* C, const int* bmask, cudaStream_t s) {
    const int ntiles = sym ? p.n_sym : p.n_full;
    if (ntiles == 0 || p.nsplit == 0) return;
    set_tc_smem_attr();
    // op(A)(m, k): row-major when not transposed; op(B)^T(n, k) = op(B)(k, n):
    // row-major storage of B^T when B is transposed
    const dim3 sg(p.nsplit, p.max_nk > 0 ? p.max_nk : 1);
    tc_split_kernel<<<sg, 256, 0, s>>>(p.tasks, p.split, A, !transA, nullptr, p.wa, bmask);
    tc_split_kernel<<<sg, 256, 0, s>>>(p.tasks, p.split, Bm, transB, dvec, p.wb, bmask);
    tc_gemm_kernel<<<ntiles, kTcThreads, kTcSmem, s>>>(p.tasks, sym ? p.tiles_sym : p.tiles_full, p.wa, p.wb, C,
                                                       bmask);
    g_kernel_launches.fetch_add(3, std::memory_order_relaxed);
}

int tc_gemm_status(bool reset) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_tc_status, sizeof(int)) != cudaSuccess) return -1;
    if (reset && v) {
        const int z = 0;
        cudaMemcpyToSymbol(g_tc_status, &z, sizeof(int));
    }
    return v;
}

void tc_gemm_status_async(int* host, cudaStream_t s) {
    cudaMemcpyFromSymbolAsync(host, g_tc_status, sizeof(int), 0, cudaMemcpyDeviceToHost, s);
}

}  // namespace v2g
