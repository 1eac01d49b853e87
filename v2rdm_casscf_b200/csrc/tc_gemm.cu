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
// One CTA computes a 128 x 64 tile of C (tcgen05.mma M = 128, N = 64) with
// its accumulator in tensor memory (64 columns).  The K dimension is walked in
// chunks of 32 through a two-stage shared-memory ring: all 128 threads load a
// chunk of A and B from global memory (FP64), split it and store the four
// TF32 tiles in the canonical K-major layout without swizzle (8-row x 16-byte
// core matrices), then one thread issues the 12 MMAs of the chunk (4 K steps
// of 8, three products each) and commits them to the stage's mbarrier, which
// releases the stage for the chunk after next.  The epilogue reads the
// accumulator with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows)
// and stores FP64.  Every wait on an mbarrier is bounded; a wait that runs out
// sets g_tc_status and the CTA still frees its tensor memory and returns.
#include <cstdint>
#include <mutex>
#include <vector>

#include "kernels.cuh"

namespace v2g {

namespace {

constexpr int kTcM = 128;        // rows of a C tile (MMA M)
constexpr int kTcN = 64;         // columns of a C tile (MMA N)
constexpr int kTcK = 32;         // K per pipeline stage
constexpr int kTcThreads = 128;  // one thread per TMEM lane / tile row
constexpr int kTileA = kTcM * kTcK * 4;            // bytes of one TF32 A tile (16 KB)
constexpr int kTileB = kTcN * kTcK * 4;            // bytes of one TF32 B tile (8 KB)
constexpr int kStage = 2 * kTileA + 2 * kTileB;    // A hi, A lo, B hi, B lo (48 KB)
constexpr int kTcSmem = 2 * kStage + 128;          // two stages + barriers and the TMEM address
constexpr long long kWaitLimit = 1ll << 26;        // polls of an mbarrier before giving up

// 0 = fine; 1 = an mbarrier wait ran out (the result of that launch is invalid)
__device__ int g_tc_status;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (row r, k) of a K-major tile with 32 K per row, in
// 8-row x 16-byte core matrices: core matrices adjacent in K are 128 B apart
// (the descriptor's leading byte offset), 8-row groups 1024 B apart (its
// stride byte offset)
__device__ __forceinline__ uint32_t kmajor_off(int r, int k) {
    return (uint32_t)((r >> 3) * 1024 + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// shared-memory matrix descriptor: start address, LBO 128 B, SBO 1024 B,
// descriptor version 1 (sm_100), no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           (1ull << 46);
}

// instruction descriptor of kind::tf32: D F32, A and B TF32, both K-major,
// N = 64, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                            ((uint32_t)(kTcM >> 4) << 24);

__device__ __forceinline__ uint32_t to_tf32(float f) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
    return r;
}

// FP64 -> (TF32 high, TF32 low) with hi + lo = float(v) to ~2^-22
__device__ __forceinline__ void split3(double v, uint32_t& hi, uint32_t& lo) {
    const float f = (float)v;
    hi = to_tf32(f);
    lo = to_tf32(f - __uint_as_float(hi));
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

// Stage chunk kc of op(A) (rows m0.., K columns kc*32..) and op(B) (K rows,
// columns n0..) into the stage at `st` as TF32 hi / lo tiles.  Each thread
// writes whole 16-byte core-matrix rows (4 K values); the 8 threads of a
// store phase cover the 8 rows of one core matrix, so the stores do not
// conflict.
__device__ __forceinline__ void stage_chunk(unsigned char* st, const double* __restrict__ A, bool transA,
                                            const double* __restrict__ Bm, bool transB,
                                            const double* __restrict__ dvec, int np, int m0, int n0, int k0) {
    unsigned char* ahi = st;
    unsigned char* alo = st + kTileA;
    unsigned char* bhi = st + 2 * kTileA;
    unsigned char* blo = st + 2 * kTileA + kTileB;
    // A: 128 rows x 8 core rows of 4 K values = 1024 pieces, 8 per thread
#pragma unroll 2
    for (int it = 0; it < (kTcM * kTcK / 4) / kTcThreads; it++) {
        const int idx = it * kTcThreads + threadIdx.x;
        const int c = (idx >> 3) & 7;              // K group of 4
        const int r = (idx & 7) + 8 * (idx >> 6);  // tile row
        const int row = m0 + r;
        uint4 h = make_uint4(0, 0, 0, 0), l = make_uint4(0, 0, 0, 0);
        if (row < np) {
            double v[4];
            const int k = k0 + 4 * c;
#pragma unroll
            for (int j = 0; j < 4; j++)
                v[j] = transA ? __ldg(A + (int64_t)(k + j) * np + row) : __ldg(A + (int64_t)row * np + k + j);
            split3(v[0], h.x, l.x);
            split3(v[1], h.y, l.y);
            split3(v[2], h.z, l.z);
            split3(v[3], h.w, l.w);
        }
        const uint32_t off = kmajor_off(r, 4 * c);
        *reinterpret_cast<uint4*>(ahi + off) = h;
        *reinterpret_cast<uint4*>(alo + off) = l;
    }
    // B^T: 64 rows (output columns) x 8 core rows = 512 pieces, 4 per thread
#pragma unroll 2
    for (int it = 0; it < (kTcN * kTcK / 4) / kTcThreads; it++) {
        const int idx = it * kTcThreads + threadIdx.x;
        const int c = (idx >> 3) & 7;
        const int r = (idx & 7) + 8 * (idx >> 6);
        const int col = n0 + r;
        const int k = k0 + 4 * c;
        double v[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            v[j] = transB ? __ldg(Bm + (int64_t)col * np + k + j) : __ldg(Bm + (int64_t)(k + j) * np + col);
            if (dvec) v[j] *= __ldg(dvec + k + j);
        }
        uint4 h, l;
        split3(v[0], h.x, l.x);
        split3(v[1], h.y, l.y);
        split3(v[2], h.z, l.z);
        split3(v[3], h.w, l.w);
        const uint32_t off = kmajor_off(r, 4 * c);
        *reinterpret_cast<uint4*>(bhi + off) = h;
        *reinterpret_cast<uint4*>(blo + off) = l;
    }
}

__global__ void __launch_bounds__(kTcThreads) tc_gemm_kernel(const BlockTask* __restrict__ tasks,
                                                             const GemmTile* __restrict__ tiles,
                                                             const double* __restrict__ A, bool transA,
                                                             const double* __restrict__ Bm, bool transB,
                                                             const double* __restrict__ dvec, double* __restrict__ C,
                                                             const int* __restrict__ bmask) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const GemmTile tl = tiles[blockIdx.x];
    if (bmask && !bmask[tl.task]) return;
    const BlockTask t = tasks[tl.task];
    const int np = t.np;
    const int m0 = tl.ti * kTcM, n0 = tl.tj * kTcN;
    const double* a = A + t.woff;
    const double* b = Bm + t.woff;
    const double* d = dvec ? dvec + t.doff : nullptr;
    double* c = C + t.woff;

    unsigned char* stage[2] = {smem, smem + kStage};
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * kStage);  // two mbarriers
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + 2 * kStage + 64);
    const uint32_t bar0 = smem_addr(&bars[0]), bar1 = smem_addr(&bars[1]);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0) {
        // 64 TMEM columns hold the 128 x 64 FP32 accumulator
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"(kTcN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    const int nk = np / kTcK;
    bool ok = true;
    for (int kc = 0; kc < nk; kc++) {
        const int s = kc & 1;
        // the MMAs of chunk kc - 2 read this stage: wait for their commit
        if (kc >= 2 && ok) ok = mbar_wait(s ? bar1 : bar0, (uint32_t)(((kc - 2) >> 1) & 1));
        if (ok) stage_chunk(stage[s], a, transA, b, transB, d, np, m0, n0, kc * kTcK);
        // generic-proxy stores become visible to the tensor cores' async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (!__syncthreads_and(ok ? 1 : 0)) {
            ok = false;
            break;
        }
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t sa = smem_addr(stage[s]);
            const uint32_t ahi = sa, alo = sa + kTileA, bhi = sa + 2 * kTileA, blo = sa + 2 * kTileA + kTileB;
#pragma unroll
            for (int ks = 0; ks < kTcK / 8; ks++) {
                const uint32_t o = ks * 256;  // two 128-byte core matrices per K step of 8
                mma_tf32(tmem, smem_desc(ahi + o), smem_desc(bhi + o), (kc > 0 || ks > 0) ? 1u : 0u);
                mma_tf32(tmem, smem_desc(ahi + o), smem_desc(blo + o), 1u);
                mma_tf32(tmem, smem_desc(alo + o), smem_desc(bhi + o), 1u);
            }
            mma_commit(s ? bar1 : bar0);
        }
    }
    // the last commit covers every MMA of the tile
    if (ok && nk > 0) {
        const int kl = nk - 1;
        ok = mbar_wait((kl & 1) ? bar1 : bar0, (uint32_t)((kl >> 1) & 1));
    }
    if (!ok && nk > 1) {
        // a wait ran out: drain the other stage's commit too (bounded), so no MMA
        // is left reading shared memory when the CTA exits
        const int kl = nk - 2;
        mbar_wait((kl & 1) ? bar1 : bar0, (uint32_t)((kl >> 1) & 1));
    }
    if (!ok && threadIdx.x == 0) atomicExch(&g_tc_status, 1);
    tc_fence_after();
    if (ok) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int h = 0; h < kTcN / 32; h++) {
            float v[32];
            tmem_ld32(taddr + h * 32, v);
            if (row < np) {
                double* out = c + (int64_t)row * np + n0 + h * 32;
#pragma unroll
                for (int j = 0; j < 32; j += 2)
                    *reinterpret_cast<double2*>(out + j) = make_double2((double)v[j], (double)v[j + 1]);
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

void launch_tc_gemm(const BlockTask* tasks, const GemmTile* tiles, int ntiles, const double* A, bool transA,
                    const double* Bm, bool transB, const double* dvec, double* C, const int* bmask, cudaStream_t s) {
    if (ntiles == 0) return;
    set_tc_smem_attr();
    tc_gemm_kernel<<<ntiles, kTcThreads, kTcSmem, s>>>(tasks, tiles, A, transA, Bm, transB, dvec, C, bmask);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
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
