// Device kernels of the boundary-point SDP solver (declarations of the
// host-side launchers).
//
// Vector layout: a group of B instances that share one constraint layout is
// stored instance-interleaved, element e of instance b at [e * B + b].  A
// gather through the shared index tables then reads B contiguous doubles per
// table entry, and the table itself is read once for all B instances.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

namespace v2g {

// Number of kernels the launchers below have issued (all threads, all devices).
extern std::atomic<long> g_kernel_launches;

// A sparse map (A or A^T) in bucketed ELL form: rows are grouped by length
// into buckets of fixed width (1, 2, 4, 8, 16, 32 slots, padding marked by
// col = -1), stored slot-major so that a warp reads its table entries
// coalesced and needs no row-pointer lookup; rows longer than 32 entries
// (traces, contractions) are kept as CSR and reduced by a whole CTA each.
constexpr int kMaxBuckets = 6;
struct DevMap {
    int64_t nrows = 0;  // output length
    int nb = 0;
    int width[kMaxBuckets] = {};
    int64_t nslots[kMaxBuckets] = {};
    int64_t row_off[kMaxBuckets] = {};  // into rows
    int64_t ent_off[kMaxBuckets] = {};  // into cols / vals
    const int32_t* rows = nullptr;
    // Entry words.  Unpacked: the column, with vals[] the coefficient.  Packed
    // (book != nullptr, vals == nullptr): column | code << kCodeShift, the
    // coefficient book[code] (the maps have a handful of distinct
    // coefficients: +-1, +-1/2, -1/sqrt 2, a few small integers), 4 bytes per
    // entry instead of 12.  Padding slots are -1 in both forms.
    const int32_t* cols = nullptr;
    const double* vals = nullptr;
    const double* book = nullptr;
    int nlong = 0;
    const int32_t* long_rows = nullptr;
    const int32_t* long_ptr = nullptr;
    const int32_t* long_col = nullptr;
    const double* long_val = nullptr;
    // kernel variant chosen by the autotuner for one instance count (-1: the
    // built-in rule); see kMapVariants
    int variant = -1;
};
constexpr int kCodeShift = 27;                 // packed entry: 27 column bits, 4 code bits
constexpr int kBookSize = 1 << (31 - kCodeShift);  // 16 coefficients at most
// Map kernel variants: instances per thread (2, 4, 8) and whether the table
// loads and output stores bypass the caches (streaming hints).
constexpr int kMapVariants = 4;  // 0: 2 plain, 1: 4 plain, 2: 4 streamed, 3: 8 streamed
const char* map_variant_name(int v);

// out[r,b] = coef[b] * (sum_k val[k] in[col[k],b] - sub[r]) + add[r,b]
// (each of sub, coef, add optional); instances with mask[b] == 0 are skipped.
void launch_spmv(const DevMap& A, int B, const double* in, double* out, const double* sub, const double* coef,
                 const double* add, const int* mask, cudaStream_t s);

// out = A in, and dot_out[b] = sum_r dotv[r,b] out[r,b] (deterministic).
void launch_spmv_dot(const DevMap& A, int B, const double* in, double* out, const double* dotv, const int* mask,
                     double* partial, double* dot_out, cudaStream_t s);

// Per-instance reductions over interleaved vectors of n elements.
enum ReduceMode {
    RED_DOT = 0,      // sum u*v
    RED_ED = 1,       // sum ((u + v) - w)^2       (dual error, v2rdm_solver.cc:1829-1832)
    RED_EP = 2,       // sum (u - row[e])^2        (primal error, v2rdm_solver.cc:1835-1837)
    RED_DOT_ROW = 3,  // sum u * row[e]            (b . y)
};
// Writes one value per instance to out[0..B).  partial must hold
// reduce_partial_size(B) doubles.  Deterministic summation order.
void launch_reduce(ReduceMode mode, int64_t n, int B, const double* u, const double* v, const double* w,
                   const double* row, double* partial, double* out, cudaStream_t s);
int64_t reduce_partial_size(int B);

// z = c - z for active instances (v2rdm_solver.cc:1789-1790)
void launch_c_minus_z(int64_t n, int B, const double* c, double* z, const int* mask, cudaStream_t s);
// out[e * B + b] = row[e] (or 0 when row is null) for the instances with mask[b] set
void launch_set_rows(int64_t n, int B, const double* row, double* out, const int* mask, cudaStream_t s);

// CG pieces (cg_solver.cc:125-177), per instance with cg_active masks.
struct CgScalars {
    double rr, pap, alpha, beta, rrnew, tol;
    double rrmin;  // smallest r.r of this solve
    int active;    // still iterating
    int iter;      // iter_ of the reference
    int do_p;      // p update pending this iteration
    int maxiter;
    int stalled;   // stopped because r.r grew past kCgGrowth * rrmin
};
// A A^T is singular (the constraint rows are dependent), so a right-hand side
// with a component in the null space of A^T above the CG tolerance (rounding
// in A(c - z) and A x) cannot be met: r stalls at that component and CG then
// diverges, with y growing without bound.  In the converging BPSDP runs
// measured, r.r never rose more than ~30x above its running minimum (|r| 5.3x
// in 4,252 CG solves); a rise past this factor stops the instance's CG with
// the current y instead.
constexpr double kCgGrowth = 1e4;
// r = rhs - Ap ; p = r
void launch_cg_init(int64_t n, int B, const double* rhs, const double* Ap, double* r, double* p, const CgScalars* cs,
                    cudaStream_t s);
// alpha = rr / pap
void launch_cg_alpha(int B, CgScalars* cs, const double* pap, cudaStream_t s);
// y += alpha p ; r -= alpha Ap ; rr_out[b] = r.r
void launch_cg_update_yr(int64_t n, int B, double* y, double* r, const double* p, const double* Ap,
                         const CgScalars* cs, double* partial, double* rr_out, cudaStream_t s);
// convergence test and beta; counts instances still active into *n_active
void launch_cg_beta(int B, CgScalars* cs, const double* rrnew, int* n_active, cudaStream_t s);
// One CG step after p.Ap (in pap): y += alpha p, r -= alpha Ap, then r.r,
// alpha, the convergence test, beta and the count of instances still
// iterating into *n_active (two launches; replaces alpha / update_yr / beta)
void launch_cg_step(int64_t n, int B, double* y, double* r, const double* p, const double* Ap, CgScalars* cs,
                    const double* pap, double* partial, int* n_active, cudaStream_t s);
// p = beta p + r
void launch_cg_update_p(int64_t n, int B, double* p, const double* r, const CgScalars* cs, cudaStream_t s);
// Sets the WHILE condition h of a device-side CG loop: ++*count, then
// continue while *n_active > 0 and *count < cap.
void launch_cg_while(cudaGraphConditionalHandle h, const int* n_active, int* count, int cap, cudaStream_t s);

// Persistent CG (maps.cu): a whole CG solve of a small group in one
// cooperative launch.  Groups of at most kLoopMaxB instances and
// kLoopMaxElems constraint elements (nc * B), where launch latency, not
// bandwidth, bounds an iteration.
constexpr int kLoopMaxB = 8;
constexpr int64_t kLoopMaxElems = 1 << 21;
bool cg_loop_fits(int64_t nc, int B);
// CTAs of the cooperative grid on this device (0: no cooperative launch)
int cg_loop_grid(int device);
// Iterates until no instance of cs is active or cap iterations: y, r, p and
// cs as the chunked path leaves them; *n_active the instances still active,
// *iters the iterations run, *err = 1 if a grid barrier wait ran out (then the
// results are invalid).  *bar must be 0 at the launch.  part_dot holds
// (row tiles + long rows of A) x B, part_rr grid x B doubles.
cudaError_t launch_cg_loop(const DevMap& A, const DevMap& AT, int B, int64_t nc, double* y, double* r, double* p,
                           double* atp, double* ap, CgScalars* cs, double* part_dot, double* part_rr,
                           unsigned int* bar, int* err, int* n_active, int* iters, int cap, int grid,
                           cudaStream_t s);
// CG start extrapolation over [e * B + b]: where mode[b] == 2,
// y <- y + (y - yprev); where mode[b] >= 1, yprev <- y (its value on entry)
void launch_cg_extrapolate(int64_t n, int B, double* y, double* yprev, const int* mode, cudaStream_t s);
// rr <- initial r.r
void launch_cg_set_rr(int B, CgScalars* cs, const double* rr, int* n_active, cudaStream_t s);

// ---- Anderson acceleration of the outer iteration --------------------------
// The state w = (x, z) of one instance is the 2 * nx rows e < nx of x and
// e >= nx of z, interleaved [e * B + b] like every vector; the history holds
// m difference columns dF_j = f_{k+1} - f_k and dG_j = g_{k+1} - g_k (f = g - w,
// g = the iterate the step produced), each 2 * nx * B doubles, column j at
// j * 2 * nx * B.
constexpr int kAndersonMax = 16;
// w <- (x, z) for the instances with mode[b] != 0
void launch_aa_save(int64_t nx, int B, const double* x, const double* z, double* w, const int* mode, cudaStream_t s);
// f = g - w; mode[b] == 2: dF[slot[b]] = f - fprev, dG[slot[b]] = g - gprev and
// dots[(2 j) * B + b] = dF[slot].dF[j], dots[(2 j + 1) * B + b] = dF[j].f for j < m;
// mode[b] >= 1: dots[(2 m) * B + b] = f.f, fprev = f, gprev = g.  partial holds
// aa_partial_size(nx, B, m) doubles; the sums are deterministic.
void launch_aa_update(int64_t nx, int B, int m, const double* x, const double* z, const double* w, double* fprev,
                      double* gprev, double* dF, double* dG, const int* mode, const int* slot, double* partial,
                      double* dots, cudaStream_t s);
int64_t aa_partial_size(int64_t nx, int B, int m);
// (x, z) <- g - sum_j gamma[b * m + j] dG_j for the instances with mix[b] set
// (columns with gamma 0 are not read)
void launch_aa_mix(int64_t nx, int B, int m, double* x, double* z, const double* dG, const double* gamma,
                   const int* mix, cudaStream_t s);

// ---- projection (Update_xz) ----------------------------------------------

// Description of one PSD block of one instance.
struct BlockTask {
    int64_t xoff;   // offset of the block in the (per-instance) primal vector
    int n;          // block dimension
    int inst;       // instance index within the group (for interleaving)
    int64_t woff;   // offset of the padded workspace matrix (large blocks)
    int np;         // padded dimension (multiple of 64, large blocks)
    int nb;         // number of 32-wide column blocks (np / 32)
    int64_t qoff;   // offset of the pair-rotation buffer (large blocks)
    int64_t doff;   // offset of the np-long weight vector (large blocks)
    int64_t toff;   // offset (32-bit words) of the split TF32 operands (tensor-core blocks)
};

// Blocks with n <= 64: form U, diagonalise in shared memory, write x and z.
// vsave (optional) keeps each block's eigenvectors (n x n at task.woff)
// across calls; warm starts the Jacobi from them.  stol (optional, per
// instance): off-diagonal entries below it are not rotated away (the
// adaptive projection's tolerance share).
void launch_small_project(const BlockTask* tasks, int ntasks, int B, const double* aty, const double* c, double* x,
                          double* z, const double* mu, const int* mask, cudaStream_t s, double* vsave = nullptr,
                          bool warm = false, const double* stol = nullptr);

// Large blocks (n > 64), block Jacobi on a padded np x np workspace.
// U = sym(A^T y - c + mu x), zero padded.
void launch_form_u(const BlockTask* tasks, int ntasks, int max_np, int B, const double* aty, const double* c,
                   const double* x, const double* mu, const int* mask, double* Uw, cudaStream_t s);
// W = U (cold start) and V = I
void launch_cold_start(const BlockTask* tasks, int ntasks, int max_np, const double* Uw, double* Ww, double* Vw,
                       const int* bmask, cudaStream_t s);
// batched 64x64-tiled FP64 GEMM on the padded workspaces:
// C = op(A) diag(d) op(B), with d optional.
struct GemmTile {
    int task;   // block task index
    int ti, tj; // tile coordinates
};
void launch_gemm(const BlockTask* tasks, const GemmTile* tiles, int ntiles, const double* A, bool transA,
                 const double* Bm, bool transB, const double* dvec, double* C, const int* bmask, cudaStream_t s);
// The same product on the tensor cores (tcgen05, 3xTF32 split, FP32
// accumulation: FP32 accuracy) over 128 x 128 tiles of C: tile (ti, tj)
// covers rows 128 ti.. and columns 128 tj..; rows and columns past np are not
// written.  The operands are first split into TF32 pairs in the MMA's shared
// memory layout, one unit (task, 128-row block) per CTA, into the plan's
// workspaces wa and wb (tc_split_words(np) words per task, at task.toff).
struct TcSplit {
    int task, rb;
};
struct TcPlan {
    const BlockTask* tasks = nullptr;
    const GemmTile* tiles_full = nullptr;  // every 128 x 128 tile
    const GemmTile* tiles_sym = nullptr;   // tiles ti <= tj (symmetric products, mirrored afterwards)
    int n_full = 0, n_sym = 0;
    const TcSplit* split = nullptr;
    int nsplit = 0;
    int max_nk = 0;  // largest np / 32 of the tasks: the split runs one CTA per (row block, K chunk)
    uint32_t* wa = nullptr;
    uint32_t* wb = nullptr;
};
int64_t tc_split_words(int np);
void launch_tc_gemm(const TcPlan& plan, bool sym, const double* A, bool transA, const double* Bm, bool transB,
                    const double* dvec, double* C, const int* bmask, cudaStream_t s);
// 0 while every tensor-core GEMM's pipeline waits ended; 1 after one ran out
// (that launch's result is invalid); reset clears the flag.
int tc_gemm_status(bool reset);
// the same flag copied into host (pinned) memory on a stream, without a device-wide sync
void tc_gemm_status_async(int* host, cudaStream_t s);
// One block-Jacobi round: solve each 64x64 pair problem, then rotate W and V.
struct PairTask {
    int task;   // block task
    int k;      // pair index within the round
};
struct WTileTask {
    int task, k1, k2;
};
struct VTileTask {
    int task, chunk, k;
};
// One round of the block Jacobi: each 64x64 pair problem is diagonalised
// into Qbuf unless its off-diagonal norm^2 is at most pthr[task] (then
// qskip marks its rotation as the identity and the update leaves it out).
void launch_bj_solve(const BlockTask* tasks, const PairTask* pt, int npt, int round, double* Ww, double* Qbuf,
                     const int* bmask, const double* pthr, int* qskip, cudaStream_t s);
void launch_bj_update_wv(const BlockTask* tasks, const WTileTask* wt, int nwt, const VTileTask* vt, int nvt, int round,
                         double* Ww, double* Vw, const double* Qbuf, const int* bmask, const int* qskip,
                         cudaStream_t s);
// Per-block off-diagonal and total Frobenius norms of W; sets bmask[t] = 0
// for blocks whose off-diagonal norm is below max(tol[t] * total, abs_tol[t])
// or that have done max_sweeps[t] sweeps, and pthr[t] = that limit squared
// over the pair problems of a sweep.
void launch_bj_check(const BlockTask* tasks, int ntasks, int max_np, const double* Ww, const double* tol,
                     const double* abs_tol, const int* max_sweeps, int sweeps_done, double* rowsum, int* bmask,
                     double* pthr, int* n_open, cudaStream_t s);
// dx = max(lam, 0) / mu and dz = max(-lam, 0) (per block, length np; zero on padding)
void launch_pos_weights(const BlockTask* tasks, int ntasks, const double* lam, const double* mu, const int* bmask,
                        double* dx, double* dz, cudaStream_t s);
// lam = diag(W)
void launch_lam_from_diag(const BlockTask* tasks, int ntasks, const double* Ww, const int* bmask, double* lam,
                          cudaStream_t s);
// Ogita-Aishima step: lam_i = s_ii / g_ii and M = I + E from S = V^T U V and
// G = V^T V; emax[t] gets max |E_ij| (as the bits of a non-negative double)
// and hard[t] is set for blocks needing the Jacobi fallback (an index
// strongly coupled to more than one other; isolated strongly coupled pairs
// are rotated exactly).  partner needs one int per padded row.
// Blocks whose eigenvectors lost orthonormality (|g_ii - 1| > 0.25) or whose
// values broke down get restart[t] = 1; blocks whose first-order step has
// ||E||_F > 0.2 are marked hard.  erow holds one double per padded row.
// gdev[t] (optional) gets max |G_ij - delta_ij| of the block (as the bits of a
// non-negative double): the distance of V from orthonormal.
void launch_oa_analyze(const BlockTask* tasks, int ntasks, int max_np, const double* S, const double* G,
                       const int* bmask, double* lam, double* scale, int* partner, double* M,
                       unsigned long long* emax, int* hard, double* erow, int* restart, unsigned long long* gdev,
                       cudaStream_t s);
void launch_oa_masks(int ntasks, const unsigned long long* emax, const int* hard, const double* tol,
                     const double* abs_tol, const double* scale, int* ref, int* upd, int* jac, int* n_ref,
                     cudaStream_t s);
void launch_copy_blocks(const BlockTask* tasks, int ntasks, int max_np, const double* src, double* dst,
                        const int* bmask, cudaStream_t s);
void launch_count(int n, const int* mask, int* out, cudaStream_t s);
// symmetric GEMM results: copy the upper tiles onto the lower ones
void launch_mirror(const BlockTask* tasks, int ntasks, int max_np, double* C, const int* bmask, cudaStream_t s);
// M = I + (I - G) / 2 (G = V^T V): V M is a Newton-Schulz step that brings V
// back to orthonormal (the distance squares)
void launch_ortho_step(const BlockTask* tasks, int ntasks, int max_np, const double* G, const int* bmask, double* M,
                       cudaStream_t s);
// bmask[t] = mask[tasks[t].inst] != 0
void launch_block_mask(const BlockTask* tasks, int ntasks, const int* mask, int* bmask, cudaStream_t s);
// max_sweeps[i] = unlimited where sel[i]
void launch_uncap(int n, const int* sel, int* max_sweeps, cudaStream_t s);
// dst[i] |= src[i]
void launch_merge_mask(int n, const int* src, int* dst, cudaStream_t s);
// x = X and z = Z (unpadded, interleaved)
void launch_write_xz(const BlockTask* tasks, int ntasks, int max_n, int B, const double* Xw, const double* Zw,
                     const int* mask, double* x, double* z, cudaStream_t s);

}  // namespace v2g
