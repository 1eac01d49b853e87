// Host driver of the B200 boundary-point SDP solver and the C ABI of
// include/v2rdm_gpu.h.
//
// The outer loop restates v2RDMSolver::compute_energy (v2rdm_solver.cc:
// 1778-1908) and CGSolver::solve (cg_solver.cc:125-177) step for step, for a
// group of B instances at once: every instance keeps its own mu, CG
// tolerance, iteration counts and stopping test, and is masked out of all
// updates once it has converged.  All vector work runs on the device; the
// host reads back four scalars per instance per outer iteration (the same
// ones the reference prints) to run the stopping test and the mu update.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/v2rdm_gpu.h"
#include "anderson.h"
#include "constraints.h"
#include "kernels.cuh"
#include "layout.h"
#include "warmstart.h"

namespace v2g {

namespace {

thread_local std::string g_last_error;

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct NoDevice : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define CK(call)                                                                                         \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            throw ::v2g::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " + __FILE__ + ":" + \
                            std::to_string(__LINE__));                                                   \
    } while (0)

// Makes a device current for the scope of a call and restores the caller's
// current device afterwards.
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        CK(cudaSetDevice(device));
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
};

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    void alloc(size_t count) {
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        if (count) {
            CK(cudaMalloc(&p, count * sizeof(T)));
            CK(cudaMemset(p, 0, count * sizeof(T)));
        }
    }
    void upload(const T* h, size_t count) {
        alloc(count);
        if (count) CK(cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice));
    }
};

// One map (A or A^T) on the device in the bucketed-ELL form of kernels.cuh.
struct MapTable {
    DevBuf<int32_t> rows, cols, long_rows, long_ptr, long_col;
    DevBuf<double> vals, long_val, book;
    DevMap dm;

    // Packs the coefficient of every ELL entry into its column word when the
    // columns fit in kCodeShift bits and the table has at most kBookSize
    // distinct coefficients (compared bit for bit, so the sums are unchanged);
    // returns the book, or an empty vector when the table stays unpacked.
    // Only tables larger than L2 are packed: there the coefficient stream is
    // HBM traffic (H50: 10 % faster maps), while for tables that stay in L2
    // the book lookup costs more than it saves (H10 and 19 x n = 20: 2-3 %
    // slower on B200).
    static constexpr size_t kPackMinBytes = size_t(128) << 20;
    static std::vector<double> pack(std::vector<int32_t>& hcols, const std::vector<double>& hvals) {
        if (hcols.size() * (sizeof(int32_t) + sizeof(double)) < kPackMinBytes) return {};
        std::map<uint64_t, int> code;
        std::vector<double> bk;
        for (size_t k = 0; k < hcols.size(); k++) {
            if (hcols[k] < 0) continue;
            if (hcols[k] >= (1 << kCodeShift)) return {};
            uint64_t bits;
            std::memcpy(&bits, &hvals[k], sizeof bits);
            if (code.count(bits)) continue;
            if ((int)bk.size() == kBookSize) return {};
            code[bits] = (int)bk.size();
            bk.push_back(hvals[k]);
        }
        if (bk.empty()) return {};
        for (size_t k = 0; k < hcols.size(); k++) {
            if (hcols[k] < 0) continue;
            uint64_t bits;
            std::memcpy(&bits, &hvals[k], sizeof bits);
            hcols[k] |= code[bits] << kCodeShift;
        }
        bk.resize(kBookSize, 0.0);
        return bk;
    }

    void build(const Csr& M) {
        static const int widths[kMaxBuckets] = {1, 2, 4, 8, 16, 32};
        std::vector<std::vector<int32_t>> brow(kMaxBuckets);
        std::vector<int32_t> lrows, lptr(1, 0), lcol;
        std::vector<double> lval;
        for (int64_t r = 0; r < M.nrows; r++) {
            const int64_t len = M.rowptr[r + 1] - M.rowptr[r];
            int w = 0;
            while (w < kMaxBuckets && widths[w] < len) w++;
            if (w < kMaxBuckets) {
                brow[w].push_back((int32_t)r);
            } else {
                lrows.push_back((int32_t)r);
                for (int64_t k = M.rowptr[r]; k < M.rowptr[r + 1]; k++) {
                    lcol.push_back(M.col[k]);
                    lval.push_back(M.val[k]);
                }
                lptr.push_back((int32_t)lcol.size());
            }
        }
        // inside a bucket, rows are ordered by their first column: rows that
        // gather from the same region of the input run in the same CTA wave,
        // so their gathers hit L2 (the output is written through rows[])
        for (int w = 0; w < kMaxBuckets; w++)
            std::stable_sort(brow[w].begin(), brow[w].end(), [&](int32_t a, int32_t b) {
                const int32_t ca = M.rowptr[a] < M.rowptr[a + 1] ? M.col[M.rowptr[a]] : -1;
                const int32_t cb = M.rowptr[b] < M.rowptr[b + 1] ? M.col[M.rowptr[b]] : -1;
                return ca < cb;
            });
        std::vector<int32_t> hrows, hcols;
        std::vector<double> hvals;
        dm = DevMap{};
        dm.nrows = M.nrows;
        for (int w = 0; w < kMaxBuckets; w++) {
            if (brow[w].empty()) continue;
            const int W = widths[w];
            const int64_t ns = (int64_t)brow[w].size();
            const int bi = dm.nb++;
            dm.width[bi] = W;
            dm.nslots[bi] = ns;
            dm.row_off[bi] = (int64_t)hrows.size();
            dm.ent_off[bi] = (int64_t)hcols.size();
            hrows.insert(hrows.end(), brow[w].begin(), brow[w].end());
            const size_t base = hcols.size();
            hcols.resize(base + (size_t)W * ns, -1);
            hvals.resize(base + (size_t)W * ns, 0.0);
            for (int64_t i = 0; i < ns; i++) {
                const int64_t r = brow[w][i];
                int k = 0;
                for (int64_t e = M.rowptr[r]; e < M.rowptr[r + 1]; e++, k++) {
                    hcols[base + (size_t)k * ns + i] = M.col[e];
                    hvals[base + (size_t)k * ns + i] = M.val[e];
                }
            }
        }
        const std::vector<double> bk = pack(hcols, hvals);
        rows.upload(hrows.data(), hrows.size());
        cols.upload(hcols.data(), hcols.size());
        if (bk.empty())
            vals.upload(hvals.data(), hvals.size());
        else
            book.upload(bk.data(), bk.size());
        long_rows.upload(lrows.data(), lrows.size());
        long_ptr.upload(lptr.data(), lptr.size());
        long_col.upload(lcol.data(), lcol.size());
        long_val.upload(lval.data(), lval.size());
        dm.rows = rows.p;
        dm.cols = cols.p;
        dm.vals = bk.empty() ? vals.p : nullptr;
        dm.book = bk.empty() ? nullptr : book.p;
        dm.nlong = (int)lrows.size();
        dm.long_rows = long_rows.p;
        dm.long_ptr = long_ptr.p;
        dm.long_col = long_col.p;
        dm.long_val = long_val.p;
    }
};

// Index tables and b for one layout, shared by every instance with it.
struct DeviceTables {
    Layout L;
    int device = 0;
    Csr hA;  // kept on the host for v2g_export_A
    MapTable mA, mAT;
    DevBuf<double> b;
    std::vector<double> hb;
    const DevMap& A() const { return mA.dm; }
    const DevMap& AT() const { return mAT.dm; }
    int max_long() const { return std::max(mA.dm.nlong, mAT.dm.nlong); }
};

std::string layout_key(const Layout& L, int device) {
    std::ostringstream s;
    const Options& o = L.opt;
    s << device << '|' << o.constrain_q2 << o.constrain_g2 << o.constrain_t1 << o.constrain_t2 << o.constrain_spin
      << o.constrain_sz << o.spin_adapt_q2 << o.spin_adapt_g2 << o.constrain_d3 << o.constrain_d4 << '|' << L.nirrep << '|';
    for (int a : L.amopi) s << a << ',';
    s << '|' << L.na << '|' << L.nb << '|' << L.multiplicity << '|';
    for (int i : L.energy_order) s << i << ',';
    return s.str();
}

std::mutex g_cache_mu;
std::map<std::string, std::weak_ptr<DeviceTables>> g_cache;

std::shared_ptr<DeviceTables> get_tables(const Layout& L, int device) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    const std::string key = layout_key(L, device);
    auto it = g_cache.find(key);
    if (it != g_cache.end())
        if (auto sp = it->second.lock()) return sp;
    auto T = std::make_shared<DeviceTables>();
    T->L = L;
    T->device = device;
    std::string err = build_A(L, T->hA);
    if (!err.empty()) throw std::invalid_argument(err);
    Csr AT;
    transpose(T->hA, AT);
    if (T->hA.nnz() >= (int64_t)INT32_MAX) throw std::invalid_argument("constraint table exceeds 2^31 entries");
    CK(cudaSetDevice(device));
    T->mA.build(T->hA);
    T->mAT.build(AT);
    build_b(L, T->hb);
    T->b.upload(T->hb.data(), T->hb.size());
    g_cache[key] = T;
    return T;
}

}  // namespace

// One active-space problem (a v2g_handle).
struct Problem {
    Options opt;
    Layout L;
    OrbitalSpaces sp;
    int device = 0;
    bool record_trace = false;
    bool profile = false;
    std::vector<double> c, x, y, z;
    double mu = 1.0;
    double efzc = 0.0, enuc = 0.0;
    bool have_c = false;
    std::shared_ptr<DeviceTables> T;
    std::vector<std::array<double, 8>> trace;
    std::vector<double> energies;  // active orbital energies, if the caller gave them
    // the integrals of an all-active C1 space (h: n x n, Lq: nq x n x n), kept
    // for the learned warm start's features
    std::vector<double> hmat, Lq;
    int nq = 0;
    // a start proposal (x holds it) that a solve with start = 2 projects onto A x = b
    bool proposal = false;
    // Loop state carried by v2g_solve_continue: outer iterations done and the
    // last eps(p), eps(d) (they set the next CG tolerance); every solve
    // updates them.  resume > 0 makes the next solve continue the loop for at
    // most that many outer iterations.
    long oiter_done = 0;
    double last_ep = 0.0, last_ed = 0.0;
    int resume = 0;

    DeviceTables& tables() {
        if (!T) T = get_tables(L, device);
        return *T;
    }
};

namespace {

// Projection tolerance down to which the mixed-precision phase runs the large
// blocks' dense products on the tensor cores (FP32 accuracy, ~1e-6 relative,
// is then two orders below what the projection has to deliver).
constexpr double kMixedRho = 1e-5;
// Smallest padded block whose products go to the tensor cores in the mixed
// phase (dimension > 448: G2aa from n = 15 on, the DQGT2 blocks, H50's blocks).
constexpr int kMixedMinNp = 512;

// Lock-step solve of B instances that share one layout.
class GroupRun {
  public:
    GroupRun(DeviceTables& T, std::vector<Problem*> probs) : T_(T), P_(std::move(probs)), B_((int)P_.size()) {
        if (B_ < 1 || B_ > 256) throw std::invalid_argument("a group holds 1..256 instances");
        CK(cudaSetDevice(T.device));
        CK(cudaStreamCreate(&s_));
        CK(cudaStreamCreate(&s_small_));
        CK(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
        nx_ = T.L.dimx;
        nc_ = T.L.ncon;
        const size_t X = (size_t)nx_ * B_, C = (size_t)nc_ * B_;
        c_.alloc(X);
        x_.alloc(X);
        z_.alloc(X);
        aty_.alloc(X);
        atp_.alloc(X);
        y_.alloc(C);
        ax_.alloc(C);
        bv_.alloc(C);
        r_.alloc(C);
        p_.alloc(C);
        ap_.alloc(C);
        partial_.alloc(reduce_partial_size(B_) + (int64_t)(T.max_long() + 8) * B_);
        red_.alloc(4 * B_);
        mu_.alloc(B_);
        coef_.alloc(B_);
        mask_.alloc(B_);
        smask1_.alloc(B_);
        smask2_.alloc(B_);
        cs_.alloc(B_);
        nact_.alloc(8);  // counters: CG, Jacobi, refinement, fallback, restart
        for (auto* p : P_) extrapolate_ = extrapolate_ || p->opt.cg_extrapolate;
        if (extrapolate_) {
            yprev_.alloc(C);
            ex_.alloc(B_);
        }
        CK(cudaMallocHost(&hscal_, sizeof(double) * 4 * B_));
        CK(cudaMallocHost(&hnact_, sizeof(int) * 8));
        CK(cudaMallocHost(&hcs_, sizeof(CgScalars) * B_));
        stage_cap_ = 1 << 20;
        CK(cudaMallocHost(&stage_, stage_cap_));
        mA_ = T.A();
        mAT_ = T.AT();
        build_projection_plan();
        upload_state();
        tune_maps();
        if (cg_loop_fits(nc_, B_)) loop_grid_ = cg_loop_grid(T.device);
        if (loop_grid_ > 0) {
            loopbar_.alloc(2);
            looppart_.alloc((size_t)loop_grid_ * B_);
        }
        alloc_anderson(X);
        if (const char* d = std::getenv("V2G_DIAG")) diag_every_ = std::atoi(d);
        if (diag_every_ > 0)
            if (const char* fn = std::getenv("V2G_DIAG_FILE")) diag_file_ = std::fopen(fn, "a");
        for (auto* p : P_) profile_ = profile_ || p->profile;
        if (profile_) {
            prof_ev_.resize(256);
            for (auto& e : prof_ev_) CK(cudaEventCreate(&e));
        }
    }
    ~GroupRun() {
        if (cg_exec_) cudaGraphExecDestroy(cg_exec_);
        if (cg_loop_exec_) cudaGraphExecDestroy(cg_loop_exec_);
        if (diag_file_) std::fclose(diag_file_);
        for (auto e : prof_ev_) cudaEventDestroy(e);
        if (hscal_) cudaFreeHost(hscal_);
        if (hnact_) cudaFreeHost(hnact_);
        if (hcs_) cudaFreeHost(hcs_);
        if (hdots_ptr_) cudaFreeHost(hdots_ptr_);
        if (stage_) cudaFreeHost(stage_);
        if (ev_fork_) cudaEventDestroy(ev_fork_);
        if (ev_join_) cudaEventDestroy(ev_join_);
        if (s_small_) cudaStreamDestroy(s_small_);
        if (s_) cudaStreamDestroy(s_);
    }

    // Interleave host vectors of all instances into [e * B + b].
    void upload_vec(DevBuf<double>& d, int64_t n, const std::vector<double> Problem::*member) {
        std::vector<double> h((size_t)n * B_);
        for (int b = 0; b < B_; b++) {
            const auto& v = P_[b]->*member;
            for (int64_t e = 0; e < n; e++) h[(size_t)e * B_ + b] = v[e];
        }
        CK(cudaMemcpy(d.p, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    void download_vec(const DevBuf<double>& d, int64_t n, std::vector<double> Problem::*member) {
        std::vector<double> h((size_t)n * B_);
        CK(cudaMemcpy(h.data(), d.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int b = 0; b < B_; b++) {
            auto& v = P_[b]->*member;
            v.resize(n);
            for (int64_t e = 0; e < n; e++) v[e] = h[(size_t)e * B_ + b];
        }
    }
    void upload_state() {
        upload_vec(c_, nx_, &Problem::c);
        upload_vec(x_, nx_, &Problem::x);
        upload_vec(z_, nx_, &Problem::z);
        upload_vec(y_, nc_, &Problem::y);
        std::vector<double> mu(B_);
        for (int b = 0; b < B_; b++) mu[b] = P_[b]->mu;
        CK(cudaMemcpy(mu_.p, mu.data(), B_ * sizeof(double), cudaMemcpyHostToDevice));
        std::vector<int> m(B_, 1);
        CK(cudaMemcpy(mask_.p, m.data(), B_ * sizeof(int), cudaMemcpyHostToDevice));
    }
    void download_state() {
        download_vec(x_, nx_, &Problem::x);
        download_vec(z_, nx_, &Problem::z);
        download_vec(y_, nc_, &Problem::y);
    }

    // Update_xz for every instance with mask set; ATy is left in aty_.
    // rho[b] > 0 lets instance b accept an eigendecomposition whose
    // off-diagonal residual is below rho[b] in absolute terms (the adaptive
    // projection, rho = 0.01 min(eps_p, eps_d) like the CG tolerance rule);
    // rho[b] = 0 asks for a converged one.  x = V D+ V^T / mu and z = V D- V^T
    // are positive semidefinite either way.
    // mixed = true runs the large blocks' dense products on the tensor cores.
    void project(const std::vector<double>& rho = {}, bool mixed = false) {
        tc_ = mixed && ntc_gtiles_ > 0;
        if (tc_) tc_projections_++;
        launch_spmv(mAT_, B_, y_.p, aty_.p, nullptr, nullptr, nullptr, mask_.p, s_);
        // The small blocks (one CTA each: a few SMs for a few hundred
        // microseconds) run on a second stream beside the large blocks' path;
        // both read A^T y, c and mu and write disjoint entries of x and z.
        // They start from their previous eigenvectors, except in the first
        // projection, after a cold restart and every kSmallCold-th projection
        // (so that rounding in the kept eigenvectors cannot build up).
        const bool small_warm = small_warm_ && (nproj_ % kSmallCold) != 0;
        const bool fork = nsmall_ > 0;
        if (fork) {
            CK(cudaEventRecord(ev_fork_, s_));
            CK(cudaStreamWaitEvent(s_small_, ev_fork_, 0));
            launch_small_project(small_d_.p, nsmall_, B_, aty_.p, c_.p, x_.p, z_.p, mu_.p, mask_.p, s_small_,
                                 vsmall_.p, small_warm);
            CK(cudaEventRecord(ev_join_, s_small_));
        }
        small_warm_ = true;
        nproj_++;
        project_large(rho);
        if (fork) CK(cudaStreamWaitEvent(s_, ev_join_, 0));
    }

    void project_large(const std::vector<double>& rho) {
        if (nlarge_ == 0) return;
        launch_form_u(large_d_.p, nlarge_, max_np_, B_, aty_.p, c_.p, x_.p, mu_.p, mask_.p, U_.p, s_);
        set_block_masks();  // bact_ = blocks of active instances
        set_block_tolerances(rho);
        if (!warm_) {
            // cold start: W = U, V = I, block Jacobi to convergence
            launch_cold_start(large_d_.p, nlarge_, max_np_, U_.p, W_.p, V_.p, bact_.p, s_);
            CK(cudaMemcpyAsync(bjac_.p, bact_.p, nlarge_ * sizeof(int), cudaMemcpyDeviceToDevice, s_));
            block_jacobi(40);
        } else {
            refine();
        }
        launch_pos_weights(large_d_.p, nlarge_, lam_.p, mu_.p, bact_.p, dw_.p, dz_.p, s_);
        gemm_sym(V_.p, false, V_.p, true, dw_.p, Tm_.p, bact_.p);
        gemm_sym(V_.p, false, V_.p, true, dz_.p, M_.p, bact_.p);
        launch_mirror(large_d_.p, nlarge_, max_np_, Tm_.p, bact_.p, s_);
        launch_mirror(large_d_.p, nlarge_, max_np_, M_.p, bact_.p, s_);
        launch_write_xz(large_d_.p, nlarge_, max_n_, B_, Tm_.p, M_.p, mask_.p, x_.p, z_.p, s_);
        warm_ = true;
    }

    // Ogita-Aishima sweeps from the previous eigenvectors; blocks with a hard
    // pair or without convergence after kMaxOa sweeps go to block Jacobi.
    void refine() {
        // in the mixed phase the products carry FP32 rounding, so the refinement's
        // residual floor is FP32's: a few sweeps, and blocks that stop above the
        // (loose) tolerance are accepted as they are instead of going to Jacobi
        const int kMaxOa = tc_ ? 3 : 6;
        CK(cudaMemcpyAsync(bref_.p, bact_.p, nlarge_ * sizeof(int), cudaMemcpyDeviceToDevice, s_));
        CK(cudaMemsetAsync(bjac_.p, 0, nlarge_ * sizeof(int), s_));
        CK(cudaMemsetAsync(restart_.p, 0, nlarge_ * sizeof(int), s_));
        CK(cudaMemsetAsync(gdev_.p, 0, nlarge_ * sizeof(unsigned long long), s_));
        int nref = 1;
        for (int sweep = 0; sweep < kMaxOa && nref > 0; sweep++) {
            // S = V^T (U V) and G = V^T V are symmetric: upper tiles, then mirrored
            gemm_full(U_.p, false, V_.p, false, nullptr, Tm_.p, bref_.p);
            gemm_sym(V_.p, true, Tm_.p, false, nullptr, W_.p, bref_.p);
            gemm_sym(V_.p, true, V_.p, false, nullptr, G_.p, bref_.p);
            launch_mirror(large_d_.p, nlarge_, max_np_, W_.p, bref_.p, s_);
            launch_mirror(large_d_.p, nlarge_, max_np_, G_.p, bref_.p, s_);
            CK(cudaMemsetAsync(emax_.p, 0, nlarge_ * sizeof(unsigned long long), s_));
            CK(cudaMemsetAsync(hard_.p, 0, nlarge_ * sizeof(int), s_));
            launch_oa_analyze(large_d_.p, nlarge_, max_np_, W_.p, G_.p, bref_.p, lam_.p, scale_.p, partner_.p,
                              M_.p, emax_.p, hard_.p, erow_.p, restart_.p, gdev_.p, s_);
            launch_oa_masks(nlarge_, emax_.p, hard_.p, otol_.p, atol_.p, scale_.p, bref_.p, bupd_.p, bjac_.p,
                            nact_.p + 2, s_);
            gemm_full(V_.p, false, M_.p, false, nullptr, Tm_.p, bupd_.p);
            launch_copy_blocks(large_d_.p, nlarge_, max_np_, Tm_.p, V_.p, bupd_.p, s_);
            CK(cudaMemcpyAsync(hnact_ + 2, nact_.p + 2, sizeof(int), cudaMemcpyDeviceToHost, s_));
            CK(cudaStreamSynchronize(s_));
            nref = hnact_[2];
            oa_sweeps_++;
        }
        // blocks still unconverged join the Jacobi set (their OA update was applied)
        if (nref > 0 && !tc_) {
            launch_merge_mask(nlarge_, bref_.p, bjac_.p, s_);
            jacobi_unconverged_ += nref;
        }
        launch_count(nlarge_, bjac_.p, nact_.p + 3, s_);
        // blocks whose eigenvectors degraded restart cold (V = I, W = U) and
        // converge fully; they leave the refinement and warm Jacobi sets
        launch_count(nlarge_, restart_.p, nact_.p + 4, s_);
        CK(cudaMemcpyAsync(hnact_ + 3, nact_.p + 3, 2 * sizeof(int), cudaMemcpyDeviceToHost, s_));
        CK(cudaStreamSynchronize(s_));
        if (hnact_[3] > 0) {
            jacobi_blocks_ += hnact_[3];
            // the refinement skipped these blocks' update, so their V carries the
            // orthogonality error of the previous iteration: two Newton-Schulz
            // steps first (Jacobi's rotations preserve V^T V, whatever it is)
            // (FP64 products even in the mixed phase: the Jacobi below converges
            // W = V^T U V to its tolerance, which FP32 rounding in W would not allow)
            const bool tc = tc_;
            tc_ = false;
            for (int k = 0; k < 2; k++) {
                gemm_sym(V_.p, true, V_.p, false, nullptr, G_.p, bjac_.p);
                launch_mirror(large_d_.p, nlarge_, max_np_, G_.p, bjac_.p, s_);
                launch_ortho_step(large_d_.p, nlarge_, max_np_, G_.p, bjac_.p, M_.p, s_);
                gemm_full(V_.p, false, M_.p, false, nullptr, Tm_.p, bjac_.p);
                launch_copy_blocks(large_d_.p, nlarge_, max_np_, Tm_.p, V_.p, bjac_.p, s_);
            }
            // warm block Jacobi on W = V^T U V with the current V
            gemm_full(U_.p, false, V_.p, false, nullptr, Tm_.p, bjac_.p);
            gemm_sym(V_.p, true, Tm_.p, false, nullptr, W_.p, bjac_.p);
            tc_ = tc;
            launch_mirror(large_d_.p, nlarge_, max_np_, W_.p, bjac_.p, s_);
        }
        if (hnact_[4] > 0) {
            restarts_ += hnact_[4];
            launch_cold_start(large_d_.p, nlarge_, max_np_, U_.p, W_.p, V_.p, restart_.p, s_);
            launch_merge_mask(nlarge_, restart_.p, bjac_.p, s_);
            launch_uncap(nlarge_, restart_.p, msw_.p, s_);
        }
        if (hnact_[3] > 0 || hnact_[4] > 0) block_jacobi(30);
    }

    // Block Jacobi on the blocks flagged in bjac_ until their relative
    // off-diagonal norm is below 1e-13; sets lam = diag(W) for them.
    void block_jacobi(int max_sweeps) {
        CK(cudaMemcpyAsync(bwork_.p, bjac_.p, nlarge_ * sizeof(int), cudaMemcpyDeviceToDevice, s_));
        for (int sweep = 0; sweep < max_sweeps; sweep++) {
            launch_bj_check(large_d_.p, nlarge_, max_np_, W_.p, jtol_.p, atol_.p, cap_ ? msw_.p : nullptr, sweep,
                            rowsum_.p, bwork_.p, pthr_.p, nact_.p + 1, s_);
            CK(cudaMemcpyAsync(hnact_ + 1, nact_.p + 1, sizeof(int), cudaMemcpyDeviceToHost, s_));
            CK(cudaStreamSynchronize(s_));
            if (hnact_[1] == 0) break;
            for (int g = 0; g < max_rounds_; g++) {
                launch_bj_solve(large_d_.p, pairs_.p, npairs_, g, W_.p, Q_.p, bwork_.p, pthr_.p, qskip_.p, s_);
                launch_bj_update_wv(large_d_.p, wtiles_.p, nwtiles_, vtiles_.p, nvtiles_, g, W_.p, V_.p, Q_.p,
                                    bwork_.p, qskip_.p, s_);
            }
            sweeps_total_++;
        }
        launch_lam_from_diag(large_d_.p, nlarge_, W_.p, bjac_.p, lam_.p, s_);
    }

    cudaStream_t stream() const { return s_; }
    DevBuf<double>& xbuf() { return x_; }
    DevBuf<double>& ybuf() { return y_; }
    DevBuf<double>& zbuf() { return z_; }
    DevBuf<double>& mubuf() { return mu_; }

    // The outer BPSDP loop.  Returns per-instance results.
    void solve(std::vector<v2g_result>& res) {
        // loop options are per instance; the shared tables only fix the layout
        auto opt = [&](int b) -> const Options& { return P_[b]->opt; };
        res.assign(B_, v2g_result{});
        std::vector<double> mu(B_), ep(B_, 0.0), ed(B_, 0.0), egap(B_, 0.0);
        std::vector<int> active(B_, 1), oiter(B_, 0);
        std::vector<long> iiter(B_, 0), stalls(B_, 0);
        std::vector<double> coef(B_);
        // the last outer iteration of this call: MAXITER, or the end of a
        // continued segment
        std::vector<int> limit(B_);
        for (int b = 0; b < B_; b++) {
            mu[b] = P_[b]->mu;
            P_[b]->trace.clear();
            res[b].status = V2G_ERR_NOT_CONVERGED;
            limit[b] = opt(b).maxiter;
            if (P_[b]->resume > 0) {
                oiter[b] = (int)P_[b]->oiter_done;
                ep[b] = P_[b]->last_ep;
                ed[b] = P_[b]->last_ed;
                limit[b] = oiter[b] + P_[b]->resume;
            }
        }
        cudaEvent_t e0, e1, e2, e3;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        CK(cudaEventCreate(&e2));
        CK(cudaEventCreate(&e3));
        double t_cg = 0, t_xz = 0;
        CK(cudaEventRecord(e3, s_));
        std::vector<CgScalars> cs(B_);
        {
            std::vector<int> fs(B_);
            bool any = false;
            // a continued loop keeps its state; its first segment starts like a solve
            // 1: least-norm feasible point; 2: the instance's proposal (the
            // learned warm start) projected onto A x = b; without a proposal,
            // start 2 falls back to 1
            for (int b = 0; b < B_; b++) {
                fs[b] = 0;
                if (oiter[b] != 0) continue;
                if (opt(b).proposal_start)
                    fs[b] = P_[b]->proposal ? 2 : 1;
                else if (opt(b).feasible_start)
                    fs[b] = 1;
                any |= fs[b] != 0;
            }
            if (any) {
                feasible_start(fs, cs);
                for (int b = 0; b < B_; b++)
                    if (fs[b]) {
                        mu[b] = fs[b] == 2 ? P_[b]->mu : 1.0;
                        P_[b]->proposal = false;  // a proposal serves one solve
                        iiter[b] += cs[b].iter;
                        stalls[b] += cs[b].stalled;
                    }
            }
        }
        // an instance whose iterate turns non-finite restarts (at most twice)
        std::vector<int> restarts_left(B_, 2), recover(B_, 0);
        // CG solutions seen per instance since its (re)start, for cg_extrapolate
        std::vector<int> ycount(B_, 0), exmode(B_, 0);
        // Anderson acceleration, per instance: f and g stored, valid columns,
        // newest ring slot, this iteration's kernel mode, mu changed
        std::vector<int> mu_changed(B_, 0);
        AndersonState aa(B_, aa_m_);
        int it = 0;
        while (true) {
            if (std::find(recover.begin(), recover.end(), 1) != recover.end()) {
                feasible_start(recover, cs);
                for (int b = 0; b < B_; b++)
                    if (recover[b]) {
                        mu[b] = 1.0;
                        iiter[b] += cs[b].iter;
                        stalls[b] += cs[b].stalled;
                        recover[b] = 0;
                        ycount[b] = 0;
                        aa.restart(b);
                    }
                warm_ = false;  // every block of the group starts its projection cold again
                small_warm_ = false;
            }
            int nactive = 0;
            for (int b = 0; b < B_; b++) nactive += active[b];
            if (nactive == 0) break;
            put(mask_.p, active.data(), B_);
            for (int b = 0; b < B_; b++) coef[b] = -opt(b).tau * mu[b];
            put(coef_.p, coef.data(), B_);
            put(mu_.p, mu.data(), B_);
            if (aa_m_ > 0) {
                // w = the (x, z) this step starts from
                for (int b = 0; b < B_; b++) aa.mode[b] = (active[b] && aa_memory(b) > 0) ? 1 : 0;
                put(amode_.p, aa.mode.data(), B_);
                launch_aa_save(nx_, B_, x_.p, z_.p, aw_.p, amode_.p, s_);
            }
            std::fill(mu_changed.begin(), mu_changed.end(), 0);
            CK(cudaEventRecord(e0, s_));
            // Ax = -tau mu (A x - b); z <- c - z; B = A z + Ax   (:1783-1794)
            launch_spmv(mA_, B_, x_.p, ax_.p, T_.b.p, coef_.p, nullptr, mask_.p, s_);
            launch_c_minus_z(nx_, B_, c_.p, z_.p, mask_.p, s_);
            launch_spmv(mA_, B_, z_.p, bv_.p, nullptr, nullptr, ax_.p, mask_.p, s_);
            // CG tolerance (:1797-1805)
            for (int b = 0; b < B_; b++) {
                const Options& o = opt(b);
                double tol;
                if (oiter[b] == 0)
                    tol = 0.01;
                else
                    tol = (ep[b] > ed[b]) ? o.cg_tol_factor * ed[b] : o.cg_tol_factor * ep[b];
                if (tol < o.cg_convergence) tol = o.cg_convergence;
                cs[b] = CgScalars{};
                cs[b].tol = tol;
                cs[b].active = active[b];
                cs[b].maxiter = o.cg_maxiter;
            }
            put(cs_.p, cs.data(), B_);
            // CG starts from y_k + (y_k - y_{k-1}) once two CG solutions exist
            // (mode 2); before that it only records y_k (mode 1)
            if (extrapolate_) {
                for (int b = 0; b < B_; b++) {
                    exmode[b] = (active[b] && opt(b).cg_extrapolate) ? (ycount[b] >= 2 ? 2 : 1) : 0;
                    if (exmode[b]) ycount[b]++;
                }
                put(ex_.p, exmode.data(), B_);
                launch_cg_extrapolate(nc_, B_, y_.p, yprev_.p, ex_.p, s_);
            }
            cg_solve();
            CK(cudaMemcpyAsync(hcs_, cs_.p, B_ * sizeof(CgScalars), cudaMemcpyDeviceToHost, s_));
            CK(cudaEventRecord(e1, s_));
            std::vector<double> rho(B_, 0.0);
            for (int b = 0; b < B_; b++)
                if (opt(b).adaptive_projection)
                    rho[b] = (oiter[b] == 0) ? 0.01 : 0.01 * std::min(ep[b], ed[b]);
            // the mixed-precision phase: every instance still iterating asked for it
            // and accepts a projection residual of at least kMixedRho
            bool mixed = false;
            for (int b = 0; b < B_; b++) {
                if (!active[b]) continue;
                if (!(opt(b).mixed_precision && rho[b] >= kMixedRho)) {
                    mixed = false;
                    break;
                }
                mixed = true;
            }
            project(rho, mixed);
            CK(cudaEventRecord(e2, s_));
            // ed = ||A^T y + z - c||, ep = ||A x - b||, E = c.x, b.y (:1826-1852)
            launch_reduce(RED_ED, nx_, B_, aty_.p, z_.p, c_.p, nullptr, partial_.p, red_.p, s_);
            launch_spmv(mA_, B_, x_.p, ax_.p, nullptr, nullptr, nullptr, mask_.p, s_);
            launch_reduce(RED_EP, nc_, B_, ax_.p, nullptr, nullptr, T_.b.p, partial_.p, red_.p + B_, s_);
            launch_reduce(RED_DOT, nx_, B_, c_.p, x_.p, nullptr, nullptr, partial_.p, red_.p + 2 * B_, s_);
            launch_reduce(RED_DOT_ROW, nc_, B_, y_.p, nullptr, nullptr, T_.b.p, partial_.p, red_.p + 3 * B_, s_);
            CK(cudaMemcpyAsync(hscal_, red_.p, 4 * B_ * sizeof(double), cudaMemcpyDeviceToHost, s_));
            if (tc_) tc_gemm_status_async(hnact_ + 5, s_);
            CK(cudaStreamSynchronize(s_));
            stage_synced();
            std::copy(hcs_, hcs_ + B_, cs.begin());
            if (tc_ && hnact_[5] != 0)
                throw CudaError("a tensor-core GEMM of the projection did not finish (pipeline wait ran out)");
            float ms_cg = 0, ms_xz = 0;
            CK(cudaEventElapsedTime(&ms_cg, e0, e1));
            CK(cudaEventElapsedTime(&ms_xz, e1, e2));
            t_cg += ms_cg * 1e-3;
            t_xz += ms_xz * 1e-3;
            for (int b = 0; b < B_; b++) {
                if (!active[b]) continue;
                Problem& P = *P_[b];
                const Options& o = opt(b);
                ed[b] = std::sqrt(hscal_[b]);
                ep[b] = std::sqrt(hscal_[B_ + b]);
                const double e_p = hscal_[2 * B_ + b], e_d = hscal_[3 * B_ + b];
                const long ii = cs[b].iter;
                iiter[b] += ii;
                stalls[b] += cs[b].stalled;
                if (oiter[b] % o.mu_update_frequency == 0 && oiter[b] > 0) {
                    mu[b] = mu[b] * ep[b] / ed[b];
                    mu_changed[b] = 1;
                }
                const double shift = P.enuc + P.efzc;
                if (P.record_trace)
                    P.trace.push_back({(double)oiter[b], (double)ii, e_p + shift, e_d + shift, std::fabs(e_p - e_d),
                                       mu[b], ep[b], ed[b]});
                oiter[b]++;
                res[b].e_primal = e_p + shift;
                res[b].e_dual = e_d + shift;
                res[b].e_total = e_p + shift;
                res[b].ep = ep[b];
                res[b].ed = ed[b];
                res[b].mu = mu[b];
                res[b].oiter = oiter[b];
                res[b].iiter = iiter[b];
                res[b].cg_stalls = stalls[b];
                res[b].efzc = P.efzc;
                res[b].enuc = P.enuc;
                if (!std::isfinite(ep[b]) || !std::isfinite(ed[b]) || !std::isfinite(e_p)) {
                    report_nonfinite(b, oiter[b], mu[b], ii);
                    if (restarts_left[b] > 0) {
                        // restart this instance from the feasible start and
                        // the whole group's projection cold (below)
                        restarts_left[b]--;
                        recover[b] = 1;
                        ep[b] = ed[b] = 1.0;  // CG and projection tolerances as in iteration 0
                        continue;
                    }
                    res[b].status = V2G_ERR_NONFINITE;
                    active[b] = 0;
                    continue;
                }
                if (oiter[b] == limit[b]) {
                    res[b].status = V2G_ERR_NOT_CONVERGED;
                    active[b] = 0;
                    continue;
                }
                egap[b] = std::fabs(e_p - e_d);
                if (!(ep[b] > o.r_convergence || ed[b] > o.r_convergence || egap[b] > o.e_convergence)) {
                    res[b].status = V2G_OK;
                    active[b] = 0;
                }
            }
            if (diag_every_ > 0 && (it % diag_every_ == 0 || any_nonfinite(ep, ed))) diagnose(it, cs, ep, ed, mu);
            if (aa_m_ > 0) anderson(active, recover, mu_changed, aa);
            it++;
        }
        CK(cudaEventRecord(e2, s_));
        CK(cudaEventSynchronize(e2));
        float ms_tot = 0;
        CK(cudaEventElapsedTime(&ms_tot, e3, e2));
        for (int b = 0; b < B_; b++) {
            res[b].t_cg = t_cg;
            res[b].t_xz = t_xz;
            res[b].t_total = ms_tot * 1e-3;
            P_[b]->mu = mu[b];
            P_[b]->oiter_done = oiter[b];
            P_[b]->last_ep = ep[b];
            P_[b]->last_ed = ed[b];
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(e2);
        cudaEventDestroy(e3);
    }

    // The Anderson history of the group (after every other buffer): (3 + 2 m)
    // state vectors.  m shrinks to what 80 % of the free device memory holds,
    // or the acceleration is switched off for this group, with a note on stderr.
    void alloc_anderson(size_t X) {
        for (auto* p : P_) aa_m_ = std::max(aa_m_, p->opt.anderson_memory);
        if (aa_m_ <= 0) return;
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        const double vec = 2.0 * (double)X * sizeof(double);
        const int fit = (int)std::floor((0.8 * (double)free_b / vec - 3.0) / 2.0);
        if (fit < aa_m_) {
            std::fprintf(stderr, "v2g: Anderson memory %d does not fit in device memory next to this group; using %d\n",
                         aa_m_, std::max(fit, 0));
            aa_m_ = std::max(fit, 0);
            if (aa_m_ == 0) return;
        }
        aw_.alloc(2 * X);
        af_.alloc(2 * X);
        ag_.alloc(2 * X);
        adF_.alloc(2 * X * aa_m_);
        adG_.alloc(2 * X * aa_m_);
        agam_.alloc((size_t)B_ * aa_m_);
        apart_.alloc(aa_partial_size(nx_, B_, aa_m_));
        adots_.alloc((size_t)(2 * aa_m_ + 1) * B_);
        amode_.alloc(B_);
        aslot_.alloc(B_);
        amix_.alloc(B_);
    }
    // An instance's history length: its anderson_memory within the group's allocation.
    int aa_memory(int b) const { return std::min(P_[b]->opt.anderson_memory, aa_m_); }

    // Anderson acceleration after a step: f = g - w enters the history of every
    // instance still iterating with anderson_memory > 0, and an instance with
    // at least one difference column continues from g - sum_j gamma_j dG_j,
    // where gamma minimises |f - sum_j gamma_j dF_j| (a Tikhonov term of
    // 1e-10 tr(dF^T dF) keeps the small system regular).  The history restarts
    // from this f after a mu change and when |f| more than doubled since the
    // previous step (the step went the wrong way; that step is not mixed).
    void anderson(const std::vector<int>& active, const std::vector<int>& recover, const std::vector<int>& mu_changed,
                  AndersonState& aa) {
        bool any = false;
        for (int b = 0; b < B_; b++) {
            aa.mode[b] = 0;
            if (!active[b] || recover[b]) continue;
            if (aa.begin(b, aa_memory(b), mu_changed[b] != 0)) any = true;
        }
        if (!any) return;
        put(amode_.p, aa.mode.data(), B_);
        put(aslot_.p, aa.slot.data(), B_);
        launch_aa_update(nx_, B_, aa_m_, x_.p, z_.p, aw_.p, af_.p, ag_.p, adF_.p, adG_.p, amode_.p, aslot_.p,
                         apart_.p, adots_.p, s_);
        const size_t ndots = (size_t)(2 * aa_m_ + 1) * B_;
        if (hdots_.size() < ndots) {
            if (hdots_ptr_) CK(cudaFreeHost(hdots_ptr_));
            hdots_ptr_ = nullptr;
            CK(cudaMallocHost(&hdots_ptr_, ndots * sizeof(double)));
            hdots_.assign(ndots, 0.0);
        }
        CK(cudaMemcpyAsync(hdots_ptr_, adots_.p, ndots * sizeof(double), cudaMemcpyDeviceToHost, s_));
        CK(cudaStreamSynchronize(s_));
        stage_synced();
        std::vector<double> dots(hdots_ptr_, hdots_ptr_ + ndots);
        std::vector<double> gamma((size_t)B_ * aa_m_, 0.0);
        std::vector<int> mix(B_, 0);
        bool anymix = false;
        for (int b = 0; b < B_; b++) {
            if (aa.finish(b, aa_memory(b), dots, &gamma[(size_t)b * aa_m_])) {
                mix[b] = 1;
                anymix = true;
            }
        }
        if (!anymix) return;
        put(agam_.p, gamma.data(), gamma.size());
        put(amix_.p, mix.data(), B_);
        launch_aa_mix(nx_, B_, aa_m_, x_.p, z_.p, adG_.p, agam_.p, amix_.p, s_);
    }

    static bool any_nonfinite(const std::vector<double>& ep, const std::vector<double>& ed) {
        for (size_t b = 0; b < ep.size(); b++)
            if (!std::isfinite(ep[b]) || !std::isfinite(ed[b])) return true;
        return false;
    }

    // Per-iteration diagnostics (V2G_DIAG = every k outer iterations, written to
    // V2G_DIAG_FILE or stderr): per instance eps(p), eps(d), mu, this
    // iteration's CG count, |y|^2, |x|^2, |z|^2; per group the largest distance
    // of the projection's eigenvectors from orthonormal (max |V^T V - I| over the
    // large blocks, as the refinement found it) and the running counts of
    // block-Jacobi fallbacks and cold restarts.
    void diagnose(int it, const std::vector<CgScalars>& cs, const std::vector<double>& ep,
                  const std::vector<double>& ed, const std::vector<double>& mu) {
        std::vector<double> sums(3 * B_);
        const DevBuf<double>* vecs[3] = {&y_, &x_, &z_};
        const int64_t lens[3] = {nc_, nx_, nx_};
        for (int k = 0; k < 3; k++) {
            launch_reduce(RED_DOT, lens[k], B_, vecs[k]->p, vecs[k]->p, nullptr, nullptr, partial_.p, red_.p, s_);
            CK(cudaMemcpyAsync(&sums[k * B_], red_.p, B_ * sizeof(double), cudaMemcpyDeviceToHost, s_));
        }
        double gmax = 0.0;
        if (nlarge_ > 0) {
            std::vector<unsigned long long> g(nlarge_);
            CK(cudaMemcpyAsync(g.data(), gdev_.p, nlarge_ * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s_));
            CK(cudaStreamSynchronize(s_));
            for (auto v : g) {
                double d;
                std::memcpy(&d, &v, sizeof(d));
                gmax = std::max(gmax, d);
            }
        }
        CK(cudaStreamSynchronize(s_));
        std::FILE* f = diag_file_ ? diag_file_ : stderr;
        std::fprintf(f, "diag it %d group n=%lld B=%d gdev %.3e jacobi_blocks %ld restarts %ld oa_sweeps %ld\n", it,
                     (long long)nx_, B_, gmax, jacobi_blocks_, restarts_, oa_sweeps_);
        for (int b = 0; b < B_; b++)
            std::fprintf(f, "diag it %d b %d ep %.3e ed %.3e mu %.4f cg %d stalled %d y2 %.3e x2 %.3e z2 %.3e\n", it, b,
                         ep[b], ed[b], mu[b], cs[b].iter, cs[b].stalled, sums[b], sums[B_ + b], sums[2 * B_ + b]);
        std::fflush(f);
    }

    // Which of y, x, z (and the CG scalars) turned non-finite, on stderr, so
    // that a failing instance can be reproduced and traced alone.
    void report_nonfinite(int b, int oiter, double mu, long cg_iters) {
        double sums[3] = {0, 0, 0};
        const DevBuf<double>* vecs[3] = {&y_, &x_, &z_};
        const int64_t lens[3] = {nc_, nx_, nx_};
        for (int k = 0; k < 3; k++) {
            launch_reduce(RED_DOT, lens[k], B_, vecs[k]->p, vecs[k]->p, nullptr, nullptr, partial_.p, red_.p, s_);
            CK(cudaMemcpyAsync(&sums[k], red_.p + b, sizeof(double), cudaMemcpyDeviceToHost, s_));
            CK(cudaStreamSynchronize(s_));
        }
        std::fprintf(stderr,
                     "v2g: instance %d of a group of %d (dimx %lld) non-finite after outer iteration %d: "
                     "|y|^2 %g, |x|^2 %g, |z|^2 %g, mu %g, CG iterations %ld\n",
                     b, B_, (long long)nx_, oiter, sums[0], sums[1], sums[2], mu, cg_iters);
    }

    // Start for the instances with fs[b] set.  fs[b] = 1: the least-norm
    // feasible point, w solves A A^T w = b by the loop's CG (to 1e-10 ||b||),
    // x = A^T w, y = z = 0, mu = 1.  fs[b] = 2: the instance's x (a proposal)
    // moved onto A x = b the same way, x += A^T w with A A^T w = b - A x,
    // y = z = 0, mu = the problem's mu.  A x = b then holds to the CG
    // tolerance and the BPSDP iteration starts from a feasible primal with
    // zero duals.
    void feasible_start(const std::vector<int>& fs, std::vector<CgScalars>& cs) {
        std::vector<int> m1(B_), m2(B_), mall(B_);
        std::vector<double> coef(B_, 0.0), mu(B_);
        for (int b = 0; b < B_; b++) {
            m1[b] = fs[b] == 1;
            m2[b] = fs[b] == 2;
            mall[b] = fs[b] != 0;
            coef[b] = -1.0;
            mu[b] = P_[b]->mu;
        }
        CK(cudaMemcpyAsync(smask1_.p, m1.data(), B_ * sizeof(int), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(smask2_.p, m2.data(), B_ * sizeof(int), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(mask_.p, mall.data(), B_ * sizeof(int), cudaMemcpyHostToDevice, s_));
        CK(cudaMemcpyAsync(coef_.p, coef.data(), B_ * sizeof(double), cudaMemcpyHostToDevice, s_));
        double bn = 0.0;
        for (double v : T_.hb) bn += v * v;
        bn = std::sqrt(bn);
        for (int b = 0; b < B_; b++) {
            cs[b] = CgScalars{};
            cs[b].tol = 1e-10 * std::max(1.0, bn);
            cs[b].active = fs[b] != 0;
            cs[b].maxiter = P_[b]->opt.cg_maxiter;
        }
        CK(cudaMemcpyAsync(cs_.p, cs.data(), B_ * sizeof(CgScalars), cudaMemcpyHostToDevice, s_));
        launch_set_rows(nc_, B_, T_.b.p, bv_.p, smask1_.p, s_);  // right-hand side b
        // b - A x for the proposals
        launch_spmv(mA_, B_, x_.p, bv_.p, T_.b.p, coef_.p, nullptr, smask2_.p, s_);
        launch_set_rows(nc_, B_, nullptr, y_.p, mask_.p, s_);  // w starts at 0
        cg_solve();
        CK(cudaMemcpyAsync(cs.data(), cs_.p, B_ * sizeof(CgScalars), cudaMemcpyDeviceToHost, s_));
        launch_spmv(mAT_, B_, y_.p, x_.p, nullptr, nullptr, nullptr, smask1_.p, s_);
        launch_spmv(mAT_, B_, y_.p, x_.p, nullptr, nullptr, x_.p, smask2_.p, s_);
        launch_set_rows(nc_, B_, nullptr, y_.p, mask_.p, s_);
        launch_set_rows(nx_, B_, nullptr, z_.p, mask_.p, s_);
        std::vector<double> dmu(B_);
        CK(cudaMemcpyAsync(dmu.data(), mu_.p, B_ * sizeof(double), cudaMemcpyDeviceToHost, s_));
        CK(cudaStreamSynchronize(s_));
        for (int b = 0; b < B_; b++)
            if (fs[b]) dmu[b] = fs[b] == 2 ? mu[b] : 1.0;
        CK(cudaMemcpyAsync(mu_.p, dmu.data(), B_ * sizeof(double), cudaMemcpyHostToDevice, s_));
        CK(cudaStreamSynchronize(s_));
    }

    long jacobi_sweeps() const { return sweeps_total_; }
    long oa_sweeps() const { return oa_sweeps_; }
    long jacobi_blocks() const { return jacobi_blocks_; }
    long jacobi_unconverged() const { return jacobi_unconverged_; }
    long tc_projections() const { return tc_projections_; }
    double map_seconds() const { return map_sec_; }
    long map_launches() const { return map_n_; }
    double map_bytes() const { return map_bytes_; }
    double h2d_bytes() const { return 8.0 * B_ * (3.0 * nx_ + nc_); }
    double d2h_bytes() const { return 8.0 * B_ * (2.0 * nx_ + nc_); }

  private:
    // The autotuner of the map kernels: for this group's layout and instance
    // count, every variant of kMapVariants is timed on A and on A^T (CUDA
    // events around a few launches on the group's stream) and the fastest is
    // kept for the process (the choice depends only on layout and B).
    void tune_maps() {
        static std::mutex mu;
        static std::map<std::tuple<const void*, int, int>, int> chosen;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        for (int which = 0; which < 2; which++) {
            DevMap& M = which == 0 ? mA_ : mAT_;
            const auto key = std::make_tuple((const void*)M.rows, B_, which);
            {
                std::lock_guard<std::mutex> lk(mu);
                auto it = chosen.find(key);
                if (it != chosen.end()) {
                    M.variant = it->second;
                    continue;
                }
            }
            if (!e0) {
                CK(cudaEventCreate(&e0));
                CK(cudaEventCreate(&e1));
            }
            const double* in = which == 0 ? x_.p : y_.p;
            double* out = which == 0 ? ax_.p : aty_.p;
            float best = 0.f;
            int bestv = -1;
            for (int v = 0; v < kMapVariants; v++) {
                DevMap m = M;
                m.variant = v;
                launch_spmv(m, B_, in, out, nullptr, nullptr, nullptr, nullptr, s_);
                CK(cudaEventRecord(e0, s_));
                for (int k = 0; k < 5; k++) launch_spmv(m, B_, in, out, nullptr, nullptr, nullptr, nullptr, s_);
                CK(cudaEventRecord(e1, s_));
                CK(cudaEventSynchronize(e1));
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                if (bestv < 0 || ms < best) {
                    best = ms;
                    bestv = v;
                }
            }
            M.variant = bestv;
            std::lock_guard<std::mutex> lk(mu);
            chosen[key] = bestv;
        }
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }

    // Host -> device copies of per-iteration scalars go through pinned
    // staging memory: cudaMemcpyAsync from pageable memory first drains the
    // stream, which would stall the pipeline at every copy.  The ring restarts
    // after a stream synchronisation (stage_synced), or synchronises itself
    // when full.
    template <class T>
    void put(T* dst, const T* src, size_t n) {
        const size_t bytes = n * sizeof(T);
        if (bytes == 0) return;
        size_t off = (stage_off_ + 15) & ~(size_t)15;
        if (off + bytes > stage_cap_) {
            CK(cudaStreamSynchronize(s_));
            off = 0;
            if (bytes > stage_cap_) {
                CK(cudaFreeHost(stage_));
                stage_ = nullptr;
                stage_cap_ = bytes;
                CK(cudaMallocHost(&stage_, stage_cap_));
            }
        }
        std::memcpy(stage_ + off, src, bytes);
        CK(cudaMemcpyAsync(dst, stage_ + off, bytes, cudaMemcpyHostToDevice, s_));
        stage_off_ = off + bytes;
    }
    void stage_synced() { stage_off_ = 0; }

    // The projection's dense products: on all tiles of C (full) or on the
    // upper tiles of a symmetric C (sym, mirrored afterwards), in FP64 or, in
    // the mixed-precision phase (tc_), as 3xTF32 products on the tensor cores.
    // In the mixed phase only blocks padded to kMixedMinNp or more go to the
    // tensor cores; smaller ones gain nothing there (a few tiles each) and stay FP64.
    void gemm_full(const double* A, bool ta, const double* Bm, bool tb, const double* d, double* C, const int* mask) {
        if (tc_) {
            launch_tc_gemm(tc_plan_, false, A, ta, Bm, tb, d, C, mask, s_);
            launch_gemm(large_d_.p, lo_gtiles_.p, nlo_gtiles_, A, ta, Bm, tb, d, C, mask, s_);
        } else {
            launch_gemm(large_d_.p, gtiles_.p, ngtiles_, A, ta, Bm, tb, d, C, mask, s_);
        }
    }
    void gemm_sym(const double* A, bool ta, const double* Bm, bool tb, const double* d, double* C, const int* mask) {
        if (tc_) {
            launch_tc_gemm(tc_plan_, true, A, ta, Bm, tb, d, C, mask, s_);
            launch_gemm(large_d_.p, lo_stiles_.p, nlo_stiles_, A, ta, Bm, tb, d, C, mask, s_);
        } else {
            launch_gemm(large_d_.p, stiles_.p, nstiles_, A, ta, Bm, tb, d, C, mask, s_);
        }
    }

    // CG map launch with optional CUDA-event timing (profile mode).
    // With dotv, also red_[b] = sum dotv[., b] * out[., b].
    void map_launch(const DevMap& M, const double* in, double* out, const double* dotv = nullptr,
                    const int* mask = nullptr) {
        auto go = [&]() {
            if (dotv)
                launch_spmv_dot(M, B_, in, out, dotv, mask, partial_.p, red_.p, s_);
            else
                launch_spmv(M, B_, in, out, nullptr, nullptr, nullptr, mask, s_);
        };
        if (!profile_) {
            go();
            return;
        }
        if (prof_used_ + 2 > prof_ev_.size()) flush_profile();
        CK(cudaEventRecord(prof_ev_[prof_used_], s_));
        go();
        CK(cudaEventRecord(prof_ev_[prof_used_ + 1], s_));
        prof_used_ += 2;
        map_bytes_ += 8.0 * (double)(M.nrows + (M.nrows == nc_ ? nx_ : nc_)) * B_;
    }
    void flush_profile() {
        if (prof_used_ == 0) return;
        CK(cudaEventSynchronize(prof_ev_[prof_used_ - 1]));
        for (size_t i = 0; i + 1 < prof_used_; i += 2) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, prof_ev_[i], prof_ev_[i + 1]));
            map_sec_ += ms * 1e-3;
            map_n_++;
        }
        prof_used_ = 0;
    }
    // CGSolver::solve for every instance whose CG scalars are active.
    void cg_solve() {
        // Ap = A A^T y ; r = B - Ap ; p = r
        map_launch(mAT_, y_.p, atp_.p, nullptr, mask_.p);
        map_launch(mA_, atp_.p, ap_.p, nullptr, mask_.p);
        launch_cg_init(nc_, B_, bv_.p, ap_.p, r_.p, p_.p, cs_.p, s_);
        launch_reduce(RED_DOT, nc_, B_, r_.p, r_.p, nullptr, nullptr, partial_.p, red_.p, s_);
        launch_cg_set_rr(B_, cs_.p, red_.p, nact_.p, s_);
        // Small groups (outside profile mode): the whole solve in one
        // cooperative launch, the phases of each iteration separated by grid
        // barriers (maps.cu), one host synchronisation per solve
        if (!profile_ && loop_grid_ > 0) {
            int cap = 1;
            for (auto* p : P_) cap = std::max(cap, p->opt.cg_maxiter);
            cap += 2;
            CK(cudaMemsetAsync(loopbar_.p, 0, 2 * sizeof(unsigned int), s_));
            CK(launch_cg_loop(mA_, mAT_, B_, nc_, y_.p, r_.p, p_.p, atp_.p, ap_.p, cs_.p, partial_.p, looppart_.p,
                              loopbar_.p, reinterpret_cast<int*>(loopbar_.p + 1), nact_.p, nact_.p + 6, cap,
                              loop_grid_, s_));
            CK(cudaMemcpyAsync(hnact_, nact_.p, sizeof(int), cudaMemcpyDeviceToHost, s_));
            CK(cudaMemcpyAsync(hnact_ + 6, nact_.p + 6, sizeof(int), cudaMemcpyDeviceToHost, s_));
            CK(cudaMemcpyAsync(hnact_ + 7, loopbar_.p + 1, sizeof(int), cudaMemcpyDeviceToHost, s_));
            CK(cudaStreamSynchronize(s_));
            if (hnact_[7] != 0) throw CudaError("a grid barrier of the persistent CG did not complete (wait ran out)");
            cg_loop_iters_ += hnact_[6];
            if (hnact_[0] == 0) return;
        }
        // Outside profile mode the iterations run as a device-side loop: a
        // CUDA graph (captured once per group) whose WHILE node repeats one
        // CG iteration until no instance iterates, bounded by the largest
        // CG_MAXITER of the group, with one host synchronisation per solve.
        // Instances that converge earlier are masked by their scalars, so the
        // result is the same as iteration by iteration.
        if (!profile_ && cg_loop_ok_) {
            if (!cg_loop_exec_) capture_cg_loop();
            if (cg_loop_exec_) {
                CK(cudaMemsetAsync(nact_.p + 6, 0, sizeof(int), s_));
                CK(cudaGraphLaunch(cg_loop_exec_, s_));
                CK(cudaMemcpyAsync(hnact_, nact_.p, sizeof(int), cudaMemcpyDeviceToHost, s_));
                CK(cudaMemcpyAsync(hnact_ + 6, nact_.p + 6, sizeof(int), cudaMemcpyDeviceToHost, s_));
                CK(cudaStreamSynchronize(s_));
                g_kernel_launches.fetch_add(cg_loop_nodes_ * (long)hnact_[6], std::memory_order_relaxed);
                if (hnact_[0] == 0) return;
            }
        }
        // Otherwise (and should the loop stop at its cap with an instance still
        // iterating) chunks of kCgChunk iterations, a CUDA graph outside
        // profile mode, with the host looking at the count of instances still
        // iterating after each chunk
        while (true) {
            if (!profile_) {
                if (!cg_exec_) capture_cg_chunk();
                CK(cudaGraphLaunch(cg_exec_, s_));
                g_kernel_launches.fetch_add(cg_chunk_nodes_, std::memory_order_relaxed);
            } else {
                for (int k = 0; k < kCgChunk; k++) cg_iteration();
            }
            CK(cudaMemcpyAsync(hnact_, nact_.p, sizeof(int), cudaMemcpyDeviceToHost, s_));
            CK(cudaStreamSynchronize(s_));
            if (hnact_[0] == 0) break;
        }
        if (profile_) flush_profile();
    }

    static constexpr int kCgChunk = 4;
    // One CG iteration (cg_solver.cc:141-177) for every instance whose scalars are active.
    void cg_iteration() {
        map_launch(mAT_, p_.p, atp_.p, nullptr, mask_.p);
        map_launch(mA_, atp_.p, ap_.p, p_.p, mask_.p);  // Ap and p.Ap (into red_)
        launch_cg_step(nc_, B_, y_.p, r_.p, p_.p, ap_.p, cs_.p, red_.p, partial_.p, nact_.p, s_);
        launch_cg_update_p(nc_, B_, p_.p, r_.p, cs_.p, s_);
    }
    // kCgChunk CG iterations captured from the stream into a graph: the
    // kernels' arguments are the group's fixed buffers, so one capture serves
    // every CG solve of the group.
    void capture_cg_chunk() {
        CK(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < kCgChunk; k++) cg_iteration();
        cudaGraph_t g = nullptr;
        CK(cudaStreamEndCapture(s_, &g));
        size_t nodes = 0;
        CK(cudaGraphGetNodes(g, nullptr, &nodes));
        // the launchers counted the captured kernels as launches; graph
        // launches are counted per replay instead
        g_kernel_launches.fetch_sub((long)nodes, std::memory_order_relaxed);
        cg_chunk_nodes_ = (long)nodes;
        const cudaError_t e = cudaGraphInstantiate(&cg_exec_, g, 0);
        cudaGraphDestroy(g);
        CK(e);
    }

    // One CG iteration and its loop condition captured as the body of a WHILE
    // node (conditional graph nodes); if the runtime refuses the conditional
    // node, the chunked graph serves instead.
    void capture_cg_loop() {
        int cap = 1;
        for (auto* p : P_) cap = std::max(cap, p->opt.cg_maxiter);
        cap += 2;  // the scalars stop every instance at its CG_MAXITER before this
        cudaGraph_t g = nullptr;
        CK(cudaGraphCreate(&g, 0));
        cudaGraphConditionalHandle h{};
        cudaGraphNodeParams cp{};
        cudaGraphNode_t node = nullptr;
        if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphDestroy(g);
            cg_loop_ok_ = false;
            return;
        }
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        if (cudaGraphAddNode(&node, g, nullptr, 0, &cp) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphDestroy(g);
            cg_loop_ok_ = false;
            return;
        }
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CK(cudaStreamBeginCaptureToGraph(s_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        cg_iteration();
        launch_cg_while(h, nact_.p, nact_.p + 6, cap, s_);
        cudaGraph_t captured = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(s_, &captured);
        size_t nodes = 0;
        if (ce == cudaSuccess) cudaGraphGetNodes(body, nullptr, &nodes);
        // the launchers counted the captured kernels; replays are counted per iteration
        g_kernel_launches.fetch_sub((long)nodes, std::memory_order_relaxed);
        cg_loop_nodes_ = (long)nodes;
        const cudaError_t ie = ce == cudaSuccess ? cudaGraphInstantiate(&cg_loop_exec_, g, 0) : ce;
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            cudaGetLastError();
            cg_loop_exec_ = nullptr;
            cg_loop_ok_ = false;
        }
    }

    // Jacobi: relative off-diagonal norm 1e-13 or the absolute rho share of
    // the block; refinement: max |E| <= 1e-7 or residual (~max|E|^2 scale)
    // below the block's rho share.
    void set_block_tolerances(const std::vector<double>& rho) {
        std::vector<int> nblk(B_, 0);
        for (int t = 0; t < nlarge_; t++) nblk[hlarge_[t].inst]++;
        std::vector<double> jt(nlarge_, 1e-13), ot(nlarge_, 1e-7), at(nlarge_, 0.0);
        for (int t = 0; t < nlarge_; t++) {
            const int b = hlarge_[t].inst;
            if (!rho.empty() && rho[b] > 0.0) at[t] = rho[b] / std::sqrt((double)nblk[b]);
        }
        // a fallback block of an instance still far from the solution takes one
        // warm sweep per outer iteration; the next iteration continues from it
        std::vector<int> ms(nlarge_, 1 << 20);
        cap_ = false;
        for (int t = 0; t < nlarge_; t++) {
            const int b = hlarge_[t].inst;
            if (!rho.empty() && rho[b] >= 1e-4) {
                ms[t] = 1;
                cap_ = true;
            }
        }
        put(msw_.p, ms.data(), nlarge_);
        put(jtol_.p, jt.data(), nlarge_);
        put(otol_.p, ot.data(), nlarge_);
        put(atol_.p, at.data(), nlarge_);
    }

    void set_block_masks() {
        // bact[t] = mask[inst(t)], on the device (no round trip through the host)
        launch_block_mask(large_d_.p, nlarge_, mask_.p, bact_.p, s_);
    }

    void build_projection_plan() {
        const Layout& L = T_.L;
        std::vector<BlockTask> small;
        int64_t woff = 0, qoff = 0, doff = 0, soff = 0;
        for (int b = 0; b < B_; b++)
            for (size_t k = 0; k < L.block_dims.size(); k++) {
                const int n = L.block_dims[k];
                if (n == 0) continue;
                BlockTask t{};
                t.xoff = L.block_off[k];
                t.n = n;
                t.inst = b;
                if (n <= 64) {
                    t.woff = soff;  // its kept eigenvectors
                    soff += (int64_t)n * n;
                    small.push_back(t);
                    continue;
                }
                t.np = (n + 63) / 64 * 64;
                t.nb = t.np / 32;
                t.woff = woff;
                t.qoff = qoff;
                t.doff = doff;
                woff += (int64_t)t.np * t.np;
                qoff += (int64_t)(t.nb / 2) * 4096;
                doff += t.np;
                hlarge_.push_back(t);
            }
        nsmall_ = (int)small.size();
        nlarge_ = (int)hlarge_.size();
        small_d_.upload(small.data(), small.size());
        vsmall_.alloc(std::max<int64_t>(soff, 1));
        large_d_.upload(hlarge_.data(), hlarge_.size());
        if (nlarge_ == 0) return;
        U_.alloc(woff);
        W_.alloc(woff);
        V_.alloc(woff);
        Tm_.alloc(woff);
        G_.alloc(woff);
        M_.alloc(woff);
        Q_.alloc(qoff);
        qskip_.alloc(qoff / 4096);
        pthr_.alloc(nlarge_);
        dw_.alloc(doff);
        dz_.alloc(doff);
        jtol_.alloc(nlarge_);
        otol_.alloc(nlarge_);
        atol_.alloc(nlarge_);
        msw_.alloc(nlarge_);
        lam_.alloc(doff);
        erow_.alloc(doff);
        restart_.alloc(nlarge_);
        rowsum_.alloc(2 * doff);
        partner_.alloc(doff);
        scale_.alloc(nlarge_);
        emax_.alloc(nlarge_);
        gdev_.alloc(nlarge_);
        hard_.alloc(nlarge_);
        bact_.alloc(nlarge_);
        bwork_.alloc(nlarge_);
        bref_.alloc(nlarge_);
        bupd_.alloc(nlarge_);
        bjac_.alloc(nlarge_);
        std::vector<GemmTile> gt, st;
        std::vector<PairTask> pt;
        std::vector<WTileTask> wt;
        std::vector<VTileTask> vt;
        for (int ti = 0; ti < nlarge_; ti++) {
            const BlockTask& t = hlarge_[ti];
            const int nt = t.np / 64, npair = t.nb / 2;
            max_np_ = std::max(max_np_, t.np);
            max_n_ = std::max(max_n_, t.n);
            max_rounds_ = std::max(max_rounds_, t.nb - 1);
            for (int i = 0; i < nt; i++)
                for (int j = 0; j < nt; j++) {
                    gt.push_back({ti, i, j});
                    if (i <= j) st.push_back({ti, i, j});
                }
            for (int k = 0; k < npair; k++) pt.push_back({ti, k});
            for (int k1 = 0; k1 < npair; k1++)
                for (int k2 = 0; k2 < npair; k2++) wt.push_back({ti, k1, k2});
            for (int ch = 0; ch < nt; ch++)
                for (int k = 0; k < npair; k++) vt.push_back({ti, ch, k});
        }
        gtiles_.upload(gt.data(), gt.size());
        stiles_.upload(st.data(), st.size());
        // 128 x 64 tiles of the tensor-core GEMM; the symmetric products need
        // every 64 x 64 upper tile, i.e. 128-row tile ti with 64-column tile tj >= 2 ti
        // 128 x 128 tiles of the tensor-core GEMM (blocks padded to kMixedMinNp or
        // more); the symmetric products need every 64 x 64 upper tile, which the
        // 128-tiles ti <= tj cover; blocks below kMixedMinNp keep FP64 tiles in
        // the mixed phase
        std::vector<GemmTile> tg, ts, lg, ls;
        std::vector<TcSplit> sp;
        int64_t toff = 0;
        for (int ti = 0; ti < nlarge_; ti++) {
            BlockTask& t = hlarge_[ti];
            if (t.np < kMixedMinNp) {
                const int nt = t.np / 64;
                for (int i = 0; i < nt; i++)
                    for (int j = 0; j < nt; j++) {
                        lg.push_back({ti, i, j});
                        if (i <= j) ls.push_back({ti, i, j});
                    }
                continue;
            }
            t.toff = toff;
            toff += tc_split_words(t.np);
            const int nr = (t.np + 127) / 128;
            for (int i = 0; i < nr; i++) {
                sp.push_back({ti, i});
                for (int j = 0; j < nr; j++) {
                    tg.push_back({ti, i, j});
                    if (i <= j) ts.push_back({ti, i, j});
                }
            }
        }
        if (toff > 0) {
            large_d_.upload(hlarge_.data(), hlarge_.size());  // with the split offsets
            tcwa_.alloc(toff);
            tcwb_.alloc(toff);
        }
        tc_gtiles_.upload(tg.data(), tg.size());
        tc_stiles_.upload(ts.data(), ts.size());
        tc_split_.upload(sp.data(), sp.size());
        lo_gtiles_.upload(lg.data(), lg.size());
        lo_stiles_.upload(ls.data(), ls.size());
        ntc_gtiles_ = (int)tg.size();
        nlo_gtiles_ = (int)lg.size();
        nlo_stiles_ = (int)ls.size();
        tc_plan_.tasks = large_d_.p;
        tc_plan_.tiles_full = tc_gtiles_.p;
        tc_plan_.tiles_sym = tc_stiles_.p;
        tc_plan_.n_full = (int)tg.size();
        tc_plan_.n_sym = (int)ts.size();
        tc_plan_.split = tc_split_.p;
        tc_plan_.nsplit = (int)sp.size();
        for (const auto& u : sp) tc_plan_.max_nk = std::max(tc_plan_.max_nk, hlarge_[u.task].np / 32);
        tc_plan_.wa = tcwa_.p;
        tc_plan_.wb = tcwb_.p;
        nstiles_ = (int)st.size();
        pairs_.upload(pt.data(), pt.size());
        wtiles_.upload(wt.data(), wt.size());
        vtiles_.upload(vt.data(), vt.size());
        ngtiles_ = (int)gt.size();
        npairs_ = (int)pt.size();
        nwtiles_ = (int)wt.size();
        nvtiles_ = (int)vt.size();
    }

    DeviceTables& T_;
    DevMap mA_, mAT_;  // the group's copies of the maps, with the tuned kernel variant
    std::vector<Problem*> P_;
    int B_;
    int64_t nx_ = 0, nc_ = 0;
    cudaStream_t s_ = nullptr;
    cudaStream_t s_small_ = nullptr;  // the small blocks' projection, beside the large blocks'
    cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
    DevBuf<double> c_, x_, z_, aty_, atp_, y_, ax_, bv_, r_, p_, ap_, partial_, red_, mu_, coef_;
    DevBuf<int> mask_, nact_, smask1_, smask2_;
    DevBuf<CgScalars> cs_;
    // CG start extrapolation (cg_extrapolate): the previous CG start and the
    // per-instance mode of the extrapolation kernel
    DevBuf<double> yprev_;
    DevBuf<int> ex_;
    bool extrapolate_ = false;
    // Anderson acceleration (anderson_memory): the saved state w, the previous
    // f and g, the difference columns, and the per-instance modes, slots,
    // mixing flags and coefficients; aa_m_ = columns allocated (the largest
    // memory of the group)
    int aa_m_ = 0;
    DevBuf<double> aw_, af_, ag_, adF_, adG_, agam_, apart_, adots_;
    DevBuf<int> amode_, aslot_, amix_;
    double* hscal_ = nullptr;
    int* hnact_ = nullptr;
    char* stage_ = nullptr;
    size_t stage_cap_ = 0, stage_off_ = 0;
    CgScalars* hcs_ = nullptr;  // pinned copy of the CG scalars after a CG solve
    double* hdots_ptr_ = nullptr;  // pinned Anderson dot products
    std::vector<double> hdots_;
    // projection plan
    std::vector<BlockTask> hlarge_;
    DevBuf<BlockTask> small_d_, large_d_;
    int nsmall_ = 0, nlarge_ = 0, max_np_ = 0, max_n_ = 0, max_rounds_ = 0;
    DevBuf<double> U_, W_, V_, Tm_, G_, M_, Q_, dw_, dz_, lam_, scale_, jtol_, otol_, atol_, rowsum_, erow_;
    DevBuf<unsigned long long> emax_, gdev_;
    DevBuf<int> hard_, bact_, bwork_, bref_, bupd_, bjac_, partner_, msw_, restart_, qskip_;
    DevBuf<double> pthr_;
    long restarts_ = 0;
    bool cap_ = false;
    long oa_sweeps_ = 0, jacobi_blocks_ = 0, jacobi_unconverged_ = 0;
    DevBuf<GemmTile> gtiles_, stiles_, tc_gtiles_, tc_stiles_, lo_gtiles_, lo_stiles_;
    int ntc_gtiles_ = 0, nlo_gtiles_ = 0, nlo_stiles_ = 0;
    DevBuf<TcSplit> tc_split_;
    DevBuf<uint32_t> tcwa_, tcwb_;  // the split operands of the tensor-core products
    TcPlan tc_plan_;
    bool tc_ = false;  // this projection's dense products on the tensor cores
    long tc_projections_ = 0;
    DevBuf<PairTask> pairs_;
    DevBuf<WTileTask> wtiles_;
    DevBuf<VTileTask> vtiles_;
    int ngtiles_ = 0, nstiles_ = 0, npairs_ = 0, nwtiles_ = 0, nvtiles_ = 0;
    bool warm_ = false;
    // kept eigenvectors of the small blocks (warm Jacobi starts)
    static constexpr long kSmallCold = 64;
    DevBuf<double> vsmall_;
    bool small_warm_ = false;
    long nproj_ = 0;
    long sweeps_total_ = 0;
    // the captured CG chunk
    cudaGraphExec_t cg_exec_ = nullptr;
    long cg_chunk_nodes_ = 0;
    // the persistent CG (small groups): cooperative grid size (0: not used),
    // barrier counter and error flag, per-CTA partials of r.r
    int loop_grid_ = 0;
    DevBuf<unsigned int> loopbar_;
    DevBuf<double> looppart_;
    long cg_loop_iters_ = 0;
    cudaGraphExec_t cg_loop_exec_ = nullptr;  // the device-side CG loop (WHILE node)
    long cg_loop_nodes_ = 0;
    bool cg_loop_ok_ = true;
    // diagnostics (V2G_DIAG)
    int diag_every_ = 0;
    std::FILE* diag_file_ = nullptr;
    // profile mode
    bool profile_ = false;
    std::vector<cudaEvent_t> prof_ev_;
    size_t prof_used_ = 0;
    double map_sec_ = 0.0, map_bytes_ = 0.0;
    long map_n_ = 0;
};

thread_local v2g_batch_stats g_stats{};

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

template <class F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const NoDevice& e) {
        return fail(V2G_ERR_NO_DEVICE, e.what());
    } catch (const CudaError& e) {
        return fail(V2G_ERR_CUDA, e.what());
    } catch (const std::invalid_argument& e) {
        return fail(V2G_ERR_ARG, e.what());
    } catch (const std::exception& e) {
        return fail(V2G_ERR_ARG, e.what());
    }
}

void require_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw NoDevice("no CUDA device visible");
}

}  // namespace
}  // namespace v2g

using v2g::Problem;

struct v2g_handle {
    Problem P;
};

extern "C" {

void v2g_default_options(v2g_options* o) {
    o->positivity = "DQG";
    o->constrain_spin = 1;
    o->constrain_sz = 1;
    o->r_convergence = 1e-4;
    o->e_convergence = 1e-4;
    o->cg_convergence = 1e-9;
    o->maxiter = 10000;
    o->cg_maxiter = 10000;
    o->tau_parameter = 1.0;
    o->mu_update_frequency = 500;
    o->device = 0;
    o->record_trace = 0;
    o->profile = 0;
    o->adaptive_projection = 0;
    o->cg_tolerance_factor = 0.01;
    o->spin_adapt_q2 = 0;
    o->spin_adapt_g2 = 0;
    o->constrain_d3 = 0;
    o->constrain_d4 = 0;
    o->start = 0;
    o->cg_extrapolate = 0;
    o->anderson_memory = 0;
    o->mixed_precision = 0;
}

const char* v2g_last_error(void) { return v2g::g_last_error.c_str(); }

int v2g_create(const v2g_options* opt, int nirrep, const int* frzcpi, const int* rstcpi, const int* amopi,
               const int* rstvpi, const int* frzvpi, int nalpha, int nbeta, int multiplicity, v2g_handle** out) {
    return v2g::guarded([&]() -> int {
        if (!opt || !amopi || !out) return v2g::fail(V2G_ERR_ARG, "null argument");
        *out = nullptr;
        v2g::Options o;
        if (!v2g::parse_positivity(opt->positivity ? opt->positivity : "", o))
            return v2g::fail(V2G_ERR_ARG, "unknown POSITIVITY");
        o.constrain_spin = opt->constrain_spin != 0;
        o.constrain_sz = opt->constrain_sz != 0;
        o.r_convergence = opt->r_convergence;
        o.e_convergence = opt->e_convergence;
        o.cg_convergence = opt->cg_convergence;
        o.maxiter = opt->maxiter;
        o.cg_maxiter = opt->cg_maxiter;
        o.tau = opt->tau_parameter;
        o.mu_update_frequency = opt->mu_update_frequency;
        o.adaptive_projection = opt->adaptive_projection != 0;
        o.cg_tol_factor = opt->cg_tolerance_factor;
        o.spin_adapt_q2 = opt->spin_adapt_q2 != 0;
        o.spin_adapt_g2 = opt->spin_adapt_g2 != 0;
        o.constrain_d4 = opt->constrain_d4 != 0;
        o.constrain_d3 = opt->constrain_d3 != 0 || o.constrain_d4;  // v2rdm_solver.cc:527-532
        if (opt->start < 0 || opt->start > 2) return v2g::fail(V2G_ERR_ARG, "start must be 0, 1 or 2");
        o.feasible_start = opt->start == 1;
        o.proposal_start = opt->start == 2;
        if (opt->cg_extrapolate != 0 && opt->cg_extrapolate != 1)
            return v2g::fail(V2G_ERR_ARG, "cg_extrapolate must be 0 or 1");
        o.cg_extrapolate = opt->cg_extrapolate == 1;
        if (opt->anderson_memory < 0 || opt->anderson_memory > v2g::kAndersonMax)
            return v2g::fail(V2G_ERR_ARG, "anderson_memory must be in 0..16");
        o.anderson_memory = opt->anderson_memory;
        if (opt->mixed_precision != 0 && opt->mixed_precision != 1)
            return v2g::fail(V2G_ERR_ARG, "mixed_precision must be 0 or 1");
        o.mixed_precision = opt->mixed_precision == 1;
        if (!(o.cg_tol_factor > 0.0 && o.cg_tol_factor < 1.0))
            return v2g::fail(V2G_ERR_ARG, "cg_tolerance_factor must be in (0, 1)");
        if (o.maxiter < 1 || o.cg_maxiter < 1 || o.mu_update_frequency < 1)
            return v2g::fail(V2G_ERR_ARG, "iteration limits must be positive");
        auto h = std::make_unique<v2g_handle>();
        Problem& P = h->P;
        P.opt = o;
        P.device = opt->device;
        P.record_trace = opt->record_trace != 0;
        P.profile = opt->profile != 0;
        std::vector<int> z(nirrep, 0);
        auto arr = [&](const int* a) { return a ? std::vector<int>(a, a + nirrep) : z; };
        P.sp.frzcpi = arr(frzcpi);
        P.sp.rstcpi = arr(rstcpi);
        P.sp.amopi = arr(amopi);
        P.sp.rstvpi = arr(rstvpi);
        P.sp.frzvpi = arr(frzvpi);
        int core = 0;
        for (int hh = 0; hh < nirrep; hh++) core += P.sp.frzcpi[hh] + P.sp.rstcpi[hh];
        const double na = nalpha - core, nb = nbeta - core;
        std::string err = v2g::build_layout(o, nirrep, P.sp.amopi, na, nb, multiplicity, P.L);
        if (!err.empty()) return v2g::fail(V2G_ERR_ARG, err);
        P.c.assign(P.L.dimx, 0.0);
        P.x.assign(P.L.dimx, 0.0);
        P.z.assign(P.L.dimx, 0.0);
        P.y.assign(P.L.ncon, 0.0);
        *out = h.release();
        return V2G_OK;
    });
}

void v2g_destroy(v2g_handle* h) { delete h; }

long v2g_dimx(const v2g_handle* h) { return h ? (long)h->P.L.dimx : -1; }
long v2g_nconstraints(const v2g_handle* h) { return h ? (long)h->P.L.ncon : -1; }
int v2g_nblocks(const v2g_handle* h) { return h ? (int)h->P.L.block_dims.size() : -1; }
int v2g_block_dims(const v2g_handle* h, int* dims) {
    if (!h || !dims) return V2G_ERR_ARG;
    for (size_t i = 0; i < h->P.L.block_dims.size(); i++) dims[i] = h->P.L.block_dims[i];
    return V2G_OK;
}

int v2g_set_hamiltonian(v2g_handle* h, const double* oei, const double* qmo, int nq, double enuc) {
    return v2g::guarded([&]() -> int {
        if (!h || !oei || (!qmo && nq > 0) || nq < 0) return v2g::fail(V2G_ERR_ARG, "bad integral arguments");
        Problem& P = h->P;
        std::string err = v2g::build_c(P.L, P.sp, oei, qmo, nq, P.c, P.efzc);
        if (!err.empty()) return v2g::fail(V2G_ERR_ARG, err);
        P.enuc = enuc;
        P.have_c = true;
        P.hmat.clear();
        P.Lq.clear();
        P.nq = 0;
        int other = 0;
        for (int hh = 0; hh < P.L.nirrep; hh++)
            other += P.sp.frzcpi[hh] + P.sp.rstcpi[hh] + P.sp.rstvpi[hh] + P.sp.frzvpi[hh];
        if (P.L.nirrep == 1 && other == 0) {
            const int n = P.L.amo;
            const size_t ntri = (size_t)n * (n + 1) / 2;
            P.hmat.assign((size_t)n * n, 0.0);
            P.Lq.assign((size_t)nq * n * n, 0.0);
            for (int p = 0; p < n; p++)
                for (int q = 0; q <= p; q++) {
                    const size_t t = (size_t)p * (p + 1) / 2 + q;  // INDEX(p, q)
                    P.hmat[p * n + q] = P.hmat[q * n + p] = oei[t];
                    for (int Q = 0; Q < nq; Q++)
                        P.Lq[((size_t)Q * n + p) * n + q] = P.Lq[((size_t)Q * n + q) * n + p] = qmo[Q * ntri + t];
                }
            P.nq = nq;
        }
        return V2G_OK;
    });
}

int v2g_get_c(const v2g_handle* h, double* c) {
    if (!h || !c) return V2G_ERR_ARG;
    std::copy(h->P.c.begin(), h->P.c.end(), c);
    return V2G_OK;
}

int v2g_get_b(const v2g_handle* h, double* b) {
    if (!h || !b) return V2G_ERR_ARG;
    std::vector<double> bb;
    v2g::build_b(h->P.L, bb);
    std::copy(bb.begin(), bb.end(), b);
    return V2G_OK;
}

double v2g_efzc(const v2g_handle* h) { return h ? h->P.efzc : 0.0; }

int v2g_guess_random(v2g_handle* h) {
    if (!h) return V2G_ERR_ARG;
    Problem& P = h->P;
    // v2rdm_solver.cc:2479-2490: srand(0); x_i, z_i interleaved, then y
    srand(0);
    for (int64_t i = 0; i < P.L.dimx; i++) {
        P.x[i] = ((double)rand() / RAND_MAX - 1.0) * 2.0;
        P.z[i] = ((double)rand() / RAND_MAX - 1.0) * 2.0;
    }
    for (int64_t i = 0; i < P.L.ncon; i++) P.y[i] = ((double)rand() / RAND_MAX - 1.0) * 2.0;
    P.mu = 1.0;
    P.proposal = false;
    return V2G_OK;
}

int v2g_set_state(v2g_handle* h, const double* x, const double* y, const double* z, double mu) {
    if (!h || !x || !y || !z || !(mu > 0.0)) return V2G_ERR_ARG;
    Problem& P = h->P;
    std::copy(x, x + P.L.dimx, P.x.begin());
    std::copy(z, z + P.L.dimx, P.z.begin());
    std::copy(y, y + P.L.ncon, P.y.begin());
    P.mu = mu;
    P.proposal = false;
    return V2G_OK;
}

// Checkpoint file: the entries of WriteCheckpointFile (checkpoint.cc:56-88),
// "MU", "PRIMAL", "DUAL 1", "DUAL 2", as named records in a small container of
// our own (Psi4's PSIO container is not reproduced):
//   magic "V2GCKPT1", int64 record count, then per record an 80-byte
//   zero-padded key, an int64 byte length and the bytes.
// A "LAYOUT" record (dimx, nconstraints) guards against restarting a
// different problem.
namespace {
const char kCkptMagic[8] = {'V', '2', 'G', 'C', 'K', 'P', 'T', '1'};

void ckpt_put(std::FILE* f, const char* key, const void* data, int64_t bytes) {
    char k[80] = {};
    std::strncpy(k, key, sizeof(k) - 1);
    if (std::fwrite(k, 1, sizeof(k), f) != sizeof(k) || std::fwrite(&bytes, sizeof(bytes), 1, f) != 1 ||
        (bytes > 0 && std::fwrite(data, 1, (size_t)bytes, f) != (size_t)bytes))
        throw std::invalid_argument("checkpoint write failed");
}
}  // namespace

int v2g_write_checkpoint(const v2g_handle* h, const char* path) {
    return v2g::guarded([&]() -> int {
        if (!h || !path) return v2g::fail(V2G_ERR_ARG, "null argument");
        const Problem& P = h->P;
        std::FILE* f = std::fopen(path, "wb");
        if (!f) return v2g::fail(V2G_ERR_ARG, std::string("cannot open ") + path + " for writing");
        try {
            const int64_t n = 5;
            const int64_t layout[2] = {P.L.dimx, P.L.ncon};
            if (std::fwrite(kCkptMagic, 1, 8, f) != 8 || std::fwrite(&n, sizeof(n), 1, f) != 1)
                throw std::invalid_argument("checkpoint write failed");
            ckpt_put(f, "LAYOUT", layout, sizeof(layout));
            ckpt_put(f, "MU", &P.mu, sizeof(double));
            ckpt_put(f, "PRIMAL", P.x.data(), (int64_t)P.x.size() * 8);
            ckpt_put(f, "DUAL 1", P.y.data(), (int64_t)P.y.size() * 8);
            ckpt_put(f, "DUAL 2", P.z.data(), (int64_t)P.z.size() * 8);
        } catch (...) {
            std::fclose(f);
            throw;
        }
        if (std::fclose(f) != 0) return v2g::fail(V2G_ERR_ARG, "checkpoint write failed");
        return V2G_OK;
    });
}

int v2g_read_checkpoint(v2g_handle* h, const char* path) {
    return v2g::guarded([&]() -> int {
        if (!h || !path) return v2g::fail(V2G_ERR_ARG, "null argument");
        Problem& P = h->P;
        std::FILE* f = std::fopen(path, "rb");
        if (!f) return v2g::fail(V2G_ERR_ARG, std::string("cannot open ") + path);
        std::map<std::string, std::vector<char>> rec;
        bool ok = true;
        char magic[8];
        int64_t n = 0;
        ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kCkptMagic, 8) == 0 &&
             std::fread(&n, sizeof(n), 1, f) == 1 && n >= 0 && n < 64;
        for (int64_t i = 0; ok && i < n; i++) {
            char k[81] = {};
            int64_t bytes = 0;
            ok = std::fread(k, 1, 80, f) == 80 && std::fread(&bytes, sizeof(bytes), 1, f) == 1 && bytes >= 0 &&
                 bytes <= (int64_t)1 << 40;
            if (!ok) break;
            std::vector<char> buf((size_t)bytes);
            ok = bytes == 0 || std::fread(buf.data(), 1, (size_t)bytes, f) == (size_t)bytes;
            rec[std::string(k)] = std::move(buf);
        }
        std::fclose(f);
        if (!ok) return v2g::fail(V2G_ERR_ARG, std::string(path) + " is not a v2g checkpoint file");
        for (const char* k : {"LAYOUT", "MU", "PRIMAL", "DUAL 1", "DUAL 2"})
            if (!rec.count(k)) return v2g::fail(V2G_ERR_ARG, std::string("checkpoint lacks the entry ") + k);
        int64_t layout[2];
        if (rec["LAYOUT"].size() != sizeof(layout)) return v2g::fail(V2G_ERR_ARG, "bad LAYOUT entry");
        std::memcpy(layout, rec["LAYOUT"].data(), sizeof(layout));
        if (layout[0] != P.L.dimx || layout[1] != P.L.ncon)
            return v2g::fail(V2G_ERR_ARG, "checkpoint belongs to a different layout (dimx " + std::to_string(layout[0]) +
                                              ", nconstraints " + std::to_string(layout[1]) + ")");
        if (rec["MU"].size() != 8 || rec["PRIMAL"].size() != (size_t)P.L.dimx * 8 ||
            rec["DUAL 1"].size() != (size_t)P.L.ncon * 8 || rec["DUAL 2"].size() != (size_t)P.L.dimx * 8)
            return v2g::fail(V2G_ERR_ARG, "checkpoint entry sizes do not match the layout");
        std::memcpy(&P.mu, rec["MU"].data(), 8);
        P.x.resize(P.L.dimx);
        P.y.resize(P.L.ncon);
        P.z.resize(P.L.dimx);
        std::memcpy(P.x.data(), rec["PRIMAL"].data(), rec["PRIMAL"].size());
        std::memcpy(P.y.data(), rec["DUAL 1"].data(), rec["DUAL 1"].size());
        std::memcpy(P.z.data(), rec["DUAL 2"].data(), rec["DUAL 2"].size());
        return V2G_OK;
    });
}

int v2g_get_state(const v2g_handle* h, double* x, double* y, double* z, double* mu) {
    if (!h) return V2G_ERR_ARG;
    const Problem& P = h->P;
    if (x) std::copy(P.x.begin(), P.x.end(), x);
    if (y) std::copy(P.y.begin(), P.y.end(), y);
    if (z) std::copy(P.z.begin(), P.z.end(), z);
    if (mu) *mu = P.mu;
    return V2G_OK;
}

static int apply_map(v2g_handle* h, const double* u, double* out, bool transpose, bool device_ptrs) {
    return v2g::guarded([&]() -> int {
        if (!h || !u || !out) return v2g::fail(V2G_ERR_ARG, "null argument");
        v2g::require_device();
        Problem& P = h->P;
        v2g::DeviceTables& T = P.tables();
        CK(cudaSetDevice(T.device));
        const int64_t nin = transpose ? P.L.ncon : P.L.dimx, nout = transpose ? P.L.dimx : P.L.ncon;
        const v2g::DevMap& M = transpose ? T.AT() : T.A();
        if (device_ptrs) {
            v2g::launch_spmv(M, 1, u, out, nullptr, nullptr, nullptr, nullptr, 0);
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(0));
            return V2G_OK;
        }
        v2g::DevBuf<double> din, dout(nout);
        din.upload(u, nin);
        v2g::launch_spmv(M, 1, din.p, dout.p, nullptr, nullptr, nullptr, nullptr, 0);
        CK(cudaGetLastError());
        CK(cudaMemcpy(out, dout.p, nout * sizeof(double), cudaMemcpyDeviceToHost));
        return V2G_OK;
    });
}

int v2g_apply_A(v2g_handle* h, const double* u, double* out) { return apply_map(h, u, out, false, false); }
int v2g_apply_AT(v2g_handle* h, const double* u, double* out) { return apply_map(h, u, out, true, false); }
int v2g_apply_A_device(v2g_handle* h, const double* u, double* out) { return apply_map(h, u, out, false, true); }
int v2g_apply_AT_device(v2g_handle* h, const double* u, double* out) { return apply_map(h, u, out, true, true); }

static int apply_batched(v2g_handle* h, int nvec, const double* u, double* out, void* stream, bool transpose) {
    return v2g::guarded([&]() -> int {
        if (!h || !u || !out || nvec < 1 || nvec > 256) return v2g::fail(V2G_ERR_ARG, "bad batched map arguments");
        v2g::require_device();
        v2g::DeviceTables& T = h->P.tables();
        CK(cudaSetDevice(T.device));
        v2g::launch_spmv(transpose ? T.AT() : T.A(), nvec, u, out, nullptr, nullptr, nullptr, nullptr,
                         (cudaStream_t)stream);
        CK(cudaGetLastError());
        return V2G_OK;
    });
}

int v2g_apply_A_batched_device(v2g_handle* h, int nvec, const double* u, double* out, void* stream) {
    return apply_batched(h, nvec, u, out, stream, false);
}
int v2g_apply_AT_batched_device(v2g_handle* h, int nvec, const double* u, double* out, void* stream) {
    return apply_batched(h, nvec, u, out, stream, true);
}

int v2g_set_active_orbital_energies(v2g_handle* h, const double* energies) {
    return v2g::guarded([&]() -> int {
        if (!h || !energies) return v2g::fail(V2G_ERR_ARG, "null argument");
        Problem& P = h->P;
        std::vector<int> order(P.L.amo);
        for (int i = 0; i < P.L.amo; i++) order[i] = i;
        // the reference takes the first strict minimum (basis.cc:211-238): ties keep Pitzer order
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return energies[a] < energies[b]; });
        v2g::Layout L;
        std::string err = v2g::build_layout(P.L.opt, P.L.nirrep, P.L.amopi, P.L.na, P.L.nb, P.L.multiplicity, L, order);
        if (!err.empty()) return v2g::fail(V2G_ERR_ARG, err);
        if (L.dimx != P.L.dimx || L.ncon != P.L.ncon) return v2g::fail(V2G_ERR_ARG, "internal error: layout changed size");
        P.L = std::move(L);
        P.T.reset();  // device tables are rebuilt for the new pair numbering
        P.energies.assign(energies, energies + P.L.amo);
        return V2G_OK;
    });
}

int v2g_spatial_density_dims(const v2g_handle* h, long* d1_dim, long* d2_dim) {
    return v2g::guarded([&]() -> int {
        if (!h || !d1_dim || !d2_dim) return v2g::fail(V2G_ERR_ARG, "null argument");
        const v2g::Layout& L = h->P.L;
        long n1 = 0, n2 = 0;
        std::vector<int> g00(L.nirrep, 0);
        for (int i = 0; i < L.amo; i++)
            for (int j = 0; j <= i; j++) g00[L.sym_pair(L.symmetry[i], L.symmetry[j])]++;
        for (int hh = 0; hh < L.nirrep; hh++) {
            n1 += (long)L.amopi[hh] * (L.amopi[hh] + 1) / 2;
            n2 += (long)g00[hh] * (g00[hh] + 1) / 2;
        }
        *d1_dim = n1;
        *d2_dim = n2;
        return V2G_OK;
    });
}

int v2g_pack_spatial_density(v2g_handle* h, const double* active_energies, double* d1, double* d2) {
    return v2g::guarded([&]() -> int {
        if (!h || !d1 || !d2) return v2g::fail(V2G_ERR_ARG, "null argument");
        v2g::require_device();
        Problem& P = h->P;
        if ((int64_t)P.x.size() != P.L.dimx) return v2g::fail(V2G_ERR_ARG, "the handle has no primal state");
        v2g::Csr M;
        int64_t n1 = 0, n2 = 0;
        v2g::build_spatial_map(P.L, active_energies ? active_energies : (P.energies.empty() ? nullptr : P.energies.data()),
                               M, n1, n2);
        CK(cudaSetDevice(P.device));
        v2g::MapTable T;
        T.build(M);
        v2g::DevBuf<double> x, out;
        x.upload(P.x.data(), P.x.size());
        out.alloc((size_t)(n1 + n2));
        v2g::launch_spmv(T.dm, 1, x.p, out.p, nullptr, nullptr, nullptr, nullptr, 0);
        CK(cudaGetLastError());
        std::vector<double> hout((size_t)(n1 + n2));
        CK(cudaMemcpy(hout.data(), out.p, hout.size() * sizeof(double), cudaMemcpyDeviceToHost));
        std::copy(hout.begin(), hout.begin() + n1, d1);
        std::copy(hout.begin() + n1, hout.end(), d2);
        return V2G_OK;
    });
}

int v2g_update_xz(v2g_handle* h, double mu) {
    return v2g::guarded([&]() -> int {
        if (!h || !(mu > 0.0)) return v2g::fail(V2G_ERR_ARG, "bad argument");
        v2g::require_device();
        Problem& P = h->P;
        P.mu = mu;
        v2g::GroupRun g(P.tables(), {&P});
        g.project();
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(g.stream()));
        g.download_state();
        return V2G_OK;
    });
}

int v2g_solve_batch(v2g_handle** hs, int count, v2g_result* res) {
    return v2g::guarded([&]() -> int {
        if (!hs || !res || count < 1) return v2g::fail(V2G_ERR_ARG, "bad batch arguments");
        v2g::require_device();
        const int device = hs[0] ? hs[0]->P.device : 0;
        CK(cudaSetDevice(device));
        cudaEvent_t t0, t1, t2, t3;
        CK(cudaEventCreate(&t0));
        CK(cudaEventCreate(&t1));
        CK(cudaEventCreate(&t2));
        CK(cudaEventCreate(&t3));
        CK(cudaEventRecord(t0, 0));
        // group handles by layout (shared tables), at most 256 per group
        std::map<v2g::DeviceTables*, std::vector<int>> groups;
        for (int i = 0; i < count; i++) {
            if (!hs[i]) return v2g::fail(V2G_ERR_ARG, "null handle in batch");
            if (!hs[i]->P.have_c) return v2g::fail(V2G_ERR_ARG, "v2g_set_hamiltonian was not called");
            if (hs[i]->P.device != device) return v2g::fail(V2G_ERR_ARG, "all handles of a batch use one device");
            groups[&hs[i]->P.tables()].push_back(i);
        }
        std::vector<std::unique_ptr<v2g::GroupRun>> runs;
        std::vector<std::vector<int>> members;
        for (auto& kv : groups) {
            const auto& idx = kv.second;
            for (size_t s0 = 0; s0 < idx.size(); s0 += 256) {
                std::vector<Problem*> probs;
                std::vector<int> which;
                for (size_t k = s0; k < idx.size() && k < s0 + 256; k++) {
                    probs.push_back(&hs[idx[k]]->P);
                    which.push_back(idx[k]);
                }
                runs.push_back(std::make_unique<v2g::GroupRun>(*kv.first, probs));
                members.push_back(which);
            }
        }
        CK(cudaDeviceSynchronize());
        CK(cudaEventRecord(t1, 0));
        const long launches0 = v2g::g_kernel_launches.load();
        // every layout group runs its own lock-step loop on its own stream
        std::vector<std::vector<v2g_result>> out(runs.size());
        std::vector<std::string> errs(runs.size());
        std::vector<std::thread> th;
        for (size_t g = 0; g < runs.size(); g++)
            th.emplace_back([&, g]() {
                try {
                    CK(cudaSetDevice(device));
                    runs[g]->solve(out[g]);
                } catch (const std::exception& e) {
                    errs[g] = e.what();
                }
            });
        for (auto& t : th) t.join();
        for (auto& e : errs)
            if (!e.empty()) throw v2g::CudaError(e);
        CK(cudaDeviceSynchronize());
        CK(cudaEventRecord(t2, 0));
        const long launches1 = v2g::g_kernel_launches.load();
        for (auto& r : runs) r->download_state();
        CK(cudaGetLastError());
        CK(cudaEventRecord(t3, 0));
        CK(cudaEventSynchronize(t3));
        float ms_dev = 0, ms_e2e = 0;
        CK(cudaEventElapsedTime(&ms_dev, t1, t2));
        CK(cudaEventElapsedTime(&ms_e2e, t0, t3));
        v2g_batch_stats st{};
        st.device_seconds = ms_dev * 1e-3;
        st.e2e_seconds = ms_e2e * 1e-3;
        st.kernel_launches = launches1 - launches0;
        st.groups = (long)runs.size();
        for (auto& r : runs) {
            st.map_seconds += r->map_seconds();
            st.map_launches += r->map_launches();
            st.map_bytes += r->map_bytes();
            st.h2d_bytes += r->h2d_bytes();
            st.d2h_bytes += r->d2h_bytes();
            st.refine_sweeps += r->oa_sweeps();
            st.jacobi_sweeps += r->jacobi_sweeps();
            st.jacobi_blocks += r->jacobi_blocks();
            st.jacobi_unconverged += r->jacobi_unconverged();
        }
        v2g::g_stats = st;
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        cudaEventDestroy(t2);
        cudaEventDestroy(t3);
        int worst = V2G_OK;
        for (size_t g = 0; g < runs.size(); g++)
            for (size_t k = 0; k < members[g].size(); k++) {
                res[members[g][k]] = out[g][k];
                if (out[g][k].status != V2G_OK && worst == V2G_OK) worst = out[g][k].status;
            }
        if (worst != V2G_OK) v2g::g_last_error = "at least one instance did not converge";
        return worst;
    });
}

int v2g_last_batch_stats(v2g_batch_stats* out) {
    if (!out) return V2G_ERR_ARG;
    *out = v2g::g_stats;
    return V2G_OK;
}

int v2g_solve(v2g_handle* h, v2g_result* res) { return v2g_solve_batch(&h, 1, res); }

int v2g_solve_continue(v2g_handle* h, int max_outer, v2g_result* res) {
    if (!h || !res || max_outer < 1) return v2g::fail(V2G_ERR_ARG, "bad arguments to v2g_solve_continue");
    h->P.resume = max_outer;
    const int st = v2g_solve_batch(&h, 1, res);  // guarded: returns a status, never throws
    h->P.resume = 0;
    return st;
}

long v2g_A_nnz(v2g_handle* h) {
    if (!h) return -1;
    v2g::Csr A;
    if (!v2g::build_A(h->P.L, A).empty()) return -1;
    return (long)A.nnz();
}

int v2g_export_A(v2g_handle* h, long* rowptr, int* col, double* val) {
    return v2g::guarded([&]() -> int {
        if (!h || !rowptr || !col || !val) return v2g::fail(V2G_ERR_ARG, "null argument");
        v2g::Csr A;
        std::string err = v2g::build_A(h->P.L, A);
        if (!err.empty()) return v2g::fail(V2G_ERR_UNSUPPORTED, err);
        for (size_t i = 0; i < A.rowptr.size(); i++) rowptr[i] = (long)A.rowptr[i];
        std::copy(A.col.begin(), A.col.end(), col);
        std::copy(A.val.begin(), A.val.end(), val);
        return V2G_OK;
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Projection step that allocates no device memory.
//
// Some host programs cannot call cudaMalloc while they run: codes that hand
// all device memory to their own pool allocator at start-up and forbid other
// allocations, programs that run under a fixed device-memory budget, and
// callers that must not take the implicit device synchronisation a
// cudaMalloc/cudaFree can cause.  v2g_update_xz_noalloc serves them for
// layouts whose blocks all take the shared-memory eigensolver (dimension
// <= 64).  Its scratch, the A^T y intermediate, the block task list and mu,
// lives in the file-scope array below: every GPU that loads this library
// holds it until the process exits, and every call shares it.
namespace {

constexpr int kNoAllocMaxTasks = 256;          // blocks per call
constexpr int64_t kNoAllocMaxDimx = 65536;     // primal length per call
constexpr size_t kNoAllocMuBytes = 256;
constexpr size_t kNoAllocTaskBytes = (kNoAllocMaxTasks * sizeof(v2g::BlockTask) + 255) / 256 * 256;
constexpr size_t kNoAllocBytes = kNoAllocMuBytes + kNoAllocTaskBytes + kNoAllocMaxDimx * sizeof(double);
constexpr int kNoAllocMaxDevices = 64;

// In host code this name only stands for the symbol; its device address
// comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device (the first call on a device does this set-up).
unsigned char* noalloc_scratch(int device) {
    if (device < 0 || device >= kNoAllocMaxDevices) throw std::invalid_argument("device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) throw v2g::CudaError(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_noalloc_addr[device] = p;
    }
    return static_cast<unsigned char*>(g_noalloc_addr[device]);
}

// The per-call inputs of the scratch (mu and the block list), passed by value
// as a kernel argument (3 KB) so that no host memory is copied per call.
struct NoAllocSetup {
    double mu;
    int nt;
    int n[kNoAllocMaxTasks];
    int64_t xoff[kNoAllocMaxTasks];
};

__global__ void noalloc_setup_kernel(NoAllocSetup p, double* s_mu, v2g::BlockTask* s_tasks) {
    for (int i = threadIdx.x; i < p.nt; i += blockDim.x) {
        v2g::BlockTask t{};
        t.xoff = p.xoff[i];
        t.n = p.n[i];
        t.inst = 0;
        s_tasks[i] = t;
    }
    if (threadIdx.x == 0) *s_mu = p.mu;
}


}  // namespace

extern "C" {

int v2g_update_xz_noalloc(v2g_handle* h, double mu, const double* d_c, const double* d_y, double* d_x, double* d_z,
                          void* stream) {
    return v2g::guarded([&]() -> int {
        if (!h || !(mu > 0.0) || !d_c || !d_y || !d_x || !d_z) return v2g::fail(V2G_ERR_ARG, "bad argument");
        v2g::require_device();
        Problem& P = h->P;
        if (!P.T)
            return v2g::fail(V2G_ERR_ARG,
                             "v2g_update_xz_noalloc: the handle's constraint tables are not on the device yet "
                             "(v2g_update_xz, a map call or a solve builds them)");
        v2g::DeviceTables& T = *P.T;
        const v2g::Layout& L = T.L;
        if (L.dimx > kNoAllocMaxDimx)
            return v2g::fail(V2G_ERR_ARG, "v2g_update_xz_noalloc: dimx " + std::to_string(L.dimx) +
                                              " exceeds the maximum of " + std::to_string(kNoAllocMaxDimx));
        NoAllocSetup setup{};
        setup.mu = mu;
        setup.nt = 0;
        for (size_t k = 0; k < L.block_dims.size(); k++) {
            const int n = L.block_dims[k];
            if (n == 0) continue;
            if (n > 64)
                return v2g::fail(V2G_ERR_ARG, "v2g_update_xz_noalloc: block of dimension " + std::to_string(n) +
                                                  " exceeds the maximum of 64 (use v2g_update_xz)");
            if (setup.nt == kNoAllocMaxTasks)
                return v2g::fail(V2G_ERR_ARG, "v2g_update_xz_noalloc: more than " +
                                                  std::to_string(kNoAllocMaxTasks) + " blocks");
            setup.n[setup.nt] = n;
            setup.xoff[setup.nt] = L.block_off[k];
            setup.nt++;
        }
        v2g::DeviceScope scope(T.device);
        unsigned char* base = noalloc_scratch(T.device);
        double* s_mu = reinterpret_cast<double*>(base);
        v2g::BlockTask* s_tasks = reinterpret_cast<v2g::BlockTask*>(base + kNoAllocMuBytes);
        double* s_aty = reinterpret_cast<double*>(base + kNoAllocMuBytes + kNoAllocTaskBytes);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        // mu and the block list are rewritten by every call; A^T y is cleared
        // first, so nothing of an earlier call's contents is read.
        noalloc_setup_kernel<<<1, 256, 0, s>>>(setup, s_mu, s_tasks);
        v2g::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
        CK(cudaMemsetAsync(s_aty, 0, L.dimx * sizeof(double), s));
        v2g::launch_spmv(T.AT(), 1, d_y, s_aty, nullptr, nullptr, nullptr, nullptr, s);
        v2g::launch_small_project(s_tasks, setup.nt, 1, s_aty, d_c, d_x, d_z, s_mu, nullptr, s);
        CK(cudaGetLastError());
        return V2G_OK;
    });
}

int v2g_time_maps(v2g_handle* h, int nvec, int reps, double* sec_A, double* sec_AT) {
    return v2g::guarded([&]() -> int {
        if (!h || nvec < 1 || nvec > 256 || reps < 1 || reps > 10000 || !sec_A || !sec_AT)
            return v2g::fail(V2G_ERR_ARG, "bad map timing arguments");
        v2g::require_device();
        v2g::DeviceTables& T = h->P.tables();
        v2g::DeviceScope scope(T.device);
        const int64_t nx = T.L.dimx, nc = T.L.ncon;
        v2g::DevBuf<double> x((size_t)nx * nvec), y((size_t)nc * nvec), ox((size_t)nx * nvec), oy((size_t)nc * nvec);
        cudaStream_t s = nullptr;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaGraphExec_t ex = nullptr;
        auto cleanup = [&]() {
            if (ex) cudaGraphExecDestroy(ex);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            if (s) cudaStreamDestroy(s);
        };
        try {
            CK(cudaEventCreate(&e0));
            CK(cudaEventCreate(&e1));
            // every kernel variant is timed and the fastest kept (the autotuner's choice)
            for (int which = 0; which < 2; which++)
                for (int v = 0; v < v2g::kMapVariants; v++) {
                    v2g::DevMap M = which == 0 ? T.A() : T.AT();
                    M.variant = v;
                    const double* in = which == 0 ? x.p : y.p;
                    double* out = which == 0 ? oy.p : ox.p;
                    for (int k = 0; k < 3; k++) v2g::launch_spmv(M, nvec, in, out, nullptr, nullptr, nullptr, nullptr, s);
                    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                    for (int k = 0; k < reps; k++)
                        v2g::launch_spmv(M, nvec, in, out, nullptr, nullptr, nullptr, nullptr, s);
                    cudaGraph_t g = nullptr;
                    CK(cudaStreamEndCapture(s, &g));
                    size_t nodes = 0;
                    cudaGraphGetNodes(g, nullptr, &nodes);
                    v2g::g_kernel_launches.fetch_sub((long)nodes, std::memory_order_relaxed);
                    const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
                    cudaGraphDestroy(g);
                    CK(ie);
                    CK(cudaGraphLaunch(ex, s));  // warm
                    CK(cudaEventRecord(e0, s));
                    CK(cudaGraphLaunch(ex, s));
                    CK(cudaEventRecord(e1, s));
                    CK(cudaEventSynchronize(e1));
                    v2g::g_kernel_launches.fetch_add(2 * (long)nodes, std::memory_order_relaxed);
                    float ms = 0.f;
                    CK(cudaEventElapsedTime(&ms, e0, e1));
                    double& best = which == 0 ? *sec_A : *sec_AT;
                    if (v == 0 || ms * 1e-3 / reps < best) best = ms * 1e-3 / reps;
                    cudaGraphExecDestroy(ex);
                    ex = nullptr;
                }
        } catch (...) {
            cleanup();
            throw;
        }
        cleanup();
        return V2G_OK;
    });
}

namespace {
// Tasks, tiles and split units of a batched block product on the device.
struct BlockGemmPlan {
    std::vector<v2g::BlockTask> tasks;
    std::vector<v2g::GemmTile> tiles;
    std::vector<v2g::TcSplit> split;
    int64_t toff = 0;
    v2g::DevBuf<v2g::BlockTask> dt;
    v2g::DevBuf<v2g::GemmTile> dg;
    v2g::DevBuf<v2g::TcSplit> ds;
    v2g::DevBuf<uint32_t> wa, wb;
    v2g::TcPlan tc;
    bool tensor_cores = false;

    // false: a dimension out of range
    bool build(int nblocks, const int* dims, bool use_tc) {
        tensor_cores = use_tc;
        tasks.resize(nblocks);
        int64_t woff = 0, doff = 0;
        for (int i = 0; i < nblocks; i++) {
            if (dims[i] < 1 || dims[i] > 16384) return false;
            v2g::BlockTask t{};
            t.n = dims[i];
            t.np = (dims[i] + 63) / 64 * 64;
            t.nb = t.np / 32;
            t.woff = woff;
            t.doff = doff;
            t.toff = toff;
            woff += (int64_t)t.np * t.np;
            doff += t.np;
            toff += v2g::tc_split_words(t.np);
            tasks[i] = t;
            if (use_tc) {
                const int nr = (t.np + 127) / 128;
                for (int a = 0; a < nr; a++) {
                    split.push_back({i, a});
                    for (int b = 0; b < nr; b++) tiles.push_back({i, a, b});
                }
            } else {
                const int nt = t.np / 64;
                for (int a = 0; a < nt; a++)
                    for (int b = 0; b < nt; b++) tiles.push_back({i, a, b});
            }
        }
        dt.upload(tasks.data(), tasks.size());
        dg.upload(tiles.data(), tiles.size());
        if (use_tc) {
            ds.upload(split.data(), split.size());
            wa.alloc(toff);
            wb.alloc(toff);
            tc.tasks = dt.p;
            tc.tiles_full = dg.p;
            tc.n_full = (int)tiles.size();
            tc.split = ds.p;
            tc.nsplit = (int)split.size();
            for (const auto& t : tasks) tc.max_nk = std::max(tc.max_nk, t.np / 32);
            tc.wa = wa.p;
            tc.wb = wb.p;
        }
        return true;
    }
    void launch(const double* A, bool transA, const double* B, bool transB, const double* d, double* C,
                cudaStream_t s) const {
        if (tensor_cores)
            v2g::launch_tc_gemm(tc, false, A, transA, B, transB, d, C, nullptr, s);
        else
            v2g::launch_gemm(dt.p, dg.p, (int)tiles.size(), A, transA, B, transB, d, C, nullptr, s);
    }
};
}  // namespace

int v2g_block_gemm_device(int nblocks, const int* dims, const double* A, int transA, const double* B, int transB,
                          const double* d, double* C, int tensor_cores, int device) {
    return v2g::guarded([&]() -> int {
        if (nblocks < 1 || !dims || !A || !B || !C) return v2g::fail(V2G_ERR_ARG, "bad block GEMM arguments");
        v2g::require_device();
        v2g::DeviceScope scope(device);
        BlockGemmPlan plan;
        if (!plan.build(nblocks, dims, tensor_cores != 0))
            return v2g::fail(V2G_ERR_ARG, "block dimension out of range");
        if (tensor_cores) v2g::tc_gemm_status(true);
        plan.launch(A, transA != 0, B, transB != 0, d, C, 0);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(0));
        if (tensor_cores && v2g::tc_gemm_status(true) != 0)
            return v2g::fail(V2G_ERR_CUDA, "a tensor-core GEMM pipeline wait ran out");
        return V2G_OK;
    });
}

int v2g_time_block_gemm(int nblocks, const int* dims, const double* A, const double* B, double* C, int tensor_cores,
                        int reps, int device, double* sec) {
    return v2g::guarded([&]() -> int {
        if (nblocks < 1 || !dims || !A || !B || !C || !sec || reps < 1 || reps > 10000)
            return v2g::fail(V2G_ERR_ARG, "bad block GEMM timing arguments");
        v2g::require_device();
        v2g::DeviceScope scope(device);
        BlockGemmPlan plan;
        if (!plan.build(nblocks, dims, tensor_cores != 0))
            return v2g::fail(V2G_ERR_ARG, "block dimension out of range");
        cudaStream_t s = nullptr;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        auto cleanup = [&]() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            if (s) cudaStreamDestroy(s);
        };
        try {
            CK(cudaEventCreate(&e0));
            CK(cudaEventCreate(&e1));
            if (tensor_cores) v2g::tc_gemm_status(true);
            for (int k = 0; k < 3; k++) plan.launch(A, false, B, false, nullptr, C, s);
            CK(cudaEventRecord(e0, s));
            for (int k = 0; k < reps; k++) plan.launch(A, false, B, false, nullptr, C, s);
            CK(cudaEventRecord(e1, s));
            CK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            *sec = ms * 1e-3 / reps;
        } catch (...) {
            cleanup();
            throw;
        }
        cleanup();
        if (tensor_cores && v2g::tc_gemm_status(true) != 0)
            return v2g::fail(V2G_ERR_CUDA, "a tensor-core GEMM pipeline wait ran out");
        return V2G_OK;
    });
}

// ---- learned warm start (warmstart.cu) --------------------------------------

namespace {
// the all-active C1 singlet the warm start works on
int ws_check(const Problem& P) {
    if (P.hmat.empty()) return v2g::fail(V2G_ERR_UNSUPPORTED, "the learned warm start needs an all-active C1 space "
                                                              "with integrals (v2g_set_hamiltonian)");
    if (P.L.na != P.L.nb) return v2g::fail(V2G_ERR_UNSUPPORTED, "the learned warm start is built for singlets");
    return V2G_OK;
}
}  // namespace

int v2g_ws_create(int hidden, int device, unsigned long long seed, v2g_warmstart** out) {
    return v2g::guarded([&]() -> int {
        if (!out || hidden < 8 || hidden > 1024) return v2g::fail(V2G_ERR_ARG, "hidden width must be in 8..1024");
        *out = nullptr;
        v2g::require_device();
        v2g::DeviceScope scope(device);
        v2g::ws_create(hidden, device, seed, out);
        return V2G_OK;
    });
}

void v2g_ws_destroy(v2g_warmstart* w) {
    if (w) v2g::ws_destroy(w);
}

long v2g_ws_num_params(const v2g_warmstart* w) { return w ? (long)v2g::ws_num_params(w) : -1; }

int v2g_ws_get_params(const v2g_warmstart* w, float* params) {
    return v2g::guarded([&]() -> int {
        if (!w || !params) return v2g::fail(V2G_ERR_ARG, "null argument");
        v2g::ws_get_params(w, params);
        return V2G_OK;
    });
}

int v2g_ws_set_params(v2g_warmstart* w, const float* params) {
    return v2g::guarded([&]() -> int {
        if (!w || !params) return v2g::fail(V2G_ERR_ARG, "null argument");
        v2g::ws_set_params(w, params);
        return V2G_OK;
    });
}

long v2g_ws_rows(const v2g_handle* h) { return h ? (long)h->P.L.amo * (h->P.L.amo + 1) / 2 : -1; }

int v2g_ws_features(const v2g_handle* h, float* features) {
    return v2g::guarded([&]() -> int {
        if (!h || !features) return v2g::fail(V2G_ERR_ARG, "null argument");
        const Problem& P = h->P;
        if (int e = ws_check(P)) return e;
        v2g::ws_features(P.L.amo, P.L.na, P.hmat.data(), P.Lq.data(), P.nq, features);
        return V2G_OK;
    });
}

int v2g_ws_targets(const v2g_handle* h, float* targets) {
    return v2g::guarded([&]() -> int {
        if (!h || !targets) return v2g::fail(V2G_ERR_ARG, "null argument");
        const Problem& P = h->P;
        if (int e = ws_check(P)) return e;
        const v2g::Layout& L = P.L;
        const int n = L.amo;
        const int64_t d1 = L.off[v2g::F_D1A][0], d2 = L.off[v2g::F_D2AB][0];
        const int64_t gab = L.gems_ab[0];
        int r = 0;
        for (int p = 0; p < n; p++)
            for (int q = p; q < n; q++, r++) {
                const int g = L.ab(0, p, q);
                targets[r * v2g::kWsOut + 0] = (float)P.x[d1 + (int64_t)p * n + q];
                targets[r * v2g::kWsOut + 1] = (float)P.x[d2 + (int64_t)g * gab + g];
                targets[r * v2g::kWsOut + 2] = (float)std::log(P.mu);
            }
        return V2G_OK;
    });
}

int v2g_ws_forward(v2g_warmstart* w, long rows, const float* features, float* out) {
    return v2g::guarded([&]() -> int {
        if (!w || rows < 1 || !features || !out) return v2g::fail(V2G_ERR_ARG, "bad forward arguments");
        v2g::ws_forward(w, rows, features, out);
        return V2G_OK;
    });
}

int v2g_ws_gradient(v2g_warmstart* w, long rows, const float* features, const float* targets, double* loss,
                    float* grad) {
    return v2g::guarded([&]() -> int {
        if (!w || rows < 1 || !features || !targets) return v2g::fail(V2G_ERR_ARG, "bad gradient arguments");
        const double l = v2g::ws_gradient(w, rows, features, targets, grad);
        if (loss) *loss = l;
        return V2G_OK;
    });
}

int v2g_ws_train(v2g_warmstart* w, long rows, const float* features, const float* targets, int epochs,
                 int batch_rows, float lr, double* loss) {
    return v2g::guarded([&]() -> int {
        if (!w || rows < 1 || !features || !targets || epochs < 1 || batch_rows < 1 || !(lr > 0.f))
            return v2g::fail(V2G_ERR_ARG, "bad training arguments");
        const double l = v2g::ws_train(w, rows, features, targets, epochs, batch_rows, lr);
        if (loss) *loss = l;
        return V2G_OK;
    });
}

int v2g_ws_propose(v2g_warmstart* w, v2g_handle* h, int use_mu) {
    return v2g::guarded([&]() -> int {
        if (!w || !h) return v2g::fail(V2G_ERR_ARG, "null argument");
        Problem& P = h->P;
        if (int e = ws_check(P)) return e;
        const v2g::Layout& L = P.L;
        const int n = L.amo;
        const long rows = (long)n * (n + 1) / 2;
        std::vector<float> feat((size_t)rows * v2g::kWsFeatures), out((size_t)rows * v2g::kWsOut);
        v2g::ws_features(n, L.na, P.hmat.data(), P.Lq.data(), P.nq, feat.data());
        v2g::ws_forward(w, rows, feat.data(), out.data());
        std::fill(P.x.begin(), P.x.end(), 0.0);
        std::fill(P.y.begin(), P.y.end(), 0.0);
        std::fill(P.z.begin(), P.z.end(), 0.0);
        const int64_t gab = L.gems_ab[0];
        double lmu = 0.0;
        int r = 0;
        for (int p = 0; p < n; p++)
            for (int q = p; q < n; q++, r++) {
                const double gam = out[r * v2g::kWsOut + 0], d2 = out[r * v2g::kWsOut + 1];
                lmu += out[r * v2g::kWsOut + 2];
                for (int f : {v2g::F_D1A, v2g::F_D1B}) {
                    P.x[L.off[f][0] + (int64_t)p * n + q] = gam;
                    P.x[L.off[f][0] + (int64_t)q * n + p] = gam;
                }
                for (int f : {v2g::F_Q1A, v2g::F_Q1B}) {
                    P.x[L.off[f][0] + (int64_t)p * n + q] = (p == q ? 1.0 : 0.0) - gam;
                    P.x[L.off[f][0] + (int64_t)q * n + p] = (p == q ? 1.0 : 0.0) - gam;
                }
                const int g1 = L.ab(0, p, q), g2 = L.ab(0, q, p);
                P.x[L.off[v2g::F_D2AB][0] + (int64_t)g1 * gab + g1] = d2;
                P.x[L.off[v2g::F_D2AB][0] + (int64_t)g2 * gab + g2] = d2;
            }
        P.mu = use_mu ? std::min(10.0, std::max(0.1, std::exp(lmu / rows))) : 1.0;
        P.proposal = true;
        return V2G_OK;
    });
}

long v2g_trace(const v2g_handle* h, double* rows, long cap) {
    if (!h) return -1;
    const auto& t = h->P.trace;
    long n = (long)t.size();
    if (rows)
        for (long i = 0; i < n && i < cap; i++)
            for (int k = 0; k < 8; k++) rows[i * 8 + k] = t[i][k];
    return n;
}

}  // extern "C"
