// Host half of the Anderson acceleration of the BPSDP outer iteration
// (option anderson_memory; the device half is the aa_* kernels of maps.cu).
//
// Type-II Anderson mixing on the state w = (x, z): after a step w -> g with
// residual f = g - w, the history holds up to m difference columns
// dF_j = f_{j+1} - f_j and dG_j = g_{j+1} - g_j in a ring of m slots, and the
// next state is g - sum_j gamma_j dG_j with
// (dF^T dF + lambda I) gamma = dF^T f, lambda = 1e-10 tr(dF^T dF).
// The history restarts after a mu change, when |f| more than doubles from
// one step to the next (that step is not mixed), and when the small system
// has no finite solution.
//
// Plain C++ (no CUDA), so that the bookkeeping is tested on the CPU.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <vector>

namespace v2g {

// The history restarts when the fixed-point residual |f| grows by more than
// this factor from one outer iteration to the next.
constexpr double kAndersonGuard = 2.0;

// Per instance b of a group of B: whether f and g of a previous step are
// stored, the number of valid difference columns and the newest ring slot,
// this step's kernel mode, |f| of the previous step, and the Gram matrix of
// the columns dF indexed by ring slot.  M = columns allocated per instance.
struct AndersonState {
    int B = 0, M = 0;
    std::vector<int> have, count, slot, mode;
    std::vector<double> fnorm;
    std::vector<double> g;  // [b][M][M]

    AndersonState(int nb, int m)
        : B(nb), M(m), have(nb, 0), count(nb, 0), slot(nb, 0), mode(nb, 0), fnorm(nb, -1.0),
          g((size_t)nb * m * m, 0.0) {}

    // Forget the history of instance b entirely (a restart of its solve).
    void restart(int b) {
        have[b] = count[b] = 0;
        fnorm[b] = -1.0;
    }

    // Mode of this step's update kernel for instance b with memory mb:
    // 0 = nothing, 1 = store f and g only, 2 = also a new column at slot[b].
    int begin(int b, int mb, bool mu_changed) {
        mode[b] = 0;
        if (mb <= 0) return 0;
        if (mu_changed) have[b] = count[b] = 0;  // |f| of the last step stays the reference
        if (have[b]) {
            slot[b] = count[b] == 0 ? 0 : (slot[b] + 1) % mb;
            count[b] = std::min(count[b] + 1, mb);
            mode[b] = 2;
        } else {
            mode[b] = 1;
            have[b] = 1;
        }
        return mode[b];
    }

    // After the update kernel, whose dots are laid out as
    // dots[(2 j) * B + b] = dF_slot . dF_j, dots[(2 j + 1) * B + b] = dF_j . f
    // (j < M) and dots[(2 M) * B + b] = f . f: the |f| guard, the Gram update
    // and the solve.  True when instance b mixes with gamma (M entries, by
    // slot, zero outside the valid columns).
    bool finish(int b, int mb, const std::vector<double>& dots, double* gamma) {
        if (mode[b] == 0) return false;
        const double fn = std::sqrt(dots[(size_t)(2 * M) * B + b]);
        const bool grew = fnorm[b] >= 0.0 && fn > kAndersonGuard * fnorm[b];
        fnorm[b] = fn;
        if (mode[b] != 2) return false;
        if (grew) {
            count[b] = 0;  // this f starts a new history; the column just written is dropped
            return false;
        }
        if (solve(b, mb, dots, gamma)) return true;
        have[b] = count[b] = 0;
        return false;
    }

  private:
    double& at(int b, int i, int j) { return g[((size_t)b * M + i) * M + j]; }

    // Enters the new column at slot[b] into the Gram matrix and solves
    // (G + lambda I) gamma = dF^T f over the count[b] valid slots of a ring
    // of mb by Gaussian elimination with partial pivoting (count <= 16).
    bool solve(int b, int mb, const std::vector<double>& dots, double* gamma) {
        const int s = slot[b], c = count[b];
        std::vector<int> sl(c);
        for (int i = 0; i < c; i++) sl[i] = (s - i + mb) % mb;
        for (int i = 0; i < c; i++) {
            const double v = dots[(size_t)(2 * sl[i]) * B + b];
            at(b, s, sl[i]) = v;
            at(b, sl[i], s) = v;
        }
        std::vector<double> a((size_t)c * c), r(c);
        double tr = 0.0;
        for (int i = 0; i < c; i++) tr += at(b, sl[i], sl[i]);
        const double lambda = 1e-10 * tr + 1e-300;
        for (int i = 0; i < c; i++) {
            for (int k = 0; k < c; k++) a[(size_t)i * c + k] = at(b, sl[i], sl[k]) + (i == k ? lambda : 0.0);
            r[i] = dots[(size_t)(2 * sl[i] + 1) * B + b];
        }
        for (int k = 0; k < c; k++) {
            int piv = k;
            for (int i = k + 1; i < c; i++)
                if (std::fabs(a[(size_t)i * c + k]) > std::fabs(a[(size_t)piv * c + k])) piv = i;
            if (!(std::fabs(a[(size_t)piv * c + k]) > 0.0)) return false;
            if (piv != k) {
                for (int j = 0; j < c; j++) std::swap(a[(size_t)k * c + j], a[(size_t)piv * c + j]);
                std::swap(r[k], r[piv]);
            }
            for (int i = k + 1; i < c; i++) {
                const double f = a[(size_t)i * c + k] / a[(size_t)k * c + k];
                for (int j = k; j < c; j++) a[(size_t)i * c + j] -= f * a[(size_t)k * c + j];
                r[i] -= f * r[k];
            }
        }
        std::vector<double> x(c);
        for (int k = c - 1; k >= 0; k--) {
            double sum = r[k];
            for (int j = k + 1; j < c; j++) sum -= a[(size_t)k * c + j] * x[j];
            x[k] = sum / a[(size_t)k * c + k];
            if (!std::isfinite(x[k])) return false;
        }
        for (int i = 0; i < c; i++) gamma[sl[i]] = x[i];
        return true;
    }
};

}  // namespace v2g
