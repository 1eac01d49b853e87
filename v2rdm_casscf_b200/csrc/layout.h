// Problem layout of the boundary-point SDP: geminal/triplet index maps, the
// primal blocks (their order, offsets and dimensions) and the constraint
// families with their row counts.
//
// The layout is the reference plugin's, so that x, y and z are exchangeable
// with it element for element:
//   * geminal maps      basis.cc:439-548 (ab pairs pushed as (j,i) with the
//                       outer loop over i; aa pairs are the ab pairs with
//                       first > second)
//   * triplet maps      basis.cc:655-757
//   * dimx / offsets    v2rdm_solver.cc:560-885
//   * constraint counts v2rdm_solver.cc:887-1127
//   * block dimensions  v2rdm_solver.cc:1129-1270
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace v2g {

// Options on the hot path (plugin.cc:66-124), with the plugin's defaults.
struct Options {
    bool constrain_q2 = true;
    bool constrain_g2 = true;
    bool constrain_t1 = false;
    bool constrain_t2 = false;
    bool constrain_spin = true;
    bool constrain_sz = true;
    double r_convergence = 1e-4;
    double e_convergence = 1e-4;
    double cg_convergence = 1e-9;
    int maxiter = 10000;
    int cg_maxiter = 10000;
    double tau = 1.0;
    int mu_update_frequency = 500;
    // Accept an eigendecomposition whose off-diagonal residual is below
    // 0.01 min(eps_p, eps_d) (the CG tolerance rule); off = every projection
    // converged, as the reference's Update_xz.
    bool adaptive_projection = false;
    // CG tolerance = cg_tol_factor * min(eps_p, eps_d) after the first
    // iteration (0.01 in the reference, v2rdm_solver.cc:1797-1805).
    double cg_tol_factor = 0.01;
    // SPIN_ADAPT_Q2 / SPIN_ADAPT_G2 (plugin.cc): Q2 and G2 in singlet and
    // triplet blocks instead of spin blocks.
    bool spin_adapt_q2 = false;
    bool spin_adapt_g2 = false;
    // CONSTRAIN_D3 (plugin.cc): 3-RDM positivity with its contractions to D2
    bool constrain_d3 = false;
    // CONSTRAIN_D4: 4-RDM positivity with its contractions to D3 (implies D3)
    bool constrain_d4 = false;
    // Start the solve from the least-norm point of {A x = b} (x = A^T w with
    // A A^T w = b, y = z = 0, mu = 1) instead of the handle's state.
    bool feasible_start = false;
    // Start from the handle's proposal (the learned warm start, v2g_ws_propose)
    // projected onto {A x = b}, y = z = 0 and the proposed mu; the least-norm
    // feasible point when the handle has no proposal.
    bool proposal_start = false;
    // Start each outer iteration's CG from y_k + (y_k - y_{k-1}), the linear
    // extrapolation of the last two CG solutions, instead of from y_k.  CG
    // still stops on the same residual test, so only its iteration count
    // changes.
    bool cg_extrapolate = false;
    // Anderson acceleration (type II) of the outer iteration on (x, z) with
    // this many difference columns; 0 = off.  The history restarts whenever mu
    // changes.
    int anderson_memory = 0;
    bool mixed_precision = false;  // tensor-core (3xTF32) projection products while rho >= 1e-5
};

// Parses POSITIVITY the way v2rdm_solver.cc:497-522 does; returns false for
// an unknown value.
bool parse_positivity(const std::string& p, Options& o);

enum Fam {
    F_D2AB, F_D2AA, F_D2BB, F_D200, F_D1A, F_D1B, F_Q1A, F_Q1B,
    F_Q2AB, F_Q2AA, F_Q2BB, F_G2AB, F_G2BA, F_G2AA,
    F_Q2S, F_Q2T, F_Q2TP, F_Q2TM,  // spin-adapted Q2: singlet, triplet M = 0, +1, -1
    F_G2S, F_G2T, F_G2TP, F_G2TM,  // spin-adapted G2
    F_T1AAA, F_T1BBB, F_T1AAB, F_T1BBA,
    F_T2AAA, F_T2BBB, F_T2AAB, F_T2BBA,
    F_D3AAA, F_D3BBB, F_D3AAB, F_D3BBA,
    F_D4AAAA, F_D4AAAB, F_D4AABB, F_D4BBBA, F_D4BBBB,
    F_COUNT
};

struct Layout {
    // active space
    int nirrep = 1;
    int amo = 0;
    std::vector<int> amopi;           // active orbitals per irrep
    std::vector<int> symmetry;        // irrep of each active orbital (Pitzer order)
    std::vector<int> pitzer_offset;   // first active orbital of each irrep
    double na = 0, nb = 0;            // active alpha / beta electrons
    int multiplicity = 1;
    Options opt;

    // geminals per irrep
    std::vector<int> gems_ab, gems_aa, gems_00;
    std::vector<std::vector<std::array<int, 2>>> bas_ab, bas_aa, bas_00;
    std::vector<std::vector<int>> ibas_00;            // [h][i*amo+j], spatial pairs in energy order
    std::vector<int> energy_order;                    // active orbitals by orbital energy
    std::vector<std::vector<int>> ibas_ab, ibas_aa;  // [h][i*amo+j], -1 if (i,j) not in irrep h
    // triplets per irrep
    std::vector<int> trip_aaa, trip_aab, trip_aba;
    std::vector<std::vector<std::array<int, 3>>> bas_aaa, bas_aab, bas_aba;
    std::vector<std::vector<int>> ibas_aaa, ibas_aab, ibas_aba;  // [h][(i*amo+j)*amo+k]

    // quartets per irrep (basis.cc:758-904): aaaa i<j<k<l, aaab i<j<k, aabb i<j & k<l
    std::vector<int> quart_aaaa, quart_aaab, quart_aabb;
    std::vector<std::vector<std::array<int, 4>>> bas_aaaa, bas_aaab, bas_aabb;
    std::vector<std::vector<int>> ibas_aaaa, ibas_aaab, ibas_aabb;  // [h][((i*amo+j)*amo+k)*amo+l]

    // primal layout
    std::array<std::vector<int64_t>, F_COUNT> off;  // per family, per irrep
    int64_t dimx = 0;
    int64_t ncon = 0;
    std::vector<int> block_dims;       // dimensions_ of the reference
    std::vector<int64_t> block_off;    // offset of each block in x

    bool singlet() const { return na == nb; }
    int sym_pair(int hi, int hj) const { return hi ^ hj; }  // abelian product table, basis.cc:58-89
    int ab(int h, int i, int j) const { return ibas_ab[h][i * amo + j]; }
    int aa(int h, int i, int j) const { return ibas_aa[h][i * amo + j]; }
    int aab(int h, int i, int j, int k) const { return ibas_aab[h][(i * amo + j) * amo + k]; }
    int aba(int h, int i, int j, int k) const { return ibas_aba[h][(i * amo + j) * amo + k]; }
    int aaa(int h, int i, int j, int k) const { return ibas_aaa[h][(i * amo + j) * amo + k]; }
    int q4(const std::vector<std::vector<int>>& m, int h, int i, int j, int k, int l) const {
        return m[h][((i * amo + j) * amo + k) * amo + l];
    }
};

// Builds the layout.  orbital_irrep lists the irrep of each active orbital in
// Pitzer order (irreps non-decreasing); na/nb are active electron counts.
// Returns an empty string on success, else the reason.
// energy_order lists the active orbitals in increasing orbital energy (it
// numbers the spatial pairs, basis.cc:626-652); empty = Pitzer order.
std::string build_layout(const Options& opt, int nirrep, const std::vector<int>& amopi, double na, double nb,
                         int multiplicity, Layout& L, const std::vector<int>& energy_order = {});

}  // namespace v2g
