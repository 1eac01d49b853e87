// Layout of the boundary-point SDP (see layout.h for the reference map).
#include "layout.h"

#include <algorithm>

namespace v2g {

bool parse_positivity(const std::string& p, Options& o) {
    // v2rdm_solver.cc:490-522
    o.constrain_q2 = true;
    o.constrain_g2 = true;
    o.constrain_t1 = false;
    o.constrain_t2 = false;
    if (p == "D") {
        o.constrain_q2 = false;
        o.constrain_g2 = false;
    } else if (p == "DQ") {
        o.constrain_g2 = false;
    } else if (p == "DG") {
        o.constrain_q2 = false;
    } else if (p == "DQG") {
    } else if (p == "DQGT1") {
        o.constrain_t1 = true;
    } else if (p == "DQGT2") {
        o.constrain_t2 = true;
    } else if (p == "DQGT1T2" || p == "DQGT") {
        o.constrain_t1 = true;
        o.constrain_t2 = true;
    } else {
        return false;
    }
    return true;
}

static void build_geminals(Layout& L) {
    const int n = L.amo, H = L.nirrep;
    L.gems_ab.assign(H, 0);
    L.gems_aa.assign(H, 0);
    L.gems_00.assign(H, 0);
    L.bas_ab.assign(H, {});
    L.bas_aa.assign(H, {});
    L.ibas_ab.assign(H, std::vector<int>(n * n, -1));
    L.ibas_aa.assign(H, std::vector<int>(n * n, -1));
    for (int h = 0; h < H; h++) {
        // basis.cc:439-450 pushes (j,i) with i the outer index; basis.cc:526-546
        // numbers ab pairs in that order and aa pairs as those with first > second.
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                if (L.sym_pair(L.symmetry[i], L.symmetry[j]) != h) continue;
                const int p = j, q = i;
                L.ibas_ab[h][p * n + q] = (int)L.bas_ab[h].size();
                L.bas_ab[h].push_back({p, q});
                if (p <= q) continue;
                const int c = (int)L.bas_aa[h].size();
                L.ibas_aa[h][p * n + q] = c;
                L.ibas_aa[h][q * n + p] = c;
                L.bas_aa[h].push_back({p, q});
            }
        L.gems_ab[h] = (int)L.bas_ab[h].size();
        L.gems_aa[h] = (int)L.bas_aa[h].size();
    }
    // spatial pairs per irrep (basis.cc:626-652): for orbitals taken in energy
    // order, each with every orbital before it (and itself)
    L.bas_00.assign(H, {});
    L.ibas_00.assign(H, std::vector<int>(n * n, -1));
    for (int ie = 0; ie < n; ie++)
        for (int je = 0; je <= ie; je++) {
            const int i = L.energy_order[ie], j = L.energy_order[je];
            const int h = L.sym_pair(L.symmetry[i], L.symmetry[j]);
            L.ibas_00[h][i * n + j] = L.gems_00[h];
            L.ibas_00[h][j * n + i] = L.gems_00[h];
            L.bas_00[h].push_back({i, j});
            L.gems_00[h]++;
        }
}

static void build_triplets(Layout& L) {
    // basis.cc:655-757: aba = all (i,j,k) of irrep h in i,j,k loop order;
    // aab = those with i < j; aaa = those with i < j < k.
    const int n = L.amo, H = L.nirrep;
    L.trip_aaa.assign(H, 0);
    L.trip_aab.assign(H, 0);
    L.trip_aba.assign(H, 0);
    L.bas_aaa.assign(H, {});
    L.bas_aab.assign(H, {});
    L.bas_aba.assign(H, {});
    L.ibas_aaa.assign(H, std::vector<int>(n * n * n, -1));
    L.ibas_aab.assign(H, std::vector<int>(n * n * n, -1));
    L.ibas_aba.assign(H, std::vector<int>(n * n * n, -1));
    auto at = [n](int i, int j, int k) { return (i * n + j) * n + k; };
    for (int h = 0; h < H; h++) {
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                const int s1 = L.sym_pair(L.symmetry[i], L.symmetry[j]);
                for (int k = 0; k < n; k++) {
                    if (L.sym_pair(s1, L.symmetry[k]) != h) continue;
                    L.ibas_aba[h][at(i, j, k)] = (int)L.bas_aba[h].size();
                    L.bas_aba[h].push_back({i, j, k});
                    if (i >= j) continue;
                    const int c = (int)L.bas_aab[h].size();
                    L.ibas_aab[h][at(i, j, k)] = c;
                    L.ibas_aab[h][at(j, i, k)] = c;
                    L.bas_aab[h].push_back({i, j, k});
                    if (j >= k) continue;
                    const int d = (int)L.bas_aaa[h].size();
                    for (auto t : {at(i, j, k), at(i, k, j), at(j, i, k), at(j, k, i), at(k, i, j), at(k, j, i)})
                        L.ibas_aaa[h][t] = d;
                    L.bas_aaa[h].push_back({i, j, k});
                }
            }
        L.trip_aaa[h] = (int)L.bas_aaa[h].size();
        L.trip_aab[h] = (int)L.bas_aab[h].size();
        L.trip_aba[h] = (int)L.bas_aba[h].size();
    }
}

static void build_quartets(Layout& L) {
    // basis.cc:758-904: all (i,j,k,l) of irrep h in loop order; each map
    // gives every permutation of its same-spin indices the same number
    const int n = L.amo, H = L.nirrep;
    const size_t n4 = (size_t)n * n * n * n;
    L.quart_aaaa.assign(H, 0);
    L.quart_aaab.assign(H, 0);
    L.quart_aabb.assign(H, 0);
    L.bas_aaaa.assign(H, {});
    L.bas_aaab.assign(H, {});
    L.bas_aabb.assign(H, {});
    L.ibas_aaaa.assign(H, std::vector<int>(n4, -1));
    L.ibas_aaab.assign(H, std::vector<int>(n4, -1));
    L.ibas_aabb.assign(H, std::vector<int>(n4, -1));
    auto at = [n](int i, int j, int k, int l) { return ((size_t)(i * n + j) * n + k) * n + l; };
    for (int h = 0; h < H; h++)
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++)
                    for (int l = 0; l < n; l++) {
                        const int s = L.sym_pair(L.sym_pair(L.symmetry[i], L.symmetry[j]),
                                                 L.sym_pair(L.symmetry[k], L.symmetry[l]));
                        if (s != h) continue;
                        if (i < j && k < l) {
                            const int c = (int)L.bas_aabb[h].size();
                            for (auto t : {at(i, j, k, l), at(j, i, k, l), at(i, j, l, k), at(j, i, l, k)})
                                L.ibas_aabb[h][t] = c;
                            L.bas_aabb[h].push_back({i, j, k, l});
                        }
                        if (i < j && j < k) {
                            const int c = (int)L.bas_aaab[h].size();
                            const int a3[3] = {i, j, k};
                            int perm[3] = {0, 1, 2};
                            do {
                                L.ibas_aaab[h][at(a3[perm[0]], a3[perm[1]], a3[perm[2]], l)] = c;
                            } while (std::next_permutation(perm, perm + 3));
                            L.bas_aaab[h].push_back({i, j, k, l});
                        }
                        if (i < j && j < k && k < l) {
                            const int c = (int)L.bas_aaaa[h].size();
                            const int a4[4] = {i, j, k, l};
                            int perm[4] = {0, 1, 2, 3};
                            do {
                                L.ibas_aaaa[h][at(a4[perm[0]], a4[perm[1]], a4[perm[2]], a4[perm[3]])] = c;
                            } while (std::next_permutation(perm, perm + 4));
                            L.bas_aaaa[h].push_back({i, j, k, l});
                        }
                    }
    for (int h = 0; h < H; h++) {
        L.quart_aaaa[h] = (int)L.bas_aaaa[h].size();
        L.quart_aaab[h] = (int)L.bas_aaab[h].size();
        L.quart_aabb[h] = (int)L.bas_aabb[h].size();
    }
}

std::string build_layout(const Options& opt, int nirrep, const std::vector<int>& amopi, double na, double nb,
                         int multiplicity, Layout& L, const std::vector<int>& energy_order) {
    if (nirrep != 1 && nirrep != 2 && nirrep != 4 && nirrep != 8) return "nirrep must be 1, 2, 4 or 8";
    if ((int)amopi.size() != nirrep) return "amopi must have nirrep entries";
    // restrictions of v2rdm_solver.cc:538-558
    if ((opt.constrain_t1 || opt.constrain_t2) && (opt.spin_adapt_q2 || opt.spin_adapt_g2))
        return "If constraining T1/T2, Q2 and G2 cannot currently be spin adapted.";
    if ((opt.spin_adapt_q2 || opt.spin_adapt_g2) && multiplicity != 1)
        return "Q2 / G2 are not spin adapted for S = M != 0";
    // the maximal spin constraint reads the G2ba block (spin.cc:470-489),
    // which the spin-adapted G2 layout does not have
    if (opt.spin_adapt_g2 && opt.constrain_spin && opt.constrain_g2)
        return "SPIN_ADAPT_G2 needs CONSTRAIN_SPIN false (the maximal spin constraint uses the G2ba block)";
    L = Layout();
    L.opt = opt;
    L.nirrep = nirrep;
    L.amopi = amopi;
    L.na = na;
    L.nb = nb;
    L.multiplicity = multiplicity;
    L.amo = 0;
    for (int h = 0; h < nirrep; h++) {
        if (amopi[h] < 0) return "negative orbital count";
        L.pitzer_offset.push_back(L.amo);
        for (int i = 0; i < amopi[h]; i++) L.symmetry.push_back(h);
        L.amo += amopi[h];
    }
    if (L.amo == 0) return "empty active space";
    if (na < 0 || nb < 0 || na > L.amo || nb > L.amo) return "electron counts outside the active space";
    if (energy_order.empty()) {
        L.energy_order.resize(L.amo);
        for (int i = 0; i < L.amo; i++) L.energy_order[i] = i;
    } else {
        std::vector<int> seen(L.amo, 0);
        if ((int)energy_order.size() != L.amo) return "energy order must list every active orbital";
        for (int i : energy_order) {
            if (i < 0 || i >= L.amo || seen[i]++) return "energy order must be a permutation of the active orbitals";
        }
        L.energy_order = energy_order;
    }
    build_geminals(L);
    if (opt.constrain_d4 && !opt.constrain_d3) return "internal error: CONSTRAIN_D4 without D3";
    if (opt.constrain_t1 || opt.constrain_t2 || opt.constrain_d3) build_triplets(L);
    if (opt.constrain_d4) build_quartets(L);

    const int H = nirrep;
    const auto& gab = L.gems_ab;
    const auto& gaa = L.gems_aa;
    const auto& amp = L.amopi;
    for (auto& v : L.off) v.assign(H, -1);
    int64_t o = 0;
    auto place = [&](Fam f, const std::vector<int>& d, int mult) {
        for (int h = 0; h < H; h++) {
            L.off[f][h] = o;
            o += (int64_t)mult * d[h] * mult * d[h];
        }
    };
    auto tsum = [&](int h) { return L.trip_aab[h] + L.trip_aba[h]; };

    // offsets in x, v2rdm_solver.cc:698-885
    place(F_D2AB, gab, 1);
    place(F_D2AA, gaa, 1);
    place(F_D2BB, gaa, 1);
    if (opt.constrain_spin) place(F_D200, gab, L.singlet() ? 1 : 2);
    place(F_D1A, amp, 1);
    place(F_D1B, amp, 1);
    place(F_Q1A, amp, 1);
    place(F_Q1B, amp, 1);
    if (opt.constrain_q2 && !opt.spin_adapt_q2) {
        place(F_Q2AB, gab, 1);
        place(F_Q2AA, gaa, 1);
        place(F_Q2BB, gaa, 1);
    } else if (opt.constrain_q2) {
        place(F_Q2S, L.gems_00, 1);
        place(F_Q2T, gaa, 1);
        place(F_Q2TP, gaa, 1);
        place(F_Q2TM, gaa, 1);
    }
    if (opt.constrain_g2 && !opt.spin_adapt_g2) {
        place(F_G2AB, gab, 1);
        place(F_G2BA, gab, 1);
        place(F_G2AA, gab, 2);
    } else if (opt.constrain_g2) {
        place(F_G2S, gab, 1);
        place(F_G2T, gab, 1);
        place(F_G2TP, gab, 1);
        place(F_G2TM, gab, 1);
    }
    if (opt.constrain_t1) {
        place(F_T1AAA, L.trip_aaa, 1);
        place(F_T1BBB, L.trip_aaa, 1);
        place(F_T1AAB, L.trip_aab, 1);
        place(F_T1BBA, L.trip_aab, 1);
    }
    if (opt.constrain_t2) {
        std::vector<int> big(H);
        for (int h = 0; h < H; h++) big[h] = tsum(h);
        place(F_T2AAA, big, 1);
        place(F_T2BBB, big, 1);
        place(F_T2AAB, L.trip_aab, 1);
        place(F_T2BBA, L.trip_aab, 1);
    }
    if (opt.constrain_d3) {  // v2rdm_solver.cc:846-862
        place(F_D3AAA, L.trip_aaa, 1);
        place(F_D3BBB, L.trip_aaa, 1);
        place(F_D3AAB, L.trip_aab, 1);
        place(F_D3BBA, L.trip_aab, 1);
    }
    if (opt.constrain_d4) {  // v2rdm_solver.cc:864-880
        place(F_D4AAAA, L.quart_aaaa, 1);
        place(F_D4AAAB, L.quart_aaab, 1);
        place(F_D4AABB, L.quart_aabb, 1);
        place(F_D4BBBA, L.quart_aaab, 1);
        place(F_D4BBBB, L.quart_aaaa, 1);
    }
    L.dimx = o;

    // constraint count, v2rdm_solver.cc:887-1127
    int64_t m = 0;
    auto sq = [](int64_t a) { return a * a; };
    m += opt.constrain_sz ? 3 : 1;
    for (int h = 0; h < H; h++) m += 2 * sq(amp[h]);
    for (int h = 0; h < H; h++) m += (opt.constrain_sz ? 4 : 2) * sq(amp[h]);
    if (opt.constrain_spin) {
        m += 1;
        if (L.singlet()) {
            for (int h = 0; h < H; h++) m += sq(amp[h]) + 3 * sq(gaa[h]) + sq(gab[h]);
        } else {
            for (int h = 0; h < H; h++) m += 4 * sq(gab[h]);
        }
        if (opt.constrain_g2) m += 2 * (int64_t)gab[0];
    }
    if (opt.constrain_q2)
        for (int h = 0; h < H; h++)
            m += opt.spin_adapt_q2 ? sq(L.gems_00[h]) + 3 * sq(gaa[h]) : sq(gab[h]) + 2 * sq(gaa[h]);
    if (opt.constrain_g2)
        for (int h = 0; h < H; h++) m += opt.spin_adapt_g2 ? 4 * sq(gab[h]) : 2 * sq(gab[h]) + sq(2 * gab[h]);
    if (opt.constrain_t1)
        for (int h = 0; h < H; h++) m += 2 * sq(L.trip_aaa[h]) + 2 * sq(L.trip_aab[h]);
    if (opt.constrain_t2)
        for (int h = 0; h < H; h++) m += 2 * sq(tsum(h)) + 2 * sq(L.trip_aab[h]);
    if (opt.constrain_d3) {  // v2rdm_solver.cc:1046-1080, with active electron counts
        for (int h = 0; h < H; h++) {
            if (na > 2) m += sq(gaa[h]);
            if (nb > 2) m += sq(gaa[h]);
            m += 2 * sq(gaa[h]);
            if (na > 1) m += sq(gab[h]);
            if (nb > 1) m += sq(gab[h]);
            if (opt.constrain_spin && L.singlet()) m += sq(L.trip_aab[h]) + 2 * sq(L.trip_aaa[h]);
        }
    }
    if (opt.constrain_d4) {
        // v2rdm_solver.cc:1084-1127.  The count lists the D4aabb contractions
        // twice while D4_constraints_Au writes them once, so the reference's
        // constraint vector ends with 2 sum trip_aab^2 empty rows (b = 0);
        // they are kept for an identical layout.
        for (int h = 0; h < H; h++) {
            const int64_t ta = sq(L.trip_aaa[h]), tb = sq(L.trip_aab[h]);
            if (na > 3) m += ta;
            if (na > 2 && nb > 0) m += ta + tb;
            if (na > 1 && nb > 1) m += 4 * tb;
            if (na > 0 && nb > 2) m += tb + ta;
            if (nb > 3) m += ta;
        }
    }
    L.ncon = m;

    // block dimensions, v2rdm_solver.cc:1129-1270 (same order as the offsets)
    auto dims = [&](const std::vector<int>& d, int mult) {
        for (int h = 0; h < H; h++) L.block_dims.push_back(mult * d[h]);
    };
    dims(gab, 1);
    dims(gaa, 1);
    dims(gaa, 1);
    if (opt.constrain_spin) dims(gab, L.singlet() ? 1 : 2);
    dims(amp, 1);
    dims(amp, 1);
    dims(amp, 1);
    dims(amp, 1);
    if (opt.constrain_q2 && !opt.spin_adapt_q2) {
        dims(gab, 1);
        dims(gaa, 1);
        dims(gaa, 1);
    } else if (opt.constrain_q2) {
        dims(L.gems_00, 1);
        dims(gaa, 1);
        dims(gaa, 1);
        dims(gaa, 1);
    }
    if (opt.constrain_g2 && !opt.spin_adapt_g2) {
        dims(gab, 1);
        dims(gab, 1);
        dims(gab, 2);
    } else if (opt.constrain_g2) {
        for (int k = 0; k < 4; k++) dims(gab, 1);
    }
    if (opt.constrain_t1) {
        dims(L.trip_aaa, 1);
        dims(L.trip_aaa, 1);
        dims(L.trip_aab, 1);
        dims(L.trip_aab, 1);
    }
    if (opt.constrain_t2) {
        std::vector<int> big(H);
        for (int h = 0; h < H; h++) big[h] = tsum(h);
        dims(big, 1);
        dims(big, 1);
        dims(L.trip_aab, 1);
        dims(L.trip_aab, 1);
    }
    if (opt.constrain_d3) {
        dims(L.trip_aaa, 1);
        dims(L.trip_aaa, 1);
        dims(L.trip_aab, 1);
        dims(L.trip_aab, 1);
    }
    if (opt.constrain_d4) {
        dims(L.quart_aaaa, 1);
        dims(L.quart_aaab, 1);
        dims(L.quart_aabb, 1);
        dims(L.quart_aaab, 1);
        dims(L.quart_aaaa, 1);
    }
    int64_t bo = 0;
    for (int d : L.block_dims) {
        L.block_off.push_back(bo);
        bo += (int64_t)d * d;
    }
    if (bo != L.dimx) return "internal error: block dimensions do not tile the primal vector";
    return "";
}

}  // namespace v2g
