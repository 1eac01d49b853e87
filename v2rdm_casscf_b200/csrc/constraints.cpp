// Constraint rows, b and c (see constraints.h).
#include "constraints.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <stdexcept>

namespace v2g {

namespace {

// Collects one row at a time; entries hitting the same primal element are
// summed, exact zeros dropped, and columns sorted.
class RowSink {
  public:
    explicit RowSink(Csr& A) : A_(A) {
        A_.rowptr.assign(1, 0);
        A_.col.clear();
        A_.val.clear();
    }
    void add(int64_t c, double v) { cur_.push_back({c, v}); }
    void end() {
        std::sort(cur_.begin(), cur_.end(), [](const E& a, const E& b) { return a.c < b.c; });
        size_t k = 0;
        while (k < cur_.size()) {
            int64_t c = cur_[k].c;
            double s = 0.0;
            while (k < cur_.size() && cur_[k].c == c) s += cur_[k++].v;
            if (s != 0.0) {
                A_.col.push_back((int32_t)c);
                A_.val.push_back(s);
            }
        }
        A_.rowptr.push_back((int64_t)A_.col.size());
        cur_.clear();
    }
    int64_t rows() const { return (int64_t)A_.rowptr.size() - 1; }

  private:
    struct E {
        int64_t c;
        double v;
    };
    Csr& A_;
    std::vector<E> cur_;
};

// D1-type element (p,q) of a family stored per irrep as amopi x amopi blocks;
// p and q are absolute active indices of the same irrep.
inline int64_t d1(const Layout& L, Fam f, int p, int q) {
    const int h = L.symmetry[p];
    const int o = L.pitzer_offset[h];
    return L.off[f][h] + (int64_t)(p - o) * L.amopi[h] + (q - o);
}
inline int64_t gem(const Layout& L, Fam f, int h, int64_t dim, int r, int c) {
    return L.off[f][h] + (int64_t)r * dim + c;
}

// d2.cc:296-547 (D2_constraints_Au)
void rows_d2(const Layout& L, RowSink& S) {
    const int n = L.amo;
    const auto& o = L.off;
    if (L.opt.constrain_sz) {
        // Tr(D2ab), Tr(D2aa), Tr(D2bb): d2.cc:301-346
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                int h = L.sym_pair(L.symmetry[i], L.symmetry[j]);
                int ij = L.ab(h, i, j);
                S.add(gem(L, F_D2AB, h, L.gems_ab[h], ij, ij), 1.0);
            }
        S.end();
        for (Fam f : {F_D2AA, F_D2BB}) {
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) {
                    if (i == j) continue;
                    int h = L.sym_pair(L.symmetry[i], L.symmetry[j]);
                    int ij = L.aa(h, i, j);
                    S.add(gem(L, f, h, L.gems_aa[h], ij, ij), 1.0);
                }
            S.end();
        }
    } else {
        // Tr(D2ab + D2aa + D2bb): d2.cc:347-367
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                int h = L.sym_pair(L.symmetry[i], L.symmetry[j]);
                int ij = L.ab(h, i, j);
                S.add(gem(L, F_D2AB, h, L.gems_ab[h], ij, ij), 2.0);
                if (i == j) continue;
                ij = L.aa(h, i, j);
                S.add(gem(L, F_D2AA, h, L.gems_aa[h], ij, ij), 1.0);
                S.add(gem(L, F_D2BB, h, L.gems_aa[h], ij, ij), 1.0);
            }
        S.end();
    }
    // D1 + Q1 = I: row (i,j) = D1(j,i) + Q1(i,j), d2.cc:369-387
    for (Fam fd : {F_D1A, F_D1B}) {
        Fam fq = (fd == F_D1A) ? F_Q1A : F_Q1B;
        for (int h = 0; h < L.nirrep; h++)
            for (int i = 0; i < L.amopi[h]; i++)
                for (int j = 0; j < L.amopi[h]; j++) {
                    S.add(o[fd][h] + (int64_t)j * L.amopi[h] + i, 1.0);
                    S.add(o[fq][h] + (int64_t)i * L.amopi[h] + j, 1.0);
                    S.end();
                }
    }
    const double na = L.na, nb = L.nb, ntot = na + nb;
    // contraction rows D2 -> D1
    auto ab_to_d1 = [&](Fam fd, double coef, bool alpha, bool with_aa, Fam faa) {
        for (int h = 0; h < L.nirrep; h++)
            for (int i = 0; i < L.amopi[h]; i++)
                for (int j = 0; j < L.amopi[h]; j++) {
                    int ii = i + L.pitzer_offset[h], jj = j + L.pitzer_offset[h];
                    S.add(o[fd][h] + (int64_t)i * L.amopi[h] + j, coef);
                    for (int k = 0; k < n; k++) {
                        int h2 = L.sym_pair(L.symmetry[ii], L.symmetry[k]);
                        int ik = alpha ? L.ab(h2, ii, k) : L.ab(h2, k, ii);
                        int jk = alpha ? L.ab(h2, jj, k) : L.ab(h2, k, jj);
                        S.add(gem(L, F_D2AB, h2, L.gems_ab[h2], ik, jk), -1.0);
                    }
                    if (with_aa) {
                        for (int k = 0; k < n; k++) {
                            if (ii == k || jj == k) continue;
                            int h2 = L.sym_pair(L.symmetry[ii], L.symmetry[k]);
                            int ik = L.aa(h2, ii, k), jk = L.aa(h2, jj, k);
                            int s = ((ii < k) ? 1 : -1) * ((jj < k) ? 1 : -1);
                            S.add(gem(L, faa, h2, L.gems_aa[h2], ik, jk), -(double)s);
                        }
                    }
                    S.end();
                }
    };
    auto aa_to_d1 = [&](Fam fd, double coef, Fam faa) {
        for (int h = 0; h < L.nirrep; h++)
            for (int i = 0; i < L.amopi[h]; i++)
                for (int j = 0; j < L.amopi[h]; j++) {
                    int ii = i + L.pitzer_offset[h], jj = j + L.pitzer_offset[h];
                    S.add(o[fd][h] + (int64_t)i * L.amopi[h] + j, coef);
                    for (int k = 0; k < n; k++) {
                        if (ii == k || jj == k) continue;
                        int h2 = L.sym_pair(L.symmetry[ii], L.symmetry[k]);
                        int ik = L.aa(h2, ii, k), jk = L.aa(h2, jj, k);
                        int s = ((ii < k) ? 1 : -1) * ((jj < k) ? 1 : -1);
                        S.add(gem(L, faa, h2, L.gems_aa[h2], ik, jk), -(double)s);
                    }
                    S.end();
                }
    };
    if (!L.opt.constrain_sz) {
        // d2.cc:395-458
        ab_to_d1(F_D1A, ntot - 1.0, true, true, F_D2AA);
        ab_to_d1(F_D1B, ntot - 1.0, false, true, F_D2BB);
    } else {
        // d2.cc:459-545
        ab_to_d1(F_D1A, nb, true, false, F_D2AA);
        ab_to_d1(F_D1B, na, false, false, F_D2AA);
        aa_to_d1(F_D1A, na - 1.0, F_D2AA);
        aa_to_d1(F_D1B, nb - 1.0, F_D2BB);
    }
}

// spin.cc:274-493 (Spin_constraints_Au)
void rows_spin(const Layout& L, RowSink& S) {
    const int n = L.amo;
    const auto& o = L.off;
    // <S^2> row, spin.cc:280-291
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            int h = L.sym_pair(L.symmetry[i], L.symmetry[j]);
            S.add(gem(L, F_D2AB, h, L.gems_ab[h], L.ab(h, i, j), L.ab(h, j, i)), 1.0);
        }
    S.end();
    const double r2 = std::sqrt(2.0);
    if (L.singlet()) {
        // D1a = D1b, spin.cc:319-324
        for (int h = 0; h < L.nirrep; h++)
            for (int64_t k = 0; k < (int64_t)L.amopi[h] * L.amopi[h]; k++) {
                S.add(o[F_D1A][h] + k, 1.0);
                S.add(o[F_D1B][h] + k, -1.0);
                S.end();
            }
        // D2aa = D2bb, spin.cc:326-331
        for (int h = 0; h < L.nirrep; h++)
            for (int64_t k = 0; k < (int64_t)L.gems_aa[h] * L.gems_aa[h]; k++) {
                S.add(o[F_D2AA][h] + k, 1.0);
                S.add(o[F_D2BB][h] + k, -1.0);
                S.end();
            }
        // D2aa / D2bb = antisymmetrised D2ab, spin.cc:332-373
        for (Fam f : {F_D2AA, F_D2BB}) {
            for (int h = 0; h < L.nirrep; h++) {
                const int ga = L.gems_aa[h], gb = L.gems_ab[h];
                for (int ij = 0; ij < ga; ij++) {
                    int i = L.bas_aa[h][ij][0], j = L.bas_aa[h][ij][1];
                    int ijb = L.ab(h, i, j), jib = L.ab(h, j, i);
                    for (int kl = 0; kl < ga; kl++) {
                        int k = L.bas_aa[h][kl][0], l = L.bas_aa[h][kl][1];
                        int klb = L.ab(h, k, l), lkb = L.ab(h, l, k);
                        S.add(gem(L, f, h, ga, ij, kl), 1.0);
                        S.add(gem(L, F_D2AB, h, gb, ijb, klb), -0.5);
                        S.add(gem(L, F_D2AB, h, gb, jib, klb), 0.5);
                        S.add(gem(L, F_D2AB, h, gb, ijb, lkb), 0.5);
                        S.add(gem(L, F_D2AB, h, gb, jib, lkb), -0.5);
                        S.end();
                    }
                }
            }
        }
        // D200 = symmetrised D2ab, spin.cc:374-394
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_ab[h];
            for (int ij = 0; ij < g; ij++) {
                int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
                int ji = L.ab(h, j, i);
                double dij = (i == j) ? r2 : 1.0;
                for (int kl = 0; kl < g; kl++) {
                    int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
                    int lk = L.ab(h, l, k);
                    double dkl = (k == l) ? r2 : 1.0;
                    double w = -0.5 / (dij * dkl);
                    S.add(gem(L, F_D200, h, g, ij, kl), 1.0);
                    S.add(gem(L, F_D2AB, h, g, ij, kl), w);
                    S.add(gem(L, F_D2AB, h, g, ji, kl), w);
                    S.add(gem(L, F_D2AB, h, g, ij, lk), w);
                    S.add(gem(L, F_D2AB, h, g, ji, lk), w);
                    S.end();
                }
            }
        }
    } else {
        // non-singlets: the 2g x 2g block of D200/D201/D210/D211, spin.cc:395-468
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_ab[h];
            for (int r = 0; r < 2 * g; r++)
                for (int cc = 0; cc < 2 * g; cc++) {
                    const int ij = r % g, kl = cc % g;
                    const bool rb = r >= g, cb = cc >= g;
                    int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
                    int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
                    int ji = L.ab(h, j, i), lk = L.ab(h, l, k);
                    double dij = (i == j) ? r2 : 1.0, dkl = (k == l) ? r2 : 1.0;
                    S.add(gem(L, F_D200, h, 2 * g, r, cc), 1.0);
                    double a, b2, c2, d;  // coefficients of (ij,kl), (ji,kl), (ij,lk), (ji,lk)
                    if (!rb && !cb) {
                        a = b2 = c2 = d = -0.5 / (dij * dkl);
                    } else if (!rb && cb) {
                        a = -0.5 / dij; c2 = 0.5 / dij; b2 = -0.5 / dij; d = 0.5 / dij;
                    } else if (rb && !cb) {
                        a = -0.5 / dkl; c2 = -0.5 / dkl; b2 = 0.5 / dkl; d = 0.5 / dkl;
                    } else {
                        a = -0.5; b2 = 0.5; c2 = 0.5; d = -0.5;
                    }
                    S.add(gem(L, F_D2AB, h, g, ij, kl), a);
                    S.add(gem(L, F_D2AB, h, g, ji, kl), b2);
                    S.add(gem(L, F_D2AB, h, g, ij, lk), c2);
                    S.add(gem(L, F_D2AB, h, g, ji, lk), d);
                    S.end();
                }
        }
    }
    if (L.opt.constrain_g2) {
        // maximal spin: sum_i G2ba(kl,ii) = 0 and sum_i G2ba(ii,kl) = 0, irrep 0
        // only, spin.cc:470-491
        const int g = L.gems_ab[0];
        for (int kl = 0; kl < g; kl++) {
            for (int i = 0; i < n; i++) S.add(gem(L, F_G2BA, 0, g, kl, L.ab(0, i, i)), 1.0);
            S.end();
        }
        for (int kl = 0; kl < g; kl++) {
            for (int i = 0; i < n; i++) S.add(gem(L, F_G2BA, 0, g, L.ab(0, i, i), kl), 1.0);
            S.end();
        }
    }
}

// q2.cc:801-950 (Q2_constraints_Au, not spin adapted)
void rows_q2(const Layout& L, RowSink& S) {
    // Q2ab: D2ab(ij,kl) - Q2ab(ij,kl) - d_jl D1a(k,i) - d_ik D1b(l,j)
    for (int h = 0; h < L.nirrep; h++) {
        const int g = L.gems_ab[h];
        for (int ij = 0; ij < g; ij++) {
            int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
            for (int kl = 0; kl < g; kl++) {
                int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
                S.add(gem(L, F_D2AB, h, g, ij, kl), 1.0);
                S.add(gem(L, F_Q2AB, h, g, ij, kl), -1.0);
                if (j == l) S.add(d1(L, F_D1A, k, i), -1.0);
                if (i == k) S.add(d1(L, F_D1B, l, j), -1.0);
                S.end();
            }
        }
    }
    // Q2aa / Q2bb
    for (int spin = 0; spin < 2; spin++) {
        Fam fd2 = spin ? F_D2BB : F_D2AA, fq2 = spin ? F_Q2BB : F_Q2AA, fd1 = spin ? F_D1B : F_D1A;
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_aa[h];
            for (int ij = 0; ij < g; ij++) {
                int i = L.bas_aa[h][ij][0], j = L.bas_aa[h][ij][1];
                for (int kl = 0; kl < g; kl++) {
                    int k = L.bas_aa[h][kl][0], l = L.bas_aa[h][kl][1];
                    S.add(gem(L, fd2, h, g, ij, kl), 1.0);
                    S.add(gem(L, fq2, h, g, ij, kl), -1.0);
                    if (j == l) S.add(d1(L, fd1, k, i), -1.0);
                    if (j == k) S.add(d1(L, fd1, l, i), 1.0);
                    if (i == l) S.add(d1(L, fd1, k, j), 1.0);
                    if (i == k) S.add(d1(L, fd1, l, j), -1.0);
                    S.end();
                }
            }
        }
    }
}

// q2.cc:260-468 (Q2_constraints_Au_spin_adapted): Q2 singlet block over the
// spatial pairs and three triplet blocks (M = 0, +1, -1) over aa pairs.
void rows_q2_spin_adapted(const Layout& L, RowSink& S) {
    auto D2 = [&](int h, int r, int c) { return gem(L, F_D2AB, h, L.gems_ab[h], r, c); };
    for (int trip = 0; trip < 2; trip++) {
        // trip = 0: Q2s (gems_00); trip = 1: Q2t, M = 0 (gems_aa)
        for (int h = 0; h < L.nirrep; h++) {
            const int g = trip ? L.gems_aa[h] : L.gems_00[h];
            const auto& bas = trip ? L.bas_aa[h] : L.bas_00[h];
            const double sg = trip ? -1.0 : 1.0;
            for (int ij = 0; ij < g; ij++) {
                const int i = bas[ij][0], j = bas[ij][1];
                const int ijd = L.ab(h, i, j), jid = L.ab(h, j, i);
                for (int kl = 0; kl < g; kl++) {
                    const int k = bas[kl][0], l = bas[kl][1];
                    const int kld = L.ab(h, k, l), lkd = L.ab(h, l, k);
                    S.add(gem(L, trip ? F_Q2T : F_Q2S, h, g, ij, kl), -1.0);
                    S.add(D2(h, kld, ijd), 0.5);
                    S.add(D2(h, lkd, ijd), 0.5 * sg);
                    S.add(D2(h, kld, jid), 0.5 * sg);
                    S.add(D2(h, lkd, jid), 0.5);
                    if (j == l) {
                        S.add(d1(L, F_Q1A, i, k), 0.5);
                        S.add(d1(L, F_D1B, i, k), -0.5);
                    }
                    if (i == k) {
                        S.add(d1(L, F_Q1A, l, j), 0.5);
                        S.add(d1(L, F_D1B, l, j), -0.5);
                    }
                    if (j == k) {
                        S.add(d1(L, F_Q1A, l, i), 0.5 * sg);
                        S.add(d1(L, F_D1B, l, i), -0.5 * sg);
                    }
                    if (i == l) {
                        S.add(d1(L, F_Q1A, k, j), 0.5 * sg);
                        S.add(d1(L, F_D1B, k, j), -0.5 * sg);
                    }
                    S.end();
                }
            }
        }
    }
    for (int beta = 0; beta < 2; beta++) {
        // Q2t, M = +1 from D2aa; M = -1 from D2bb
        const Fam fq = beta ? F_Q2TM : F_Q2TP, fd = beta ? F_D2BB : F_D2AA, fq1 = beta ? F_Q1B : F_Q1A,
                  fd1 = beta ? F_D1B : F_D1A;
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_aa[h];
            for (int ij = 0; ij < g; ij++) {
                const int i = L.bas_aa[h][ij][0], j = L.bas_aa[h][ij][1];
                for (int kl = 0; kl < g; kl++) {
                    const int k = L.bas_aa[h][kl][0], l = L.bas_aa[h][kl][1];
                    S.add(gem(L, fq, h, g, ij, kl), -1.0);
                    S.add(gem(L, fd, h, g, kl, ij), 1.0);
                    if (j == l) S.add(d1(L, fq1, i, k), 1.0);
                    if (j == k) S.add(d1(L, fd1, l, i), 1.0);
                    if (i == l) S.add(d1(L, fq1, j, k), -1.0);
                    if (i == k) S.add(d1(L, fd1, l, j), -1.0);
                    S.end();
                }
            }
        }
    }
}

// g2.cc:235-455 (G2_constraints_Au_spin_adapted): singlet and triplet
// (M = 0, +1, -1) G2 blocks over ab pairs.
void rows_g2_spin_adapted(const Layout& L, RowSink& S) {
    for (int trip = 0; trip < 2; trip++) {
        // trip = 0: G2s; trip = 1: G2t, M = 0 (the D2ab terms change sign)
        const double sab = trip ? -0.5 : 0.5;
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_ab[h];
            for (int ij = 0; ij < g; ij++) {
                const int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
                for (int kl = 0; kl < g; kl++) {
                    const int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
                    S.add(gem(L, trip ? F_G2T : F_G2S, h, g, ij, kl), -1.0);
                    if (j == l) {
                        S.add(d1(L, F_D1A, i, k), 0.5);
                        S.add(d1(L, F_D1B, i, k), 0.5);
                    }
                    const int h2 = L.sym_pair(L.symmetry[i], L.symmetry[l]);
                    if (i != l && k != j) {
                        const double sgn = (i < l ? 1.0 : -1.0) * (k < j ? 1.0 : -1.0);
                        const int ga = L.gems_aa[h2];
                        S.add(gem(L, F_D2AA, h2, ga, L.aa(h2, i, l), L.aa(h2, k, j)), -0.5 * sgn);
                        S.add(gem(L, F_D2BB, h2, ga, L.aa(h2, i, l), L.aa(h2, k, j)), -0.5 * sgn);
                    }
                    const int g2 = L.gems_ab[h2];
                    S.add(gem(L, F_D2AB, h2, g2, L.ab(h2, i, l), L.ab(h2, j, k)), sab);
                    S.add(gem(L, F_D2AB, h2, g2, L.ab(h2, l, i), L.ab(h2, k, j)), sab);
                    S.end();
                }
            }
        }
    }
    for (int beta = 0; beta < 2; beta++) {
        // G2t, M = +1: D1a(i,k) d_jl - D2ab(il,kj); M = -1: D1b(i,k) d_jl - D2ab(li,jk)
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_ab[h];
            for (int ij = 0; ij < g; ij++) {
                const int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
                for (int kl = 0; kl < g; kl++) {
                    const int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
                    S.add(gem(L, beta ? F_G2TM : F_G2TP, h, g, ij, kl), -1.0);
                    if (j == l) S.add(d1(L, beta ? F_D1B : F_D1A, i, k), 1.0);
                    const int h2 = L.sym_pair(L.symmetry[i], L.symmetry[l]);
                    const int g2 = L.gems_ab[h2];
                    if (!beta)
                        S.add(gem(L, F_D2AB, h2, g2, L.ab(h2, i, l), L.ab(h2, k, j)), -1.0);
                    else
                        S.add(gem(L, F_D2AB, h2, g2, L.ab(h2, l, i), L.ab(h2, j, k)), -1.0);
                    S.end();
                }
            }
        }
    }
}

// g2.cc:1061-1260 (G2_constraints_Au, not spin adapted)
void rows_g2(const Layout& L, RowSink& S) {
    // G2ab: -G2ab(ij,kl) + d_jl D1a(i,k) - D2ab(il,kj)
    // G2ba: -G2ba(ij,kl) + d_jl D1b(i,k) - D2ab(li,jk)
    for (int which = 0; which < 2; which++) {
        Fam fg = which ? F_G2BA : F_G2AB, fd1 = which ? F_D1B : F_D1A;
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_ab[h];
            for (int ij = 0; ij < g; ij++) {
                int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
                for (int kl = 0; kl < g; kl++) {
                    int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
                    S.add(gem(L, fg, h, g, ij, kl), -1.0);
                    if (j == l) S.add(d1(L, fd1, i, k), 1.0);
                    int h2 = L.sym_pair(L.symmetry[i], L.symmetry[l]);
                    int g2 = L.gems_ab[h2];
                    if (!which)
                        S.add(gem(L, F_D2AB, h2, g2, L.ab(h2, i, l), L.ab(h2, k, j)), -1.0);
                    else
                        S.add(gem(L, F_D2AB, h2, g2, L.ab(h2, l, i), L.ab(h2, j, k)), -1.0);
                    S.end();
                }
            }
        }
    }
    // G2 2g x 2g block: aaaa | aabb / bbaa | bbbb, g2.cc:1131-1257
    for (int h = 0; h < L.nirrep; h++) {
        const int g = L.gems_ab[h];
        for (int r = 0; r < 2 * g; r++)
            for (int cc = 0; cc < 2 * g; cc++) {
                const int ij = r % g, kl = cc % g;
                const bool rb = r >= g, cb = cc >= g;
                int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
                int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
                int h2 = L.sym_pair(L.symmetry[i], L.symmetry[l]);
                S.add(gem(L, F_G2AA, h, 2 * g, r, cc), -1.0);
                if (rb == cb) {
                    // G2aaaa / G2bbbb
                    if (j == l) S.add(d1(L, rb ? F_D1B : F_D1A, i, k), 1.0);
                    if (i != l && k != j) {
                        int s = ((i < l) ? 1 : -1) * ((k < j) ? 1 : -1);
                        int ga = L.gems_aa[h2];
                        S.add(gem(L, rb ? F_D2BB : F_D2AA, h2, ga, L.aa(h2, i, l), L.aa(h2, k, j)), -(double)s);
                    }
                } else if (!rb) {
                    // G2aabb: + D2ab(il,jk)
                    S.add(gem(L, F_D2AB, h2, L.gems_ab[h2], L.ab(h2, i, l), L.ab(h2, j, k)), 1.0);
                } else {
                    // G2bbaa: + D2ab(li,kj)
                    S.add(gem(L, F_D2AB, h2, L.gems_ab[h2], L.ab(h2, l, i), L.ab(h2, k, j)), 1.0);
                }
                S.end();
            }
    }
}

// Element (r, c) of a geminal-indexed family in irrep h; throws when an
// index does not exist, which would mean a wrong restatement.
struct Gem {
    const Layout& L;
    int64_t at(Fam f, int h, int64_t dim, int r, int c) const {
        if (r < 0 || c < 0) throw std::logic_error("constraint row refers to a missing geminal");
        return gem(L, f, h, dim, r, c);
    }
    int hp(int p, int q) const { return L.sym_pair(L.symmetry[p], L.symmetry[q]); }
    // D2ab-type (ab geminals), D2aa-type (aa geminals), G2 2g x 2g
    int64_t ab(Fam f, int p, int q, int r, int s) const {
        const int h = hp(p, q);
        return at(f, h, L.gems_ab[h], L.ab(h, p, q), L.ab(h, r, s));
    }
    int64_t aa(Fam f, int p, int q, int r, int s) const {
        const int h = hp(p, q);
        return at(f, h, L.gems_aa[h], L.aa(h, p, q), L.aa(h, r, s));
    }
    int64_t g2(bool beta, int p, int q, int r, int s) const {
        const int h = hp(p, q), g = L.gems_ab[h], o = beta ? g : 0;
        if (L.ab(h, p, q) < 0 || L.ab(h, r, s) < 0) throw std::logic_error("constraint row refers to a missing geminal");
        return at(F_G2AA, h, 2 * g, L.ab(h, p, q) + o, L.ab(h, r, s) + o);
    }
};

// Sign of the antisymmetric pair (p,q) stored as its p > q geminal.
inline int pair_sign(int p, int q) { return p > q ? -1 : 1; }

// t1.cc:433-811 (T1_constraints_Au).  Row order aab, bba, aaa, bbb; every
// row is -T1(ijk,lmn) plus Q2 / D2 / G2 / D1 terms selected by coincident
// indices.
void rows_t1(const Layout& L, RowSink& S) {
    const Gem G{L};
    for (int beta = 0; beta < 2; beta++) {
        const Fam ft = beta ? F_T1BBA : F_T1AAB, fq = beta ? F_Q2BB : F_Q2AA, fg = beta ? F_G2AB : F_G2BA;
        for (int h = 0; h < L.nirrep; h++) {
            const int nt = L.trip_aab[h];
            for (int I = 0; I < nt; I++) {
                const int i = L.bas_aab[h][I][0], j = L.bas_aab[h][I][1], k = L.bas_aab[h][I][2];
                for (int J = 0; J < nt; J++) {
                    const int l = L.bas_aab[h][J][0], m = L.bas_aab[h][J][1], n = L.bas_aab[h][J][2];
                    S.add(G.at(ft, h, nt, I, J), -1.0);
                    if (k == n) S.add(G.aa(fq, i, j, l, m), 1.0);
                    if (!beta) {
                        if (j == l) S.add(G.ab(F_D2AB, m, n, i, k), -1.0);
                        if (l == i) S.add(G.ab(F_D2AB, m, n, j, k), 1.0);
                    } else {
                        if (j == l) S.add(G.ab(F_D2AB, n, m, k, i), -1.0);
                        if (l == i) S.add(G.ab(F_D2AB, n, m, k, j), 1.0);
                    }
                    if (j == m) S.add(G.ab(fg, n, i, k, l), -1.0);
                    if (i == m) S.add(G.ab(fg, n, j, k, l), 1.0);
                    S.end();
                }
            }
        }
    }
    for (int beta = 0; beta < 2; beta++) {
        const Fam ft = beta ? F_T1BBB : F_T1AAA, fq = beta ? F_Q2BB : F_Q2AA, fd = beta ? F_D2BB : F_D2AA,
                  f1 = beta ? F_D1B : F_D1A;
        for (int h = 0; h < L.nirrep; h++) {
            const int nt = L.trip_aaa[h];
            for (int I = 0; I < nt; I++) {
                const int i = L.bas_aaa[h][I][0], j = L.bas_aaa[h][I][1], k = L.bas_aaa[h][I][2];
                for (int J = 0; J < nt; J++) {
                    const int l = L.bas_aaa[h][J][0], m = L.bas_aaa[h][J][1], n = L.bas_aaa[h][J][2];
                    S.add(G.at(ft, h, nt, I, J), -1.0);
                    if (k == n) S.add(G.aa(fq, i, j, l, m), 1.0);
                    if (j == n && G.hp(i, k) == G.hp(l, m)) S.add(G.aa(fq, i, k, l, m), -1.0);
                    if (i == n && G.hp(j, k) == G.hp(l, m)) S.add(G.aa(fq, j, k, l, m), 1.0);
                    if (l == k && G.hp(j, i) == G.hp(n, m)) S.add(G.aa(fd, n, m, j, i), 1.0);
                    if (j == l) S.add(G.aa(fd, n, m, k, i), -1.0);
                    if (l == i) S.add(G.aa(fd, n, m, k, j), 1.0);
                    if (k == m) {
                        if (j == l) S.add(d1(L, f1, n, i), -1.0);
                        S.add(G.g2(beta, n, i, j, l), 1.0);
                    }
                    if (j == m) {
                        if (k == l) S.add(d1(L, f1, n, i), 1.0);
                        S.add(G.g2(beta, n, i, k, l), -1.0);
                    }
                    if (i == m) {
                        if (k == l) S.add(d1(L, f1, n, j), -1.0);
                        S.add(G.g2(beta, n, j, k, l), 1.0);
                    }
                    S.end();
                }
            }
        }
    }
}

// t2.cc:1251-1862 (T2_constraints_Au_slow, the form the reference calls).
// Row order aab, bba, then the two (aab + aba)-dimensional blocks aaa/abb
// and bbb/baa, each walked row by row over its four sub-blocks.
void rows_t2(const Layout& L, RowSink& S) {
    const Gem G{L};
    for (int beta = 0; beta < 2; beta++) {
        const Fam ft = beta ? F_T2BBA : F_T2AAB, fd = beta ? F_D2BB : F_D2AA, f1 = beta ? F_D1A : F_D1B;
        for (int h = 0; h < L.nirrep; h++) {
            const int nt = L.trip_aab[h];
            for (int I = 0; I < nt; I++) {
                const int i = L.bas_aab[h][I][0], j = L.bas_aab[h][I][1], k = L.bas_aab[h][I][2];
                for (int J = 0; J < nt; J++) {
                    const int l = L.bas_aab[h][J][0], m = L.bas_aab[h][J][1], n = L.bas_aab[h][J][2];
                    S.add(G.at(ft, h, nt, I, J), -1.0);
                    if (k == n) S.add(G.aa(fd, i, j, l, m), 1.0);
                    if (j == m && i == l) S.add(d1(L, f1, n, k), 1.0);
                    if (j == l && i == m) S.add(d1(L, f1, n, k), -1.0);
                    if (!beta) {
                        if (i == l) S.add(G.ab(F_D2AB, j, n, m, k), -1.0);
                        if (j == l) S.add(G.ab(F_D2AB, i, n, m, k), 1.0);
                        if (i == m) S.add(G.ab(F_D2AB, j, n, l, k), 1.0);
                        if (j == m) S.add(G.ab(F_D2AB, i, n, l, k), -1.0);
                    } else {
                        if (i == l) S.add(G.ab(F_D2AB, n, j, k, m), -1.0);
                        if (j == l) S.add(G.ab(F_D2AB, n, i, k, m), 1.0);
                        if (i == m) S.add(G.ab(F_D2AB, n, j, k, l), 1.0);
                        if (j == m) S.add(G.ab(F_D2AB, n, i, k, l), -1.0);
                    }
                    S.end();
                }
            }
        }
    }
    for (int beta = 0; beta < 2; beta++) {
        // beta = 0: aaa/abb block (same-spin D2aa, D1a; mixed D2ab, D2bb)
        // beta = 1: bbb/baa block (same-spin D2bb, D1b; mixed D2ab, D2aa)
        const Fam ft = beta ? F_T2BBB : F_T2AAA;
        const Fam fs = beta ? F_D2BB : F_D2AA, fo = beta ? F_D2AA : F_D2BB;
        const Fam f1s = beta ? F_D1B : F_D1A, f1o = beta ? F_D1A : F_D1B;
        for (int h = 0; h < L.nirrep; h++) {
            const int na = L.trip_aab[h], nt = L.trip_aab[h] + L.trip_aba[h];
            for (int I = 0; I < nt; I++) {
                const bool ri = I >= na;
                const auto& tI = ri ? L.bas_aba[h][I - na] : L.bas_aab[h][I];
                const int i = tI[0], j = tI[1], k = tI[2];
                for (int J = 0; J < nt; J++) {
                    const bool cj = J >= na;
                    const auto& tJ = cj ? L.bas_aba[h][J - na] : L.bas_aab[h][J];
                    const int l = tJ[0], m = tJ[1], n = tJ[2];
                    S.add(G.at(ft, h, nt, I, J), -1.0);
                    if (!ri && !cj) {
                        // same-spin triplets
                        if (k == n) S.add(G.aa(fs, i, j, l, m), 1.0);
                        if (j == m && i == l) S.add(d1(L, f1s, n, k), 1.0);
                        if (j == l && i == m) S.add(d1(L, f1s, n, k), -1.0);
                        if (i == l && n != j && k != m)
                            S.add(G.aa(fs, n, j, k, m), -(double)(pair_sign(n, j) * pair_sign(k, m)));
                        if (j == l && n != i && k != m)
                            S.add(G.aa(fs, n, i, k, m), (double)(pair_sign(n, i) * pair_sign(k, m)));
                        if (i == m && n != j && k != l)
                            S.add(G.aa(fs, n, j, k, l), (double)(pair_sign(n, j) * pair_sign(k, l)));
                        if (j == m && n != i && k != l)
                            S.add(G.aa(fs, n, i, k, l), -(double)(pair_sign(n, i) * pair_sign(k, l)));
                    } else if (!ri && cj) {
                        if (!beta) {
                            if (i == l) S.add(G.ab(F_D2AB, j, n, k, m), 1.0);
                            if (j == l) S.add(G.ab(F_D2AB, i, n, k, m), -1.0);
                        } else {
                            if (i == l) S.add(G.ab(F_D2AB, n, j, m, k), 1.0);
                            if (j == l) S.add(G.ab(F_D2AB, n, i, m, k), -1.0);
                        }
                    } else if (ri && !cj) {
                        if (!beta) {
                            if (i == l) S.add(G.ab(F_D2AB, n, j, m, k), 1.0);
                            if (i == m) S.add(G.ab(F_D2AB, n, j, l, k), -1.0);
                        } else {
                            if (i == l) S.add(G.ab(F_D2AB, j, n, k, m), 1.0);
                            if (i == m) S.add(G.ab(F_D2AB, j, n, k, l), -1.0);
                        }
                    } else {
                        // mixed-spin triplets on both sides
                        if (!beta) {
                            if (k == n) S.add(G.ab(F_D2AB, i, j, l, m), 1.0);
                        } else {
                            if (k == n) S.add(G.ab(F_D2AB, j, i, m, l), 1.0);
                        }
                        if (j == m && i == l) S.add(d1(L, f1o, n, k), 1.0);
                        if (i == l && n != j && k != m)
                            S.add(G.aa(fo, n, j, k, m), -(double)(pair_sign(n, j) * pair_sign(k, m)));
                        if (!beta) {
                            if (j == m) S.add(G.ab(F_D2AB, i, n, l, k), -1.0);
                        } else {
                            if (j == m) S.add(G.ab(F_D2AB, n, i, k, l), -1.0);
                        }
                    }
                    S.end();
                }
            }
        }
    }
}

// d3.cc:57-298 (D3_constraints_Au): the partial traces of D3 onto D2, with
// the active electron counts, and for singlets with CONSTRAIN_SPIN the
// D3aab = D3bba and D3aaa / D3bbb <- D3aab / D3bba relations.
void rows_d3(const Layout& L, RowSink& S) {
    const Gem G{L};
    const int n = L.amo;
    const double na = L.na, nb = L.nb;
    auto aaa = [&](int h, int i, int j, int k) {
        const int v = L.aaa(h, i, j, k);
        if (v < 0) throw std::logic_error("constraint row refers to a missing triplet");
        return v;
    };
    auto aab = [&](int h, int i, int j, int k) {
        const int v = L.aab(h, i, j, k);
        if (v < 0) throw std::logic_error("constraint row refers to a missing triplet");
        return v;
    };
    // D3aaa -> D2aa (na > 2), D3bbb -> D2bb (nb > 2)
    for (int beta = 0; beta < 2; beta++) {
        const double ne = beta ? nb : na;
        if (!(ne > 2)) continue;
        const Fam f2 = beta ? F_D2BB : F_D2AA, f3 = beta ? F_D3BBB : F_D3AAA;
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_aa[h];
            for (int ij = 0; ij < g; ij++) {
                const int i = L.bas_aa[h][ij][0], j = L.bas_aa[h][ij][1];
                for (int kl = 0; kl < g; kl++) {
                    const int k = L.bas_aa[h][kl][0], l = L.bas_aa[h][kl][1];
                    S.add(gem(L, f2, h, g, ij, kl), ne - 2.0);
                    for (int p = 0; p < n; p++) {
                        if (i == p || j == p || k == p || l == p) continue;
                        const int h2 = L.sym_pair(h, L.symmetry[p]);
                        const int s = ((p < i) ^ (p < j) ^ (p < k) ^ (p < l)) ? -1 : 1;
                        S.add(G.at(f3, h2, L.trip_aaa[h2], aaa(h2, i, j, p), aaa(h2, k, l, p)), -(double)s);
                    }
                    S.end();
                }
            }
        }
    }
    // D3aab -> D2aa (times nb), D3bba -> D2bb (times na)
    for (int beta = 0; beta < 2; beta++) {
        const double ne = beta ? na : nb;
        const Fam f2 = beta ? F_D2BB : F_D2AA, f3 = beta ? F_D3BBA : F_D3AAB;
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_aa[h];
            for (int ij = 0; ij < g; ij++) {
                const int i = L.bas_aa[h][ij][0], j = L.bas_aa[h][ij][1];
                for (int kl = 0; kl < g; kl++) {
                    const int k = L.bas_aa[h][kl][0], l = L.bas_aa[h][kl][1];
                    S.add(gem(L, f2, h, g, ij, kl), ne);
                    for (int p = 0; p < n; p++) {
                        const int h2 = L.sym_pair(h, L.symmetry[p]);
                        S.add(G.at(f3, h2, L.trip_aab[h2], aab(h2, i, j, p), aab(h2, k, l, p)), -1.0);
                    }
                    S.end();
                }
            }
        }
    }
    // D3aab -> D2ab (na > 1), D3bba -> D2ab (nb > 1)
    for (int beta = 0; beta < 2; beta++) {
        const double ne = beta ? nb : na;
        if (!(ne > 1)) continue;
        const Fam f3 = beta ? F_D3BBA : F_D3AAB;
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_ab[h];
            for (int ij = 0; ij < g; ij++) {
                const int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
                for (int kl = 0; kl < g; kl++) {
                    const int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
                    S.add(gem(L, F_D2AB, h, g, ij, kl), ne - 1.0);
                    // alpha pair (i, p) with beta j; beta: beta pair (j, p) with alpha i
                    const int a = beta ? j : i, c = beta ? l : k;
                    const int o1 = beta ? i : j, o2 = beta ? k : l;
                    for (int p = 0; p < n; p++) {
                        if (a == p || c == p) continue;
                        const int h2 = L.sym_pair(h, L.symmetry[p]);
                        const int s = ((p < a) ^ (p < c)) ? -1 : 1;
                        S.add(G.at(f3, h2, L.trip_aab[h2], aab(h2, a, p, o1), aab(h2, c, p, o2)), -(double)s);
                    }
                    S.end();
                }
            }
        }
    }
    if (!(L.opt.constrain_spin && L.singlet())) return;
    // D3aab = D3bba
    for (int h = 0; h < L.nirrep; h++) {
        const int t = L.trip_aab[h];
        for (int r = 0; r < t; r++)
            for (int c = 0; c < t; c++) {
                S.add(G.at(F_D3AAB, h, t, r, c), 1.0);
                S.add(G.at(F_D3BBA, h, t, r, c), -1.0);
                S.end();
            }
    }
    // D3aaa <- D3aab, D3bbb <- D3bba: D3aaa(pqr,stu) - 1/3 sum of the nine
    // antisymmetrised D3aab elements
    for (int beta = 0; beta < 2; beta++) {
        const Fam f3 = beta ? F_D3BBB : F_D3AAA, fm = beta ? F_D3BBA : F_D3AAB;
        for (int h = 0; h < L.nirrep; h++) {
            const int t = L.trip_aaa[h], tb = L.trip_aab[h];
            for (int r = 0; r < t; r++) {
                const int p = L.bas_aaa[h][r][0], q = L.bas_aaa[h][r][1], rr = L.bas_aaa[h][r][2];
                const int row[3] = {aab(h, p, q, rr), aab(h, p, rr, q), aab(h, q, rr, p)};
                const double rs[3] = {1.0, -1.0, 1.0};
                for (int c = 0; c < t; c++) {
                    const int s_ = L.bas_aaa[h][c][0], tt = L.bas_aaa[h][c][1], u = L.bas_aaa[h][c][2];
                    const int col[3] = {aab(h, s_, tt, u), aab(h, s_, u, tt), aab(h, tt, u, s_)};
                    const double cs[3] = {1.0, -1.0, 1.0};
                    S.add(G.at(f3, h, t, r, c), 1.0);
                    for (int x = 0; x < 3; x++)
                        for (int y = 0; y < 3; y++) S.add(G.at(fm, h, tb, row[x], col[y]), -(1.0 / 3.0) * rs[x] * cs[y]);
                    S.end();
                }
            }
        }
    }
}

// d4.cc:55-312 (D4_constraints_Au): partial traces of D4 onto D3 with the
// active electron counts; the reference's constraint count adds two empty
// blocks after them (see build_layout).
void rows_d4(const Layout& L, RowSink& S) {
    const Gem G{L};
    const int n = L.amo;
    const double na = L.na, nb = L.nb;
    auto chk = [](int v) {
        if (v < 0) throw std::logic_error("constraint row refers to a missing quartet");
        return v;
    };
    auto q = [&](const std::vector<std::vector<int>>& m, int h, int a, int b, int c, int d) {
        return chk(L.q4(m, h, a, b, c, d));
    };
    auto parity = [](int p, std::initializer_list<int> xs) {
        int c = 0;
        for (int x : xs) c += p < x;
        return (c & 1) ? -1.0 : 1.0;
    };
    // rows over same-spin triplets (bas_aaa): D4aaaa/bbbb (p distinct, signed) or
    // D4aaab/bbba (all p, unsigned)
    auto aaa_rows = [&](Fam f3, double coef, Fam f4, bool four_same) {
        for (int h = 0; h < L.nirrep; h++) {
            const int t = L.trip_aaa[h];
            for (int r = 0; r < t; r++) {
                const int i = L.bas_aaa[h][r][0], j = L.bas_aaa[h][r][1], k = L.bas_aaa[h][r][2];
                for (int c = 0; c < t; c++) {
                    const int l = L.bas_aaa[h][c][0], m = L.bas_aaa[h][c][1], nn = L.bas_aaa[h][c][2];
                    S.add(G.at(f3, h, t, r, c), coef);
                    for (int p = 0; p < n; p++) {
                        const int h2 = L.sym_pair(h, L.symmetry[p]);
                        if (four_same) {
                            if (p == i || p == j || p == k || p == l || p == m || p == nn) continue;
                            S.add(G.at(f4, h2, L.quart_aaaa[h2], q(L.ibas_aaaa, h2, i, j, k, p),
                                       q(L.ibas_aaaa, h2, l, m, nn, p)),
                                  -parity(p, {i, j, k, l, m, nn}));
                        } else {
                            S.add(G.at(f4, h2, L.quart_aaab[h2], q(L.ibas_aaab, h2, i, j, k, p),
                                       q(L.ibas_aaab, h2, l, m, nn, p)),
                                  -1.0);
                        }
                    }
                    S.end();
                }
            }
        }
    };
    // rows over mixed triplets (bas_aab) from D4aaab / D4bbba: the same-spin
    // pair (i,j) gains p
    auto aab_rows_3 = [&](Fam f3, double coef, Fam f4) {
        for (int h = 0; h < L.nirrep; h++) {
            const int t = L.trip_aab[h];
            for (int r = 0; r < t; r++) {
                const int i = L.bas_aab[h][r][0], j = L.bas_aab[h][r][1], k = L.bas_aab[h][r][2];
                for (int c = 0; c < t; c++) {
                    const int l = L.bas_aab[h][c][0], m = L.bas_aab[h][c][1], nn = L.bas_aab[h][c][2];
                    S.add(G.at(f3, h, t, r, c), coef);
                    for (int p = 0; p < n; p++) {
                        if (p == i || p == j || p == l || p == m) continue;
                        const int h2 = L.sym_pair(h, L.symmetry[p]);
                        S.add(G.at(f4, h2, L.quart_aaab[h2], q(L.ibas_aaab, h2, i, j, p, k),
                                   q(L.ibas_aaab, h2, l, m, p, nn)),
                              -parity(p, {i, j, l, m}));
                    }
                    S.end();
                }
            }
        }
    };
    if (na > 3) aaa_rows(F_D3AAA, na - 3.0, F_D4AAAA, true);
    if (na > 2 && nb > 0) {
        aaa_rows(F_D3AAA, nb, F_D4AAAB, false);
        aab_rows_3(F_D3AAB, na - 2.0, F_D4AAAB);
    }
    if (na > 1 && nb > 1) {
        // D4aabb -> D3aab (times nb - 1) and -> D3bba (times na - 1)
        for (int beta = 0; beta < 2; beta++) {
            for (int h = 0; h < L.nirrep; h++) {
                const int t = L.trip_aab[h];
                for (int r = 0; r < t; r++) {
                    const int i = L.bas_aab[h][r][0], j = L.bas_aab[h][r][1], k = L.bas_aab[h][r][2];
                    for (int c = 0; c < t; c++) {
                        const int l = L.bas_aab[h][c][0], m = L.bas_aab[h][c][1], nn = L.bas_aab[h][c][2];
                        S.add(G.at(beta ? F_D3BBA : F_D3AAB, h, t, r, c), beta ? na - 1.0 : nb - 1.0);
                        for (int p = 0; p < n; p++) {
                            const int h2 = L.sym_pair(h, L.symmetry[p]);
                            if (p == k || p == nn) continue;
                            const int a = beta ? q(L.ibas_aabb, h2, k, p, i, j) : q(L.ibas_aabb, h2, i, j, k, p);
                            const int b = beta ? q(L.ibas_aabb, h2, nn, p, l, m) : q(L.ibas_aabb, h2, l, m, nn, p);
                            S.add(G.at(F_D4AABB, h2, L.quart_aabb[h2], a, b), -parity(p, {k, nn}));
                        }
                        S.end();
                    }
                }
            }
        }
    }
    if (na > 0 && nb > 2) {
        aaa_rows(F_D3BBB, na, F_D4BBBA, false);
        aab_rows_3(F_D3BBA, nb - 2.0, F_D4BBBA);
    }
    if (nb > 3) aaa_rows(F_D3BBB, nb - 3.0, F_D4BBBB, true);
    // the empty rows the reference's count adds (v2rdm_solver.cc:1108-1115)
    if (na > 1 && nb > 1)
        for (int h = 0; h < L.nirrep; h++)
            for (int64_t r = 0; r < 2 * (int64_t)L.trip_aab[h] * L.trip_aab[h]; r++) S.end();
}

}  // namespace

std::string build_A(const Layout& L, Csr& A) {
    if (L.dimx >= (int64_t)INT32_MAX) return "primal vector too long for 32-bit column indices";
    RowSink S(A);
    rows_d2(L, S);
    if (L.opt.constrain_spin) rows_spin(L, S);
    if (L.opt.constrain_q2) (L.opt.spin_adapt_q2 ? rows_q2_spin_adapted : rows_q2)(L, S);
    if (L.opt.constrain_g2) (L.opt.spin_adapt_g2 ? rows_g2_spin_adapted : rows_g2)(L, S);
    if (L.opt.constrain_t1) rows_t1(L, S);
    if (L.opt.constrain_t2) rows_t2(L, S);
    if (L.opt.constrain_d3) rows_d3(L, S);
    if (L.opt.constrain_d4) rows_d4(L, S);
    A.nrows = S.rows();
    A.ncols = L.dimx;
    if (A.nrows != L.ncon) return "internal error: constraint row count mismatch";
    return "";
}

void transpose(const Csr& A, Csr& AT) {
    AT.nrows = A.ncols;
    AT.ncols = A.nrows;
    AT.rowptr.assign(AT.nrows + 1, 0);
    for (int32_t c : A.col) AT.rowptr[c + 1]++;
    for (int64_t r = 0; r < AT.nrows; r++) AT.rowptr[r + 1] += AT.rowptr[r];
    AT.col.resize(A.col.size());
    AT.val.resize(A.val.size());
    std::vector<int64_t> fill(AT.rowptr.begin(), AT.rowptr.end() - 1);
    for (int64_t r = 0; r < A.nrows; r++)
        for (int64_t k = A.rowptr[r]; k < A.rowptr[r + 1]; k++) {
            int64_t dst = fill[A.col[k]]++;
            AT.col[dst] = (int32_t)r;
            AT.val[dst] = A.val[k];
        }
}

void build_b(const Layout& L, std::vector<double>& b) {
    b.assign(L.ncon, 0.0);
    int64_t o = 0;
    const double na = L.na, nb = L.nb, ntot = na + nb;
    if (L.opt.constrain_sz) {
        b[o++] = na * nb;
        b[o++] = na * (na - 1.0);
        b[o++] = nb * (nb - 1.0);
    } else {
        b[o++] = ntot * (ntot - 1.0);
    }
    for (int s = 0; s < 2; s++)
        for (int h = 0; h < L.nirrep; h++) {
            for (int i = 0; i < L.amopi[h]; i++)
                for (int j = 0; j < L.amopi[h]; j++) b[o + (int64_t)i * L.amopi[h] + j] = (i == j);
            o += (int64_t)L.amopi[h] * L.amopi[h];
        }
    for (int h = 0; h < L.nirrep; h++) o += (L.opt.constrain_sz ? 4 : 2) * (int64_t)L.amopi[h] * L.amopi[h];
    if (L.opt.constrain_spin) {
        // "funny ab trace": N/2 + Ms^2 - Ms(Ms+1), v2rdm_solver.cc:2616-2618
        double ms = (L.multiplicity - 1.0) / 2.0;
        b[o++] = 0.5 * (na + nb) + ms * ms - ms * (ms + 1.0);
        for (int h = 0; h < L.nirrep; h++) {
            if (L.singlet())
                o += (int64_t)L.amopi[h] * L.amopi[h] + 3 * (int64_t)L.gems_aa[h] * L.gems_aa[h] +
                     (int64_t)L.gems_ab[h] * L.gems_ab[h];
            else
                o += 4 * (int64_t)L.gems_ab[h] * L.gems_ab[h];
        }
        if (L.opt.constrain_g2) o += 2 * (int64_t)L.gems_ab[0];
    }
    if (L.opt.constrain_q2 && !L.opt.spin_adapt_q2) {  // spin-adapted Q2 rows have b = 0
        // v2rdm_solver.cc:2650-2695
        for (int h = 0; h < L.nirrep; h++) {
            const int g = L.gems_ab[h];
            for (int ij = 0; ij < g; ij++)
                for (int kl = 0; kl < g; kl++) {
                    int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
                    int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
                    b[o + (int64_t)ij * g + kl] = -(double)((i == k) * (j == l));
                }
            o += (int64_t)g * g;
        }
        for (int s = 0; s < 2; s++)
            for (int h = 0; h < L.nirrep; h++) {
                const int g = L.gems_aa[h];
                for (int ij = 0; ij < g; ij++)
                    for (int kl = 0; kl < g; kl++) {
                        int i = L.bas_aa[h][ij][0], j = L.bas_aa[h][ij][1];
                        int k = L.bas_aa[h][kl][0], l = L.bas_aa[h][kl][1];
                        b[o + (int64_t)ij * g + kl] = -(double)((i == k) * (j == l)) + (double)((i == l) * (j == k));
                    }
                o += (int64_t)g * g;
            }
    }
    // G2, T1 and T2 rows have b = 0.
}

std::string build_c(const Layout& L, const OrbitalSpaces& sp, const double* oei, const double* qmo, int nq,
                    std::vector<double>& c, double& efzc) {
    const int H = L.nirrep;
    if ((int)sp.frzcpi.size() != H || (int)sp.rstcpi.size() != H || (int)sp.amopi.size() != H ||
        (int)sp.rstvpi.size() != H || (int)sp.frzvpi.size() != H)
        return "orbital space arrays must have nirrep entries";
    for (int h = 0; h < H; h++)
        if (sp.amopi[h] != L.amopi[h]) return "active orbitals per irrep differ from the layout";
    // "full" space = all orbitals except frozen virtuals, Pitzer order.
    std::vector<int> nfull(H), full_off(H), oei_off(H);
    int nf = 0, no = 0;
    for (int h = 0; h < H; h++) {
        nfull[h] = sp.frzcpi[h] + sp.rstcpi[h] + sp.amopi[h] + sp.rstvpi[h];
        full_off[h] = nf;
        oei_off[h] = no;
        nf += nfull[h];
        no += nfull[h] * (nfull[h] + 1) / 2;
    }
    const int64_t ntri = (int64_t)nf * (nf + 1) / 2;
    auto idx = [](int64_t i, int64_t j) { return i > j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; };
    // TEI via the three-index factors, tei.cc:315-321
    auto tei = [&](int i, int j, int k, int l) {
        const double* a = qmo + idx(i, j);
        const double* b = qmo + idx(k, l);
        double s = 0.0;
        for (int q = 0; q < nq; q++) s += a[q * ntri] * b[q * ntri];
        return s;
    };
    // active orbital -> full-space index (basis.cc:122-129)
    std::vector<int> full_basis(L.amo);
    for (int h = 0; h < H; h++)
        for (int i = 0; i < L.amopi[h]; i++)
            full_basis[L.pitzer_offset[h] + i] = full_off[h] + sp.frzcpi[h] + sp.rstcpi[h] + i;

    c.assign(L.dimx, 0.0);
    // FrozenCoreEnergy, tei.cc:230-313
    efzc = 0.0;
    for (int h = 0; h < H; h++)
        for (int i = 0; i < sp.frzcpi[h] + sp.rstcpi[h]; i++) {
            int ifull = i + full_off[h];
            efzc += 2.0 * oei[oei_off[h] + idx(i, i)];
            for (int h2 = 0; h2 < H; h2++)
                for (int j = 0; j < sp.frzcpi[h2] + sp.rstcpi[h2]; j++) {
                    int jfull = j + full_off[h2];
                    efzc += 2.0 * tei(ifull, ifull, jfull, jfull) - tei(ifull, jfull, ifull, jfull);
                }
        }
    for (int h = 0; h < H; h++) {
        const int core = sp.frzcpi[h] + sp.rstcpi[h];
        for (int i = core; i < core + sp.amopi[h]; i++)
            for (int j = core; j < core + sp.amopi[h]; j++) {
                int ifull = i + full_off[h], jfull = j + full_off[h];
                double dum = 0.0;
                for (int h2 = 0; h2 < H; h2++)
                    for (int k = 0; k < sp.frzcpi[h2] + sp.rstcpi[h2]; k++) {
                        int kfull = k + full_off[h2];
                        dum += 2.0 * tei(ifull, jfull, kfull, kfull) - tei(ifull, kfull, jfull, kfull);
                    }
                double v = oei[oei_off[h] + idx(i, j)] + dum;
                int64_t e = (int64_t)(i - core) * L.amopi[h] + (j - core);
                c[L.off[F_D1A][h] + e] = v;
                c[L.off[F_D1B][h] + e] = v;
            }
    }
    // RepackIntegrals two-electron part, tei.cc:144-228
    for (int h = 0; h < H; h++) {
        const int g = L.gems_ab[h];
        for (int ij = 0; ij < g; ij++) {
            int ii = full_basis[L.bas_ab[h][ij][0]], jj = full_basis[L.bas_ab[h][ij][1]];
            for (int kl = 0; kl < g; kl++) {
                int kk = full_basis[L.bas_ab[h][kl][0]], ll = full_basis[L.bas_ab[h][kl][1]];
                c[L.off[F_D2AB][h] + (int64_t)ij * g + kl] = tei(ii, kk, jj, ll);
            }
        }
        const int ga = L.gems_aa[h];
        for (int ij = 0; ij < ga; ij++) {
            int ii = full_basis[L.bas_aa[h][ij][0]], jj = full_basis[L.bas_aa[h][ij][1]];
            for (int kl = 0; kl < ga; kl++) {
                int kk = full_basis[L.bas_aa[h][kl][0]], ll = full_basis[L.bas_aa[h][kl][1]];
                double v = tei(ii, kk, jj, ll) - tei(ii, ll, jj, kk);
                c[L.off[F_D2AA][h] + (int64_t)ij * ga + kl] = v;
                c[L.off[F_D2BB][h] + (int64_t)ij * ga + kl] = v;
            }
        }
    }
    return "";
}

void build_spatial_map(const Layout& L, const double* active_energies, Csr& P, int64_t& d1_dim, int64_t& d2_dim) {
    const int n = L.amo, H = L.nirrep;
    // active orbitals in energy order; ties keep Pitzer order (the reference
    // takes the first strict minimum, basis.cc:211-238)
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    if (active_energies)
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return active_energies[a] < active_energies[b]; });
    // spatial pairs (basis.cc:626-652)
    std::vector<int> g00(H, 0);
    std::vector<std::vector<int>> i00(H, std::vector<int>((size_t)n * n, -1));
    for (int ie = 0; ie < n; ie++)
        for (int je = 0; je <= ie; je++) {
            const int i = order[ie], j = order[je];
            const int h = L.sym_pair(L.symmetry[i], L.symmetry[j]);
            i00[h][(size_t)i * n + j] = g00[h];
            i00[h][(size_t)j * n + i] = g00[h];
            g00[h]++;
        }
    auto tri = [](int64_t a, int64_t b) { return a > b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; };
    std::vector<int64_t> off2(H + 1, 0), off1(H + 1, 0);
    for (int h = 0; h < H; h++) {
        off2[h + 1] = off2[h] + (int64_t)g00[h] * (g00[h] + 1) / 2;
        off1[h + 1] = off1[h] + (int64_t)L.amopi[h] * (L.amopi[h] + 1) / 2;
    }
    d1_dim = off1[H];
    d2_dim = off2[H];
    // the last (h, ij, kl) of the reference's loop that writes each element
    std::vector<int64_t> win((size_t)d2_dim, -1);
    int64_t gmax = 1;
    for (int h = 0; h < H; h++) gmax = std::max<int64_t>(gmax, L.gems_ab[h]);
    for (int h = 0; h < H; h++)
        for (int ij = 0; ij < L.gems_ab[h]; ij++) {
            const int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
            for (int kl = 0; kl < L.gems_ab[h]; kl++) {
                const int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
                const int hik = L.sym_pair(L.symmetry[i], L.symmetry[k]);
                const int ik = i00[hik][(size_t)i * n + k], jl = i00[hik][(size_t)j * n + l];
                win[(size_t)(off2[hik] + tri(ik, jl))] = ((int64_t)h * gmax + ij) * gmax + kl;
            }
        }
    P = Csr();
    P.nrows = d1_dim + d2_dim;
    P.ncols = L.dimx;
    P.rowptr.assign(1, 0);
    // d1: D1a(i,j) + D1b(i,j), i <= j, element INDEX(i,j) of irrep h
    std::vector<std::array<int64_t, 2>> r1((size_t)d1_dim, {-1, -1});
    for (int h = 0; h < H; h++)
        for (int i = 0; i < L.amopi[h]; i++)
            for (int j = i; j < L.amopi[h]; j++) {
                const int64_t e = (int64_t)i * L.amopi[h] + j;
                r1[(size_t)(off1[h] + tri(i, j))] = {L.off[F_D1A][h] + e, L.off[F_D1B][h] + e};
            }
    for (const auto& r : r1) {
        for (int64_t c : r) {
            P.col.push_back((int32_t)c);
            P.val.push_back(1.0);
        }
        P.rowptr.push_back((int64_t)P.col.size());
    }
    // d2: the sixteen terms of v2rdm_solver.cc:3713-3742 in their order
    auto ab = [&](int h, int p, int q) { return L.ab(h, p, q); };
    auto aa = [&](int h, int p, int q) { return L.aa(h, p, q); };
    for (int64_t id = 0; id < d2_dim; id++) {
        const int64_t w = win[(size_t)id];
        if (w >= 0) {
            const int h = (int)(w / (gmax * gmax)), ij = (int)((w / gmax) % gmax), kl = (int)(w % gmax);
            const int i = L.bas_ab[h][ij][0], j = L.bas_ab[h][ij][1];
            const int k = L.bas_ab[h][kl][0], l = L.bas_ab[h][kl][1];
            const int hik = L.sym_pair(L.symmetry[i], L.symmetry[k]);
            const int hkj = L.sym_pair(L.symmetry[k], L.symmetry[j]);
            const bool diag = i00[hik][(size_t)i * n + k] == i00[hik][(size_t)j * n + l];
            const double half = diag ? 0.5 : 1.0;
            const bool lj = l == j, ikq = i == k;
            const int64_t gh = L.gems_ab[h], gk = L.gems_ab[hkj], ah = L.gems_aa[h], ak = L.gems_aa[hkj];
            auto put = [&](int64_t col, double coef) {
                P.col.push_back((int32_t)col);
                P.val.push_back(coef);
            };
            const int64_t dab = L.off[F_D2AB][h], dabk = L.off[F_D2AB][hkj];
            const int ijab = ab(h, i, j), jiab = ab(h, j, i), klab = ab(h, k, l), lkab = ab(h, l, k);
            const int kjab = ab(hkj, k, j), ilab = ab(hkj, i, l), jkab = ab(hkj, j, k), liab = ab(hkj, l, i);
            put(dab + ijab * gh + klab, half);
            if (!lj) put(dabk + kjab * gk + ilab, half);
            if (!ikq) put(dabk + ilab * gk + kjab, half);
            if (!lj && !ikq) put(dab + klab * gh + ijab, half);
            put(dab + jiab * gh + lkab, half);
            if (!lj) put(dabk + jkab * gk + liab, half);
            if (!ikq) put(dabk + liab * gk + jkab, half);
            if (!lj && !ikq) put(dab + lkab * gh + jiab, half);
            if (i != j && k != l) {
                const double s = half * (i < j ? 1 : -1) * (k < l ? 1 : -1);
                const int ijaa = aa(h, i, j), klaa = aa(h, k, l);
                put(L.off[F_D2AA][h] + ijaa * ah + klaa, s);
                if (!lj && !ikq) put(L.off[F_D2AA][h] + klaa * ah + ijaa, s);
                put(L.off[F_D2BB][h] + ijaa * ah + klaa, s);
                if (!lj && !ikq) put(L.off[F_D2BB][h] + klaa * ah + ijaa, s);
            }
            if (k != j && i != l) {
                const double s = half * (k < j ? 1 : -1) * (i < l ? 1 : -1);
                const int kjaa = aa(hkj, k, j), ilaa = aa(hkj, i, l);
                if (!lj) put(L.off[F_D2AA][hkj] + kjaa * ak + ilaa, s);
                if (!ikq) put(L.off[F_D2AA][hkj] + ilaa * ak + kjaa, s);
                if (!lj) put(L.off[F_D2BB][hkj] + kjaa * ak + ilaa, s);
                if (!ikq) put(L.off[F_D2BB][hkj] + ilaa * ak + kjaa, s);
            }
        }
        P.rowptr.push_back((int64_t)P.col.size());
    }
}

}  // namespace v2g
