/*
 * Oracle harness around the reference's own BPSDP hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file links against the reference sources
 * compiled from the reference tree (d2.cc, spin.cc, q2.cc, g2.cc, t1.cc, t2.cc,
 * d3.cc, d4.cc, basis.cc, tei.cc, cg_solver.cc and the hot-path pieces of
 * v2rdm_solver.cc, see gen_ref_sources.py) and exposes them through a plain C
 * ABI so that Python tests and the CPU baseline can call them.  Only tests/,
 * the smoke check and bench.py's CPU-baseline leg load the resulting
 * oracle/_ref/libv2rdm_ref.so; the product never does.
 *
 * What the harness itself provides (everything else is the reference's code):
 *   * the Psi4-wavefunction part of v2RDMSolver::common_init
 *     (v2rdm_solver.cc:206-486) is replaced by setting the same members from
 *     explicit per-irrep orbital counts (oref_create);
 *   * the outer BPSDP loop of v2RDMSolver::compute_energy
 *     (v2rdm_solver.cc:1778-1908) is restated in oref_solve with the orbital
 *     optimisation branch off (all-active spaces have no rotations), calling
 *     the reference's bpsdp_Au, bpsdp_ATu, CGSolver::solve and Update_xz.
 */
#include <omp.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cg_solver.h"
#include "psi4/libmints/vector.h"
#include "v2rdm_solver.h"

void* oracle_evaluate_Ap_ptr();

namespace psi {
namespace v2rdm_casscf {

// The real constructor reads a Psi4 wavefunction; the oracle sets members
// itself (OracleSolver::setup) and then runs the generated common_init body.
v2RDMSolver::v2RDMSolver(SharedWavefunction, Options& options) : Wavefunction(options) {}
v2RDMSolver::~v2RDMSolver() {}
double v2RDMSolver::compute_energy() { return 0.0; }

// tei.cc's GetIntegrals references these; the oracle supplies integrals
// directly and never calls them.
SharedMatrix v2RDMSolver::GetOEI() { throw PsiException("GetOEI is not available in the oracle", __FILE__, __LINE__); }
void v2RDMSolver::GetTEIFromDisk() { throw PsiException("GetTEIFromDisk is not available in the oracle", __FILE__, __LINE__); }

std::vector<double> g_next_eps;  // orbital energies for the next setup (Pitzer order)
int g_next_spin_adapt[4] = {0, 0, 0, 0};  // SPIN_ADAPT_Q2, SPIN_ADAPT_G2, CONSTRAIN_D3, CONSTRAIN_D4 (next setup)

class OracleSolver : public v2RDMSolver {
  public:
    explicit OracleSolver(Options& o) : v2RDMSolver(SharedWavefunction(), o) {}

    // Members that common_init derives from the Psi4 wavefunction
    // (v2rdm_solver.cc:227-455), set from explicit counts.
    void setup(int nirrep, const int* nmopi, const int* frzcpi, const int* rstcpi, const int* rstvpi,
               const int* frzvpi, const int* doccpi, const int* soccpi, int multiplicity) {
        nirrep_ = nirrep;
        rstcpi_ = (int*)calloc(nirrep, sizeof(int));
        rstvpi_ = (int*)calloc(nirrep, sizeof(int));
        amopi_ = (int*)calloc(nirrep, sizeof(int));
        nmo_ = 0;
        nalpha_ = 0;
        nbeta_ = 0;
        for (int h = 0; h < nirrep; h++) {
            nmopi_[h] = nmopi[h];
            nsopi_[h] = nmopi[h];
            frzcpi_[h] = frzcpi[h];
            frzvpi_[h] = frzvpi[h];
            rstcpi_[h] = rstcpi[h];
            rstvpi_[h] = rstvpi[h];
            doccpi_[h] = doccpi[h];
            soccpi_[h] = soccpi[h];
            nalphapi_[h] = doccpi[h] + soccpi[h];
            nbetapi_[h] = doccpi[h];
            nmo_ += nmopi[h];
            nalpha_ += doccpi[h] + soccpi[h];
            nbeta_ += doccpi[h];
        }
        nso_ = nmo_;
        multiplicity_ = multiplicity;
        amo_ = nfrzc_ = nfrzv_ = nrstc_ = nrstv_ = 0;
        for (int h = 0; h < nirrep; h++) {
            nfrzc_ += frzcpi_[h];
            nrstc_ += rstcpi_[h];
            nrstv_ += rstvpi_[h];
            nfrzv_ += frzvpi_[h];
            amopi_[h] = nmopi_[h] - frzcpi_[h] - rstcpi_[h] - rstvpi_[h] - frzvpi_[h];
            amo_ += amopi_[h];
        }
        // Orbital energies only order orbitals inside BuildBasis (the energy
        // order sets the numbering of the spatial pairs that PackSpatialDensity
        // writes); default i + 0.001 h, or the values given to
        // oref_set_next_energies (all orbitals, Pitzer order).
        epsilon_a_ = SharedVector(new Vector(nirrep_, (int*)nmopi_));
        epsilon_b_ = SharedVector(new Vector(nirrep_, (int*)nmopi_));
        for (int h = 0, k = 0; h < nirrep; h++)
            for (int i = 0; i < nmopi[h]; i++, k++) {
                const double e = (k < (int)g_next_eps.size()) ? g_next_eps[k] : i + 0.001 * h;
                epsilon_a_->pointer(h)[i] = e;
                epsilon_b_->pointer(h)[i] = e;
            }
        g_next_eps.clear();
        is_df_ = true;
        is_doci_ = false;
        doci_alpha_ = 1.0;
        doci_ref_ = 1.0;
        enuc_ = 0.0;
        efzc_ = 0.0;

        common_init();  // the reference's layout code (generated unit)

        Ax = SharedVector(new Vector("A . x", nconstraints_));
        ATy = SharedVector(new Vector("A^T . y", dimx_));
        x = SharedVector(new Vector("primal solution", dimx_));
        c = SharedVector(new Vector("OEI and TEI", dimx_));
        y = SharedVector(new Vector("dual solution", nconstraints_));
        z = SharedVector(new Vector("dual solution 2", dimx_));
        b = SharedVector(new Vector("constraints", nconstraints_));
        tau = 1.0;
        mu = 1.0;
        ep = ed = 0.0;
    }

    void set_integrals(const double* oei_packed, const double* qmo, int nq, double enuc) {
        long ntri = (long)(nmo_ - nfrzv_) * (nmo_ - nfrzv_ + 1) / 2;
        long noei = 0;
        for (int h = 0; h < nirrep_; h++) noei += (long)(nmopi_[h] - frzvpi_[h]) * (nmopi_[h] - frzvpi_[h] + 1) / 2;
        oei_.assign(oei_packed, oei_packed + noei);
        qmo_.assign(qmo, qmo + (long)nq * ntri);
        oei_full_sym_ = oei_.data();
        Qmo_ = qmo_.data();
        tei_full_sym_ = Qmo_;
        nQ_ = nq;
        enuc_ = enuc;
        c->zero();
        RepackIntegrals();  // tei.cc:144, with FrozenCoreEnergy tei.cc:230
    }

    SharedVector vec(const std::string& w) {
        if (w == "x") return x;
        if (w == "y") return y;
        if (w == "z") return z;
        if (w == "c") return c;
        if (w == "b") return b;
        throw PsiException("unknown vector " + w, __FILE__, __LINE__);
    }

    // Outer loop of v2rdm_solver.cc:1778-1908 (OPTIMIZE_ORBITALS false).
    int solve(double tau_in, double mu_in, int mu_update_frequency, int max_outer, double* res, double* trace,
              int trace_cap) {
        tau = tau_in;
        mu = mu_in;
        long N = nconstraints_;
        SharedVector B(new Vector("compound B", nconstraints_));
        CGSolver cg(N);
        cg.set_max_iter(cg_maxiter_);
        typedef void (*cb_t)(long, SharedVector, SharedVector, void*);
        cb_t cb = (cb_t)oracle_evaluate_Ap_ptr();

        double energy_primal = C_DDOT(dimx_, c->pointer(), 1, x->pointer(), 1);
        double energy_dual = 0.0, egap = 0.0, current_energy = energy_primal;
        int oiter = 0;
        long iiter_total = 0;
        double t_cg = 0.0, t_xz = 0.0;
        double t_start = omp_get_wtime();
        int limit = (max_outer > 0 && max_outer < maxiter_) ? max_outer : maxiter_;
        bool hit_limit = false;
        do {
            double t0 = omp_get_wtime();
            bpsdp_Au(Ax, x);
            Ax->subtract(b);
            Ax->scale(-tau * mu);
            z->scale(-1.0);
            z->add(c);
            bpsdp_Au(B, z);
            B->add(Ax);
            double cg_conv_i;
            if (oiter == 0)
                cg_conv_i = 0.01;
            else
                cg_conv_i = (ep > ed) ? 0.01 * ed : 0.01 * ep;
            if (cg_conv_i < cg_convergence_) cg_conv_i = cg_convergence_;
            cg.set_convergence(cg_conv_i);
            cg.solve(N, Ax, y, B, cb, (void*)this);
            int iiter = cg.total_iterations();
            double t1 = omp_get_wtime();
            t_cg += t1 - t0;
            iiter_total += iiter;

            Update_xz();
            double t2 = omp_get_wtime();
            t_xz += t2 - t1;

            bpsdp_ATu(ATy, y);
            ATy->add(z);
            ATy->subtract(c);
            ed = ATy->norm();
            bpsdp_Au(Ax, x);
            Ax->subtract(b);
            ep = Ax->norm();
            if (oiter % mu_update_frequency == 0 && oiter > 0) mu = mu * ep / ed;
            current_energy = C_DDOT(dimx_, c->pointer(), 1, x->pointer(), 1);
            energy_dual = C_DDOT(nconstraints_, b->pointer(), 1, y->pointer(), 1);
            if (trace && oiter < trace_cap) {
                double* t = trace + 8L * oiter;
                t[0] = oiter;
                t[1] = iiter;
                t[2] = current_energy + enuc_ + efzc_;
                t[3] = energy_dual + efzc_ + enuc_;
                t[4] = fabs(current_energy - energy_dual);
                t[5] = mu;
                t[6] = ep;
                t[7] = ed;
            }
            oiter++;
            if (oiter == limit) {
                hit_limit = true;
                break;
            }
            egap = fabs(current_energy - energy_dual);
            energy_primal = current_energy;
        } while (ep > r_convergence_ || ed > r_convergence_ || egap > e_convergence_);
        double t_end = omp_get_wtime();
        // As in the reference (v2rdm_solver.cc:1910-1912), reaching the
        // iteration limit means "did not converge".
        bool converged = !hit_limit;
        res[0] = current_energy + enuc_ + efzc_;
        res[1] = energy_dual + enuc_ + efzc_;
        res[2] = ep;
        res[3] = ed;
        res[4] = mu;
        res[5] = oiter;
        res[6] = (double)iiter_total;
        res[7] = t_cg;
        res[8] = t_xz;
        res[9] = t_end - t_start;
        res[10] = efzc_;
        return converged ? 0 : 1;
    }

    // Layout introspection for parity of the product's tables.
    int offsets(const std::string& fam, int* out) {
        int* p = nullptr;
        if (fam == "d2ab") p = d2aboff;
        else if (fam == "d2aa") p = d2aaoff;
        else if (fam == "d2bb") p = d2bboff;
        else if (fam == "d200") p = d200off;
        else if (fam == "d1a") p = d1aoff;
        else if (fam == "d1b") p = d1boff;
        else if (fam == "q1a") p = q1aoff;
        else if (fam == "q1b") p = q1boff;
        else if (fam == "q2ab") p = constrain_q2_ ? q2aboff : nullptr;
        else if (fam == "q2aa") p = constrain_q2_ ? q2aaoff : nullptr;
        else if (fam == "q2bb") p = constrain_q2_ ? q2bboff : nullptr;
        else if (fam == "g2ab") p = constrain_g2_ ? g2aboff : nullptr;
        else if (fam == "g2ba") p = constrain_g2_ ? g2baoff : nullptr;
        else if (fam == "g2aa") p = constrain_g2_ ? g2aaoff : nullptr;
        else if (fam == "t1aaa") p = constrain_t1_ ? t1aaaoff : nullptr;
        else if (fam == "t1bbb") p = constrain_t1_ ? t1bbboff : nullptr;
        else if (fam == "t1aab") p = constrain_t1_ ? t1aaboff : nullptr;
        else if (fam == "t1bba") p = constrain_t1_ ? t1bbaoff : nullptr;
        else if (fam == "t2aaa") p = constrain_t2_ ? t2aaaoff : nullptr;
        else if (fam == "t2bbb") p = constrain_t2_ ? t2bbboff : nullptr;
        else if (fam == "t2aab") p = constrain_t2_ ? t2aaboff : nullptr;
        else if (fam == "t2bba") p = constrain_t2_ ? t2bbaoff : nullptr;
        if (!p) return 0;
        for (int h = 0; h < nirrep_; h++) out[h] = p[h];
        return nirrep_;
    }
    int counts(const std::string& what, int* out) {
        int* p = nullptr;
        if (what == "gems_ab") p = gems_ab;
        else if (what == "gems_aa") p = gems_aa;
        else if (what == "gems_00") p = gems_00;
        else if (what == "trip_aab") p = trip_aab;
        else if (what == "trip_aba") p = trip_aba;
        else if (what == "trip_aaa") p = trip_aaa;
        else if (what == "amopi") p = amopi_;
        if (!p) return 0;
        for (int h = 0; h < nirrep_; h++) out[h] = p[h];
        return nirrep_;
    }
    // ibas_ab / ibas_aa / bas maps for irrep h, flattened.
    void ibas(const std::string& what, int h, int* out) {
        int*** p = (what == "ab") ? ibas_ab_sym : ibas_aa_sym;
        for (int i = 0; i < amo_; i++)
            for (int j = 0; j < amo_; j++) out[i * amo_ + j] = p[h][i][j];
    }

    long dimx() const { return dimx_; }
    long ncon() const { return nconstraints_; }
    const std::vector<int>& dims() const { return dimensions_; }
    void do_update_xz(double mu_in) {
        mu = mu_in;
        Update_xz();
    }
    void do_Au(SharedVector out, SharedVector in) { bpsdp_Au(out, in); }
    void do_ATu(SharedVector out, SharedVector in) { bpsdp_ATu(out, in); }
    void do_guess() { Guess(); }
    // Packed spatial densities of PackSpatialDensity (v2rdm_solver.cc:3664),
    // sized as tei.cc:91-110 sizes them.
    long d1_dim() const {
        long n = 0;
        for (int h = 0; h < nirrep_; h++) n += (long)amopi_[h] * (amopi_[h] + 1) / 2;
        return n;
    }
    long d2_dim() const {
        long n = 0;
        for (int h = 0; h < nirrep_; h++) n += (long)gems_00[h] * (gems_00[h] + 1L) / 2L;
        return n;
    }
    void do_pack(double* d1, double* d2) {
        std::vector<double> a(d1_dim() + 1), b(d2_dim() + 1);
        d1_act_spatial_sym_ = a.data();
        d2_act_spatial_sym_ = b.data();
        d1_act_spatial_dim_ = d1_dim();  // PackSpatialDensity clears d2 by this size
        d2_act_spatial_dim_ = d2_dim();
        PackSpatialDensity();
        memcpy(d1, a.data(), sizeof(double) * d1_dim());
        memcpy(d2, b.data(), sizeof(double) * d2_dim());
        d1_act_spatial_sym_ = nullptr;
        d2_act_spatial_sym_ = nullptr;
    }
    void do_build_constraints() { BuildConstraints(); }
    double efzc() const { return efzc_; }
    int* symmetry_of_active() { return symmetry; }

  private:
    std::vector<double> oei_, qmo_;
};

}  // namespace v2rdm_casscf
}  // namespace psi

using psi::v2rdm_casscf::OracleSolver;

namespace {
struct Handle {
    psi::Options opts;
    OracleSolver* s = nullptr;
};
thread_local std::string g_err;
}  // namespace

extern "C" {

const char* oref_last_error() { return g_err.c_str(); }

void oref_set_next_spin_adapt(int q2, int g2, int d3, int d4) {
    psi::v2rdm_casscf::g_next_spin_adapt[0] = q2;
    psi::v2rdm_casscf::g_next_spin_adapt[1] = g2;
    psi::v2rdm_casscf::g_next_spin_adapt[2] = d3;
    psi::v2rdm_casscf::g_next_spin_adapt[3] = d4;
}
void oref_set_next_energies(const double* eps, int n) { psi::v2rdm_casscf::g_next_eps.assign(eps, eps + n); }
long oref_spatial_dims(void* h, long* d1, long* d2) {
    *d1 = ((Handle*)h)->s->d1_dim();
    *d2 = ((Handle*)h)->s->d2_dim();
    return 0;
}
void oref_pack_spatial(void* h, double* d1, double* d2) { ((Handle*)h)->s->do_pack(d1, d2); }

void* oref_create(int nirrep, const int* nmopi, const int* frzcpi, const int* rstcpi, const int* rstvpi,
                  const int* frzvpi, const int* doccpi, const int* soccpi, int multiplicity, const char* positivity,
                  int constrain_spin, int constrain_sz, double r_conv, double e_conv, double cg_conv, int maxiter,
                  int cg_maxiter) {
    Handle* hd = new Handle();
    try {
        hd->opts.set_str("POSITIVITY", positivity);
        hd->opts.set_num("CONSTRAIN_SPIN", constrain_spin);
        hd->opts.set_num("CONSTRAIN_SZ", constrain_sz);
        hd->opts.set_num("CONSTRAIN_D3", psi::v2rdm_casscf::g_next_spin_adapt[2]);
        hd->opts.set_num("CONSTRAIN_D4", psi::v2rdm_casscf::g_next_spin_adapt[3]);
        hd->opts.set_num("SPIN_ADAPT_G2", psi::v2rdm_casscf::g_next_spin_adapt[1]);
        hd->opts.set_num("SPIN_ADAPT_Q2", psi::v2rdm_casscf::g_next_spin_adapt[0]);
        psi::v2rdm_casscf::g_next_spin_adapt[0] = psi::v2rdm_casscf::g_next_spin_adapt[1] = 0;
        psi::v2rdm_casscf::g_next_spin_adapt[2] = psi::v2rdm_casscf::g_next_spin_adapt[3] = 0;
        hd->opts.set_num("R_CONVERGENCE", r_conv);
        hd->opts.set_num("E_CONVERGENCE", e_conv);
        hd->opts.set_num("CG_CONVERGENCE", cg_conv);
        hd->opts.set_num("MAXITER", maxiter);
        hd->opts.set_num("CG_MAXITER", cg_maxiter);
        hd->opts.set_num("DIIS_MAX_VECS", 8);
        hd->opts.set_str("TPDM_GUESS", "RANDOM");
        hd->opts.set_str("RESTART_FROM_CHECKPOINT_FILE", "");
        hd->s = new OracleSolver(hd->opts);
        hd->s->setup(nirrep, nmopi, frzcpi, rstcpi, rstvpi, frzvpi, doccpi, soccpi, multiplicity);
    } catch (const std::exception& e) {
        g_err = e.what();
        delete hd->s;
        delete hd;
        return nullptr;
    }
    return hd;
}

void oref_destroy(void* h) {
    Handle* hd = (Handle*)h;
    if (!hd) return;
    delete hd->s;
    delete hd;
}

long oref_dimx(void* h) { return ((Handle*)h)->s->dimx(); }
long oref_ncon(void* h) { return ((Handle*)h)->s->ncon(); }
int oref_nblocks(void* h) { return (int)((Handle*)h)->s->dims().size(); }
void oref_block_dims(void* h, int* out) {
    auto& d = ((Handle*)h)->s->dims();
    for (size_t i = 0; i < d.size(); i++) out[i] = d[i];
}
int oref_offsets(void* h, const char* fam, int* out) { return ((Handle*)h)->s->offsets(fam, out); }
int oref_counts(void* h, const char* what, int* out) { return ((Handle*)h)->s->counts(what, out); }
void oref_ibas(void* h, const char* what, int irrep, int* out) { ((Handle*)h)->s->ibas(what, irrep, out); }

int oref_set_integrals(void* h, const double* oei_packed, const double* qmo, int nq, double enuc) {
    try {
        ((Handle*)h)->s->set_integrals(oei_packed, qmo, nq, enuc);
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
    return 0;
}
double oref_efzc(void* h) { return ((Handle*)h)->s->efzc(); }

int oref_get(void* h, const char* which, double* out) {
    try {
        auto v = ((Handle*)h)->s->vec(which);
        memcpy(out, v->pointer(), sizeof(double) * v->dim());
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
    return 0;
}
int oref_set(void* h, const char* which, const double* in) {
    try {
        auto v = ((Handle*)h)->s->vec(which);
        memcpy(v->pointer(), in, sizeof(double) * v->dim());
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
    return 0;
}
void oref_guess(void* h) { ((Handle*)h)->s->do_guess(); }
void oref_build_constraints(void* h) { ((Handle*)h)->s->do_build_constraints(); }

void oref_Au(void* h, const double* u, double* out) {
    OracleSolver* s = ((Handle*)h)->s;
    psi::SharedVector in(new psi::Vector(s->dimx()));
    psi::SharedVector o(new psi::Vector(s->ncon()));
    memcpy(in->pointer(), u, sizeof(double) * s->dimx());
    s->do_Au(o, in);
    memcpy(out, o->pointer(), sizeof(double) * s->ncon());
}
void oref_ATu(void* h, const double* u, double* out) {
    OracleSolver* s = ((Handle*)h)->s;
    psi::SharedVector in(new psi::Vector(s->ncon()));
    psi::SharedVector o(new psi::Vector(s->dimx()));
    memcpy(in->pointer(), u, sizeof(double) * s->ncon());
    s->do_ATu(o, in);
    memcpy(out, o->pointer(), sizeof(double) * s->dimx());
}
void oref_update_xz(void* h, double mu) { ((Handle*)h)->s->do_update_xz(mu); }

int oref_solve(void* h, double tau, double mu0, int mu_update_frequency, int max_outer, double* res, double* trace,
               int trace_cap) {
    try {
        return ((Handle*)h)->s->solve(tau, mu0, mu_update_frequency, max_outer, res, trace, trace_cap);
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

void oref_set_threads(int n) { omp_set_num_threads(n); }
}
