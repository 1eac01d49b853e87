// Constraint matrix A of the boundary-point SDP as a sparse row list, the
// right-hand side b, and the cost vector c.
//
// A is generated row by row in the reference's row order (bpsdp_Au,
// v2rdm_solver.cc:3020-3065), one family at a time.  Each family's rows
// restate the reference's *_Au loop for that family (cited at each emitter);
// A^T is obtained by transposing A, which makes the two maps exact adjoints
// by construction instead of restating the reference's scatter loops.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "layout.h"

namespace v2g {

struct Csr {
    int64_t nrows = 0, ncols = 0;
    std::vector<int64_t> rowptr;  // nrows + 1
    std::vector<int32_t> col;
    std::vector<double> val;
    int64_t nnz() const { return (int64_t)col.size(); }
};

// Builds A (ncon x dimx).  Returns "" on success.
std::string build_A(const Layout& L, Csr& A);

// Transpose (dimx x ncon), rows sorted by column index.
void transpose(const Csr& A, Csr& AT);

// b of BuildConstraints (v2rdm_solver.cc:2518-3017).
void build_b(const Layout& L, std::vector<double>& b);

// Full-space orbital description needed to turn integrals into c
// (per irrep: frozen core, restricted core, active, restricted virtual,
// frozen virtual).  The active counts must equal the layout's amopi.
struct OrbitalSpaces {
    std::vector<int> frzcpi, rstcpi, amopi, rstvpi, frzvpi;
};

// c and the frozen-core energy from one-electron integrals packed per irrep
// (lower triangle, frozen virtuals excluded) and three-index integrals
// Qmo[Q * ntri + INDEX(p,q)] over the non-frozen-virtual orbitals in Pitzer
// order: RepackIntegrals + FrozenCoreEnergy (tei.cc:144-313, TEI tei.cc:315).
std::string build_c(const Layout& L, const OrbitalSpaces& sp, const double* oei_packed, const double* qmo, int nq,
                    std::vector<double>& c, double& efzc);

// PackSpatialDensity (v2rdm_solver.cc:3664-3773) as a gather map P
// ((d1_dim + d2_dim) x dimx): row r < d1_dim is element r of the packed
// spin-summed 1-RDM, row d1_dim + r element r of the packed spin-free 2-RDM
// handed to focas.  The spatial pairs are numbered in the energy order of the
// active orbitals (basis.cc:626-652; energies in Pitzer order, NULL = Pitzer
// order).  Each row lists its terms in the reference's summation order with
// coefficients +-0.5 (+-1 for off-diagonal pairs, the reference's final
// doubling), so an in-order FP64 sum reproduces the reference bit for bit.
void build_spatial_map(const Layout& L, const double* active_energies, Csr& P, int64_t& d1_dim, int64_t& d2_dim);

}  // namespace v2g
