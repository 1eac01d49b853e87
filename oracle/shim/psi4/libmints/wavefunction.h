/*
 * Oracle shim (test infrastructure only): the Wavefunction base class that
 * v2RDMSolver derives from, reduced to the data members the hot-path sources
 * read (orbital counts per irrep, orbital energies, options).
 */
#ifndef ORACLE_SHIM_WAVEFUNCTION_H
#define ORACLE_SHIM_WAVEFUNCTION_H

#include <memory>
#include <string>
#include <vector>

#include "psi4/liboptions/liboptions.h"
#include "psi4/libmints/matrix.h"
#include "psi4/libmints/vector.h"
#include "psi4/psi4-dec.h"

namespace psi {

// Per-irrep orbital counts; Psi4 calls this Dimension.
class Dimension {
  public:
    Dimension() : v_(8, 0) {}
    int& operator[](int h) { return v_[h]; }
    int operator[](int h) const { return v_[h]; }
    operator int*() { return v_.data(); }

  private:
    std::vector<int> v_;
};

class Wavefunction;
typedef std::shared_ptr<Wavefunction> SharedWavefunction;

class Wavefunction {
  public:
    explicit Wavefunction(Options& options) : options_(options) {}
    virtual ~Wavefunction() = default;

  protected:
    Options& options_;
    std::string name_;
    double energy_ = 0.0;
    double efzc_ = 0.0;
    long memory_ = 0;
    int nirrep_ = 1;
    int nso_ = 0;
    int nmo_ = 0;
    Dimension nsopi_, nmopi_, frzcpi_, frzvpi_, doccpi_, soccpi_, nalphapi_, nbetapi_;
    SharedVector epsilon_a_, epsilon_b_;
    bool same_a_b_orbs_ = true;
    bool same_a_b_dens_ = true;
};

}  // namespace psi

#endif
