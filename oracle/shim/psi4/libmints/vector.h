/*
 * Oracle shim (test infrastructure only): Psi4-style Vector, blocked by irrep,
 * with the handful of methods the reference hot-path sources call.
 */
#ifndef ORACLE_SHIM_VECTOR_H
#define ORACLE_SHIM_VECTOR_H

#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace psi {

class Vector;
typedef std::shared_ptr<Vector> SharedVector;

class Vector {
  public:
    explicit Vector(long n) { blocks_.resize(1); blocks_[0].assign(n > 0 ? n : 0, 0.0); }
    Vector(const std::string&, long n) : Vector(n) {}
    Vector(int nirrep, const int* dimpi) {
        blocks_.resize(nirrep);
        for (int h = 0; h < nirrep; h++) blocks_[h].assign(dimpi[h] > 0 ? dimpi[h] : 0, 0.0);
    }
    double* pointer(int h = 0) { return blocks_[h].data(); }
    const double* pointer(int h = 0) const { return blocks_[h].data(); }
    long dim(int h = 0) const { return (long)blocks_[h].size(); }
    void zero() {
        for (auto& b : blocks_) std::fill(b.begin(), b.end(), 0.0);
    }
    void scale(double a) {
        for (auto& b : blocks_)
            for (auto& v : b) v *= a;
    }
    void add(const SharedVector& o) { axpy(1.0, *o); }
    void subtract(const SharedVector& o) { axpy(-1.0, *o); }
    void axpy(double a, const Vector& o) {
        for (size_t h = 0; h < blocks_.size(); h++)
            for (size_t i = 0; i < blocks_[h].size(); i++) blocks_[h][i] += a * o.blocks_[h][i];
    }
    double norm() const {
        double s = 0.0;
        for (auto& b : blocks_)
            for (double v : b) s += v * v;
        return std::sqrt(s);
    }
    void copy(const Vector* o) { blocks_ = o->blocks_; }

  private:
    std::vector<std::vector<double>> blocks_;
};

}  // namespace psi

#endif
