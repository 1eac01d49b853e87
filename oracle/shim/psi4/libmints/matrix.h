/*
 * Oracle shim (test infrastructure only): Psi4-style square Matrix with
 * row-pointer access and a symmetric eigensolver.
 *
 * diagonalize() follows Psi4's convention as the reference's Update_xz
 * relies on it (v2rdm_solver.cc:3248-3264): eigenvalues ascending, and
 * eigvec->pointer()[q][j] is component q of eigenvector j.  It calls
 * LAPACK dsyev from the OpenBLAS build shipped with scipy.
 */
#ifndef ORACLE_SHIM_MATRIX_H
#define ORACLE_SHIM_MATRIX_H

#include <memory>
#include <string>
#include <vector>

#include "psi4/libmints/vector.h"

namespace psi {

class Matrix;
typedef std::shared_ptr<Matrix> SharedMatrix;

class Matrix {
  public:
    Matrix(int rows, int cols) : rows_(rows), cols_(cols), data_((size_t)rows * cols, 0.0) {
        rowp_.resize(rows);
        for (int i = 0; i < rows; i++) rowp_[i] = data_.data() + (size_t)i * cols;
    }
    Matrix(const std::string&, int rows, int cols) : Matrix(rows, cols) {}
    double** pointer(int h = 0) { return rowp_.data(); }
    int rowdim() const { return rows_; }
    int coldim() const { return cols_; }
    void diagonalize(SharedMatrix& eigvec, SharedVector& eigval);

  private:
    int rows_, cols_;
    std::vector<double> data_;
    std::vector<double*> rowp_;
};

}  // namespace psi

#endif
