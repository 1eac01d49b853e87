/*
 * Oracle shim implementation (test infrastructure only).
 *
 * Implements the Psi4 pieces declared under oracle/shim/psi4/ and the BLAS
 * entry points that the reference's blas.h declares (psi::fnocc::F_DGEMM,
 * Fortran-mangled dgemm_/ddot_/...).  Dense linear algebra is forwarded to the
 * LP64 OpenBLAS build that scipy ships (symbols prefixed "scipy_"), whose path
 * the oracle Makefile passes at link time.
 */
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <vector>

#include "psi4/libmints/matrix.h"
#include "psi4/libmints/vector.h"
#include "psi4/libqt/qt.h"
#include "psi4/psi4-dec.h"

extern "C" {
void scipy_dgemm_(const char* ta, const char* tb, const int* m, const int* n, const int* k, const double* alpha,
                  const double* a, const int* lda, const double* b, const int* ldb, const double* beta, double* c,
                  const int* ldc);
void scipy_dsyev_(const char* jobz, const char* uplo, const int* n, double* a, const int* lda, double* w,
                  double* work, const int* lwork, int* info);
void scipy_openblas_set_num_threads(int n);
}

namespace psi {

std::shared_ptr<PsiOutStream> outfile = std::make_shared<PsiOutStream>();

void PsiOutStream::Printf(const char* fmt, ...) {
    static const bool verbose = std::getenv("ORACLE_VERBOSE") != nullptr;
    if (!verbose) return;
    va_list ap;
    va_start(ap, fmt);
    vfprintf(stdout, fmt, ap);
    va_end(ap);
}

void C_DCOPY(size_t n, const double* x, int incx, double* y, int incy) {
    for (size_t i = 0; i < n; i++) y[i * incy] = x[i * incx];
}
void C_DAXPY(size_t n, double a, const double* x, int incx, double* y, int incy) {
    for (size_t i = 0; i < n; i++) y[i * incy] += a * x[i * incx];
}
void C_DSCAL(size_t n, double a, double* x, int incx) {
    for (size_t i = 0; i < n; i++) x[i * incx] *= a;
}
double C_DDOT(size_t n, const double* x, int incx, const double* y, int incy) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += x[i * incx] * y[i * incy];
    return s;
}
double C_DNRM2(size_t n, const double* x, int incx) {
    double s = 0.0;
    for (size_t i = 0; i < n; i++) s += x[i * incx] * x[i * incx];
    return std::sqrt(s);
}

void Matrix::diagonalize(SharedMatrix& eigvec, SharedVector& eigval) {
    const int n = rows_;
    if (n == 0) return;
    // A symmetric row-major matrix reads the same in column-major order.
    std::vector<double> a(data_);
    double* w = eigval->pointer();
    int lwork = -1, info = 0;
    double wq = 0.0;
    scipy_dsyev_("V", "U", &n, a.data(), &n, w, &wq, &lwork, &info);
    lwork = (int)wq;
    std::vector<double> work(lwork > 1 ? lwork : 1);
    scipy_dsyev_("V", "U", &n, a.data(), &n, w, work.data(), &lwork, &info);
    if (info != 0) throw std::runtime_error("dsyev failed in oracle shim");
    // LAPACK returns eigenvector j as column j (column-major); store it so that
    // ev[q][j] is component q of eigenvector j.
    double** ev = eigvec->pointer();
    for (int j = 0; j < n; j++)
        for (int q = 0; q < n; q++) ev[q][j] = a[(size_t)j * n + q];
}

namespace fnocc {

// Fortran-ordered dgemm with the reference's long-int BLAS integers (blas.h:34).
void F_DGEMM(char transa, char transb, long m, long n, long k, double alpha, double* A, long lda, double* B,
             long ldb, double beta, double* C, long ldc) {
    if (m == 0 || n == 0) return;
    int im = (int)m, in = (int)n, ik = (int)k, ilda = (int)lda, ildb = (int)ldb, ildc = (int)ldc;
    if (k == 0) {
        // BLAS semantics: C = beta*C when the inner dimension is empty, and C is
        // overwritten without being read when beta is zero.
        for (long j = 0; j < n; j++)
            for (long i = 0; i < m; i++) C[j * ldc + i] = (beta == 0.0) ? 0.0 : beta * C[j * ldc + i];
        return;
    }
    scipy_dgemm_(&transa, &transb, &im, &in, &ik, &alpha, A, &ilda, B, &ildb, &beta, C, &ildc);
}

}  // namespace fnocc
}  // namespace psi

extern "C" void oracle_set_blas_threads(int n) { scipy_openblas_set_num_threads(n); }
