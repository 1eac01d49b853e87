/*
 * Oracle shim (test infrastructure only): the Psi4 libqt BLAS-1 wrappers and
 * the packed lower-triangle INDEX macro used by the reference hot path.
 *
 * INDEX(i,j) is the position of element (max(i,j), min(i,j)) in a packed
 * lower triangle, the layout the reference's three-index integrals use
 * (tei.cc:321).
 */
#ifndef ORACLE_SHIM_QT_H
#define ORACLE_SHIM_QT_H

#include <cstddef>

#define INDEX(i, j) \
    ((i) > (j) ? ((long)(i) * ((long)(i) + 1) / 2 + (long)(j)) : ((long)(j) * ((long)(j) + 1) / 2 + (long)(i)))

namespace psi {

void C_DCOPY(size_t n, const double* x, int incx, double* y, int incy);
void C_DAXPY(size_t n, double a, const double* x, int incx, double* y, int incy);
void C_DSCAL(size_t n, double a, double* x, int incx);
double C_DDOT(size_t n, const double* x, int incx, const double* y, int incy);
double C_DNRM2(size_t n, const double* x, int incx);

}  // namespace psi

#endif
