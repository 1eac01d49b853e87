/* Oracle shim (test infrastructure only): empty stand-in for a Psi4 header
 * that the reference hot-path sources include but do not use. */
#ifndef ORACLE_SHIM_LIBPSI4UTIL_PROCESS_H
#define ORACLE_SHIM_LIBPSI4UTIL_PROCESS_H
#include "psi4/psi4-dec.h"
#endif
