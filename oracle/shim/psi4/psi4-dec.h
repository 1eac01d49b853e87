/*
 * Minimal stand-in for the Psi4 declarations that the v2RDM-CASSCF hot-path
 * sources include.  TEST INFRASTRUCTURE ONLY: it exists so that the
 * reference's own constraint-map, CG and projection sources compile here,
 * unmodified, into the oracle library under oracle/_ref/.  Nothing in the
 * product links against it.
 *
 * Only the small slice of Psi4's interface that those sources touch is
 * provided: an output stream with Printf, PsiException, and the shared
 * pointer typedefs.
 */
#ifndef ORACLE_SHIM_PSI4_DEC_H
#define ORACLE_SHIM_PSI4_DEC_H

#include <cstdarg>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>

#include "psi4/liboptions/liboptions.h"

namespace psi {

class PsiOutStream {
  public:
    // Output is discarded unless ORACLE_VERBOSE is set in the environment.
    void Printf(const char* fmt, ...);
};
extern std::shared_ptr<PsiOutStream> outfile;

class PsiException : public std::runtime_error {
  public:
    PsiException(const std::string& msg, const char* file, int line)
        : std::runtime_error(msg + " (" + file + ":" + std::to_string(line) + ")") {}
};

}  // namespace psi

#endif
