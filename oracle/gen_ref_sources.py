#!/usr/bin/env python3
"""Assemble the compile unit for the reference solver pieces (oracle build step).

TEST INFRASTRUCTURE ONLY.  v2rdm_solver.cc as a whole needs most of Psi4
(molden writers, integral transforms, PSIO), which is absent.  Its hot-path
functions do not: this script copies them, unmodified and at build time, from
the reference tree into ``oracle/_ref/gen/v2rdm_solver_hotpath.cc`` (a
git-ignored build directory).  Nothing from the reference is committed.

Pieces taken from v2rdm_solver.cc, located by anchor lines and checked:
  * evaluate_Ap, the CG callback trampoline         (v2rdm_solver.cc:119-126)
  * common_init's options-to-layout section, from "pick conditions" through
    the convergence parameters (v2rdm_solver.cc:487-1285); it is wrapped as
    the body of v2RDMSolver::common_init(), whose earlier part (reading the
    Psi4 wavefunction) the harness replaces by setting the same members
  * SymmetryPair / TotalSym                        (v2rdm_solver.cc:1677-1682)
  * Guess, BuildConstraints, bpsdp_Au/ATu(_slow), cg_Ax, Update_xz
                                                   (v2rdm_solver.cc:2386-3289)
  * PackSpatialDensity, the RDM hand-off to focas  (v2rdm_solver.cc:3664-3773)

Usage: gen_ref_sources.py <reference_dir> <out_file>
"""
import sys


def find_unique(lines, needle, start=0):
    hits = [i for i in range(start, len(lines)) if needle in lines[i]]
    if len(hits) != 1:
        raise SystemExit(f"anchor {needle!r} found {len(hits)} times; reference layout changed")
    return hits[0]


def main():
    ref_dir, out = sys.argv[1], sys.argv[2]
    src = open(f"{ref_dir}/v2rdm_solver.cc").read().split("\n")

    # evaluate_Ap: from its signature to the closing brace before the namespace.
    a0 = find_unique(src, "static void evaluate_Ap(")
    a1 = a0
    while src[a1].strip() != "}":
        a1 += 1

    # common_init layout section.
    c0 = find_unique(src, "// pick conditions.  default is dqg")
    c1 = find_unique(src, "// memory check happens here")

    # SymmetryPair/TotalSym.
    s0 = find_unique(src, "int v2RDMSolver::SymmetryPair(int i,int j)")
    s1 = find_unique(src, "int v2RDMSolver::TotalSym(")
    while src[s1].strip() != "}":
        s1 += 1

    # Guess .. end of Update_xz.
    g0 = find_unique(src, "void v2RDMSolver::Guess(){")
    g1 = find_unique(src, "void v2RDMSolver::Update_xz_nonsymmetric() {")
    while not src[g1].startswith("}"):
        g1 -= 1

    # PackSpatialDensity: up to the line before RotateOrbitals.
    p0 = find_unique(src, "void v2RDMSolver::PackSpatialDensity() {")
    p1 = find_unique(src, "void v2RDMSolver::RotateOrbitals(){")
    while not src[p1].startswith("}"):
        p1 -= 1

    def block(a, b):
        return "\n".join(src[a:b + 1])

    parts = [
        "// Generated at build time by oracle/gen_ref_sources.py from the reference's",
        "// v2rdm_solver.cc.  Build artefact: not committed.",
        '#include <stdio.h>',
        '#include <stdlib.h>',
        '#include <string.h>',
        '#include <math.h>',
        '#include <psi4/psi4-dec.h>',
        '#include <psi4/liboptions/liboptions.h>',
        '#include <psi4/libqt/qt.h>',
        '#include <psi4/libmints/vector.h>',
        '#include <psi4/libmints/matrix.h>',
        '#include "blas.h"',
        '#include "cg_solver.h"',
        '#include "v2rdm_solver.h"',
        '#include <omp.h>',
        "using namespace psi;",
        "using namespace fnocc;",
        f"#line {a0 + 1} \"v2rdm_solver.cc\"",
        block(a0, a1),
        "namespace psi{ namespace v2rdm_casscf{",
        "void v2RDMSolver::common_init(){",
        f"#line {c0 + 1} \"v2rdm_solver.cc\"",
        block(c0, c1 - 1),
        "}",
        f"#line {s0 + 1} \"v2rdm_solver.cc\"",
        block(s0, s1),
        f"#line {g0 + 1} \"v2rdm_solver.cc\"",
        block(g0, g1),
        f"#line {p0 + 1} \"v2rdm_solver.cc\"",
        block(p0, p1),
        "}}",
        "// accessor so that the harness drives CG through the reference trampoline",
        "void* oracle_evaluate_Ap_ptr() { return (void*)&evaluate_Ap; }",
        "",
    ]
    with open(out, "w") as f:
        f.write("\n".join(parts))


if __name__ == "__main__":
    main()
