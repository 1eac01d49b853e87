"""Builds the solver library in-tree: v2rdm_casscf_b200/lib/libv2rdm_b200.so.

Every CUDA source is compiled for sm_100a only (B200); host sources go through
nvcc's host compiler.  The library exports the C ABI of include/v2rdm_gpu.h.

    python -m v2rdm_casscf_b200.build        # or build() from Python
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libv2rdm_b200.so")
OBJDIR = os.path.join(ROOT, "_build", "obj")

CU_SOURCES = ["maps.cu", "eig.cu", "tc_gemm.cu", "mlp.cu", "warmstart.cu", "solver.cu"]
CPP_SOURCES = ["layout.cpp", "constraints.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r.stdout + r.stderr


def build(verbose=False, ptxas_info=False):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    nv = nvcc()
    host_cc = ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo"] + host_cc
    objs = []
    log = ""
    for src in CU_SOURCES:
        obj = os.path.join(OBJDIR, src + ".o")
        cmd = [nv] + ARCH + common + ["-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        log += _run(cmd)
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = os.path.join(OBJDIR, src + ".o")
        log += _run([nv] + common + ["-x", "c++", "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    tmp = LIB + ".tmp"
    log += _run([nv] + ARCH + host_cc + ["-shared", "-o", tmp] + objs + ["-lcudart"])
    os.replace(tmp, LIB)
    if verbose:
        print(log)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
