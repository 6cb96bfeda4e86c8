"""Build the engine (libluthe.so, sm_100a) and the CPU oracle (liboracle.so).

Both libraries are built in-tree so that they travel with the source tree.
`python -m luthe_b200.build` builds both; nvcc cross-compiles without a GPU.
"""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "luthe_b200")
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libluthe.so")
ORACLE_SRC = os.path.join(ROOT, "oracle", "tfhe_oracle.c")
ORACLE_LIB = os.path.join(ROOT, "oracle", "liboracle.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["kernels.cu", "api.cu", "serve.cu", "probe.cu", "keygen.cpp"]


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _deps():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    out.append(os.path.join(ROOT, "include", "luthe.h"))
    return out


def build_engine(force=False, verbose=False):
    if not force and _newer(LIB, _deps()):
        return LIB
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-fopenmp",
           "-I", os.path.join(ROOT, "include"), "-o", LIB]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    cmd += ["-lgomp"]
    subprocess.run(cmd, check=True)
    return LIB


def build_oracle(force=False):
    if not force and _newer(ORACLE_LIB, [ORACLE_SRC]):
        return ORACLE_LIB
    cc = os.environ.get("LUTHE_CC", "/usr/bin/gcc")
    subprocess.run([cc, "-O2", "-fopenmp", "-shared", "-fPIC", "-o", ORACLE_LIB, ORACLE_SRC, "-lm"], check=True)
    return ORACLE_LIB


def build_all(force=False, verbose=False):
    build_oracle(force)
    build_engine(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
    print(ORACLE_LIB)
