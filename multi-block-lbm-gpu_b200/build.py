"""Builds the in-tree shared libraries.

  mblbm/libmblbm.so   the product: CUDA kernels for sm_100a plus the C ABI
                      (include/mblbm.h), compiled with nvcc;
  ../oracle/liboracle.so   the FP64 C oracle (test infrastructure), gcc + OpenMP.

Run as `python build.py [--oracle-only|--lib-only]`; __graft_entry__.build()
calls build_all().  Outputs are written next to the sources so that they
travel with the repository snapshot.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "mblbm", "libmblbm.so")
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def build_lib(force=False, verbose_ptxas=False):
    srcs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cpp"))]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(REPO, "include", "mblbm.h"))
    if not force and _newer(LIB, deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [NVCC, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-c", s, "-o", o] + ARCH
        if s.endswith(".cu"):
            cmd += ["--expt-relaxed-constexpr"]
            if verbose_ptxas:
                cmd += ["-Xptxas", "-v"]
        else:
            cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-I/usr/local/cuda/include", "-c", s, "-o", o]
        _run(cmd)
        objs.append(o)
    tmp = LIB + ".tmp"
    _run([NVCC, "-shared", "-o", tmp] + objs + ARCH + ["-lcudart"])
    os.replace(tmp, LIB)  # a reader never sees a half-written library
    return LIB


APP_SRC = os.path.join(HERE, "apps", "mblbm_run.c")
APP = os.path.join(HERE, "apps", "mblbm_run")


def build_app(force=False):
    """The C driver (apps/mblbm_run.c), linked against libmblbm.so."""
    if not force and _newer(APP, [APP_SRC, LIB]):
        return APP
    _run(["gcc", "-O2", "-std=c11", APP_SRC, "-o", APP, "-L" + os.path.dirname(LIB), "-lmblbm",
          "-Wl,-rpath,$ORIGIN/../mblbm"])
    return APP


def build_oracle(force=False):
    src = os.path.join(ORACLE_DIR, "oracle.c")
    deps = [src, os.path.join(ORACLE_DIR, "oracle.h"), os.path.join(REPO, "include", "mblbm.h")]
    if not force and _newer(ORACLE_LIB, deps):
        return ORACLE_LIB
    _run(["gcc", "-O2", "-std=c11", "-fopenmp", "-fPIC", "-shared", src, "-o", ORACLE_LIB, "-lm"])
    return ORACLE_LIB


def build_all(force=False):
    build_oracle(force)
    build_lib(force)
    build_app(force)


if __name__ == "__main__":
    force = "--force" in sys.argv
    if "--oracle-only" in sys.argv:
        build_oracle(force)
    elif "--lib-only" in sys.argv:
        build_lib(force, verbose_ptxas="--ptxas" in sys.argv)
    else:
        build_oracle(force)
        build_lib(force, verbose_ptxas="--ptxas" in sys.argv)
        build_app(force)
