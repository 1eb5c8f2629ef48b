"""Builds the native library in-tree.

Outputs (under ppc_b200/lib/ and ppc_b200/bin/):
  libppcb.so   C ABI (include/ppc_b200.h) + drop-in C++ API (include/xppc.h)
  libxppc.so   the same objects under the name the reference's library has
               (gpu/Makefile:12-13), for programs linked against it (llh/DirectFit)
  ppc          the command-line program (reference CLI, gpu/ppc.cu:524-598)

CUDA code is compiled for sm_100a only.  Host code is compiled with IEEE float
semantics (no fast-math, no contraction) so that the table build matches the reference
bit for bit (see tests/test_config_pin.py).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")
INC = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
# The system driver links libstdc++ as a shared library, the same one Python and numpy
# load; a toolchain that links it statically into the .so clashes with theirs at run time.
CXX = os.environ.get("PPCB_CXX", "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v", "-I" + INC]
CXXFLAGS = ["-O2", "-ffp-contract=off", "-fPIC", "-std=c++17", "-Wall", "-Wno-unused-result",
            "-I" + os.path.join(CUDA_HOME, "include"), "-I" + INC]

CU = ["propagate.cu", "engine.cu", "noalloc.cu", "batch.cu", "gradient.cu", "peak.cu", "backend.cu", "llh.cu",
      "frontend.cu"]
CPP = ["config.cpp", "session.cpp", "capi.cpp", "capi_batch.cpp", "capi_llh.cpp", "xppc.cpp", "llh.cpp"]
# Fast math everywhere but in the front end, whose bunch templates follow the host front
# end's float arithmetic (no approximate logf/powf, no contraction).  The likelihood
# (llh.cu) repeats the back end's acceptance decisions, so it keeps the back end's flags.
CU_EXTRA = {"frontend.cu": ["--fmad=false"]}
CU_FAST_MATH = ["--use_fast_math"]
CU_EXACT = {"frontend.cu"}
CLI = ["ppc_cli.cpp"]
HEADERS = ["ppcb_types.h", "config.h", "engine.h", "propagate.cuh", "session.h", "ctx.h", "tilt.h", "batch.h",
           "backend.cuh", "llh.h", "strgrid.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, log=None):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build failed: " + os.path.basename(cmd[-1]))
    if log is not None:
        with open(log, "w") as f:
            f.write(r.stdout + r.stderr)
    return r


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    hdrs = [os.path.join(SRC, h) for h in HEADERS] + [os.path.join(INC, "ppc_b200.h"), os.path.join(INC, "xppc.h")]
    objs = []
    for f in CU:
        src, obj = os.path.join(SRC, f), os.path.join(OBJ, f + ".o")
        if _newer(obj, [src] + hdrs):
            fast = [] if f in CU_EXACT else CU_FAST_MATH
            _run([NVCC] + NVFLAGS + fast + CU_EXTRA.get(f, []) + ["-c", src, "-o", obj],
                 log=os.path.join(OBJ, f + ".ptxas.txt"))
        objs.append(obj)
    for f in CPP:
        src, obj = os.path.join(SRC, f), os.path.join(OBJ, f + ".o")
        if _newer(obj, [src] + hdrs):
            _run([CXX] + CXXFLAGS + ["-c", src, "-o", obj])
        objs.append(obj)
    libs = ["-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    for name, soname in (("libppcb.so", "libppcb.so"), ("libxppc.so", "libxppc.so")):
        out = os.path.join(LIB, name)
        if _newer(out, objs):
            _run([CXX, "-shared", "-o", out] + objs + ["-Wl,-soname," + soname] + libs)
    cli_objs = []
    for f in CLI:
        src, obj = os.path.join(SRC, f), os.path.join(OBJ, f + ".o")
        if _newer(obj, [src] + hdrs):
            _run([CXX] + CXXFLAGS + ["-c", src, "-o", obj])
        cli_objs.append(obj)
    exe = os.path.join(BIN, "ppc")
    if _newer(exe, objs + cli_objs):
        _run([CXX, "-o", exe] + cli_objs + objs + libs)
    mwc_src, mwc = os.path.join(SRC, "mwc_multipliers.c"), os.path.join(BIN, "mwc_multipliers")
    if _newer(mwc, [mwc_src]):
        _run(["gcc", "-O2", "-fopenmp", mwc_src, "-o", mwc])
    if verbose:
        with open(os.path.join(OBJ, "propagate.cu.ptxas.txt")) as f:
            sys.stdout.write(f.read())
    return os.path.join(LIB, "libppcb.so")


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
