"""Builds the in-tree shared library skirt7_b200/libskirt_b200.so for sm_100a.

The library is plain nvcc/g++ output (no torch extension): the C ABI of include/skirt_b200.h is
loaded with ctypes by the Python package and can be linked by any C/C++ host.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
LIB = os.path.join(HERE, "libskirt_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH

# The path harness is compiled without FMA contraction: its FP64 steppers must round every
# multiply and add separately, as the reference's host build does.
UNITS = [
    ("skg_trace.cu", ["--fmad=false"]),
    ("skg_tracer.cu", []),
    ("skg_setup.cu", []),
    ("skg_voronoi.cu", []),
    ("skg_api.cu", []),
]
CXX_UNITS = ["skg_host.cpp", "skg_serve.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r.stdout + r.stderr


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "skirt_b200.h"))
    objs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s, __file__] + headers):
            cmd = [nvcc] + NVCC_COMMON + extra + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", "-o", o, s]
            out = _run(cmd)
            if verbose or ptxas_info:
                sys.stdout.write(out)
    for src in CXX_UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s, __file__] + headers):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-pthread", "-ffp-contract=off", "-I" + CUDA_INC, "-c", "-o", o,
                  s])
    if _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-Xcompiler", "-pthread"])
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
