"""Build libep2d.so (and the drop-in CLI) in-tree for sm_100a.

Kernels are compiled by nvcc; the host orchestration by the host C++ compiler with
-ffp-contract=off, so host-side arithmetic rounds exactly like the reference's host code.
The CUDA runtime is linked statically: the library needs only the NVIDIA driver.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libep2d.so")
NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")

CU_SOURCES = ["ep2d_kernels.cu", "ep2d_noalloc.cu"]
CPP_SOURCES = ["ep2d_rve.cpp", "ep2d_api.cpp", "ep2d_batch.cpp"]
HEADERS = ["ep2d_device.cuh", "ep2d_stencil.cuh", "ep2d_iter_f64.cuh", "ep2d_iter_stream.cuh", "ep2d_types.hpp", "ep2d_rve.hpp", "ep2d_batch.hpp"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r.stdout


def build_lib(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "ep2d.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + hdrs):
            out = _run([NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xptxas", "-v", "-Xcompiler", "-fPIC",
                        "-I" + INCLUDE, "-I" + CSRC, "-c", s, "-o", o])
            if verbose:
                sys.stdout.write(out)
        objs.append(o)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + hdrs):
            _run([CXX, "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
                  "-I" + INCLUDE, "-I" + CSRC, "-I" + CUDA_INC, "-c", s, "-o", o])
        objs.append(o)
    if force or _newer(LIB, objs):
        _run([NVCC, "-shared", *ARCH, "-cudart", "static", "-o", LIB, *objs])
    return LIB


if __name__ == "__main__":
    print(build_lib(verbose="-v" in sys.argv, force="-f" in sys.argv))


DROPIN = os.path.join(CSRC, "dropin")
CLI = os.path.join(HERE, "ep2d_cli")


def build_cli_unity(macros, out, force=False):
    """The self-contained drop-in CLI: the reference's nvcc line plus -DEP2D_UNITY, the
    library sources compiled into the binary (no libep2d.so needed at run time)."""
    srcs = [os.path.join(DROPIN, s) for s in ("EffPlast2D.cu", "main.cu")]
    deps = srcs + [os.path.join(DROPIN, "EffPlast2D.h")] + [os.path.join(CSRC, h) for h in HEADERS] + \
        [os.path.join(CSRC, s) for s in ("ep2d_kernels.cu", "ep2d_rve.cpp", "ep2d_api.cpp")]
    if force or _newer(out, deps):
        flags = ["-D%s=%s" % (k, v) for k, v in macros.items()]
        _run([NVCC, "-O3", "-std=c++17", *ARCH, "-DEP2D_UNITY", *flags, "-I" + INCLUDE, "-I" + CSRC, "-o", out,
              *srcs])
    return out


def build_cli(macros=None, out=None, force=False):
    """Build the drop-in CLI (the reference's main.cu + EffPlast2D class contract) from
    csrc/dropin with the reference's compile-time macros (NL, NGRID, NITER, EITER,
    NPARS, DEVICE_IDX), as eff_props_2D.m:45 passes them."""
    srcs = [os.path.join(DROPIN, s) for s in ("EffPlast2D.cu", "main.cu")]
    if not all(os.path.exists(s) for s in srcs):
        return None
    lib = build_lib()
    out = out or CLI
    deps = srcs + [os.path.join(DROPIN, "EffPlast2D.h"), lib]
    if force or macros or _newer(out, deps):
        flags = ["-D%s=%s" % (k, v) for k, v in (macros or {}).items()]
        _run([NVCC, "-std=c++17", "-O3", *ARCH, *flags, "-I" + INCLUDE, "-I" + DROPIN, "-o", out, *srcs,
              "-L" + HERE, "-lep2d", "-Xlinker", "-rpath=" + HERE])
    return out
