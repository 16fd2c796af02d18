"""Builds the in-tree CUDA library seticore_b200/_lib/libseticore_b200.so for sm_100a.

Run as `python -m seticore_b200.build` (or through __graft_entry__.build()).  The
library is a plain C-ABI shared object (include/seticore_b200.h); nothing is JIT
compiled at import time, so the built file travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libseticore_b200.so")
SOURCES = ["dd_api.cu", "dd_tree.cu", "dd_stats.cu", "dd_order.cu", "dd_hits.cu", "dd_levels.cu", "dd_noalloc.cu", "dd_precision.cu",
           "dd_exec.cu",
           "dd_pool.cu", "dd_io.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose_ptxas=False):
    os.makedirs(LIBDIR, exist_ok=True)
    gen = os.path.join(CSRC, "generated", "taylor_stream_gen.cuh")
    os.makedirs(os.path.dirname(gen), exist_ok=True)
    sys.path.insert(0, CSRC)
    try:
        import gen_taylor_stream
        gen_taylor_stream.main(gen)
    finally:
        sys.path.pop(0)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [gen, os.path.join(CSRC, "generated", "taylor_direct_gen.cuh"), os.path.join(CSRC, "dd_common.cuh"),
                   os.path.join(CSRC, "dd_internal.h"), os.path.join(ROOT, "include", "seticore_b200.h")]
    objdir = os.path.join(HERE, "_lib", "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"),
                    "-I" + CSRC]
    if verbose_ptxas:
        flags += ["-Xptxas", "-v"]
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        if force or _stale(o, [s] + deps[len(srcs):]):
            _run([NVCC] + flags + ["-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs)
    # The reference's dedoppler unit test against the header-only C++ drop-in.
    cpp = os.path.join(ROOT, "tests", "cpp", "dedoppler_api_test.cpp")
    exe = os.path.join(LIBDIR, "dedoppler_api_test")
    hpp = os.path.join(ROOT, "include", "seticore_b200", "dedoppler.hpp")
    if os.path.exists(cpp) and (force or _stale(exe, [cpp, hpp, LIB])):
        _run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", cpp,
              "-o", exe, "-L" + LIBDIR, "-lseticore_b200", "-L/usr/local/cuda/lib64", "-lcudart",
              "-Wl,-rpath,$ORIGIN", "-Wl,-rpath,/usr/local/cuda/lib64"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
