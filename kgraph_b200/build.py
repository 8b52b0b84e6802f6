"""Compiles the library in-tree for sm_100a.

    libkgraph_b200.so   CUDA kernels + C-ABI (include/kgraph_b200.h) + C++ API (include/kgraph.h)
    _kgraph*.so         Python module (pybind11) over the C++ API
    bin/index, bin/search, bin/prune, bin/resave   the command-line tools (the reference's), over the C++ API

Run as ``python -m kgraph_b200.build`` or through ``__graft_entry__.build()``.
nvcc cross-compiles without a GPU.
"""
import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libkgraph_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CUDA_SOURCES = ["kg_ctx.cu", "kg_search.cu", "kg_build.cu", "kg_graph.cu", "kg_noalloc.cu", "kg_router.cu",
                "kg_join_tc.cu", "kg_precision.cu", "kg_gemm.cu", "kg_checks.cu", "kg_bruteforce.cu"]
CXX_SOURCES = ["kgraph_api.cpp"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    # The canonical distance uses explicit _rn intrinsics; no other contraction either.
    "--fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    "-I" + os.path.join(ROOT, "include"),
]
HEADERS = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + [
    os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def _compile(src):
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ, src + ".o")
    if _stale(obj, [path] + HEADERS):
        if src.endswith(".cu"):
            _run([NVCC] + NVCC_FLAGS + ["-Xptxas", "-v", "-c", path, "-o", obj])
        else:
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-I" + os.path.join(ROOT, "include"),
                  "-I/usr/local/cuda/include", "-c", path, "-o", obj])
    return obj


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(4) as ex:
        objs = list(ex.map(_compile, CUDA_SOURCES + CXX_SOURCES))
    if _stale(LIB, objs):
        _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static", "-o", LIB] + objs)
    import pybind11
    ext = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    mod = os.path.join(PKG, "_kgraph" + ext)
    src = os.path.join(CSRC, "pykgraph.cpp")
    if _stale(mod, [src, LIB] + HEADERS):
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall",
              "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
              "-I" + os.path.join(ROOT, "include"), src, "-o", mod,
              "-L" + PKG, "-lkgraph_b200", "-Wl,-rpath,$ORIGIN"])
    bindir = os.path.join(PKG, "bin")
    os.makedirs(bindir, exist_ok=True)
    cli = os.path.join(PKG, "cli")
    for tool in ("index", "search", "prune", "resave"):
        src = os.path.join(cli, tool + ".cpp")
        exe = os.path.join(bindir, tool)
        if _stale(exe, [src, LIB, os.path.join(cli, "cli_args.h")] + HEADERS):
            _run(["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), src, "-o", exe,
                  "-L" + PKG, "-lkgraph_b200", "-Wl,-rpath,$ORIGIN/.."])
    if verbose:
        print("built", LIB, mod, bindir)
    return LIB, mod


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
