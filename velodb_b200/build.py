"""Build recipe for the sm_100a library ``velodb_b200/libvelo_obl.so``.

Every ``csrc/*.cu`` / ``csrc/*.cpp`` is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` (cross-compiles without a GPU),
objects go to ``velodb_b200/_build/`` and are linked into one shared library
that exports the C ABI declared in ``include/velo_obl.h``.  The library is
built in-tree so it travels with the repository snapshot.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libvelo_obl.so")
HOST = os.path.join(PKG, "host")
OPS_LIB = os.path.join(PKG, "libvelo_operators.so")
TRACE_LIB = os.path.join(PKG, "libvelo_obl_trace.so")
TRACE_BUILD = os.path.join(PKG, "_build_trace")
CXX = os.environ.get("VELO_CXX", "g++")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "--extended-lambda",
          "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(obj, src, hdr_mtime):
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    return os.path.getmtime(src) > m or hdr_mtime > m


def _compile(src, extra, build_dir=BUILD):
    obj = os.path.join(build_dir, os.path.basename(src) + ".o")
    cmd = [NVCC] + ARCH + CFLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def _build_lib(lib, build_dir, extra, link_extra, verbose):
    os.makedirs(build_dir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [os.path.getmtime(__file__)])
    todo = [s for s in srcs if _stale(os.path.join(build_dir, os.path.basename(s) + ".o"), s, hdr_mtime)]
    if verbose and todo:
        print("compiling:", ", ".join(os.path.basename(s) for s in todo), file=sys.stderr)
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
        list(ex.map(lambda s: _compile(s, extra, build_dir), todo))
    objs = [os.path.join(build_dir, os.path.basename(s) + ".o") for s in srcs]
    if todo or not os.path.exists(lib) or any(os.path.getmtime(o) > os.path.getmtime(lib) for o in objs):
        cmd = [NVCC] + ARCH + link_extra + ["-shared", "-o", lib] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


def build(verbose: bool = False, extra_flags=None) -> str:
    """Compile stale sources and relink.  Returns the library path."""
    _build_lib(LIB, BUILD, list(extra_flags or []), [], verbose)
    build_operators(verbose)
    return LIB


def build_trace(verbose: bool = False) -> str:
    """The address-trace test library libvelo_obl_trace.so: the same sources
    with -DVELO_TRACE, as relocatable device code so that the trace buffers
    are one set of device globals for every translation unit."""
    return _build_lib(TRACE_LIB, TRACE_BUILD, ["-DVELO_TRACE", "-rdc=true"], ["-rdc=true"], verbose)


def build_operators(verbose: bool = False) -> str:
    """The C++ operator layer (host/*.cpp) as libvelo_operators.so, linked
    against libvelo_obl.so only (no CUDA headers or runtime of its own)."""
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    deps = srcs + [os.path.join(INCLUDE, "velo_operator.hpp"), os.path.join(INCLUDE, "velo_obl.h"), LIB]
    if os.path.exists(OPS_LIB) and all(os.path.getmtime(d) <= os.path.getmtime(OPS_LIB) for d in deps):
        return OPS_LIB
    if verbose:
        print("compiling: " + ", ".join(os.path.basename(x) for x in srcs), file=sys.stderr)
    cmd = [CXX, "-std=c++17", "-O2", "-g", "-fPIC", "-shared", "-Wall", "-Wextra", "-I", INCLUDE] + srcs + \
        ["-L", PKG, "-lvelo_obl", "-Wl,-rpath,$ORIGIN", "-o", OPS_LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"operator layer build failed:\n{r.stdout}\n{r.stderr}")
    return OPS_LIB


if __name__ == "__main__":
    print(build(verbose=True))
    if "--trace" in sys.argv:
        print(build_trace(verbose=True))
