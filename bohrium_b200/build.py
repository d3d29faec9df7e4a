"""Build the native libraries of the B200 Bohrium stack in-tree.

    python -m bohrium_b200.build          # or: python bohrium_b200/build.py

Produces (under bohrium_b200/lib/):
  libbh_core.so     data model, config parser, component/extmethod loaders, the jitk fuser and
                    the flat C bridge (include/bh_b200.h)
  libbh_ve_cuda.so  the `cuda` vector engine component (NVRTC code generation for sm_100a plus
                    the hand-written sm_100a kernels compiled here with nvcc)
  libbh_vem_node.so the pass-through `node` component
  libbh_filter_bcexp.so, libbh_filter_bccon.so the bytecode filter components
  libbh_ext_cublas.so BLAS extension methods (blas_gemm, blas_gemmt) on cuBLAS for the cuda engine

C++ sources are compiled with g++ (-std=c++17 -O2 -fPIC); .cu sources with
nvcc -gencode arch=compute_100a,code=sm_100a. Objects are rebuilt when a source or any header
under include/ or the source's directory is newer.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import time

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
OBJ = os.path.join(PKG, "lib", "obj")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-Wall", "-Wno-unused-function", "-I" + INCLUDE,
            "-I" + os.path.join(CUDA_HOME, "include")]
NVCCFLAGS = ["-ccbin", CXX, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE] + ARCH


def _headers(src_dir: str) -> list[str]:
    hs = glob.glob(os.path.join(INCLUDE, "**", "*.h*"), recursive=True)
    hs += glob.glob(os.path.join(src_dir, "*.h*"))
    hs += glob.glob(os.path.join(CSRC, "jitk", "*.hpp"))
    return hs


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))


def _compile(src: str, verbose: bool) -> str:
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    obj = os.path.join(OBJ, rel + ".o")
    if _stale(obj, [src] + _headers(os.path.dirname(src))):
        os.makedirs(OBJ, exist_ok=True)
        if src.endswith(".cu"):
            cmd = [NVCC] + NVCCFLAGS + ["-c", "-o", obj, src]
        else:
            cmd = [CXX] + CXXFLAGS + ["-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return obj


def _link(target: str, objs: list[str], libs: list[str], verbose: bool) -> None:
    if not _stale(target, objs):
        return
    cmd = [CXX, "-shared", "-o", target] + objs + ["-Wl,-rpath,$ORIGIN", "-Wl,--no-undefined", "-L" + LIB] + libs
    if verbose:
        print(" ".join(cmd))
    _run(cmd)


def sources(sub: str) -> list[str]:
    d = os.path.join(CSRC, sub)
    return sorted(glob.glob(os.path.join(d, "*.cpp")) + glob.glob(os.path.join(d, "*.cu")))


def build(verbose: bool = False) -> dict:
    t0 = time.time()
    os.makedirs(LIB, exist_ok=True)
    core_objs = [_compile(s, verbose) for s in sources("core") + sources("jitk") + sources("capi")]
    core = os.path.join(LIB, "libbh_core.so")
    _link(core, core_objs, ["-ldl"], verbose)

    cuda_objs = [_compile(s, verbose) for s in sources("ve_cuda")]
    ve = os.path.join(LIB, "libbh_ve_cuda.so")
    cuda_lib = os.path.join(CUDA_HOME, "lib64")
    # .cu objects are compiled without relocatable device code, so g++ links them (against
    # cudart_static, which registers their fat binaries) with --no-undefined like the rest.
    _link(ve, cuda_objs, ["-lbh_core", "-L" + cuda_lib, "-lcudart_static", "-lnvrtc", "-ldl", "-lpthread", "-lrt"],
          verbose)

    ext_objs = [_compile(s, verbose) for s in sources("ext_cublas")]
    ext = os.path.join(LIB, "libbh_ext_cublas.so")
    _link(ext, ext_objs, ["-lbh_core", "-L" + cuda_lib, "-lcublas", "-lcudart_static", "-ldl", "-lpthread", "-lrt"],
          verbose)

    filters = {}
    for name in ("bcexp", "bccon"):
        obj = _compile(os.path.join(CSRC, "filter", name + ".cpp"), verbose)
        filters[name] = os.path.join(LIB, "libbh_filter_" + name + ".so")
        _link(filters[name], [obj], ["-lbh_core"], verbose)

    node_objs = [_compile(s, verbose) for s in sources("vem_node")]
    node = os.path.join(LIB, "libbh_vem_node.so")
    _link(node, node_objs, ["-lbh_core"], verbose)
    return {"core": core, "ve_cuda": ve, "vem_node": node, "ext_cublas": ext, **filters, "seconds": time.time() - t0}


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
