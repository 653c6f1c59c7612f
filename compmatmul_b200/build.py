"""Builds the native parts of compmatmul_b200 in-tree.

* ``libcmm_b200.so``   -- CUDA kernels + host runtime + C ABI (nvcc, sm_100a)
* ``compmatmul*.so``   -- pybind11 module ``compmatmul``: the drop-in for the
                          reference's Python binding, calling the C ABI

Run ``python -m compmatmul_b200.build`` (or ``__graft_entry__.build()``).
Objects go to ``compmatmul_b200/_build`` (git-ignored); the .so files sit in
the package directory so they travel with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libcmm_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]
# extra flags for instrumented builds, e.g. CMM_EXTRA_NVFLAGS=-DCMM_PHASE_CLOCKS
# (per-phase cycle counts of the cluster sketch kernel)
NVFLAGS += os.environ.get("CMM_EXTRA_NVFLAGS", "").split()

CUDA_SOURCES = ["cmm_sketch.cu", "cmm_sketch_v1.cu", "cmm_sketch_mixed.cu", "cmm_sketch_cluster.cu",
                "cmm_plan.cu", "cmm_recover.cu", "cmm_noalloc.cu", "cmm_probe.cu", "cmm_batch.cu", "cmm_serve.cu",
                "cmm_wht_tc.cu"]
HOST_SOURCES = ["cmm_hashparams.cpp", "cmm_capi.cpp", "cmm_hostcopy.cpp"]


def _run(cmd, verbose=False):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "compmatmul_b200.h"))
    objs = []
    for src in CUDA_SOURCES + HOST_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if _stale(obj, [path] + headers) or ptxas_info:
            extra = ["-Xptxas", "-v"] if (ptxas_info and src.endswith(".cu")) else []
            out = _run([NVCC] + NVFLAGS + extra + ["-c", path, "-o", obj], verbose)
            if ptxas_info and out:
                print(out)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl",
                                                               "-lpthread"], verbose)
    return LIB


def build_module(verbose=False):
    import pybind11

    ext = sysconfig.get_config_var("EXT_SUFFIX")
    target = os.path.join(PKG, "compmatmul" + ext)
    src = os.path.join(CSRC, "compmatmul_module.cpp")
    if not _stale(target, [src, LIB, os.path.join(INCLUDE, "compmatmul_b200.h")]):
        return target
    cmd = ["g++", "-std=c++20", "-O2", "-shared", "-fPIC", "-I" + INCLUDE,
           "-I" + sysconfig.get_paths()["include"], "-I" + pybind11.get_include(), src,
           "-o", target, "-L" + PKG, "-l:libcmm_b200.so", "-Wl,-rpath,$ORIGIN"]
    _run(cmd, verbose)
    return target


CLI = os.path.join(PKG, "cmm_multiply")


def build_cli(verbose=False):
    """The `multiply` command-line program (csrc/multiply_main.cpp)."""
    src = os.path.join(CSRC, "multiply_main.cpp")
    if not _stale(CLI, [src, LIB, os.path.join(INCLUDE, "compmatmul_b200.h")]):
        return CLI
    cuda = os.path.dirname(os.path.dirname(NVCC)) if os.path.isabs(NVCC) else "/usr/local/cuda"
    cmd = ["g++", "-std=c++17", "-O2", "-I" + INCLUDE, "-I" + os.path.join(cuda, "include"), src, "-o", CLI,
           "-L" + PKG, "-l:libcmm_b200.so", "-L" + os.path.join(cuda, "lib64"), "-lcudart",
           "-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.join(cuda, "lib64")]
    _run(cmd, verbose)
    return CLI


def build(verbose=False):
    build_lib(verbose)
    build_module(verbose)
    build_cli(verbose)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    if "--ptxas" in sys.argv:
        build_lib(verbose=False, ptxas_info=True)
