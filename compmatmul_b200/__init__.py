"""compmatmul_b200 -- Pagh's compressed matrix multiplication on NVIDIA B200.

Layers:

* ``libcmm_b200.so`` (C ABI, ``include/compmatmul_b200.h``): CUDA kernels for
  sm_100a and the host runtime.  Loaded with ctypes by :func:`lib`.
* ``compmatmul_b200.compmatmul``: the pybind11 drop-in for the reference's
  ``compmatmul`` module (``gemm``, ``matmul_fft``, ``matmul_fwht``).
* :mod:`compmatmul_b200.device`: device-resident API over torch CUDA tensors
  (sketch only, dense decompression, top-K recovery) for callers that keep
  their matrices on the GPU.

There is no CPU fallback: if the native library is missing, importing the
drop-in raises ImportError.
"""
from __future__ import annotations

import ctypes as _C
import os as _os

__all__ = ["lib", "CmmError", "HASH_KINDS", "VARIANTS", "LIB_PATH", "load_dropin"]

_PKG = _os.path.dirname(_os.path.abspath(__file__))
LIB_PATH = _os.path.join(_PKG, "libcmm_b200.so")

# compmatmul.cpp:97-104 hash strings -> cmm_hash_kind
HASH_KINDS = {None: 1, "multiply shift": 0, "multiply add shift": 1, "tabulation8": 2,
              "tabulation16": 3}
VARIANTS = {"fft": 0, "fwht": 1}

# symbols declared in include/compmatmul_b200.h
EXPORTED = [
    "cmm_last_error", "cmm_version", "cmm_device_count", "cmm_max_buckets", "cmm_matmul",
    "cmm_compressed_product", "cmm_decompress", "cmm_gemm", "cmm_hash_codes",
    "cmm_dev_compressed_product", "cmm_dev_decompress_dense", "cmm_dev_matmul", "cmm_dev_topk",
    "cmm_dev_gemm", "cmm_profile_enable", "cmm_profile_reset", "cmm_profile_read",
    "cmm_launch_count", "cmm_dev_compressed_product_f32", "cmm_dev_matmul_f32",
    "cmm_compressed_product_f32", "cmm_matmul_f32", "cmm_dev_compressed_product_noalloc",
    "cmm_last_sketch_kernel", "cmm_probe_fma_tflops", "cmm_batch_create", "cmm_batch_run",
    "cmm_batch_info", "cmm_batch_config", "cmm_batch_destroy", "cmm_server_create", "cmm_server_submit",
    "cmm_server_wait", "cmm_server_stats_get", "cmm_server_destroy", "cmm_dev_decompress_entries",
    "cmm_dev_sketch_topk", "cmm_rng_seed", "cmm_rng_next", "cmm_time_millis", "cmm_hash_params",
    "cmm_cluster_phase_cycles", "cmm_dev_wht_rows_f32",
]


class CmmError(RuntimeError):
    """A failing C ABI call; ``status`` is the cmm_status code."""

    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


_lib = None


def lib():
    """The loaded libcmm_b200.so with argument types declared."""
    global _lib
    if _lib is not None:
        return _lib
    if not _os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m compmatmul_b200.build`")
    L = _C.CDLL(LIB_PATH)
    i64, u64, i32 = _C.c_int64, _C.c_uint64, _C.c_int
    vp, dp = _C.c_void_p, _C.c_void_p
    L.cmm_last_error.restype = _C.c_char_p
    L.cmm_version.restype = _C.c_char_p
    L.cmm_last_sketch_kernel.restype = _C.c_char_p
    L.cmm_probe_fma_tflops.argtypes = [_C.c_int, _C.POINTER(_C.c_double)]
    L.cmm_batch_create.argtypes = [vp, i32, i32, i32, _C.POINTER(_C.c_void_p)]
    L.cmm_batch_run.argtypes = [vp, vp]
    L.cmm_batch_info.argtypes = [vp, _C.POINTER(_C.c_int64), _C.POINTER(_C.c_int), _C.POINTER(_C.c_int)]
    L.cmm_batch_config.argtypes = [vp, i32, _C.POINTER(_C.c_int), _C.POINTER(_C.c_int),
                                   _C.POINTER(_C.c_int), _C.POINTER(_C.c_int)]
    L.cmm_batch_destroy.argtypes = [vp]
    L.cmm_server_create.argtypes = [vp, _C.POINTER(_C.c_void_p)]
    L.cmm_server_submit.argtypes = [vp, vp, _C.POINTER(_C.c_uint64)]
    L.cmm_server_wait.argtypes = [vp, u64, _C.c_double, _C.POINTER(_C.c_int), _C.POINTER(_C.c_double)]
    L.cmm_server_stats_get.argtypes = [vp, vp]
    L.cmm_server_destroy.argtypes = [vp]
    L.cmm_dev_decompress_entries.argtypes = [i32, i32, i32, i32, u64, dp, i64, vp, vp, dp, vp]
    L.cmm_dev_sketch_topk.argtypes = [i32, i32, i64, i64, i32, i32, u64, dp, i32, _C.c_size_t, vp, vp, dp, vp]
    L.cmm_device_count.restype = i32
    L.cmm_max_buckets.restype = i32
    L.cmm_matmul.argtypes = [i32, i32, i64, i64, i64, dp, dp, dp, i32, i32, i32, u64]
    L.cmm_compressed_product.argtypes = [i32, i32, i64, i64, i64, dp, dp, i32, i32, i32, u64, dp, vp]
    L.cmm_decompress.argtypes = [i32, i32, i32, i32, u64, dp, i64, vp, vp, dp]
    L.cmm_gemm.argtypes = [i64, i64, i64, dp, dp, dp]
    L.cmm_hash_codes.argtypes = [i32, i32, i32, u64, i32, i64, vp]
    L.cmm_dev_compressed_product.argtypes = [i32, i32, i64, i64, i64, dp, dp, i32, i32, u64, dp, vp]
    L.cmm_dev_compressed_product_noalloc.argtypes = [i32, i32, i64, i64, i64, dp, dp, i32, i32, u64,
                                                     dp, vp]
    L.cmm_dev_decompress_dense.argtypes = [i32, i32, i64, i64, i32, i32, u64, dp, dp, vp]
    L.cmm_dev_matmul.argtypes = [i32, i32, i64, i64, i64, dp, dp, dp, i32, i32, u64, vp]
    L.cmm_dev_topk.argtypes = [dp, i64, i64, i32, vp, vp, dp, vp]
    L.cmm_dev_gemm.argtypes = [i64, i64, i64, dp, dp, dp, vp]
    L.cmm_dev_compressed_product_f32.argtypes = [i32, i32, i64, i64, i64, dp, dp, i32, i32, u64, dp, vp]
    L.cmm_dev_matmul_f32.argtypes = [i32, i32, i64, i64, i64, dp, dp, dp, i32, i32, u64, vp]
    L.cmm_compressed_product_f32.argtypes = [i32, i32, i64, i64, i64, dp, dp, i32, i32, i32, u64, dp, vp]
    L.cmm_matmul_f32.argtypes = [i32, i32, i64, i64, i64, dp, dp, dp, i32, i32, i32, u64]
    L.cmm_dev_wht_rows_f32.argtypes = [vp, vp, i64, i32, i32, vp]
    L.cmm_profile_enable.argtypes = [i32]
    L.cmm_profile_enable.restype = None
    L.cmm_profile_reset.restype = None
    L.cmm_profile_read.argtypes = [_C.c_char_p, _C.POINTER(_C.c_double), _C.POINTER(i64)]
    L.cmm_launch_count.restype = i64
    L.cmm_rng_seed.argtypes = [u64, vp]
    L.cmm_rng_seed.restype = None
    L.cmm_rng_next.argtypes = [vp]
    L.cmm_rng_next.restype = u64
    L.cmm_time_millis.restype = u64
    L.cmm_hash_params.argtypes = [i32, i32, u64, u64, vp, _C.c_size_t]
    L.cmm_cluster_phase_cycles.argtypes = [_C.POINTER(_C.c_double), _C.POINTER(_C.c_double)]
    for name in EXPORTED:
        if name not in ("cmm_last_error", "cmm_version", "cmm_profile_enable", "cmm_last_sketch_kernel",
                        "cmm_profile_reset", "cmm_launch_count", "cmm_rng_seed", "cmm_rng_next",
                        "cmm_time_millis"):
            getattr(L, name).restype = i32
    _lib = L
    return L


def check(status):
    """Raise the exception type the reference would raise for a status."""
    if status == 0:
        return
    msg = lib().cmm_last_error().decode()
    if status == 1:
        raise ValueError(msg)
    if status == 3:
        raise MemoryError(msg)
    raise CmmError(status, msg)


def profile_read(family):
    """(total_ms, launches) of a kernel family since the last reset."""
    ms = _C.c_double(0.0)
    n = _C.c_int64(0)
    check(lib().cmm_profile_read(family.encode(), _C.byref(ms), _C.byref(n)))
    return ms.value, n.value


def load_dropin():
    """The pybind11 drop-in module (same API as the reference's `compmatmul`)."""
    from . import compmatmul  # noqa: F401  (native extension)
    return compmatmul
