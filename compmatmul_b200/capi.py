"""numpy front end of the C ABI (include/compmatmul_b200.h).

Thin, typed wrappers: host numpy arrays in, host numpy arrays out.  The
pybind11 module `compmatmul` is the drop-in for the reference's Python
binding; these functions expose the rest of the ABI (sketch only,
decompression of listed entries, hash codes) for tests and tools.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import HASH_KINDS, VARIANTS, check, lib


def _kind(h):
    if isinstance(h, int):
        return h
    return HASH_KINDS[h]


def _var(v):
    return v if isinstance(v, int) else VARIANTS[v]


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None and a.size else C.c_void_p(0)


def hash_codes(hash_name, d, b, seed, side, n):
    """d x n uint32 codes: bucket | (sign == +1) << 31 (hashing.hpp)."""
    out = np.empty((d, n), dtype=np.uint32)
    check(lib().cmm_hash_codes(_kind(hash_name), d, b, seed, side, n, _p(out)))
    return out


def compressed_product(variant, hash_name, AT, B, d, b, seed=None):
    """(p, seed): matmul_compressed_product_{fft,fwht} (matmul_fft.hpp:26)."""
    AT = np.ascontiguousarray(AT, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    q, n_a = AT.shape
    n_b = B.shape[1]
    p = np.empty((d, b))
    used = C.c_uint64(0)
    check(lib().cmm_compressed_product(_var(variant), _kind(hash_name), n_a, q, n_b, _p(AT), _p(B),
                                       d, b, 0 if seed is None else 1, 0 if seed is None else seed,
                                       _p(p), C.byref(used)))
    return p, used.value


def matmul(variant, hash_name, AT, B, d, b, seed=None):
    """Dense C: matmul_{fft,fwht} (matmul_fft.hpp:156)."""
    AT = np.ascontiguousarray(AT, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    q, n_a = AT.shape
    n_b = B.shape[1]
    Cm = np.empty((n_a, n_b))
    check(lib().cmm_matmul(_var(variant), _kind(hash_name), n_a, q, n_b, _p(Cm), _p(AT), _p(B), d,
                           b, 0 if seed is None else 1, 0 if seed is None else seed))
    return Cm


def decompress(variant, hash_name, p, d, b, seed, i, j):
    """Estimates for listed entries: matmul_decompress_{fft,fwht}."""
    p = np.ascontiguousarray(p, dtype=np.float64)
    i = np.ascontiguousarray(i, dtype=np.uint32)
    j = np.ascontiguousarray(j, dtype=np.uint32)
    out = np.empty(i.size)
    check(lib().cmm_decompress(_var(variant), _kind(hash_name), d, b, seed, _p(p), i.size, _p(i),
                               _p(j), _p(out)))
    return out


def gemm(AT, B):
    AT = np.ascontiguousarray(AT, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    q, n_a = AT.shape
    n_b = B.shape[1]
    Cm = np.empty((n_a, n_b))
    check(lib().cmm_gemm(n_a, q, n_b, _p(Cm), _p(AT), _p(B)))
    return Cm


def compressed_product_f32(variant, hash_name, AT, B, d, b, seed=None):
    """Mixed precision sketch from FP32 inputs; p is FP64 (d x b)."""
    AT = np.ascontiguousarray(AT, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    q, n_a = AT.shape
    n_b = B.shape[1]
    p = np.empty((d, b))
    used = C.c_uint64(0)
    check(lib().cmm_compressed_product_f32(_var(variant), _kind(hash_name), n_a, q, n_b, _p(AT),
                                           _p(B), d, b, 0 if seed is None else 1,
                                           0 if seed is None else seed, _p(p), C.byref(used)))
    return p, used.value


def matmul_f32(variant, hash_name, AT, B, d, b, seed=None):
    """Mixed precision dense estimate (FP64 output) from FP32 inputs."""
    AT = np.ascontiguousarray(AT, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    q, n_a = AT.shape
    n_b = B.shape[1]
    Cm = np.empty((n_a, n_b))
    check(lib().cmm_matmul_f32(_var(variant), _kind(hash_name), n_a, q, n_b, _p(Cm), _p(AT), _p(B),
                               d, b, 0 if seed is None else 1, 0 if seed is None else seed))
    return Cm
