"""ctypes front end of the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Two checkers live under oracle/:

* ``Oracle`` -- the plain-C restatement ``cmm_oracle.c`` of the reference
  algorithm (rng.hpp, hashing.hpp, matmul_sketch.hpp, matmul_fft.hpp,
  matmul_fwht.hpp, array.hpp::median), single threaded, FP64.
* ``RefLib`` -- the reference's own headers compiled unchanged against the
  project shims (``oracle/_ref/libcmm_ref.so``, OpenMP).  Present only when
  ``make -C oracle ref`` ran in a tree that had the reference sources.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libcmm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcmm_ref.so")

HASHES = {None: 1, "multiply shift": 0, "multiply add shift": 1, "tabulation8": 2, "tabulation16": 3}
VARIANTS = {"fft": 0, "fwht": 1}

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int)
_u64p = C.POINTER(C.c_uint64)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Oracle:
    """The C restatement.  All arrays are numpy, C-contiguous."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        L.cmo_rng_seed.argtypes = [_u64p, C.c_uint64]
        L.cmo_rng_next.argtypes = [_u64p]
        L.cmo_rng_next.restype = C.c_uint64
        L.cmo_drng_next.argtypes = [_u64p]
        L.cmo_drng_next.restype = C.c_double
        L.cmo_hash_param_bytes.argtypes = [C.c_int]
        L.cmo_hash_param_bytes.restype = C.c_size_t
        L.cmo_hash_draw.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_void_p]
        L.cmo_hash_bucket.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_uint32]
        L.cmo_hash_bucket.restype = C.c_uint32
        L.cmo_hash_sign.argtypes = [C.c_int, C.c_void_p, C.c_uint32]
        L.cmo_hash_sign.restype = C.c_int
        L.cmo_fft_r2c.argtypes = [C.c_int, _dp, _dp]
        L.cmo_fft_c2r.argtypes = [C.c_int, _dp, _dp]
        L.cmo_fwht.argtypes = [C.c_int, _dp]
        L.cmo_sketch_codes.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int64, _u32p]
        L.cmo_compressed_product.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int64,
                                             _dp, _dp, C.c_int, C.c_int, C.c_uint64, _dp]
        L.cmo_decompress_rows.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, _dp,
                                          C.c_int64, C.c_int64, C.c_int64, C.c_int64, _dp]
        L.cmo_matmul.argtypes = [C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int64, _dp, _dp, _dp,
                                 C.c_int, C.c_int, C.c_uint64]
        L.cmo_gemm.argtypes = [C.c_int64, C.c_int64, C.c_int64, _dp, _dp, _dp]
        L.cmo_median.argtypes = [C.c_int, _dp]
        L.cmo_median.restype = C.c_double
        L.cmo_seed_from_time_millis.argtypes = [C.c_uint64]
        L.cmo_seed_from_time_millis.restype = C.c_uint64
        self.L = L

    # rng.hpp
    def rng(self, seed, count):
        s = (C.c_uint64 * 4)()
        self.L.cmo_rng_seed(s, seed)
        return [self.L.cmo_rng_next(s) for _ in range(count)]

    def drng(self, seed, count):
        s = (C.c_uint64 * 4)()
        self.L.cmo_rng_seed(s, seed)
        return np.array([self.L.cmo_drng_next(s) for _ in range(count)])

    # hashing.hpp
    def hash_draw(self, kind, n, seed):
        nb = self.L.cmo_hash_param_bytes(kind)
        buf = (C.c_ubyte * (nb * n))()
        self.L.cmo_hash_draw(kind, n, seed, buf)
        return buf, nb

    def hash_params_u64(self, kind, n, seed):
        buf, nb = self.hash_draw(kind, n, seed)
        return list(np.frombuffer(bytes(buf), dtype=np.uint64))

    def hash_eval(self, kind, n, b, seed, keys):
        """(buckets[t][key], signs[t][key]) for the n functions drawn with seed."""
        buf, nb = self.hash_draw(kind, n, seed)
        base = C.addressof(buf)
        hs = np.empty((n, len(keys)), dtype=np.uint32)
        ss = np.empty((n, len(keys)), dtype=np.int32)
        for t in range(n):
            fn = C.c_void_p(base + nb * t)
            for e, key in enumerate(keys):
                hs[t, e] = self.L.cmo_hash_bucket(kind, fn, b, int(key))
                ss[t, e] = self.L.cmo_hash_sign(kind, fn, int(key))
        return hs, ss

    def sketch_codes(self, kind, d, b, seed, side, n):
        out = np.empty((d, n), dtype=np.uint32)
        self.L.cmo_sketch_codes(kind, d, b, seed, side, n, _ptr(out, _u32p))
        return out

    # transform.hpp semantics
    def fft_r2c(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = x.size
        X = np.empty(2 * (n // 2 + 1))
        self.L.cmo_fft_r2c(n, _ptr(x), _ptr(X))
        return X[0::2] + 1j * X[1::2]

    def fft_c2r(self, X, n):
        Xi = np.empty(2 * (n // 2 + 1))
        Xi[0::2] = np.real(X)
        Xi[1::2] = np.imag(X)
        x = np.empty(n)
        self.L.cmo_fft_c2r(n, _ptr(Xi), _ptr(x))
        return x

    def fwht(self, x):
        y = np.array(x, dtype=np.float64, copy=True)
        self.L.cmo_fwht(y.size, _ptr(y))
        return y

    # matmul_sketch / matmul_fft / matmul_fwht
    def compressed_product(self, variant, hash_name, AT, B, d, b, seed):
        AT = np.ascontiguousarray(AT, dtype=np.float64)
        B = np.ascontiguousarray(B, dtype=np.float64)
        q, p_ = AT.shape
        r = B.shape[1]
        out = np.empty((d, b))
        self.L.cmo_compressed_product(VARIANTS[variant], HASHES[hash_name], p_, q, r, _ptr(AT),
                                      _ptr(B), d, b, seed, _ptr(out))
        return out

    def decompress(self, variant, hash_name, sketch_p, d, b, seed, n_a, n_b, rows=None):
        i0, i1 = (0, n_a) if rows is None else rows
        C_ = np.zeros((n_a, n_b))
        sp = np.ascontiguousarray(sketch_p, dtype=np.float64)
        self.L.cmo_decompress_rows(VARIANTS[variant], HASHES[hash_name], d, b, seed, _ptr(sp),
                                   n_a, n_b, i0, i1, _ptr(C_))
        return C_

    def matmul(self, variant, hash_name, AT, B, d, b, seed):
        AT = np.ascontiguousarray(AT, dtype=np.float64)
        B = np.ascontiguousarray(B, dtype=np.float64)
        q, p_ = AT.shape
        r = B.shape[1]
        C_ = np.empty((p_, r))
        self.L.cmo_matmul(VARIANTS[variant], HASHES[hash_name], p_, q, r, _ptr(C_), _ptr(AT),
                          _ptr(B), d, b, seed)
        return C_

    def gemm(self, AT, B):
        AT = np.ascontiguousarray(AT, dtype=np.float64)
        B = np.ascontiguousarray(B, dtype=np.float64)
        q, p_ = AT.shape
        r = B.shape[1]
        C_ = np.empty((p_, r))
        self.L.cmo_gemm(p_, q, r, _ptr(C_), _ptr(AT), _ptr(B))
        return C_

    def median(self, xs):
        a = np.array(xs, dtype=np.float64)
        return self.L.cmo_median(a.size, _ptr(a))

    def seed_from_time_millis(self, ms):
        return self.L.cmo_seed_from_time_millis(ms)


class RefLib:
    """The reference's own headers (compiled with shims), OpenMP threaded."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        L.ref_num_threads.restype = C.c_int
        L.ref_matmul.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp,
                                 C.c_int, C.c_int, C.c_uint64]
        L.ref_compressed_product.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp,
                                             C.c_int, C.c_int, C.c_uint64, _dp]
        L.ref_decompress_rows.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, _dp,
                                          C.c_int, C.c_int, C.c_int, _dp]
        L.ref_hash_codes.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, _u32p, _i32p]
        L.ref_gemm.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
        L.ref_fft_fwd.argtypes = [C.c_int, _dp, _dp]
        L.ref_fft_inv.argtypes = [C.c_int, _dp, _dp]
        L.ref_fwht_fwd.argtypes = [C.c_int, _dp]
        L.ref_rng_first.argtypes = [C.c_uint64]
        L.ref_rng_first.restype = C.c_uint64
        self.L = L

    @staticmethod
    def available(path=REF_SO):
        return os.path.exists(path)

    def num_threads(self):
        return self.L.ref_num_threads()

    def compressed_product(self, variant, hash_name, AT, B, d, b, seed):
        AT = np.ascontiguousarray(AT, dtype=np.float64)
        B = np.ascontiguousarray(B, dtype=np.float64)
        q, p_ = AT.shape
        r = B.shape[1]
        out = np.empty((d, b))
        rc = self.L.ref_compressed_product(VARIANTS[variant], HASHES[hash_name], p_, q, r,
                                           _ptr(AT), _ptr(B), d, b, seed, _ptr(out))
        assert rc == 0
        return out

    def decompress_rows(self, variant, hash_name, sketch_p, d, b, seed, n_b, i0, i1, C_):
        sp = np.ascontiguousarray(sketch_p, dtype=np.float64)
        rc = self.L.ref_decompress_rows(VARIANTS[variant], HASHES[hash_name], d, b, seed,
                                        _ptr(sp), n_b, i0, i1, _ptr(C_))
        assert rc == 0

    def matmul(self, variant, hash_name, AT, B, d, b, seed):
        AT = np.ascontiguousarray(AT, dtype=np.float64)
        B = np.ascontiguousarray(B, dtype=np.float64)
        q, p_ = AT.shape
        r = B.shape[1]
        C_ = np.empty((p_, r))
        rc = self.L.ref_matmul(VARIANTS[variant], HASHES[hash_name], p_, q, r, _ptr(C_),
                               _ptr(AT), _ptr(B), d, b, seed)
        assert rc == 0
        return C_

    def hash_codes(self, hash_name, d, b, seed, n):
        hs = np.empty((d, n), dtype=np.uint32)
        ss = np.empty((d, n), dtype=np.int32)
        self.L.ref_hash_codes(HASHES[hash_name], d, b, seed, n, _ptr(hs, _u32p), _ptr(ss, _i32p))
        return hs, ss

    def fft_fwd(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        X = np.empty(2 * (x.size // 2 + 1))
        self.L.ref_fft_fwd(x.size, _ptr(x), _ptr(X))
        return X[0::2] + 1j * X[1::2]

    def fwht(self, x):
        y = np.array(x, dtype=np.float64, copy=True)
        self.L.ref_fwht_fwd(y.size, _ptr(y))
        return y
