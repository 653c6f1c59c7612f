"""CPU-only checks of the boundary: the C ABI library loads and exports
every symbol include/compmatmul_b200.h declares; the drop-in module rejects
bad arguments with the reference binding's exception types and messages
(compmatmul.cpp:13-105) before touching a GPU."""
import os
import re

import numpy as np
import pytest

from conftest import aligned_alloc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "compmatmul_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:const\s+)?\w+\*?\s+\**(cmm_\w+)\s*\(", src, re.M)))


def test_header_declares_api():
    syms = declared_symbols()
    assert "cmm_matmul" in syms and "cmm_dev_topk" in syms and len(syms) >= 14


def test_library_exports_every_declared_symbol():
    import ctypes
    import compmatmul_b200
    L = ctypes.CDLL(compmatmul_b200.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert set(declared_symbols()) == set(compmatmul_b200.EXPORTED)


def test_library_calls_without_gpu_are_safe():
    import compmatmul_b200
    L = compmatmul_b200.lib()
    assert L.cmm_version().startswith(b"compmatmul_b200")
    assert L.cmm_max_buckets() == 1 << 24
    assert L.cmm_device_count() >= 0


def test_argument_errors_before_gpu():
    import compmatmul_b200
    L = compmatmul_b200.lib()
    # invalid b / d / hash are rejected by the ABI itself (no device touched)
    st = L.cmm_compressed_product(0, 1, 4, 4, 4, None, None, 1, 3, 1, 0, None, None)
    assert st == 1 and b"b must be power of 2 greater than 1 (got 3)" in L.cmm_last_error()
    st = L.cmm_compressed_product(0, 1, 4, 4, 4, None, None, 0, 8, 1, 0, None, None)
    assert st == 1 and b"d must be positive (got 0)" in L.cmm_last_error()
    st = L.cmm_compressed_product(0, 7, 4, 4, 4, None, None, 1, 8, 1, 0, None, None)
    assert st == 1
    st = L.cmm_compressed_product(0, 1, 4, 4, 4, None, None, 1, 1 << 25, 1, 0, None, None)
    assert st == 5  # CMM_ERR_UNSUPPORTED: beyond this build's limits


def test_wht_rows_argument_errors_before_gpu():
    import compmatmul_b200
    L = compmatmul_b200.lib()
    assert L.cmm_dev_wht_rows_f32(None, None, 4, 10, 1, None) == 5  # row length beyond 2^11..2^13
    assert b"2^11, 2^12 or 2^13" in L.cmm_last_error()
    assert L.cmm_dev_wht_rows_f32(None, None, 4, 13, 2, None) == 1  # unknown method
    assert L.cmm_dev_wht_rows_f32(None, None, -1, 13, 1, None) == 1
    assert L.cmm_dev_wht_rows_f32(None, None, 4, 13, 1, None) == 1  # null rows
    assert L.cmm_dev_wht_rows_f32(8, 16, 4, 13, 0, None) == 1  # not 16-byte aligned
    assert b"16-byte aligned" in L.cmm_last_error()
    assert L.cmm_dev_wht_rows_f32(None, None, 0, 13, 1, None) == 0  # nothing to do


def _bad_calls(mod):
    """(callable, expected exception) pairs mirroring compmatmul.cpp checks."""
    A = aligned_alloc((4, 4))
    A[...] = 1.0
    C = aligned_alloc((4, 4))
    f32 = aligned_alloc((4, 4), np.float32)
    vec = aligned_alloc((16,))
    nc = aligned_alloc((4, 8))[:, ::2]
    mis = aligned_alloc((17,))[1:].reshape(4, 4)
    big = aligned_alloc((4, 5))
    return [
        (lambda: mod.matmul_fft(C, f32, A, 1, 8), ValueError),
        (lambda: mod.matmul_fft(vec, A, A, 1, 8), ValueError),
        (lambda: mod.matmul_fft(C, nc, A, 1, 8), ValueError),
        (lambda: mod.matmul_fft(C, A, big, 1, 8), ValueError),
        (lambda: mod.matmul_fft(C, mis, A, 1, 8), ValueError),
        (lambda: mod.matmul_fft(C, A, mis, 1, 8), ValueError),
        (lambda: mod.matmul_fft(mis, A, A, 1, 8), ValueError),
        (lambda: mod.matmul_fft(C, A, A, 1, 12), ValueError),
        (lambda: mod.matmul_fft(C, A, A, 1, 1), ValueError),
        (lambda: mod.matmul_fwht(C, A, A, 0, 8), ValueError),
        (lambda: mod.matmul_fwht(C, A, A, 1, 8, 5, "crc32"), ValueError),
        (lambda: mod.gemm(C, f32, A), ValueError),
        (lambda: mod.matmul_fft(C, A, A, 1.5, 8), TypeError),
        (lambda: mod.matmul_fft(C, A, A, 1, 8, -1), TypeError),
    ]


def test_dropin_argument_errors(cm):
    for call, exc in _bad_calls(cm):
        with pytest.raises(exc):
            call()


def test_dropin_messages_match_reference(cm):
    """Same exception type and message as the reference binding built from
    its own sources (oracle/_ref), for every invalid call."""
    import sys
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    if not os.path.isdir(ref_dir) or not any(f.startswith("compmatmul") for f in os.listdir(ref_dir)):
        pytest.skip("reference binding not built here")
    sys.path.insert(0, ref_dir)
    try:
        import importlib
        ref = importlib.import_module("compmatmul")
    finally:
        sys.path.remove(ref_dir)
    assert ref.__file__.startswith(ref_dir)
    mine, theirs = _bad_calls(cm), _bad_calls(ref)
    for (c1, _), (c2, _) in zip(mine, theirs):
        with pytest.raises(Exception) as e1:
            c1()
        with pytest.raises(Exception) as e2:
            c2()
        assert type(e1.value) is type(e2.value)
        if isinstance(e1.value, ValueError):
            assert str(e1.value) == str(e2.value)


def test_dropin_signatures(cm):
    doc = cm.matmul_fft.__doc__
    assert "seed" in doc and "hash" in doc
    assert cm.gemm.__doc__.startswith("gemm(C")
