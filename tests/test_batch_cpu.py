"""Batched-products C ABI on the CPU: argument errors are reported before
any CUDA call, with the product index and the reference's message."""
import ctypes as C

from compmatmul_b200 import lib
from compmatmul_b200.batch import _Prod


def _create(prods):
    arr = (_Prod * len(prods))(*prods)
    h = C.c_void_p()
    rc = lib().cmm_batch_create(C.cast(arr, C.c_void_p), len(prods), 0, 0, C.byref(h))
    return rc, lib().cmm_last_error().decode(), h


def _ok(**kw):
    q = dict(variant=0, hash_kind=1, d=3, b=256, n_a=8, n_inner=4, n_b=8, seed=1, AT=16, B=16, p=16, C=None)
    q.update(kw)
    return _Prod(**q)


def test_batch_rejects_bad_b():
    rc, msg, h = _create([_ok(), _ok(b=1000)])
    assert rc == 1 and "product 1: b must be power of 2 greater than 1 (got 1000)" in msg
    assert h.value is None


def test_batch_rejects_bad_d_hash_and_null_buffers():
    rc, msg, _ = _create([_ok(d=0)])
    assert rc == 1 and "product 0: d must be positive" in msg
    rc, msg, _ = _create([_ok(), _ok(), _ok(hash_kind=7)])
    assert rc == 1 and "product 2: Invalid hash provided" in msg
    rc, msg, _ = _create([_ok(p=None)])
    assert rc == 1 and "p is null" in msg
    rc, msg, _ = _create([_ok(AT=None)])
    assert rc == 1 and "AT is null" in msg


def test_batch_rejects_too_large_b():
    rc, msg, _ = _create([_ok(b=1 << 25)])
    assert rc == 5 and "2^24" in msg


def test_batch_null_handle_calls():
    L = lib()
    assert L.cmm_batch_run(None, None) == 1
    assert "null" in L.cmm_last_error().decode()
    assert L.cmm_batch_destroy(None) == 0


def test_server_null_handle_calls():
    L = lib()
    rid = C.c_uint64()
    assert L.cmm_server_submit(None, None, C.byref(rid)) == 1
    assert "null" in L.cmm_last_error().decode()
    assert L.cmm_server_destroy(None) == 0
