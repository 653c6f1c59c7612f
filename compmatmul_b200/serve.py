"""Serving engine (cmm_server_* of the C ABI): continuous batching of
independent compressed products under a device-memory admission cap.

    srv = Server(mem_cap_bytes=40 << 30, f32=True, streams=4, max_wave=32, cache_bytes=4 << 30)
    rid = srv.submit(AT, B, d, b, seed, variant="fft")   # returns at once
    p = srv.result(rid)                                    # waits; d x b float64
    srv.close()

AT and B are 2-D contiguous arrays of the server's precision (float32 when
f32, else float64): numpy arrays (host; pinned torch CPU tensors copy
asynchronously) or torch CUDA tensors (used in place).  They and the output
stay referenced here until the request completes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import HASH_KINDS, VARIANTS, check, lib


class _Config(C.Structure):
    _fields_ = [("mem_cap_bytes", C.c_size_t), ("f32", C.c_int), ("streams", C.c_int), ("max_wave", C.c_int),
                ("cache_bytes", C.c_size_t)]


class _Request(C.Structure):
    _fields_ = [("variant", C.c_int), ("hash_kind", C.c_int), ("d", C.c_int), ("b", C.c_int),
                ("n_a", C.c_int64), ("n_inner", C.c_int64), ("n_b", C.c_int64), ("seed", C.c_uint64),
                ("AT", C.c_void_p), ("B", C.c_void_p), ("inputs_on_device", C.c_int), ("p", C.c_void_p)]


class _Stats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("queued", C.c_int64),
                ("in_flight", C.c_int64), ("waves", C.c_int64), ("max_waves_in_flight", C.c_int64),
                ("mem_in_use", C.c_size_t), ("max_mem_in_use", C.c_size_t), ("cache_hits", C.c_int64),
                ("cache_misses", C.c_int64), ("cache_in_use", C.c_size_t)]


def _info(x, dtype):
    """(pointer, shape, on_device) of a 2-D array or tensor."""
    if hasattr(x, "data_ptr"):  # torch tensor
        import torch
        want = torch.float32 if dtype == np.float32 else torch.float64
        if x.dtype != want or not x.is_contiguous() or x.dim() != 2:
            raise ValueError(f"inputs must be contiguous 2-D {want} tensors")
        return (x.data_ptr() if x.numel() else None), tuple(x.shape), bool(x.is_cuda)
    a = np.asarray(x)
    if a.dtype != dtype or not a.flags.c_contiguous or a.ndim != 2:
        raise ValueError(f"inputs must be C-contiguous 2-D {np.dtype(dtype).name} arrays")
    return (a.ctypes.data if a.size else None), a.shape, False


class Server:
    def __init__(self, mem_cap_bytes=40 << 30, f32=True, streams=4, max_wave=32, cache_bytes=0):
        self.f32 = bool(f32)
        self._dtype = np.float32 if f32 else np.float64
        cfg = _Config(int(mem_cap_bytes), int(self.f32), int(streams), int(max_wave), int(cache_bytes))
        h = C.c_void_p()
        check(lib().cmm_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._live = {}

    def submit(self, AT, B, d, b, seed, variant="fft", hash=None):
        pa, sa, da = _info(AT, self._dtype)
        pb, sb, db = _info(B, self._dtype)
        if da != db:
            raise ValueError("AT and B must both be on the device or both on the host")
        if sa[0] != sb[0]:
            raise ValueError("Shape mismatch! Note that AT is assumed to be transposed")
        p = np.empty((d, b), dtype=np.float64)
        req = _Request(VARIANTS[variant], HASH_KINDS[hash], d, b, sa[1], sa[0], sb[1], seed, pa, pb, int(da),
                       p.ctypes.data)
        rid = C.c_uint64()
        check(lib().cmm_server_submit(self._h, C.byref(req), C.byref(rid)))
        self._live[rid.value] = (AT, B, p)
        return rid.value

    def wait(self, rid, timeout=None):
        """(done, latency seconds); timeout None waits without limit."""
        done, lat = C.c_int(), C.c_double()
        check(lib().cmm_server_wait(self._h, rid, -1.0 if timeout is None else float(timeout), C.byref(done),
                                    C.byref(lat)))
        return bool(done.value), lat.value

    def result(self, rid, timeout=None):
        done, _ = self.wait(rid, timeout)
        if not done:
            raise TimeoutError(f"request {rid} not done")
        return self._live.pop(rid)[2]

    def latency(self, rid):
        done, lat = self.wait(rid, 0.0)
        return lat if done else None

    def stats(self):
        s = _Stats()
        check(lib().cmm_server_stats_get(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in _Stats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            h, self._h = self._h, None
            check(lib().cmm_server_destroy(h))
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
