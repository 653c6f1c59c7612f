"""Batched products over torch CUDA tensors (cmm_batch_* of the C ABI).

A plan fixes a list of independent compressed products of uneven shape,
each with its own variant, hash family, d, b, seed and device buffers, and
runs them all per ``run()``: one persistent sketch launch over a work queue,
captured with the rest of the sequence in a CUDA graph on the first run.
``f32=True`` takes float32 inputs (the mixed-precision kernels); otherwise
inputs are float64.  Outputs are float64: the d x b sketch ``p`` and, when
``dense=True``, the n_a x n_b median estimate ``C``.
"""
from __future__ import annotations

import ctypes as C

from . import HASH_KINDS, VARIANTS, check, lib


class _Prod(C.Structure):
    _fields_ = [("variant", C.c_int), ("hash_kind", C.c_int), ("d", C.c_int), ("b", C.c_int),
                ("n_a", C.c_int64), ("n_inner", C.c_int64), ("n_b", C.c_int64),
                ("seed", C.c_uint64), ("AT", C.c_void_p), ("B", C.c_void_p),
                ("p", C.c_void_p), ("C", C.c_void_p)]


def _ptr(t):
    return t.data_ptr() if t is not None and t.numel() else None


class BatchPlan:
    """products: list of dicts with keys AT, B (contiguous 2-D CUDA tensors,
    AT is n_inner x n_a, B is n_inner x n_b), d, b, seed, and optional
    variant ("fft"/"fwht"), hash (a reference hash string or None).  The
    tensors must stay alive, with the same storage, for the plan's lifetime;
    their contents may change between runs."""

    def __init__(self, products, f32=False, tune=True, dense=True):
        import torch
        self.f32 = bool(f32)
        dt = torch.float32 if f32 else torch.float64
        self.products = []
        arr = (_Prod * max(1, len(products)))()
        for i, q in enumerate(products):
            AT, B = q["AT"], q["B"]
            for name, t in (("AT", AT), ("B", B)):
                if not t.is_cuda or t.dtype != dt or not t.is_contiguous() or t.dim() != 2:
                    raise ValueError(f"product {i}: {name} must be a contiguous 2-D {dt} CUDA tensor")
            if AT.shape[0] != B.shape[0]:
                raise ValueError(f"product {i}: Shape mismatch! Note that AT is assumed to be transposed")
            n_inner, n_a = AT.shape
            n_b = B.shape[1]
            p = torch.empty((q["d"], q["b"]), dtype=torch.float64, device=AT.device)
            Cm = torch.empty((n_a, n_b), dtype=torch.float64, device=AT.device) if dense else None
            self.products.append(dict(q, p=p, C=Cm))
            arr[i] = _Prod(VARIANTS[q.get("variant", "fft")], HASH_KINDS[q.get("hash")], q["d"], q["b"],
                           n_a, n_inner, n_b, q["seed"], _ptr(AT), _ptr(B), _ptr(p), _ptr(Cm))
        self._arr = arr
        h = C.c_void_p()
        check(lib().cmm_batch_create(C.cast(arr, C.c_void_p), len(products), int(self.f32), int(tune),
                                     C.byref(h)))
        self._h = h

    def run(self, stream=None):
        """Enqueue one run of every product on ``stream`` (a torch stream;
        default: the current stream of the first product's device)."""
        import torch
        if stream is None:
            dev = self.products[0]["AT"].device if self.products else torch.device("cuda")
            stream = torch.cuda.current_stream(dev)
        check(lib().cmm_batch_run(self._h, C.c_void_p(stream.cuda_stream)))

    def info(self):
        items, ctas, launches = C.c_int64(), C.c_int(), C.c_int()
        check(lib().cmm_batch_info(self._h, C.byref(items), C.byref(ctas), C.byref(launches)))
        return {"items": items.value, "ctas": ctas.value, "launches": launches.value}

    def config(self, i):
        ls, rx, g, tu = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().cmm_batch_config(self._h, i, C.byref(ls), C.byref(rx), C.byref(g), C.byref(tu)))
        return {"slab": 1 << ls.value, "radix": rx.value, "groups": g.value, "tuned": bool(tu.value)}

    def close(self):
        if getattr(self, "_h", None):
            check(lib().cmm_batch_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
