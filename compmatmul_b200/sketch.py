"""Device-resident sketch object: the compressed product kept on the GPU
and queried without the dense n_a x n_b estimate (the reference's
matmul_sketch + matmul_decompress_*, matmul_sketch.hpp / matmul_fft.hpp:135-147,
matmul_fwht.hpp:122-134, on the device).

    s = Sketch.compute(AT, B, d=9, b=1 << 16, seed=7, variant="fft")
    i, j, v = s.topk(256)            # recovered entries, no dense matrix
    vals = s.entries(i, j)           # median estimates of listed entries
    C = s.dense()                    # the full estimate, when wanted
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import HASH_KINDS, VARIANTS, check, lib
from . import device as _dev


class Sketch:
    def __init__(self, p, n_a, n_b, d, b, seed, variant="fft", hash=None):
        self.p, self.n_a, self.n_b, self.d, self.b = p, int(n_a), int(n_b), int(d), int(b)
        self.seed, self.variant, self.hash = int(seed), variant, hash

    @classmethod
    def compute(cls, AT, B, d, b, seed, variant="fft", hash=None):
        """The sketch of AT^T B on the inputs' device (float32 inputs take the
        mixed-precision path; the sketch is float64 either way)."""
        p = _dev.compressed_product(AT, B, d, b, seed, variant, hash)
        return cls(p, AT.shape[1], B.shape[1], d, b, seed, variant, hash)

    def _stream(self):
        import torch
        return C.c_void_p(torch.cuda.current_stream(self.p.device).cuda_stream)

    def entries(self, i, j):
        """Median estimates at (i[e], j[e]) as a float64 numpy array."""
        import torch
        ti = torch.as_tensor(np.asarray(i, dtype=np.uint32).astype(np.int32), device=self.p.device)
        tj = torch.as_tensor(np.asarray(j, dtype=np.uint32).astype(np.int32), device=self.p.device)
        out = torch.empty(ti.numel(), dtype=torch.float64, device=self.p.device)
        check(lib().cmm_dev_decompress_entries(VARIANTS[self.variant], HASH_KINDS[self.hash], self.d, self.b,
                                               self.seed, C.c_void_p(self.p.data_ptr()), ti.numel(),
                                               C.c_void_p(ti.data_ptr()), C.c_void_p(tj.data_ptr()),
                                               C.c_void_p(out.data_ptr()), self._stream()))
        return out.cpu().numpy()

    def topk(self, K, scratch_bytes=0):
        """Top-K estimates (value descending, ties by (i, j)) as numpy
        (i, j, v), decompressing row tiles of at most scratch_bytes."""
        import torch
        oi = torch.empty(K, dtype=torch.int32, device=self.p.device)
        oj = torch.empty(K, dtype=torch.int32, device=self.p.device)
        ov = torch.empty(K, dtype=torch.float64, device=self.p.device)
        check(lib().cmm_dev_sketch_topk(VARIANTS[self.variant], HASH_KINDS[self.hash], self.n_a, self.n_b, self.d,
                                        self.b, self.seed, C.c_void_p(self.p.data_ptr()), K, int(scratch_bytes),
                                        C.c_void_p(oi.data_ptr()), C.c_void_p(oj.data_ptr()),
                                        C.c_void_p(ov.data_ptr()), self._stream()))
        return (oi.cpu().numpy().astype(np.int64), oj.cpu().numpy().astype(np.int64), ov.cpu().numpy())

    def dense(self, out=None):
        return _dev.decompress_dense(self.p, self.n_a, self.n_b, self.d, self.b, self.seed, self.variant,
                                     self.hash, out=out)
