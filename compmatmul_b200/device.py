"""Device-resident API over torch CUDA tensors.

For callers that keep A and B in HBM: the compressed product, dense
decompression and top-K recovery run on the tensors' device and the
current torch stream, with no host round trip (top-K reads back its
candidate count and synchronises).  torch supplies device memory and
streams only; every kernel is this package's own (libcmm_b200.so).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import HASH_KINDS, VARIANTS, check, lib


def _stream(t):
    import torch
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t.numel() else C.c_void_p(0)


def _f64_contig(t, name):
    import torch
    if not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous() or t.dim() != 2:
        raise ValueError(f"{name} must be a contiguous 2-D float64 CUDA tensor")


def _in_contig(t, name):
    """float64 (plain path) or float32 (mixed-precision path) inputs."""
    import torch
    if not t.is_cuda or t.dtype not in (torch.float64, torch.float32) or not t.is_contiguous() \
            or t.dim() != 2:
        raise ValueError(f"{name} must be a contiguous 2-D float64/float32 CUDA tensor")


def compressed_product(AT, B, d, b, seed, variant="fft", hash=None, out=None):
    """Sketch p (d x b float64 CUDA tensor) of AT^T-layout inputs.  float32
    inputs take the mixed-precision path."""
    import torch
    _in_contig(AT, "AT")
    _in_contig(B, "B")
    if AT.dtype != B.dtype:
        raise ValueError("AT and B must have the same dtype")
    q, n_a = AT.shape
    n_b = B.shape[1]
    if B.shape[0] != q:
        raise ValueError("Shape mismatch! Note that AT is assumed to be transposed")
    p = out if out is not None else torch.empty((d, b), dtype=torch.float64, device=AT.device)
    fn = lib().cmm_dev_compressed_product if AT.dtype == torch.float64 else \
        lib().cmm_dev_compressed_product_f32
    check(fn(VARIANTS[variant], HASH_KINDS[hash], n_a, q, n_b, _ptr(AT), _ptr(B), d, b, seed,
             _ptr(p), _stream(AT)))
    return p


def decompress_dense(p, n_a, n_b, d, b, seed, variant="fft", hash=None, out=None):
    import torch
    Cm = out if out is not None else torch.empty((n_a, n_b), dtype=torch.float64, device=p.device)
    check(lib().cmm_dev_decompress_dense(VARIANTS[variant], HASH_KINDS[hash], n_a, n_b, d, b, seed,
                                         _ptr(p), _ptr(Cm), _stream(p)))
    return Cm


def matmul(AT, B, d, b, seed, variant="fft", hash=None, out=None):
    """Dense estimate C (n_a x n_b, float64) = matmul_{fft,fwht} on the
    device.  float32 inputs take the mixed-precision path."""
    import torch
    _in_contig(AT, "AT")
    _in_contig(B, "B")
    if AT.dtype != B.dtype:
        raise ValueError("AT and B must have the same dtype")
    q, n_a = AT.shape
    n_b = B.shape[1]
    if B.shape[0] != q:
        raise ValueError("Shape mismatch! Note that AT is assumed to be transposed")
    Cm = out if out is not None else torch.empty((n_a, n_b), dtype=torch.float64, device=AT.device)
    fn = lib().cmm_dev_matmul if AT.dtype == torch.float64 else lib().cmm_dev_matmul_f32
    check(fn(VARIANTS[variant], HASH_KINDS[hash], n_a, q, n_b, _ptr(Cm), _ptr(AT), _ptr(B), d, b,
             seed, _stream(AT)))
    return Cm


def topk(Cm, K, as_numpy=True):
    """Top-K entries of a dense float64 CUDA matrix: value descending, ties
    by (i, j) ascending.  Returns (i, j, v)."""
    import torch
    _f64_contig(Cm, "C")
    n_a, n_b = Cm.shape
    oi = torch.empty(K, dtype=torch.int32, device=Cm.device)
    oj = torch.empty(K, dtype=torch.int32, device=Cm.device)
    ov = torch.empty(K, dtype=torch.float64, device=Cm.device)
    check(lib().cmm_dev_topk(_ptr(Cm), n_a, n_b, K, _ptr(oi), _ptr(oj), _ptr(ov), _stream(Cm)))
    if not as_numpy:
        return oi, oj, ov
    return (oi.cpu().numpy().astype(np.int64), oj.cpu().numpy().astype(np.int64),
            ov.cpu().numpy())


def gemm(AT, B, out=None):
    import torch
    _f64_contig(AT, "AT")
    _f64_contig(B, "B")
    q, n_a = AT.shape
    n_b = B.shape[1]
    Cm = out if out is not None else torch.empty((n_a, n_b), dtype=torch.float64, device=AT.device)
    check(lib().cmm_dev_gemm(n_a, q, n_b, _ptr(Cm), _ptr(AT), _ptr(B), _stream(AT)))
    return Cm


WHT_METHODS = {"cuda": 0, "tensor": 1}


def wht_rows(x, method="tensor", out=None):
    """Forward natural-order Walsh-Hadamard transform of every row of a
    contiguous 2-D float32 CUDA tensor (rows of 2^11, 2^12 or 2^13), the
    reference's fwht_transformer::forward (transform.hpp:94-144) on FP32.
    method "tensor": the Hadamard-16 stages as tcgen05 MMAs on BF16
    hi/mid/lo splits; "cuda": every stage on CUDA cores.  out may be x
    (in place).  Returns once the rows are transformed."""
    import torch
    if not x.is_cuda or x.dtype != torch.float32 or not x.is_contiguous() or x.dim() != 2:
        raise ValueError("x must be a contiguous 2-D float32 CUDA tensor")
    rows, n = x.shape
    log2n = n.bit_length() - 1
    if n != 1 << log2n:
        raise ValueError("the row length must be a power of two")
    y = out if out is not None else torch.empty_like(x)
    if y.shape != x.shape or y.dtype != x.dtype or not y.is_contiguous():
        raise ValueError("out must match x")
    check(lib().cmm_dev_wht_rows_f32(_ptr(x), _ptr(y), rows, log2n, WHT_METHODS[method], _stream(x)))
    return y
