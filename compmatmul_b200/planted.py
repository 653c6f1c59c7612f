"""Synthetic planted-entry problems for the compressed product.

A = noise + planted, B = noise + planted, with noise i.i.d. N(0, sigma^2)
and K planted triples (i_t, k_t, j_t): A[i_t, k_t] += big and
B[k_t, j_t] += big, so (A B)[i_t, j_t] ~ big^2.  The k_t are drawn without
replacement (and so are the i_t and the j_t), so no two triples share an
inner index and the planted entries do not create extra large products.
Matrices are returned in the reference's layout: AT (n_inner x n_a, row k
= column k of A) and B (n_inner x n_b), both 64-byte aligned as the
reference binding requires (compmatmul.cpp:65-73).

The named workloads follow the benchmark configurations of this project:
  config1   n=512,   K=32,   FFT,  b=4096,  d=5   (CPU-runnable case)
  config2   n=4096 / 16384, K=256, b=2^16, d=9, FFT and FWHT, FP64
  config3   n=16384, K=1024, b=2^18, d=9, FP32 inputs (mixed precision)
"""
from __future__ import annotations

import numpy as np

WORKLOADS = {
    "config1": dict(n=512, K=32, b=4096, d=5, variants=("fft",), gen_seed=51201, seed=9001),
    "config2_n4096": dict(n=4096, K=256, b=1 << 16, d=9, variants=("fft", "fwht"), gen_seed=409601,
                          seed=9002),
    "config2_n16384": dict(n=16384, K=256, b=1 << 16, d=9, variants=("fft", "fwht"),
                           gen_seed=1638401, seed=9003),
    "config3": dict(n=16384, K=1024, b=1 << 18, d=9, variants=("fft", "fwht"), gen_seed=1638403,
                    seed=9004, dtype="float32"),
}


def aligned_empty(shape, dtype=np.float64, alignment=64):
    elem = np.dtype(dtype).itemsize
    nbytes = int(np.prod(shape)) * elem
    raw = np.empty(nbytes + alignment, np.uint8)
    off = (alignment - raw.ctypes.data % alignment) % alignment
    return raw[off:off + nbytes].view(dtype).reshape(shape)


def planted_problem(n_a, n_inner, n_b, K, gen_seed, sigma=0.01, big=10.0, dtype=np.float64):
    """(AT, B, planted) with planted = (i, k, j) index arrays of length K."""
    if K > min(n_a, n_inner, n_b):
        raise ValueError("K must not exceed any matrix dimension")
    rng = np.random.default_rng(gen_seed)
    AT = aligned_empty((n_inner, n_a), np.float64)
    B = aligned_empty((n_inner, n_b), np.float64)
    rng.standard_normal(out=AT)
    rng.standard_normal(out=B)
    AT *= sigma
    B *= sigma
    ks = rng.choice(n_inner, size=K, replace=False)
    is_ = rng.choice(n_a, size=K, replace=False)
    js = rng.choice(n_b, size=K, replace=False)
    AT[ks, is_] += big
    B[ks, js] += big
    if dtype != np.float64:
        AT2 = aligned_empty(AT.shape, dtype)
        B2 = aligned_empty(B.shape, dtype)
        AT2[...] = AT
        B2[...] = B
        AT, B = AT2, B2
    return AT, B, (is_, ks, js)


def topk_dense_host(C, K):
    """Top-K of a dense array by value descending, ties by (i, j) ascending.
    Returns (i, j, v) arrays.  Host helper for fixtures and tests."""
    flat = C.ravel()
    K = min(K, flat.size)
    cand = np.argpartition(-flat, K - 1)[:K]
    kth = flat[cand].min()
    # include every tie of the K-th value, then order deterministically
    cand = np.nonzero(flat >= kth)[0]
    order = np.lexsort((cand, -flat[cand]))
    sel = cand[order][:K]
    n_b = C.shape[1]
    return sel // n_b, sel % n_b, flat[sel]


def batch_shapes(count=256, seed=4004, lo=256, hi=4096):
    """Shapes of the batched-products workload (config 4): m, n, p each
    log-uniform in [lo, hi] (m = rows of C, n = inner, p = columns of C),
    K = max(8, m // 64) planted entries, b = the next power of two >= 4 K 64,
    d uniform in {5, 7, 9}, FFT or FWHT with probability 1/2 each."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m, n, p = (int(round(float(np.exp(rng.uniform(np.log(lo), np.log(hi)))))) for _ in range(3))
        K = max(8, m // 64)
        K = min(K, m, n, p)
        b = 1 << int(np.ceil(np.log2(4 * K * 64)))
        d = int(rng.choice([5, 7, 9]))
        variant = "fft" if rng.random() < 0.5 else "fwht"
        out.append(dict(m=m, n=n, p=p, K=K, b=b, d=d, variant=variant, gen_seed=seed * 1000 + i,
                        seed=seed + 17 * i))
    return out


def planted_problem_device(n_a, n_inner, n_b, K, gen_seed, dtype="float32", device="cuda",
                           sigma=0.01, big=10.0):
    """The planted generator of planted_problem with the noise drawn on the
    device (torch generator seeded with gen_seed) and the planted triples
    drawn on the host (numpy, gen_seed): returns (AT, B, (i, k, j))."""
    import torch
    dt = torch.float32 if dtype == "float32" else torch.float64
    g = torch.Generator(device=device).manual_seed(int(gen_seed))
    AT = torch.randn((n_inner, n_a), generator=g, device=device, dtype=dt) * sigma
    B = torch.randn((n_inner, n_b), generator=g, device=device, dtype=dt) * sigma
    rng = np.random.default_rng(gen_seed)
    K = min(K, n_a, n_inner, n_b)
    ks = rng.choice(n_inner, size=K, replace=False)
    is_ = rng.choice(n_a, size=K, replace=False)
    js = rng.choice(n_b, size=K, replace=False)
    kt = torch.as_tensor(ks, device=device)
    AT[kt, torch.as_tensor(is_, device=device)] += big
    B[kt, torch.as_tensor(js, device=device)] += big
    return AT, B, (is_, ks, js)
