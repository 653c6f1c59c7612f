"""Allocation-free compressed product, cmm_dev_compressed_product_noalloc.

This file is named to be collected last, so that the entry point is also
exercised after every other test has used the allocating paths.  Each GPU
case calls the entry twice in a row through the C ABI and compares both
results with cmm_dev_compressed_product (the allocating entry point) on the
same device inputs, and the second result with the CPU oracle.  Tolerance:
1e-11 * max|p| absolute, as for the sketch parity tests (the entries may sum
the k groups in a different order).
The CPU test checks the size limit, which is enforced before any CUDA call.
"""
import ctypes as C

import numpy as np
import pytest

from compmatmul_b200 import HASH_KINDS, VARIANTS, lib

CMM_ERR_UNSUPPORTED = 5
SCRATCH = 32 << 20


def p_tol(p_ref):
    return 1e-11 * max(float(np.abs(p_ref).max()), 1e-300)


def test_noalloc_rejects_oversize():
    L = lib()
    # FFT, d = 9, b = 2^20: partials + inverse work alone need 3 * 9 * 2^20 * 16 bytes
    rc = L.cmm_dev_compressed_product_noalloc(VARIANTS["fft"], HASH_KINDS["multiply shift"], 64, 8,
                                              64, None, None, 9, 1 << 20, 1, None, None)
    assert rc == CMM_ERR_UNSUPPORTED
    msg = L.cmm_last_error().decode()
    assert "bytes of scratch" in msg and str(SCRATCH) in msg
    # tabulation16 parameters alone exceed the scratch for d = 17
    rc = L.cmm_dev_compressed_product_noalloc(VARIANTS["fwht"], HASH_KINDS["tabulation16"], 64, 8,
                                              64, None, None, 17, 1024, 1, None, None)
    assert rc == CMM_ERR_UNSUPPORTED
    # argument errors keep the reference's messages
    rc = L.cmm_dev_compressed_product_noalloc(0, 0, 64, 8, 64, None, None, 5, 1000, 1, None, None)
    assert rc == 1 and "b must be power of 2 greater than 1" in L.cmm_last_error().decode()


# (variant, hash, n_a, n_inner, n_b, d, b, seed); b = 2^15, d = 9 FFT fills
# the scratch so that fewer k groups fit than the allocating path uses
CASES = [
    ("fft", "multiply shift", 300, 200, 250, 5, 1024, 11),
    ("fwht", "multiply add shift", 300, 200, 250, 7, 2048, 12),
    ("fft", "tabulation8", 257, 333, 129, 9, 4096, 13),
    ("fwht", "tabulation16", 200, 64, 300, 3, 8192, 14),
    ("fft", "multiply add shift", 512, 256, 512, 9, 1 << 15, 15),
    ("fwht", "multiply shift", 512, 256, 512, 9, 1 << 16, 16),
    ("fft", "multiply shift", 100, 0, 90, 5, 512, 17),
]


@pytest.mark.gpu
@pytest.mark.parametrize("variant,h,n_a,n_inner,n_b,d,b,seed", CASES)
def test_noalloc_matches_allocating_entry(gpu, oracle, variant, h, n_a, n_inner, n_b, d, b, seed):
    import torch
    L = gpu
    dev = torch.device("cuda:0")
    g = torch.Generator(device="cpu").manual_seed(seed)
    AT = torch.randn((n_inner, n_a), generator=g, dtype=torch.float64).to(dev)
    B = torch.randn((n_inner, n_b), generator=g, dtype=torch.float64).to(dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t.numel() else C.c_void_p(0)
    args = (VARIANTS[variant], HASH_KINDS[h], n_a, n_inner, n_b, ptr(AT), ptr(B), d, b, seed)

    p_ref = torch.empty((d, b), dtype=torch.float64, device=dev)
    assert L.cmm_dev_compressed_product(*args, ptr(p_ref), stream) == 0, L.cmm_last_error()
    torch.cuda.synchronize()
    ref = p_ref.cpu().numpy()
    for call in range(2):
        p = torch.full((d, b), float("nan"), dtype=torch.float64, device=dev)
        rc = L.cmm_dev_compressed_product_noalloc(*args, ptr(p), stream)
        assert rc == 0, L.cmm_last_error().decode()
        torch.cuda.synchronize()
        np.testing.assert_allclose(p.cpu().numpy(), ref, rtol=0, atol=p_tol(ref),
                                   err_msg=f"call {call + 1}")
    # and directly against the CPU oracle on the same inputs
    want = oracle.compressed_product(variant, h, AT.cpu().numpy(), B.cpu().numpy(), d, b, seed)
    np.testing.assert_allclose(p.cpu().numpy(), want, rtol=0, atol=p_tol(want))
