"""Host-pointer entry points stream the rows of AT and B to the device while
the sketch works on earlier chunks of the inner index (a second stream, one
event per chunk, the FFT row scales computed per chunk).

With a small materialization budget the products below run several chunks
through that feed, on every sketch kernel family.  Each launch splits its own chunk into k-groups, so the host path
sums the inner indices in a different grouping than the single launch of
the device entry point: the two agree within 1e-13 * max|p| (FP64) or
1e-7 * max|p| (mixed; bit-identical when both run one launch), and both are
within the usual tolerance of the oracle: FP64 sketch within 1e-11 * max|p|,
mixed within 2e-5 * max|p|.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [("fft", 1 << 16, False), ("fwht", 1 << 16, False), ("fwht", 1 << 17, False), ("fft", 4096, False),
         ("fft", 1 << 16, True), ("fwht", 1 << 16, True), ("fft", 1 << 18, True)]


@pytest.mark.parametrize("variant,b,f32", CASES)
def test_streamed_rows_match_device_path(gpu, oracle, variant, b, f32, monkeypatch):
    import torch

    from compmatmul_b200 import capi, device, lib
    monkeypatch.setenv("CMM_MATERIALIZE_BYTES", str(256 * 1024))
    rng = np.random.default_rng(b + (7 if f32 else 0))
    AT = rng.standard_normal((77, 310))
    B = rng.standard_normal((77, 290)) * 1e-3
    AT[[0, 40, 76]] = 0.0  # skipped rows inside and at the ends of chunks
    dt = np.float32 if f32 else np.float64
    AT, B = AT.astype(dt), B.astype(dt)
    d, seed = 3, 99
    if f32:
        p_host, _ = capi.compressed_product_f32(variant, None, AT, B, d, b, seed)
    else:
        p_host, _ = capi.compressed_product(variant, None, AT, B, d, b, seed)
    kern = lib().cmm_last_sketch_kernel().decode()
    p_dev = device.compressed_product(torch.from_numpy(AT).cuda(), torch.from_numpy(B).cuda(), d, b, seed,
                                      variant).cpu().numpy()
    # FP32 transforms round each grouping's partial sums differently
    agree = 1e-7 if f32 else 1e-13
    np.testing.assert_allclose(p_host, p_dev, rtol=0, atol=agree * float(np.abs(p_dev).max()), err_msg=kern)
    ref = oracle.compressed_product(variant, None, AT.astype(np.float64), B.astype(np.float64), d, b, seed)
    tol = 2e-5 if f32 else 1e-11
    np.testing.assert_allclose(p_host, ref, rtol=0, atol=tol * float(np.abs(ref).max()), err_msg=kern)


def test_streamed_dense_estimate(gpu, monkeypatch):
    """Chunked host rows (several accumulating launches) against the device
    entry point's single launch: the same estimates within 1e-12 relative."""
    import torch

    from compmatmul_b200 import capi, device
    monkeypatch.setenv("CMM_MATERIALIZE_BYTES", str(256 * 1024))
    rng = np.random.default_rng(3)
    AT = rng.standard_normal((64, 120))
    B = rng.standard_normal((64, 100))
    C_host = capi.matmul("fft", None, AT, B, 5, 1 << 16, 17)
    C_dev = device.matmul(torch.from_numpy(AT).cuda(), torch.from_numpy(B).cuda(), 5, 1 << 16, 17, "fft")
    C_dev = C_dev.cpu().numpy()
    np.testing.assert_allclose(C_host, C_dev, rtol=1e-12, atol=1e-13 * float(np.abs(C_dev).max()))


@pytest.mark.parametrize("variant,d,n_a", [("fwht", 17, 130), ("fft", 9, 1), ("fft", 5, 77)])
def test_dense_estimate_row_blocks(gpu, variant, d, n_a):
    """The host entry point decompresses C in row blocks (each copied to the
    host while later blocks are computed); it must equal the device entry
    point's single-launch decompression, for the fixed-d and the generic-d
    kernels and row counts that do not fill the last block.  b = 2^16 runs
    sketch kernels without atomics, so both sketches are bit-identical."""
    import torch

    from compmatmul_b200 import capi, device
    rng = np.random.default_rng(n_a + d)
    AT = rng.standard_normal((30, n_a))
    B = rng.standard_normal((30, 45))
    C_host = capi.matmul(variant, None, AT, B, d, 1 << 16, 5)
    C_dev = device.matmul(torch.from_numpy(AT).cuda(), torch.from_numpy(B).cuda(), d, 1 << 16, 5, variant)
    assert np.array_equal(C_host, C_dev.cpu().numpy())


@pytest.mark.parametrize("variant", ["fft", "fwht"])
def test_pinned_and_pageable_host_buffers_agree(gpu, variant):
    """The host entry point copies page-locked buffers directly and pageable
    ones through its pinned staging slots (several host threads): the same
    chunks, so the same sketch and dense estimate bit for bit.  The product
    is larger than one 64 MB staging slot per matrix, so several slots are
    in flight."""
    import ctypes as C

    import torch

    from compmatmul_b200 import HASH_KINDS, VARIANTS, capi, lib
    rng = np.random.default_rng(23)
    AT = rng.standard_normal((2100, 4096))
    B = rng.standard_normal((2100, 4000))
    d, b, seed = 3, 1 << 15, 5
    C_page = capi.matmul(variant, None, AT, B, d, b, seed)
    hAT, hB = torch.from_numpy(AT).pin_memory(), torch.from_numpy(B).pin_memory()
    hC = torch.empty((4096, 4000), dtype=torch.float64).pin_memory()
    rc = lib().cmm_matmul(VARIANTS[variant], HASH_KINDS[None], 4096, 2100, 4000, C.c_void_p(hC.data_ptr()),
                          C.c_void_p(hAT.data_ptr()), C.c_void_p(hB.data_ptr()), d, b, 1, seed)
    assert rc == 0, lib().cmm_last_error()
    assert np.array_equal(C_page, hC.numpy())
