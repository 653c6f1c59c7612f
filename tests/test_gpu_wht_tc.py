"""Batched FP32 Walsh-Hadamard transform of rows (cmm_dev_wht_rows_f32):
the tensor-core form (Hadamard-16 stages as tcgen05 MMAs on BF16
hi/mid/lo splits, FP32 accumulators in tensor memory) and the CUDA-core
form, through the C ABI.

Pins: the reference's 32-point golden transform (tests.cpp:621-671) placed
on three bit ranges of a length-8192 row, so that every stage of the
kernel meets it; random rows against the FP64 oracle (oracle/cmm_oracle.c
cmo_fwht, natural order as transform.hpp:94-144) on the same FP32 inputs.

Tolerances: golden 1e-5 absolute (the golden values carry 8 digits and the
transform runs in FP32); random rows within 2e-6 * max|ref| (FP32
arithmetic over 13 add/sub stages; the two forms differ by 2.4e-7 of
max|y| on B200)."""
import numpy as np
import pytest

from golden.ref_vectors import FWHT_X, FWHT_XHAT

pytestmark = pytest.mark.gpu

METHODS = ["tensor", "cuda"]


def wht(x, method, out=None):
    from compmatmul_b200 import device
    return device.wht_rows(x, method, out=out)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("shift", [0, 4, 8])
def test_golden_on_every_stage(gpu, method, shift):
    """x[e] = u[e >> shift] on the multiples of 2^shift below 32 * 2^shift:
    H x repeats the 32-point golden U on every index whose bits [shift,
    shift + 5) give its position."""
    import torch
    L = 8192
    x = np.zeros(L, np.float32)
    x[(np.arange(32) << shift)] = FWHT_X.astype(np.float32)
    y = wht(torch.from_numpy(x[None, :].copy()).cuda(), method).cpu().numpy()[0]
    expect = FWHT_XHAT[(np.arange(L) >> shift) & 31]
    np.testing.assert_allclose(y, expect, rtol=0, atol=1e-5)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("log2n", [11, 12, 13])
def test_random_rows_vs_oracle(gpu, oracle, method, log2n):
    import torch
    rng = np.random.default_rng(100 + log2n)
    rows = 37
    x = rng.standard_normal((rows, 1 << log2n)).astype(np.float32)
    x[3] *= 1e-20  # tiny and huge rows: the BF16 split is relative to each value
    x[5] *= 1e20
    y = wht(torch.from_numpy(x).cuda(), method).cpu().numpy()
    for r in range(rows):
        ref = oracle.fwht(x[r].astype(np.float64))
        err = np.abs(y[r] - ref).max()
        assert err <= 2e-6 * np.abs(ref).max(), (r, err, np.abs(ref).max())


def test_tensor_cores_match_cuda_cores_in_place(gpu):
    """Both forms on the same rows, the tensor-core one in place (x == y),
    many rows (every CTA of the persistent grid takes several)."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randn((4096, 8192), device="cuda", generator=g, dtype=torch.float32)
    ref = wht(x, "cuda")
    y = x.clone()
    wht(y, "tensor", out=y)
    scale = ref.abs().max().item()
    assert (y - ref).abs().max().item() <= 2e-6 * scale
    # a second call on the same buffers gives the same result again
    y2 = wht(x, "tensor")
    assert torch.equal(y2, y)
