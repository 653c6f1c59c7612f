"""Mixed-precision path (FP32 inputs, FP32 transforms with compensated
accumulation, tensor-core Hadamard stages for the FWHT, FP64 reduction and
inverse) against the FP64 oracle on the same FP32-valued inputs.

Tolerances: sketch p within 2e-5 * max|p| (FP32 transforms); recovered
(top-K) values within 1e-5 relative of the FP64 oracle and the same
recovered (i, j) sets."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def capi():
    from compmatmul_b200 import capi as c
    return c


@pytest.mark.parametrize("variant", ["fft", "fwht"])
@pytest.mark.parametrize("b", [1024, 8192, 1 << 16, 1 << 18])
@pytest.mark.parametrize("h", [None, "multiply shift", "tabulation8", "tabulation16"])
def test_mixed_sketch_vs_oracle(gpu, oracle, variant, b, h):
    rng = np.random.default_rng(b + (0 if variant == "fft" else 1))
    AT = rng.standard_normal((50, 37)).astype(np.float32)
    B = (rng.standard_normal((50, 41)) * 1e-3).astype(np.float32)
    p, _ = capi().compressed_product_f32(variant, h, AT, B, 3, b, 99)
    ref = oracle.compressed_product(variant, h, AT.astype(np.float64), B.astype(np.float64), 3, b, 99)
    np.testing.assert_allclose(p, ref, rtol=0, atol=2e-5 * np.abs(ref).max())


@pytest.mark.parametrize("variant", ["fft", "fwht"])
def test_mixed_recovery_planted(gpu, oracle, variant):
    """Same recovered set as FP64; max relative error of recovered values <= 1e-5."""
    import torch
    from compmatmul_b200 import device
    from compmatmul_b200.planted import planted_problem, topk_dense_host
    n, K, d, b, seed = 768, 16, 7, 1 << 16, 4242
    AT, B, planted = planted_problem(n, n, n, K, 2024, dtype=np.float32)
    AT64, B64 = AT.astype(np.float64), B.astype(np.float64)
    C32 = device.matmul(torch.from_numpy(AT).cuda(), torch.from_numpy(B).cuda(), d, b, seed,
                        variant=variant).cpu().numpy()
    p = oracle.compressed_product(variant, None, AT64, B64, d, b, seed)
    C64 = oracle.decompress(variant, None, p, d, b, seed, n, n)
    i32, j32, v32 = topk_dense_host(C32, K)
    i64, j64, v64 = topk_dense_host(C64, K)
    assert set(zip(i32, j32)) == set(zip(i64, j64))
    assert set(zip(i64, j64)) == set(zip(planted[0], planted[2]))
    rel = np.abs(C32[i64, j64] - v64) / np.abs(v64)
    assert rel.max() <= 1e-5, rel.max()


def test_mixed_small_b_falls_back_to_fp64_kernels(gpu, oracle):
    rng = np.random.default_rng(5)
    AT = rng.integers(-9, 10, (20, 10)).astype(np.float32)
    B = rng.integers(-9, 10, (20, 12)).astype(np.float32)
    p, _ = capi().compressed_product_f32("fwht", None, AT, B, 3, 256, 1)
    ref = oracle.compressed_product("fwht", None, AT.astype(np.float64), B.astype(np.float64), 3, 256, 1)
    assert np.array_equal(p, ref)
