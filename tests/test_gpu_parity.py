"""GPU parity: the CUDA path (through the C ABI and the drop-in module)
against the CPU oracle and the reference-generated golden fixtures.

Tolerances: integer/byte/index results (hash codes, buckets, signs,
recovered index sets, FWHT on integer inputs) are compared for equality.
Floating point: sketch p within 1e-11 * max|p| absolute (FP64 FFTs of
different radix/order), recovered values within 1e-10 relative.
"""
import os

import numpy as np
import pytest

from conftest import aligned_alloc, as_aligned
from golden import ref_vectors as G

pytestmark = pytest.mark.gpu

HASHES = [None, "multiply shift", "multiply add shift", "tabulation8", "tabulation16"]
KIND = {None: 1, "multiply shift": 0, "multiply add shift": 1, "tabulation8": 2, "tabulation16": 3}
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def capi():
    from compmatmul_b200 import capi as c
    return c


def p_tol(p_ref):
    return 1e-11 * max(float(np.abs(p_ref).max()), 1e-300)


# ------------------------------------------------------------- hash codes
@pytest.mark.parametrize("h", ["multiply shift", "multiply add shift", "tabulation8", "tabulation16"])
@pytest.mark.parametrize("b", [2, 32, 4096, 1 << 16, 1 << 24])
def test_hash_codes_bit_exact(gpu, oracle, h, b):
    d, seed = 3, 987654321
    n = 70000 if h == "tabulation16" else 5000
    for side in (0, 1):
        got = capi().hash_codes(h, d, b, seed, side, n)
        ref = oracle.sketch_codes(KIND[h], d, b, seed, side, n)
        assert np.array_equal(got, ref)


# ---------------------------------------------------- compressed product
SHAPES = [(7, 5, 6), (40, 24, 31), (1, 1, 1), (33, 17, 9), (300, 129, 77)]


@pytest.mark.parametrize("variant", ["fft", "fwht"])
@pytest.mark.parametrize("h", HASHES)
@pytest.mark.parametrize("d,b", [(1, 2), (3, 8), (5, 64), (2, 4096), (3, 8192), (4, 1 << 16)])
def test_sketch_vs_oracle(gpu, oracle, variant, h, d, b):
    rng = np.random.default_rng(abs(hash((variant, h, d, b))) % (1 << 32))
    for q, n_a, n_b in SHAPES[:3] if b >= 8192 else SHAPES:
        AT = rng.standard_normal((q, n_a))
        B = rng.standard_normal((q, n_b))
        seed = int(rng.integers(0, 1 << 62))
        p_gpu, used = capi().compressed_product(variant, h, AT, B, d, b, seed)
        assert used == seed
        p_ref = oracle.compressed_product(variant, h, AT, B, d, b, seed)
        np.testing.assert_allclose(p_gpu, p_ref, rtol=0, atol=p_tol(p_ref))


@pytest.mark.parametrize("h", HASHES)
@pytest.mark.parametrize("b", [32, 1024, 1 << 16])
def test_fwht_integer_inputs_exact(gpu, oracle, h, b):
    rng = np.random.default_rng(b)
    AT = rng.integers(-9, 10, (50, 20)).astype(np.float64)
    B = rng.integers(-9, 10, (50, 23)).astype(np.float64)
    p_gpu, _ = capi().compressed_product("fwht", h, AT, B, 3, b, 31337)
    p_ref = oracle.compressed_product("fwht", h, AT, B, 3, b, 31337)
    assert np.array_equal(p_gpu, p_ref)


@pytest.mark.parametrize("variant", ["fft", "fwht"])
def test_large_b_multi_slab(gpu, oracle, variant):
    # b = 2^18: FFT runs 64 slabs of 4096, FWHT 32 slabs of 8192
    rng = np.random.default_rng(18)
    AT = rng.standard_normal((6, 40))
    B = rng.standard_normal((6, 50))
    p_gpu, _ = capi().compressed_product(variant, None, AT, B, 2, 1 << 18, 5)
    p_ref = oracle.compressed_product(variant, None, AT, B, 2, 1 << 18, 5)
    np.testing.assert_allclose(p_gpu, p_ref, rtol=0, atol=p_tol(p_ref))


def test_fft_unbalanced_row_scales(gpu, oracle):
    # A rows ~1e6, B rows ~1e-6: the per-k power-of-two balancing keeps the
    # (Z^2 - conj Z(-f)^2)/4i combination exact to FP64 rounding
    rng = np.random.default_rng(3)
    AT = rng.standard_normal((30, 40)) * 1e6
    B = rng.standard_normal((30, 35)) * 1e-6
    AT[3] *= 1e8
    p_gpu, _ = capi().compressed_product("fft", None, AT, B, 3, 1024, 11)
    p_ref = oracle.compressed_product("fft", None, AT, B, 3, 1024, 11)
    np.testing.assert_allclose(p_gpu, p_ref, rtol=0, atol=p_tol(p_ref))


@pytest.mark.parametrize("b", [64, 8192])
def test_zero_and_empty_inner(gpu, oracle, b):
    AT = np.zeros((5, 8))
    B = np.ones((5, 9))
    for v in ("fft", "fwht"):
        p, _ = capi().compressed_product(v, None, AT, B, 3, b, 1)
        assert np.array_equal(p, np.zeros((3, b)))
        p0, _ = capi().compressed_product(v, None, np.zeros((0, 8)), np.zeros((0, 9)), 3, b, 1)
        assert np.array_equal(p0, np.zeros((3, b)))
        C = capi().matmul(v, None, np.zeros((0, 8)), np.zeros((0, 9)), 3, b, 1)
        assert np.array_equal(C, np.zeros((8, 9)))
        # one side empty (n_a = 0 / n_b = 0)
        pa, _ = capi().compressed_product(v, None, np.ones((4, 0)), np.ones((4, 6)), 2, b, 3)
        assert np.array_equal(pa, np.zeros((2, b)))
        pb, _ = capi().compressed_product(v, None, np.ones((4, 6)), np.ones((4, 0)), 2, b, 3)
        assert np.array_equal(pb, np.zeros((2, b)))


# ----------------------------------------------------------- dense matmul
@pytest.mark.parametrize("variant", ["fft", "fwht"])
@pytest.mark.parametrize("h", HASHES)
@pytest.mark.parametrize("d", [1, 2, 5, 9, 16, 17, 20])
def test_matmul_vs_oracle(gpu, oracle, variant, h, d):
    rng = np.random.default_rng(d * 7 + KIND[h])
    AT = rng.standard_normal((60, 33))
    B = rng.standard_normal((60, 45))
    seed = 4000 + d
    b = 256
    C_gpu = capi().matmul(variant, h, AT, B, d, b, seed)
    p_ref = oracle.compressed_product(variant, h, AT, B, d, b, seed)
    C_ref = oracle.decompress(variant, h, p_ref, d, b, seed, 33, 45)
    np.testing.assert_allclose(C_gpu, C_ref, rtol=0, atol=p_tol(p_ref))


@pytest.mark.parametrize("variant", ["fft", "fwht"])
def test_decompress_list_vs_oracle(gpu, oracle, variant):
    rng = np.random.default_rng(9)
    AT = rng.standard_normal((20, 30))
    B = rng.standard_normal((20, 25))
    for d in (4, 9, 23):
        p_ref = oracle.compressed_product(variant, "tabulation8", AT, B, d, 128, 77)
        C_ref = oracle.decompress(variant, "tabulation8", p_ref, d, 128, 77, 30, 25)
        i = rng.integers(0, 30, 500)
        j = rng.integers(0, 25, 500)
        got = capi().decompress(variant, "tabulation8", p_ref, d, 128, 77, i, j)
        assert np.array_equal(got, C_ref[i, j])


def test_small_cases_golden(gpu, cm):
    """140 cases generated by the reference's own binding (make_golden.py)."""
    z = np.load(os.path.join(GOLD, "small_cases.npz"))
    n = len([k for k in z.files if k.endswith("_meta")])
    for c in range(n):
        d, b, seed, var, hidx, integer = [int(x) for x in z[f"c{c}_meta"]]
        AT = as_aligned(z[f"c{c}_AT"])
        B = as_aligned(z[f"c{c}_B"])
        C_ref = z[f"c{c}_C"]
        h = HASHES[hidx]
        C = aligned_alloc(C_ref.shape)
        (cm.matmul_fft if var == 0 else cm.matmul_fwht)(C, AT, B, d, b, seed, h)
        if f"c{c}_P" in z.files:
            p_ref = z[f"c{c}_P"]
            p_gpu, _ = capi().compressed_product(var, h, AT, B, d, b, seed)
            tol = p_tol(p_ref)
            if var == 1 and integer:
                assert np.array_equal(p_gpu, p_ref), c
            else:
                np.testing.assert_allclose(p_gpu, p_ref, rtol=0, atol=tol, err_msg=str(c))
        if var == 1 and integer:
            assert np.array_equal(C, C_ref), c
        else:
            scale = max(np.abs(C_ref).max(), 1.0)
            np.testing.assert_allclose(C, C_ref, rtol=0, atol=1e-10 * scale, err_msg=str(c))


# ---------------------------------------- the reference's own test suites
def test_reference_small_products(gpu, cm):
    # tests.cpp:842-942 and 1052-1150 through the drop-in
    for variant, dbs in (("fft", G.SMALL_DB_FFT), ("fwht", G.SMALL_DB_FWHT)):
        fn = cm.matmul_fft if variant == "fft" else cm.matmul_fwht
        for d, b in dbs:
            if not (d > 1 and b >= 32):
                continue
            for AT, B, Cc in G.SMALL_PRODUCTS:
                C = aligned_alloc(Cc.shape)
                fn(C, as_aligned(AT), as_aligned(B), d, b, G.SMALL_SEED)
                if variant == "fwht":
                    assert np.array_equal(C, Cc)
                else:
                    assert np.allclose(C, Cc, atol=1e-6, rtol=0)


def test_reference_random16(gpu, cm, oracle):
    # tests.cpp:944-1003, 1152-1211: 16x16 drng(15954), 1e-12 abs vs dgemm
    vals = oracle.drng(G.RAND16_SEED, 2 * 256)
    AT = as_aligned(vals[0::2].reshape(16, 16))
    B = as_aligned(vals[1::2].reshape(16, 16))
    C1 = aligned_alloc((16, 16))
    cm.gemm(C1, AT, B)
    for variant, cases in (("fft", G.RAND16_FFT), ("fwht", G.RAND16_FWHT)):
        fn = cm.matmul_fft if variant == "fft" else cm.matmul_fwht
        for h, d, b, off in cases:
            C = aligned_alloc((16, 16))
            fn(C, AT, B, d, b, G.RAND16_SEED + off, h)
            np.testing.assert_allclose(C, C1, atol=1e-12, rtol=0)


def test_reference_gemm_exact(gpu, cm):
    for AT, B, Cc in G.SMALL_PRODUCTS:  # tests.cpp:722-750
        C = aligned_alloc(Cc.shape)
        cm.gemm(C, as_aligned(AT), as_aligned(B))
        assert np.array_equal(C, Cc)


def test_reference_test_py(gpu, cm):
    """test.py:51-161 verbatim semantics through the drop-in module."""
    for (AT, B, C_correct) in G.py_fixtures():
        AT, B = as_aligned(AT), as_aligned(B)
        for algo in ("gemm", "fft", "fwht"):
            for h in HASHES:
                if algo == "gemm" and h is not None:
                    continue
                C = aligned_alloc(C_correct.shape)
                if algo == "gemm":
                    cm.gemm(C, AT, B)
                    assert np.array_equal(C, C_correct)
                elif algo == "fft":
                    d, b = G.PY_PARAMS_SMALL[(algo, h)]
                    cm.matmul_fft(C, AT, B, d, b, G.PY_SEED, h)
                    assert np.allclose(C, C_correct)
                else:
                    d, b = G.PY_PARAMS_SMALL[(algo, h)]
                    cm.matmul_fwht(C, AT, B, d, b, G.PY_SEED, h)
                    assert np.array_equal(C, C_correct)
    AT, B = as_aligned(G.PY_AT_4x2), as_aligned(G.PY_B_4x8)
    C1, C2, C3 = (aligned_alloc((2, 8)) for _ in range(3))
    for fn, eq in ((cm.matmul_fft, np.allclose), (cm.matmul_fwht, np.array_equal)):
        fn(C1, AT, B, 3, 8, G.PY_SEED1)
        fn(C2, AT, B, 3, 8, G.PY_SEED2)
        fn(C3, AT, B, 3, 8, G.PY_SEED1)
        assert eq(C1, C3)
        assert not np.allclose(C1, C2)
        fn(C2, AT, B, 3, 8, G.PY_SEED1)
        assert eq(C1, C2)
        fn(C3, AT, B, 3, 8, G.PY_SEED1, "multiply shift")
        fn(C2, AT, B, 3, 8, G.PY_SEED1, "multiply add shift")
        assert not np.allclose(C1, C3)
        assert eq(C1, C2)
    AT, B, C_correct = G.py_int16()
    AT, B = as_aligned(AT), as_aligned(B)
    for algo in ("gemm", "fft", "fwht"):
        for h in HASHES:
            if algo == "gemm" and h is not None:
                continue
            C = aligned_alloc(C_correct.shape)
            if algo == "gemm":
                cm.gemm(C, AT, B)
                assert np.array_equal(C, C_correct)
            elif algo == "fft":
                d, b = G.PY_PARAMS_16[(algo, h)]
                cm.matmul_fft(C, AT, B, d, b, G.PY_SEED, h)
                assert np.allclose(C, C_correct)
            else:
                d, b = G.PY_PARAMS_16[(algo, h)]
                cm.matmul_fwht(C, AT, B, d, b, G.PY_SEED, h)
                assert np.array_equal(C, C_correct)


def test_seed_none_is_time_seeded(gpu, cm):
    # seed=None draws rng()() from the ms clock: two calls normally differ
    AT, B = as_aligned(G.PY_AT_4x2), as_aligned(G.PY_B_4x8)
    C = aligned_alloc((2, 8))
    cm.matmul_fft(C, AT, B, 3, 8)  # must not raise
    p1, s1 = capi().compressed_product("fft", None, AT, B, 3, 8, None)
    assert p1.shape == (3, 8) and isinstance(s1, int)


# ------------------------------------------------- planted workloads + top-K
def _topk_gpu(C_host, K):
    import torch
    from compmatmul_b200 import device
    Ct = torch.from_numpy(C_host).cuda()
    return device.topk(Ct, K)


@pytest.mark.parametrize("name", ["config1", "config2_n4096", "config2_n16384"])
def test_planted_workload_recovery(gpu, cm, name):
    """Recovered top-K (i, j) set bit-exact vs the reference run on the same
    seeded inputs; values within 1e-10 relative."""
    path = os.path.join(GOLD, f"{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{name}.npz not generated")
    z = np.load(path)
    n, K, b, d, gen_seed, seed = [int(x) for x in z["meta"]]
    from compmatmul_b200.planted import planted_problem
    AT, B, planted = planted_problem(n, n, n, K, gen_seed)
    assert np.array_equal(planted[0], z["planted_i"])
    for variant in ("fft", "fwht"):
        if f"{variant}_top_i" not in z.files:
            continue
        C = aligned_alloc((n, n))
        (cm.matmul_fft if variant == "fft" else cm.matmul_fwht)(C, AT, B, d, b, seed)
        ti, tj, tv = _topk_gpu(C, K)
        assert np.array_equal(ti, z[f"{variant}_top_i"])
        assert np.array_equal(tj, z[f"{variant}_top_j"])
        np.testing.assert_allclose(tv, z[f"{variant}_top_v"], rtol=1e-10, atol=0)
        np.testing.assert_allclose(C[z[f"{variant}_sample_i"], z[f"{variant}_sample_j"]],
                                   z[f"{variant}_sample_v"], rtol=0,
                                   atol=1e-10 * np.abs(z[f"{variant}_top_v"]).max())
        p_gpu, _ = capi().compressed_product(variant, None, AT, B, d, b, seed)
        np.testing.assert_allclose(p_gpu[:, :64], z[f"{variant}_p_head"], rtol=0,
                                   atol=p_tol(z[f"{variant}_p_head"]))
        np.testing.assert_allclose(p_gpu.sum(axis=1), z[f"{variant}_p_sum"], rtol=1e-9)


def test_topk_ties_and_order(gpu):
    """Ties broken by (i, j) ascending, including > 4096 equal values."""
    import torch
    from compmatmul_b200 import device
    C = np.zeros((300, 200))
    C[5, 7] = 3.0
    C[1, 2] = 2.0
    C[0, 9] = 2.0
    ti, tj, tv = device.topk(torch.from_numpy(C).cuda(), 10)
    assert list(zip(ti[:3], tj[:3])) == [(5, 7), (0, 9), (1, 2)]
    assert list(zip(ti[3:], tj[3:])) == [(0, 0), (0, 1), (0, 2), (0, 3), (0, 4), (0, 5), (0, 6)]
    assert list(tv) == [3.0, 2.0, 2.0] + [0.0] * 7
    rng = np.random.default_rng(0)
    C = rng.standard_normal((513, 257))
    ti, tj, tv = device.topk(torch.from_numpy(C).cuda(), 100)
    flat = C.ravel()
    order = np.lexsort((np.arange(flat.size), -flat))[:100]
    assert np.array_equal(ti * 257 + tj, order)
