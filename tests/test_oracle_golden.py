"""Pins the CPU oracle (oracle/cmm_oracle.c) against the reference's own
golden vectors (tests.cpp, test.py) and, where oracle/_ref was built,
against the reference's headers compiled with the project shims."""
import os

import numpy as np
import pytest

from golden import ref_vectors as G

HERE = os.path.dirname(os.path.abspath(__file__))

MS, MAS, TAB8, TAB16 = 0, 1, 2, 3


def test_rng_golden(oracle):
    assert oracle.rng(1234, 4) == G.RNG_1234  # tests.cpp:90-96


def test_ilog2_via_bucket_shift(oracle):
    # bucket of multiply-shift with a = 2^63 + 1 and key 1 keeps log2(b) top bits
    for lg in range(1, 31):
        buf = np.array([(1 << 63) | 1], dtype=np.uint64)
        h = oracle.L.cmo_hash_bucket(MS, buf.ctypes.data, 1 << lg, 1)
        assert h == 1 << (lg - 1)


def test_multiply_shift_golden(oracle):
    assert oracle.hash_params_u64(MS, 1, G.MS_SEED)[0] == G.MS_A  # tests.cpp:146-183
    assert oracle.hash_params_u64(MS, 2, G.MS2_SEED) == G.MS2_A  # tests.cpp:185-222
    keys = np.arange(0, 1025)
    hs, ss = oracle.hash_eval(MS, 2, 32, G.MS2_SEED, keys)
    for t, a in enumerate(G.MS2_A):
        w = (a * keys.astype(object)) % (1 << 64)
        assert list(hs[t]) == [int(x) >> 59 for x in w]
        assert list(ss[t]) == [1 if int(x) >> 63 else -1 for x in w]


def test_multiply_add_shift_golden(oracle):
    p = oracle.hash_params_u64(MAS, 1, G.MAS_SEED)
    assert tuple(p) == G.MAS_AB  # tests.cpp:228-267
    p2 = oracle.hash_params_u64(MAS, 2, G.MAS2_SEED)
    assert [tuple(p2[0:2]), tuple(p2[2:4])] == G.MAS2_AB  # tests.cpp:269-307
    keys = np.arange(0, 2049)
    hs, ss = oracle.hash_eval(MAS, 2, 128, G.MAS2_SEED, keys)
    for t, (a, b) in enumerate(G.MAS2_AB):
        w = [(a * int(k) + b) % (1 << 64) for k in keys]
        assert list(hs[t]) == [x >> 57 for x in w]
        assert list(ss[t]) == [1 if x >> 63 else -1 for x in w]


def test_mas_draw_one_and_hashes(oracle):
    # tests.cpp:797-814: draw_one(32, 8876) -> (a, b); 100 keys from rng(32149)
    assert tuple(oracle.hash_params_u64(MAS, 1, G.MAS3_SEED)) == G.MAS3_AB
    a, b = G.MAS3_AB
    keys = [x & 0xffffffff for x in oracle.rng(G.MAS3_KEY_SEED, 100)]
    hs, ss = oracle.hash_eval(MAS, 1, 32, G.MAS3_SEED, keys)
    for e, k in enumerate(keys):
        h = ((a * k + b) % (1 << 64)) >> 59
        assert hs[0, e] == h
        assert ss[0, e] == (1 if (h >> 4) else -1)


def test_sketch_seed_derivation(oracle):
    # tests.cpp:816-840: h1 <- seed, h2 <- seed+1, s1 <- seed+2, s2 <- seed+3
    for off, name in enumerate(["h1", "h2", "s1", "s2"]):
        p = oracle.hash_params_u64(MAS, 2, G.SKETCH_SEED + off)
        assert [tuple(p[0:2]), tuple(p[2:4])] == G.SKETCH_AB[name]


@pytest.mark.parametrize("seed", [G.TAB_SEED_A, G.TAB_SEED_B])
def test_tabulation_tables_from_stream(oracle, seed):
    # tests.cpp:312-461: tables are consecutive u32-truncated rng outputs
    stream = oracle.rng(seed, 1024 * 2)
    buf, nb = oracle.hash_draw(TAB8, 2, seed)
    T = np.frombuffer(bytes(buf), dtype=np.uint32)
    assert list(T) == [x & 0xffffffff for x in stream]
    keys = [x & 0xffffffff for x in oracle.rng(seed + 99, 300)]
    hs, ss = oracle.hash_eval(TAB8, 2, 128, seed, keys)
    for t in range(2):
        Tt = T[t * 1024:(t + 1) * 1024].reshape(4, 256)
        for e, k in enumerate(keys):
            h = int(Tt[0][k & 0xff] ^ Tt[1][(k >> 8) & 0xff] ^ Tt[2][(k >> 16) & 0xff] ^ Tt[3][k >> 24])
            assert hs[t, e] == h >> 25
            assert ss[t, e] == (1 if h >> 31 else -1)
    stream16 = oracle.rng(seed + 1, 2 * 65536)
    buf16, _ = oracle.hash_draw(TAB16, 1, seed + 1)
    T16 = np.frombuffer(bytes(buf16), dtype=np.uint32)
    assert list(T16[:1000]) == [x & 0xffffffff for x in stream16[:1000]]
    assert int(T16[-1]) == stream16[-1] & 0xffffffff
    hs, ss = oracle.hash_eval(TAB16, 1, 256, seed + 1, keys)
    T16 = T16.reshape(2, 65536)
    for e, k in enumerate(keys):
        h = int(T16[0][k & 0xffff] ^ T16[1][k >> 16])
        assert hs[0, e] == h >> 24
        assert ss[0, e] == (1 if h >> 31 else -1)


def test_fft_golden(oracle):
    X = oracle.fft_r2c(G.FFT_X)  # tests.cpp:576-615
    np.testing.assert_allclose(X.real, G.FFT_XHAT.real, atol=1e-6)
    np.testing.assert_allclose(X.imag, G.FFT_XHAT.imag, atol=1e-6)
    x = oracle.fft_c2r(X, 32) / 32
    np.testing.assert_allclose(x, G.FFT_X, atol=1e-6)


def test_fwht_golden(oracle):
    X = oracle.fwht(G.FWHT_X)  # tests.cpp:621-671
    np.testing.assert_allclose(X, G.FWHT_XHAT, atol=1e-6)
    np.testing.assert_allclose(oracle.fwht(X) / 32, G.FWHT_X, atol=1e-6)


def test_median_is_upper_middle(oracle):
    assert oracle.median([3.0, 1.0]) == 3.0  # array.hpp:323-328: element size/2
    assert oracle.median([5.0, 1.0, 3.0]) == 3.0
    assert oracle.median([4.0, 1.0, 3.0, 2.0]) == 3.0


def test_gemm_exact(oracle):
    for AT, B, C in G.SMALL_PRODUCTS:  # tests.cpp:722-750
        assert np.array_equal(oracle.gemm(AT, B), C)


@pytest.mark.parametrize("variant", ["fft", "fwht"])
def test_small_products(oracle, variant):
    # tests.cpp:842-942 / 1052-1150
    dbs = G.SMALL_DB_FFT if variant == "fft" else G.SMALL_DB_FWHT
    for d, b in dbs:
        if not (d > 1 and b >= 32):
            continue
        for AT, B, C in G.SMALL_PRODUCTS:
            got = oracle.matmul(variant, None, AT, B, d, b, G.SMALL_SEED)
            if variant == "fwht":
                assert np.array_equal(got, C)
            else:
                assert np.allclose(got, C, atol=1e-6, rtol=0)


@pytest.mark.parametrize("variant", ["fft", "fwht"])
def test_random16_vs_gemm(oracle, variant):
    # tests.cpp:944-1003 / 1152-1211: drng(15954) 16x16, 1e-12 abs
    vals = oracle.drng(G.RAND16_SEED, 2 * 256)
    AT = vals[0::2].reshape(16, 16)
    B = vals[1::2].reshape(16, 16)
    C = oracle.gemm(AT, B)
    cases = G.RAND16_FFT if variant == "fft" else G.RAND16_FWHT
    for h, d, b, off in cases:
        got = oracle.matmul(variant, h, AT, B, d, b, G.RAND16_SEED + off)
        np.testing.assert_allclose(got, C, atol=1e-12, rtol=0)


def test_python_suite_cases(oracle):
    # test.py:51-119 restated against the oracle
    for AT, B, C in G.py_fixtures():
        for (algo, h), (d, b) in G.PY_PARAMS_SMALL.items():
            got = oracle.matmul(algo, h, AT, B, d, b, G.PY_SEED)
            if algo == "fft":
                assert np.allclose(got, C)
            else:
                assert np.array_equal(got, C)
    AT, B = G.PY_AT_4x2, G.PY_B_4x8
    for algo in ("fft", "fwht"):
        c1 = oracle.matmul(algo, None, AT, B, 3, 8, G.PY_SEED1)
        c2 = oracle.matmul(algo, None, AT, B, 3, 8, G.PY_SEED2)
        c3 = oracle.matmul(algo, None, AT, B, 3, 8, G.PY_SEED1)
        assert np.array_equal(c1, c3) and not np.allclose(c1, c2)
        ms = oracle.matmul(algo, "multiply shift", AT, B, 3, 8, G.PY_SEED1)
        mas = oracle.matmul(algo, "multiply add shift", AT, B, 3, 8, G.PY_SEED1)
        assert not np.allclose(c1, ms) and np.array_equal(c1, mas)
    AT, B, C = G.py_int16()
    for (algo, h), (d, b) in G.PY_PARAMS_16.items():
        got = oracle.matmul(algo, h, AT, B, d, b, G.PY_SEED)
        if algo == "fft":
            assert np.allclose(got, C)
        else:
            assert np.array_equal(got, C)


# ---------------------------------------------------------- vs reference
def test_ref_transforms_match_golden(reflib):
    X = reflib.fft_fwd(G.FFT_X)
    np.testing.assert_allclose(X.real, G.FFT_XHAT.real, atol=1e-6)
    np.testing.assert_allclose(X.imag, G.FFT_XHAT.imag, atol=1e-6)
    np.testing.assert_allclose(reflib.fwht(G.FWHT_X), G.FWHT_XHAT, atol=1e-6)


@pytest.mark.parametrize("h", [None, "multiply shift", "tabulation8", "tabulation16"])
def test_oracle_codes_match_reference(oracle, reflib, h):
    from oracle.oracle import HASHES
    kind = HASHES[h]
    for side, off in ((0, 0), (1, 1)):
        hb, _ = reflib.hash_codes(h, 3, 1024, 777 + off, 5000)
        _, sg = reflib.hash_codes(h, 3, 1024, 777 + off + 2, 5000)
        codes = oracle.sketch_codes(kind, 3, 1024, 777, side, 5000)
        assert np.array_equal(codes & 0x7fffffff, hb)
        assert np.array_equal((codes >> 31).astype(np.int32), (sg > 0).astype(np.int32))


@pytest.mark.parametrize("variant", ["fft", "fwht"])
@pytest.mark.parametrize("h", [None, "multiply shift", "tabulation8", "tabulation16"])
def test_oracle_matches_reference_sketch(oracle, reflib, variant, h):
    rng = np.random.default_rng(5)
    AT = rng.standard_normal((40, 24))
    B = rng.standard_normal((40, 31))
    po = oracle.compressed_product(variant, h, AT, B, 5, 64, 4242)
    pr = reflib.compressed_product(variant, h, AT, B, 5, 64, 4242)
    np.testing.assert_allclose(po, pr, atol=1e-12 * np.abs(pr).max(), rtol=0)
    co = oracle.decompress(variant, h, pr, 5, 64, 4242, 24, 31)
    cr = np.zeros((24, 31))
    reflib.decompress_rows(variant, h, pr, 5, 64, 4242, 31, 0, 24, cr)
    assert np.array_equal(co, cr)



@pytest.mark.parametrize("variant", ["fft", "fwht"])
@pytest.mark.parametrize("d,b", [(9, 1 << 16), (9, 1 << 18)])
def test_oracle_matches_reference_at_config_geometry(oracle, reflib, variant, d, b):
    """The oracle against the reference's own code at the buckets and
    repetitions of the configurations (b = 2^16 with d = 9, and b = 2^18),
    on a few inner indices: sketches within 1e-12 of max|p|, dense
    decompression of the reference's sketch bit-identical."""
    rng = np.random.default_rng(b + d)
    AT = rng.standard_normal((6, 200))
    B = rng.standard_normal((6, 180))
    po = oracle.compressed_product(variant, None, AT, B, d, b, 2718)
    pr = reflib.compressed_product(variant, None, AT, B, d, b, 2718)
    np.testing.assert_allclose(po, pr, atol=1e-12 * np.abs(pr).max(), rtol=0)
    co = oracle.decompress(variant, None, pr, d, b, 2718, 200, 180)
    cr = np.zeros((200, 180))
    reflib.decompress_rows(variant, None, pr, d, b, 2718, 180, 0, 200, cr)
    assert np.array_equal(co, cr)

_ONE_THREAD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from oracle.oracle import Oracle
o = Oracle()
rng = np.random.default_rng(12)
out = []
for variant in ("fft", "fwht"):
    AT = rng.standard_normal((9, 70)); B = rng.standard_normal((9, 50))
    p = o.compressed_product(variant, "tabulation8", AT, B, 7, 1 << 12, 31)
    out += [p, o.decompress(variant, "tabulation8", p, 7, 1 << 12, 31, 70, 50)]
np.savez(sys.argv[2], *out)
"""


def test_oracle_results_independent_of_thread_count(oracle, tmp_path):
    """The oracle runs its repetitions and decompression rows on OpenMP
    threads with every sum in the reference's order: one thread and many
    give bit-identical sketches and dense estimates."""
    import subprocess
    import sys
    root = os.path.dirname(HERE)
    out = str(tmp_path / "one.npz")
    env = dict(os.environ, OMP_NUM_THREADS="1")
    subprocess.run([sys.executable, "-c", _ONE_THREAD, root, out], env=env, check=True, timeout=300)
    one = np.load(out)
    rng = np.random.default_rng(12)
    k = 0
    for variant in ("fft", "fwht"):
        AT = rng.standard_normal((9, 70))
        B = rng.standard_normal((9, 50))
        p = oracle.compressed_product(variant, "tabulation8", AT, B, 7, 1 << 12, 31)
        C = oracle.decompress(variant, "tabulation8", p, 7, 1 << 12, 31, 70, 50)
        assert np.array_equal(p, one[f"arr_{k}"])
        assert np.array_equal(C, one[f"arr_{k + 1}"])
        k += 2
