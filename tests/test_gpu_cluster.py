"""Cluster sketch kernels (FFT and FWHT, FP64 and mixed) against the oracle.

The shapes are chosen so that the automatic dispatch takes the cluster
kernels (asserted through cmm_last_sketch_kernel) and cover:
  * groups of 16 CTAs (radix-16 combine split over lane pairs) and of 8;
  * R1 <= 2 (real DIF weights: the two sides scatter into the real and
    imaginary parts at once) and R1 > 2 (complex weights, sides one after
    the other);
  * the sub-spectra exchanged through global memory, double-buffered;
  * several work items per group and several k-groups;
  * all-zero rows, which every CTA of a group skips, including at the
    start and end of the inner range (the staged next row must follow);
  * chunked materialization (accumulating launches), on device inputs and
    on streamed host rows;
  * each slot's sign applied once, on rows of very different scales.
Tolerances: FP64 sketch within 1e-11 * max|p| absolute; mixed within
2e-5 * max|p|.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def capi():
    from compmatmul_b200 import capi as c
    return c


def kernel():
    from compmatmul_b200 import lib
    return lib().cmm_last_sketch_kernel().decode()


def check(variant, h, AT, B, d, b, seed, oracle, f32=False):
    if f32:
        A32, B32 = AT.astype(np.float32), B.astype(np.float32)
        p, _ = capi().compressed_product_f32(variant, h, A32, B32, d, b, seed)
        ref = oracle.compressed_product(variant, h, A32.astype(np.float64), B32.astype(np.float64), d, b, seed)
        tol = 2e-5
    else:
        p, _ = capi().compressed_product(variant, h, AT, B, d, b, seed)
        ref = oracle.compressed_product(variant, h, AT, B, d, b, seed)
        tol = 1e-11
    assert kernel() == "cluster", kernel()
    np.testing.assert_allclose(p, ref, rtol=0, atol=tol * max(float(np.abs(ref).max()), 1e-300))


@pytest.mark.parametrize("b,h", [(1 << 15, None), (1 << 16, "multiply shift"), (1 << 17, "tabulation16"),
                                 (1 << 18, "tabulation8")])
def test_fft_fp64(gpu, oracle, b, h):
    rng = np.random.default_rng(b)
    AT = rng.standard_normal((23, 300))
    B = rng.standard_normal((23, 260)) * 1e-2
    check("fft", h, AT, B, 3, b, 1234, oracle)


@pytest.mark.parametrize("b", [1 << 17, 1 << 19])
def test_fwht_fp64(gpu, oracle, b):
    rng = np.random.default_rng(b + 1)
    AT = rng.standard_normal((17, 280))
    B = rng.standard_normal((17, 310))
    check("fwht", "multiply add shift", AT, B, 2, b, 77, oracle)


def test_fft_many_items_and_groups(gpu, oracle):
    rng = np.random.default_rng(5)
    AT = rng.standard_normal((70, 90))
    B = rng.standard_normal((70, 80))
    # d = 9 at b = 2^18: more (r1, t) items than co-resident clusters
    check("fft", None, AT, B, 9, 1 << 18, 9, oracle)
    # d = 1: the planner splits the inner range into k-groups
    check("fft", None, AT, B, 1, 1 << 16, 10, oracle)


@pytest.mark.parametrize("side", ["A", "B"])
def test_fft_zero_rows_skipped(gpu, oracle, side):
    rng = np.random.default_rng(11)
    AT = rng.standard_normal((41, 200))
    B = rng.standard_normal((41, 150))
    M = AT if side == "A" else B
    M[[0, 1, 2, 7, 8, 20, 39, 40]] = 0.0
    check("fft", "tabulation8", AT, B, 2, 1 << 16, 3, oracle)


def test_fft_all_rows_zero(gpu, oracle):
    AT = np.zeros((9, 50))
    B = np.random.default_rng(2).standard_normal((9, 60))
    p, _ = capi().compressed_product("fft", None, AT, B, 2, 1 << 16, 4)
    assert kernel() == "cluster"
    assert float(np.abs(p).max()) == 0.0


@pytest.mark.parametrize("variant,b", [("fft", 1 << 16), ("fwht", 1 << 17)])
def test_chunked_materialization(gpu, oracle, variant, b, monkeypatch):
    # a small budget runs several materialize + sketch launches that accumulate
    monkeypatch.setenv("CMM_MATERIALIZE_BYTES", str(300 * 1024))
    rng = np.random.default_rng(b + 7)
    AT = rng.standard_normal((64, 400))
    B = rng.standard_normal((64, 380))
    check(variant, None, AT, B, 3, b, 21, oracle)


@pytest.mark.parametrize("variant,b", [("fft", 1 << 15), ("fwht", 1 << 16)])
def test_chunked_launches_accumulate(gpu, oracle, variant, b):
    # the host entry point streams the rows in chunks (the first one an
    # eighth of the copy budget): several cluster launches, each adding to
    # the k-group partials of the previous ones
    rng = np.random.default_rng(b + 7)
    AT = rng.standard_normal((600, 120))
    B = rng.standard_normal((600, 100))
    AT[[0, 8, 9, 599]] = 0.0  # skipped rows at chunk edges
    check(variant, None, AT, B, 3, b, 21, oracle)


def test_unbalanced_rows_and_signs(gpu, oracle):
    """Each slot's sign is applied once, by the row copy: rows of very
    different scales in A and B (the FFT row balance) and a planted large
    entry, both variants."""
    rng = np.random.default_rng(19)
    AT = rng.standard_normal((50, 333)) * np.logspace(-3, 3, 50)[:, None]
    B = rng.standard_normal((50, 277)) * np.logspace(3, -3, 50)[:, None]
    AT[10, 5] += 1e4
    B[10, 7] += 1e4
    check("fft", None, AT, B, 5, 1 << 16, 8, oracle)
    check("fwht", None, AT, B, 5, 1 << 16, 8, oracle)


@pytest.mark.parametrize("b", [1 << 16, 1 << 18])
def test_fft_mixed(gpu, oracle, b):
    rng = np.random.default_rng(b + 3)
    AT = rng.standard_normal((31, 240))
    B = rng.standard_normal((31, 220)) * 1e3
    check("fft", "multiply shift", AT, B, 3, b, 5, oracle, f32=True)


@pytest.mark.parametrize("b", [1 << 16, 1 << 18])
def test_fwht_mixed(gpu, oracle, b):
    rng = np.random.default_rng(b + 4)
    AT = rng.standard_normal((29, 250))
    B = rng.standard_normal((29, 230)) * 1e-2
    check("fwht", "multiply shift", AT, B, 3, b, 6, oracle, f32=True)


def test_group_wait_that_runs_out_is_reported(gpu, oracle, monkeypatch):
    """A group barrier wait is bounded: with the test hook every wait needs
    one arrival more than the group makes, so each CTA gives up after a
    short spin, the launch ends, its partials are NaN and the synchronous
    entry point raises.  The next product is unaffected."""
    rng = np.random.default_rng(77)
    AT = rng.standard_normal((20, 120))
    B = rng.standard_normal((20, 110))
    monkeypatch.setenv("CMM_TEST_GROUP_WAIT_EXTRA", "1")
    with pytest.raises(RuntimeError, match="group barrier wait ran out"):
        capi().compressed_product("fft", None, AT, B, 3, 1 << 16, 9)
    monkeypatch.delenv("CMM_TEST_GROUP_WAIT_EXTRA")
    check("fft", None, AT, B, 3, 1 << 16, 9, oracle)


_ALT_FORM = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from compmatmul_b200 import capi, lib
rng = np.random.default_rng(int(sys.argv[3]))
AT = rng.standard_normal((29, 250))
B = rng.standard_normal((29, 230)) * 1e-2
if sys.argv[4] == "f32":
    p, _ = capi.compressed_product_f32(sys.argv[5], None, AT.astype(np.float32), B.astype(np.float32), 3, 1 << 16, 6)
else:
    p, _ = capi.compressed_product(sys.argv[5], None, AT, B, 3, 1 << 16, 6)
assert lib().cmm_last_sketch_kernel().decode() == "cluster"
np.save(sys.argv[2], p)
"""


@pytest.mark.parametrize("env,prec,variant", [("CMM_MIXED_WHT=tc", "f32", "fwht"),
                                              ("CMM_GROUP_THREADS=256", "f64", "fft"),
                                              ("CMM_GROUP_THREADS=256", "f64", "fwht")])
def test_alternative_forms(gpu, oracle, tmp_path, env, prec, variant):
    """The forms that the dispatch does not pick by default, each in a child
    process (the choice is read once per process): the mixed FWHT with its
    Hadamard-16 stages on the tensor cores (BF16 hi/mid/lo), and the FP64
    kernels with 256-thread CTAs, two per SM."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = tmp_path / "p.npy"
    key, val = env.split("=")
    run_env = dict(os.environ, **{key: val})
    subprocess.run([sys.executable, "-c", _ALT_FORM, root, str(out), "6", prec, variant], env=run_env,
                   check=True, timeout=300)
    p = np.load(out)
    rng = np.random.default_rng(6)
    AT = rng.standard_normal((29, 250))
    B = rng.standard_normal((29, 230)) * 1e-2
    if prec == "f32":
        AT, B = AT.astype(np.float32).astype(np.float64), B.astype(np.float32).astype(np.float64)
    ref = oracle.compressed_product(variant, None, AT, B, 3, 1 << 16, 6)
    tol = 2e-5 if prec == "f32" else 1e-11
    np.testing.assert_allclose(p, ref, rtol=0, atol=tol * float(np.abs(ref).max()))
