"""cmm_multiply: the `multiply` command-line program over the C ABI
(options and messages of the reference's multiply.cpp).

CPU tests cover the argument and .npy checks, which run before any device
use; GPU tests compare the output files with numpy (gemm, exact) and with
the oracle's dense estimate (fft / fwht with a fixed seed, 1e-11 * max|p|
scaled to C's entries), for C- and Fortran-ordered inputs."""
import os
import subprocess

import numpy as np
import pytest

from compmatmul_b200.build import CLI


def run(*args):
    r = subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=300)
    return r.returncode, r.stdout + r.stderr


@pytest.fixture
def files(tmp_path):
    rng = np.random.default_rng(3)
    A = rng.standard_normal((40, 30))
    B = rng.standard_normal((40, 20))
    pa, pb, pc = tmp_path / "A.npy", tmp_path / "B.npy", tmp_path / "C.npy"
    np.save(pa, A)
    np.save(pb, B)
    return A, B, pa, pb, pc


def test_cli_parameter_errors(files):
    A, B, pa, pb, pc = files
    rc, out = run("-a", "fft", "-d", "3", pa, pb, pc)
    assert rc == 1 and "Got algorithm `fft' but the parameter b is not set!" in out
    rc, out = run("-a", "fwht", "-b", "100", "-d", "3", pa, pb, pc)
    assert rc == 1 and "The parameter b must be a positive power of 2 (got 100)" in out
    rc, out = run("-a", "fft", "-b", "64", pa, pb, pc)
    assert rc == 1 and "Got algorithm `fft' but the parameter d is not set!" in out
    rc, out = run("-a", "fft", "-b", "64", "-d", "0", pa, pb, pc)
    assert rc == 1 and "The parameter d must be positive (got 0)" in out
    rc, out = run("-a", "lsh", pa, pb, pc)
    assert rc == 1 and "gemm|fft|fwht" in out
    rc, out = run(pa, pb)
    assert rc == 1 and "expected <A.npy> <B.npy> <C.npy>" in out


def test_cli_refuses_to_overwrite(files):
    A, B, pa, pb, pc = files
    pc.write_bytes(b"x")
    rc, out = run(pa, pb, pc)
    assert rc == 1 and "already exists!" in out


def test_cli_npy_checks(files, tmp_path):
    A, B, pa, pb, pc = files
    p3 = tmp_path / "A3.npy"
    np.save(p3, np.zeros((2, 3, 4)))
    rc, out = run(p3, pb, pc)
    assert rc == 1 and "Dimension mismatch: A has 3 dims, but 2 expected!" in out
    p4 = tmp_path / "A4.npy"
    np.save(p4, np.zeros((40, 30), dtype=np.float32))
    rc, out = run(p4, pb, pc)
    assert rc == 1 and "Word size mismatch: A is expected to have word size of 8, but got 4" in out
    p5 = tmp_path / "A5.npy"
    np.save(p5, np.zeros((40, 30), dtype=np.int64))
    rc, out = run(p5, pb, pc)
    assert rc == 1 and "float64" in out


@pytest.mark.gpu
def test_cli_gemm_and_compressed(gpu, oracle, files, tmp_path):
    A, B, pa, pb, pc = files
    rc, out = run(pa, pb, pc)
    assert rc == 0, out
    np.testing.assert_allclose(np.load(pc), A.T @ B, rtol=1e-12, atol=1e-12)
    for variant in ("fft", "fwht"):
        rc, out = run("-f", "-a", variant, "-b", "256", "-d", "5", "--seed", "4242", pa, pb, pc)
        assert rc == 0, out
        ref = oracle.matmul(variant, None, A, B, 5, 256, 4242)
        got = np.load(pc)
        assert got.shape == (30, 20)
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-10 * max(float(np.abs(ref).max()), 1.0))


@pytest.mark.gpu
def test_cli_fortran_order_inputs(gpu, files, tmp_path):
    A, B, pa, pb, pc = files
    fa, fb = tmp_path / "FA.npy", tmp_path / "FB.npy"
    np.save(fa, np.asfortranarray(A))
    np.save(fb, np.asfortranarray(B))
    c2 = tmp_path / "C2.npy"
    assert run("-a", "fft", "-b", "128", "-d", "3", "--seed", "9", pa, pb, pc)[0] == 0
    assert run("-a", "fft", "-b", "128", "-d", "3", "--seed", "9", fa, fb, c2)[0] == 0
    np.testing.assert_allclose(np.load(c2), np.load(pc), rtol=0, atol=1e-12 * float(np.abs(np.load(pc)).max()))
