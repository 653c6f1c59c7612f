"""The C++ header entry points (include/compmatmul_b200.hpp): the program
builds here, checks the host-side hash objects here (no GPU needed) and
runs the reference's small exact products through the sketch type on the
GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_header_api.cpp")
PKG = os.path.join(ROOT, "compmatmul_b200")


def build(tmp_path):
    exe = str(tmp_path / "test_header_api")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L" + PKG, "-l:libcmm_b200.so", "-Wl,-rpath," + PKG], check=True)
    return exe


def test_header_compiles(tmp_path):
    assert os.path.exists(build(tmp_path))


def test_header_hash_objects_match_reference(tmp_path):
    """Host-side part (no GPU): rng, the hash families, sign hashes and the
    sketch's drawn functions against the reference's own values."""
    exe = build(tmp_path)
    r = subprocess.run([exe, "hash"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")


@pytest.mark.gpu
def test_header_runs_reference_cases(tmp_path, gpu):
    exe = build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("ok")
