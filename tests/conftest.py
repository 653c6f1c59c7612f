import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def aligned_alloc(shape, dtype=np.float64, alignment=64):
    """64-byte aligned numpy array (the reference binding rejects others,
    compmatmul.cpp:65-73); same helper as the reference's test.py:8-15."""
    elem = np.dtype(dtype).itemsize
    nbytes = int(np.prod(shape)) * elem
    raw = np.empty(nbytes + alignment, np.uint8)
    off = (alignment - raw.ctypes.data % alignment) % alignment
    return raw[off:off + nbytes].view(dtype).reshape(shape)


def as_aligned(a, alignment=64):
    a = np.ascontiguousarray(a)
    if a.ctypes.data % alignment == 0:
        return a
    out = aligned_alloc(a.shape, a.dtype, alignment)
    out[...] = a
    return out


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reflib():
    from oracle.oracle import RefLib
    if not RefLib.available():
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    return RefLib()


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cm():
    """The drop-in module; on a GPU test run the native path must load."""
    import compmatmul_b200
    return compmatmul_b200.load_dropin()


@pytest.fixture(scope="session")
def gpu():
    if not _has_gpu():
        pytest.fail("GPU test collected on a machine without a CUDA device")
    import compmatmul_b200
    L = compmatmul_b200.lib()
    assert L.cmm_device_count() >= 1
    return L
