"""k-sharded compressed product (compmatmul_b200/sharded.py): each rank
sketches its slice of the inner index and one all-reduce of the d x b
sketches completes the product.

CPU (gloo, two ranks): the slices' sketches come from the CPU oracle on each
rank's rows (the product's kernels need a GPU), so this checks the split and
the reduction plumbing, and that the reduced sketch equals the oracle's
sketch of the whole product within 1e-12 * max|p|.
GPU (one device, no process group): the sum of the device sketches of the
slices equals the device sketch of the whole product within 1e-11 * max|p|,
the linearity the sharded form relies on, with this package's kernels."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem():
    rng = np.random.default_rng(31)
    return rng.standard_normal((37, 50)), rng.standard_normal((37, 44))


def _rank(rank, world, port, variant, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from compmatmul_b200.sharded import reduce_sketch, slice_bounds
    from oracle.oracle import Oracle
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    AT, B = _problem()
    k0, k1 = slice_bounds(AT.shape[0], world, rank)
    p = Oracle().compressed_product(variant, None, AT[k0:k1], B[k0:k1], 5, 512, 77)
    t = torch.from_numpy(np.ascontiguousarray(p))
    reduce_sketch(t)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, (k0, k1), t.numpy()))


@pytest.mark.parametrize("variant", ["fft", "fwht"])
def test_sharded_sketch_two_gloo_ranks(oracle, variant):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(k, 2, port, variant, out)) for k in range(2)]
    for p in procs:
        p.start()
    res = sorted([out.get(timeout=120) for _ in procs], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [(0, 19), (19, 37)]
    AT, B = _problem()
    want = oracle.compressed_product(variant, None, AT, B, 5, 512, 77)
    for _, _, p in res:
        np.testing.assert_allclose(p, want, rtol=0, atol=1e-12 * np.abs(want).max())


def test_slice_bounds_cover_the_range():
    from compmatmul_b200.sharded import slice_bounds
    for n, w in [(10, 3), (7, 8), (16384, 8), (0, 2)]:
        b = [slice_bounds(n, w, r) for r in range(w)]
        assert b[0][0] == 0 and b[-1][1] == n
        assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))
        assert max(e - s for s, e in b) - min(e - s for s, e in b) <= 1


@pytest.mark.gpu
@pytest.mark.parametrize("variant,b", [("fft", 1 << 16), ("fwht", 1 << 16), ("fft", 4096)])
def test_slice_sketches_sum_to_the_product(gpu, variant, b):
    import torch

    from compmatmul_b200 import device
    from compmatmul_b200.sharded import slice_bounds
    rng = np.random.default_rng(b)
    AT = torch.from_numpy(rng.standard_normal((300, 400))).cuda()
    B = torch.from_numpy(rng.standard_normal((300, 350))).cuda()
    full = device.compressed_product(AT, B, 7, b, 5, variant).cpu().numpy()
    parts = np.zeros_like(full)
    for r in range(4):
        k0, k1 = slice_bounds(300, 4, r)
        parts += device.compressed_product(AT[k0:k1].contiguous(), B[k0:k1].contiguous(), 7, b, 5,
                                           variant).cpu().numpy()
    np.testing.assert_allclose(parts, full, rtol=0, atol=1e-11 * np.abs(full).max())
