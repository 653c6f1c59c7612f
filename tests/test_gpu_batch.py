"""Batched products (cmm_batch_*): one persistent sketch launch over a work
queue of uneven products, replayed from a CUDA graph.

Each product of a batch must equal the single-product device path on the
same inputs:
  * FP64 plan: sketch p within 1e-11 * max|p| absolute of
    cmm_dev_compressed_product, dense C within the same bound, and both
    against the oracle for the small products;
  * FP32 (mixed) plan: p within 2e-5 * max|p| of the FP64 path on the same
    FP32-valued inputs; recovered top-K sets equal, values within 1e-5
    relative (the mixed-precision bar).
Graph replay with changed input contents, the autotuner's choices and its
cache, empty products, and the config-4 shape generator are covered too.
"""
import numpy as np
import pytest

from compmatmul_b200 import device
from compmatmul_b200.batch import BatchPlan
from compmatmul_b200.planted import batch_shapes, planted_problem_device

HASHES = [None, "multiply shift", "multiply add shift", "tabulation8", "tabulation16"]


def p_tol(p_ref, rel):
    return rel * max(float(np.abs(p_ref).max()), 1e-300)


def _mixed_products(torch, dtype, seed=5, count=10):
    rng = np.random.default_rng(seed)
    prods = []
    for i in range(count):
        n_a, n_inner, n_b = (int(x) for x in rng.integers(24, 400, size=3))
        b = int(rng.choice([64, 256, 1024, 2048, 4096, 8192, 16384]))
        d = int(rng.integers(1, 10))
        g = torch.Generator(device="cuda").manual_seed(100 + i)
        AT = torch.randn((n_inner, n_a), generator=g, device="cuda", dtype=dtype)
        B = torch.randn((n_inner, n_b), generator=g, device="cuda", dtype=dtype)
        if i % 3 == 0:  # unbalanced row scales exercise the FFT row balance
            AT *= 1e3
            B *= 1e-2
        prods.append(dict(AT=AT, B=B, d=d, b=b, seed=int(rng.integers(1, 1 << 40)),
                          variant="fft" if i % 2 == 0 else "fwht", hash=HASHES[i % 5]))
    return prods


@pytest.mark.gpu
def test_batch_fp64_matches_single_product(gpu):
    import torch
    prods = _mixed_products(torch, torch.float64)
    plan = BatchPlan(prods, f32=False, tune=False, dense=True)
    plan.run()
    torch.cuda.synchronize()
    for i, q in enumerate(plan.products):
        p_ref = device.compressed_product(q["AT"], q["B"], q["d"], q["b"], q["seed"], q["variant"], q["hash"])
        C_ref = device.decompress_dense(p_ref, q["AT"].shape[1], q["B"].shape[1], q["d"], q["b"], q["seed"],
                                        q["variant"], q["hash"])
        pr = p_ref.cpu().numpy()
        np.testing.assert_allclose(q["p"].cpu().numpy(), pr, rtol=0, atol=p_tol(pr, 1e-11), err_msg=str(i))
        np.testing.assert_allclose(q["C"].cpu().numpy(), C_ref.cpu().numpy(), rtol=0,
                                   atol=p_tol(pr, 1e-11), err_msg=str(i))
    info = plan.info()
    assert info["items"] > 0 and info["ctas"] > 0
    plan.close()


@pytest.mark.gpu
def test_batch_fp64_matches_oracle(gpu, oracle):
    import torch
    prods = _mixed_products(torch, torch.float64, seed=9, count=6)
    plan = BatchPlan(prods, f32=False, tune=False, dense=False)
    plan.run()
    torch.cuda.synchronize()
    for i, q in enumerate(plan.products):
        AT = q["AT"].cpu().numpy()
        B = q["B"].cpu().numpy()
        p_ref = oracle.compressed_product(q["variant"], q["hash"], AT, B, q["d"], q["b"], q["seed"])
        np.testing.assert_allclose(q["p"].cpu().numpy(), p_ref, rtol=0, atol=p_tol(p_ref, 1e-11), err_msg=str(i))


@pytest.mark.gpu
def test_batch_mixed_matches_fp64(gpu):
    import torch
    prods = _mixed_products(torch, torch.float32, seed=11)
    plan = BatchPlan(prods, f32=True, tune=False, dense=False)
    plan.run()
    torch.cuda.synchronize()
    for i, q in enumerate(plan.products):
        p_ref = device.compressed_product(q["AT"].double(), q["B"].double(), q["d"], q["b"], q["seed"],
                                          q["variant"], q["hash"]).cpu().numpy()
        np.testing.assert_allclose(q["p"].cpu().numpy(), p_ref, rtol=0, atol=p_tol(p_ref, 2e-5), err_msg=str(i))


@pytest.mark.gpu
def test_batch_mixed_planted_recovery(gpu):
    """Config-4 style shapes (scaled down): the mixed batch recovers the same
    top-K sets as the FP64 path on the same inputs, values within 1e-5."""
    import torch
    shapes = batch_shapes(count=12, seed=77, lo=256, hi=1024)
    prods = []
    for s in shapes:
        AT, B, _ = planted_problem_device(s["m"], s["n"], s["p"], s["K"], s["gen_seed"], "float32")
        prods.append(dict(AT=AT, B=B, d=s["d"], b=s["b"], seed=s["seed"], variant=s["variant"], K=s["K"]))
    plan = BatchPlan(prods, f32=True, tune=True, dense=True)
    plan.run()
    torch.cuda.synchronize()
    for i, q in enumerate(plan.products):
        C64 = device.matmul(q["AT"].double(), q["B"].double(), q["d"], q["b"], q["seed"], q["variant"])
        i64, j64, v64 = device.topk(C64, q["K"])
        im, jm, vm = device.topk(q["C"], q["K"])
        assert set(zip(i64.tolist(), j64.tolist())) == set(zip(im.tolist(), jm.tolist())), i
        np.testing.assert_allclose(vm, v64, rtol=1e-5, atol=0, err_msg=str(i))


@pytest.mark.gpu
def test_batch_graph_replay_follows_input_contents(gpu):
    import torch
    prods = _mixed_products(torch, torch.float64, seed=13, count=5)
    plan = BatchPlan(prods, f32=False, tune=False, dense=False)
    plan.run()
    plan.run()  # the second run replays the captured graph
    torch.cuda.synchronize()
    first = [q["p"].cpu().numpy().copy() for q in plan.products]
    for q in plan.products:
        q["AT"].mul_(2.0)  # same storage, new contents
    plan.run()
    torch.cuda.synchronize()
    for i, q in enumerate(plan.products):
        np.testing.assert_allclose(q["p"].cpu().numpy(), 2.0 * first[i], rtol=0,
                                   atol=p_tol(first[i], 4e-11), err_msg=str(i))


@pytest.mark.gpu
def test_batch_autotuner_choices_and_cache(gpu):
    import torch
    prods = _mixed_products(torch, torch.float32, seed=17, count=6)
    plan = BatchPlan(prods, f32=True, tune=True, dense=False)
    cfg = [plan.config(i) for i in range(len(prods))]
    for q, c in zip(prods, cfg):
        assert c["tuned"] and c["radix"] in (4, 8) and c["groups"] >= 1
        assert c["slab"] <= q["b"] and c["slab"] <= (4096 if q["variant"] == "fft" else 8192)
    plan2 = BatchPlan(prods, f32=True, tune=False, dense=False)  # classes come from the cache
    assert [(c["slab"], c["radix"]) for c in cfg] == \
        [(plan2.config(i)["slab"], plan2.config(i)["radix"]) for i in range(len(prods))]
    plan2.run()
    plan.run()
    torch.cuda.synchronize()
    for a, b in zip(plan.products, plan2.products):
        np.testing.assert_allclose(a["p"].cpu().numpy(), b["p"].cpu().numpy(), rtol=0,
                                   atol=p_tol(b["p"].cpu().numpy(), 2e-5))


@pytest.mark.gpu
def test_batch_empty_and_degenerate_products(gpu):
    import torch
    z = lambda r, c: torch.zeros((r, c), dtype=torch.float64, device="cuda")
    prods = [dict(AT=z(0, 7), B=z(0, 5), d=3, b=64, seed=1, variant="fft"),
             dict(AT=z(4, 0), B=torch.randn((4, 6), dtype=torch.float64, device="cuda"), d=2, b=32, seed=2,
                  variant="fwht"),
             dict(AT=z(9, 11), B=z(9, 13), d=5, b=256, seed=3, variant="fft")]
    plan = BatchPlan(prods, f32=False, tune=False, dense=True)
    plan.run()
    torch.cuda.synchronize()
    for q in plan.products:
        assert float(q["p"].abs().max()) == 0.0
        if q["C"].numel():
            assert float(q["C"].abs().max()) == 0.0
