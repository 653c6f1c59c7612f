"""Serving engine (cmm_server_*): continuous batching under a device-memory
admission cap.

* A request's sketch is bit-identical alone and in a mix of other requests
  (its work items and summation order depend on the request alone), and
  within the mixed-precision tolerance (2e-5 * max|p|) of the FP64
  single-product path on the same inputs.
* Waves overlap: with several streams, more than one wave is in flight.
* The admission cap bounds the device bytes held; a request larger than
  the cap is rejected.
* FP64 serving matches the oracle within 1e-11 * max|p|; host (pageable
  numpy and pinned torch) and device inputs are all accepted.
"""
import numpy as np
import pytest

from compmatmul_b200 import device
from compmatmul_b200.planted import batch_shapes, planted_problem_device
from compmatmul_b200.serve import Server


def p_tol(p_ref, rel):
    return rel * max(float(np.abs(p_ref).max()), 1e-300)


def _requests(count, seed, lo=128, hi=768):
    out = []
    for s in batch_shapes(count=count, seed=seed, lo=lo, hi=hi):
        AT, B, _ = planted_problem_device(s["m"], s["n"], s["p"], s["K"], s["gen_seed"], "float32")
        out.append(dict(AT=AT, B=B, d=s["d"], b=s["b"], seed=s["seed"], variant=s["variant"]))
    return out


@pytest.mark.gpu
def test_serve_alone_equals_mix(gpu):
    import torch
    reqs = _requests(24, seed=31)
    srv = Server(mem_cap_bytes=8 << 30, f32=True, streams=3, max_wave=6)
    x = reqs[10]
    alone = srv.result(srv.submit(x["AT"], x["B"], x["d"], x["b"], x["seed"], x["variant"]))
    ids = [srv.submit(q["AT"], q["B"], q["d"], q["b"], q["seed"], q["variant"]) for q in reqs]
    outs = [srv.result(i) for i in ids]
    st = srv.stats()
    srv.close()
    np.testing.assert_array_equal(outs[10], alone)
    assert st["completed"] == 25 and st["queued"] == 0 and st["in_flight"] == 0
    assert st["max_waves_in_flight"] >= 2, st
    for q, p in zip(reqs, outs):
        ref = device.compressed_product(q["AT"].double(), q["B"].double(), q["d"], q["b"], q["seed"],
                                        q["variant"]).cpu().numpy()
        np.testing.assert_allclose(p, ref, rtol=0, atol=p_tol(ref, 2e-5))
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_serve_admission_cap(gpu):
    import torch
    reqs = _requests(16, seed=41, lo=256, hi=512)
    cap = 64 << 20
    srv = Server(mem_cap_bytes=cap, f32=True, streams=2, max_wave=4)
    # host payloads (pinned) count against the cap too
    hreqs = [dict(q, AT=q["AT"].cpu().pin_memory(), B=q["B"].cpu().pin_memory()) for q in reqs]
    ids = [srv.submit(q["AT"], q["B"], q["d"], q["b"], q["seed"], q["variant"]) for q in hreqs]
    outs = [srv.result(i) for i in ids]
    st = srv.stats()
    assert 0 < st["max_mem_in_use"] <= cap, st
    big = torch.zeros((4096, 4096), dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError, match="admission cap"):
        srv.submit(big, big, 9, 1 << 16, 1, "fft")
    srv.close()
    for q, p in zip(reqs, outs):
        ref = device.compressed_product(q["AT"].double(), q["B"].double(), q["d"], q["b"], q["seed"],
                                        q["variant"]).cpu().numpy()
        np.testing.assert_allclose(p, ref, rtol=0, atol=p_tol(ref, 2e-5))


@pytest.mark.gpu
def test_serve_fp64_matches_oracle(gpu, oracle):
    rng = np.random.default_rng(7)
    srv = Server(mem_cap_bytes=1 << 30, f32=False, streams=2, max_wave=3)
    cases = []
    for i in range(6):
        n_a, n_inner, n_b = (int(x) for x in rng.integers(16, 300, size=3))
        AT = rng.standard_normal((n_inner, n_a))
        B = rng.standard_normal((n_inner, n_b))
        d, b = int(rng.integers(1, 8)), int(rng.choice([64, 512, 4096, 16384]))
        variant = "fft" if i % 2 == 0 else "fwht"
        hs = [None, "multiply shift", "tabulation8"][i % 3]
        cases.append((AT, B, d, b, 100 + i, variant, hs, srv.submit(AT, B, d, b, 100 + i, variant, hs)))
    for AT, B, d, b, seed, variant, hs, rid in cases:
        p = srv.result(rid)
        ref = oracle.compressed_product(variant, hs, AT, B, d, b, seed)
        np.testing.assert_allclose(p, ref, rtol=0, atol=p_tol(ref, 1e-11))
    srv.close()


@pytest.mark.gpu
def test_serve_code_plan_cache(gpu):
    """Requests with the same (hash, seed, d, b, sizes) share resident hash
    codes and sorted plans: hits after the first, identical results."""
    reqs = _requests(3, seed=53)
    order = [0, 1, 2, 0, 1, 2, 2, 1, 0, 0]
    plain = Server(mem_cap_bytes=4 << 30, f32=True, streams=2, max_wave=4)
    want = [plain.result(plain.submit(q["AT"], q["B"], q["d"], q["b"], q["seed"], q["variant"])) for q in reqs]
    plain.close()
    srv = Server(mem_cap_bytes=4 << 30, f32=True, streams=2, max_wave=4, cache_bytes=1 << 30)
    got = []
    for k in order:  # one at a time: every repeat finds its entry resident
        q = reqs[k]
        got.append(srv.result(srv.submit(q["AT"], q["B"], q["d"], q["b"], q["seed"], q["variant"])))
    st = srv.stats()
    srv.close()
    assert st["cache_misses"] == 3 and st["cache_hits"] == len(order) - 3, st
    assert 0 < st["cache_in_use"] <= 1 << 30
    for k, p in zip(order, got):
        np.testing.assert_array_equal(p, want[k])
