"""Generates tests/golden/*.npz from the REFERENCE itself: the reference's
pybind module `compmatmul` (compmatmul.cpp) and headers, compiled unchanged
against the project shims into oracle/_ref (`make -C oracle ref`).

Run here (needs /root/reference at build time of oracle/_ref):
    python tests/golden/make_golden.py [small|config1|config2_n4096|config2_n16384|all]

Fixtures:
  small_cases.npz   dense C and sketch p of small seeded problems (all 4
                    hashes, both variants, several (d, b)), via the
                    reference's own Python binding.
  <workload>.npz    planted-entry workloads (compmatmul_b200.planted):
                    top-K (i, j, value) of the reference's dense estimate and
                    per-repetition checksums of its sketch p, per variant.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))

from compmatmul_b200.planted import WORKLOADS, aligned_empty, planted_problem, topk_dense_host  # noqa: E402
from oracle.oracle import RefLib  # noqa: E402

HASHES = [None, "multiply shift", "multiply add shift", "tabulation8", "tabulation16"]

# (n_inner, n_a, n_b, d, b) small shapes; values integer or real
SMALL = [
    (7, 5, 6, 3, 8), (40, 24, 31, 5, 64), (33, 17, 9, 4, 2), (64, 64, 64, 9, 4096),
    (20, 12, 15, 7, 8192), (16, 16, 16, 1, 32), (12, 30, 10, 2, 16),
]


def small():
    import compmatmul as ref  # the reference's own binding
    rl = RefLib()
    out = {}
    rng = np.random.default_rng(1234)
    case = 0
    for (q, p_, r, d, b) in SMALL:
        for integer in (True, False):
            if integer:
                AT = rng.integers(-9, 10, (q, p_)).astype(np.float64)
                B = rng.integers(-9, 10, (q, r)).astype(np.float64)
            else:
                AT = rng.standard_normal((q, p_))
                B = rng.standard_normal((q, r))
            ATa = aligned_empty(AT.shape); ATa[...] = AT
            Ba = aligned_empty(B.shape); Ba[...] = B
            for variant in ("fft", "fwht"):
                for h in HASHES:
                    seed = 1000 + case
                    C = aligned_empty((p_, r))
                    fn = ref.matmul_fft if variant == "fft" else ref.matmul_fwht
                    fn(C, ATa, Ba, d, b, seed, h)
                    P = rl.compressed_product(variant, h, ATa, Ba, d, b, seed)
                    key = f"c{case}"
                    out[key + "_AT"] = AT
                    out[key + "_B"] = B
                    out[key + "_C"] = np.array(C)
                    if d * b <= 8192:  # keep the fixture small
                        out[key + "_P"] = P
                    out[key + "_meta"] = np.array([d, b, seed, 0 if variant == "fft" else 1,
                                                   HASHES.index(h), int(integer)], dtype=np.int64)
                    case += 1
    np.savez_compressed(os.path.join(HERE, "small_cases.npz"), **out)
    print("small:", case, "cases")


def workload(name):
    import compmatmul as ref
    rl = RefLib()
    w = WORKLOADS[name]
    n = w["n"]
    t0 = time.time()
    AT, B, planted = planted_problem(n, n, n, w["K"], w["gen_seed"])
    out = {"planted_i": planted[0], "planted_k": planted[1], "planted_j": planted[2],
           "meta": np.array([n, w["K"], w["b"], w["d"], w["gen_seed"], w["seed"]], dtype=np.int64)}
    for variant in w["variants"]:
        t1 = time.time()
        P = rl.compressed_product(variant, None, AT, B, w["d"], w["b"], w["seed"])
        t2 = time.time()
        C = aligned_empty((n, n))
        fn = ref.matmul_fft if variant == "fft" else ref.matmul_fwht
        fn(C, AT, B, w["d"], w["b"], w["seed"])
        t3 = time.time()
        ii, jj, vv = topk_dense_host(C, w["K"])
        out[f"{variant}_top_i"] = ii
        out[f"{variant}_top_j"] = jj
        out[f"{variant}_top_v"] = vv
        out[f"{variant}_p_sum"] = P.sum(axis=1)
        out[f"{variant}_p_sumsq"] = (P * P).sum(axis=1)
        out[f"{variant}_p_head"] = P[:, :64].copy()
        # a fixed sample of dense entries (independent of the top-K)
        srng = np.random.default_rng(77)
        si = srng.integers(0, n, 2048)
        sj = srng.integers(0, n, 2048)
        out[f"{variant}_sample_i"] = si
        out[f"{variant}_sample_j"] = sj
        out[f"{variant}_sample_v"] = C[si, sj]
        if n <= 512:
            out[f"{variant}_P"] = P
        print(f"{name} {variant}: sketch {t2 - t1:.1f}s, matmul {t3 - t2:.1f}s, "
              f"threads {rl.num_threads()}", flush=True)
        del C
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: total {time.time() - t0:.1f}s")


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("small", "all"):
        small()
    for name in WORKLOADS:
        if what in (name, "all") and not (what == "all" and name == "config2_n16384"):
            workload(name)
