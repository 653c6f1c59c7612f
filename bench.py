"""Benchmark of the compressed product on B200.

One step = one compressed product of a planted-entry workload: hash codes,
per-k balancing, fused sketch/transform/accumulate, inverse, dense median
decompression of all n_a x n_b entries into HBM, and device top-K recovery
(K = planted count).  Default workload: n = 16384 square FP64, b = 2^16,
d = 9, FFT variant, K = 256 (inputs 4.3 GB > L2, so no flush is needed).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--variant fft|fwht]
                  [--workload config2_n16384|config2_n4096|config1]
                  [--impl reference]

--gpus N > 1 runs under torchrun, one rank per GPU, each rank an
independent product (weak scaling, no collective on the data path; the
path has none -- one product fits one GPU).  Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "compressed products/s"
HBM_PEAK_FALLBACK = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config2_n16384")
    ap.add_argument("--variant", default="fft", choices=["fft", "fwht"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--n", type=int, default=0, help="override the workload size (profiling)")
    ap.add_argument("--compare-fp64", type=int, default=0,
                    help="also time N steps of the plain FP64 path on the same inputs")
    ap.add_argument("--batch-count", type=int, default=256, help="products of the config4 batch")
    ap.add_argument("--batch-tune", type=int, default=1, help="config4: run the autotuner (0: defaults)")
    ap.add_argument("--batch-variant", default="both", choices=["both", "fft", "fwht"],
                    help="config4: draw the variants as specified (both) or force one")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="config5: Poisson arrival rate (req/s)")
    ap.add_argument("--serve-seconds", type=float, default=30.0, help="config5: arrival window (s)")
    ap.add_argument("--serve-cap-gb", type=float, default=40.0, help="config5: admission cap (GB)")
    ap.add_argument("--serve-streams", type=int, default=4, help="config5: waves in flight")
    ap.add_argument("--serve-max-wave", type=int, default=64, help="config5: requests per wave")
    ap.add_argument("--serve-cache-gb", type=float, default=4.0,
                    help="config5: resident hash codes + plans across requests (0: off)")
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed"],
                    help="fp64 = plain path; mixed = FP32 inputs (default for config3)")
    return ap.parse_args()


# DRAM traffic of one sketch-kernel launch relative to its algorithmic bytes
# (the row pairs it must read once per repetition), from one ncu capture of
# the same kernel on a small case: dram__bytes_read.sum + dram__bytes_write.sum
# over d * k_chunk * (n_a + n_b) * element bytes, scaled to a full launch by
# the units it processes (the row reads dominate and grow in proportion).
# Source: profiles/k_sketch_cluster_fft_config2_small.md.
TRAFFIC_RATIO = {("cluster", "fft", "f64"): 1.352 / 1.208}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            m = json.load(f)
        return float(m.get("hbm_gbs", HBM_PEAK_FALLBACK)), "measured"
    return HBM_PEAK_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks + throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def fft_flops(n_a, n_inner, n_b, d, b):
    lb = np.log2(b)
    return n_inner * d * (2 * 2.5 * b * lb + 8 * (b / 2 + 1) + 2 * (n_a + n_b)) + d * 2.5 * b * lb


def fwht_ops(n_a, n_inner, n_b, d, b):
    lb = np.log2(b)
    return n_inner * d * (2 * b * lb + 2 * b + 2 * (n_a + n_b)) + d * b * lb


# ------------------------------------------------------------- CPU legs
def cpu_reference_sample(AT, B, n, d, b, variant, seed, budget_s):
    """Time the reference's own CPU path (headers compiled with shims,
    oracle/_ref) on a bounded sample and extrapolate to one product:
    sketch over the first ks inner indices, decompression of the first
    rows.  Returns (seconds_per_product, threads, sample description)."""
    from oracle.oracle import RefLib
    rl = RefLib()
    thr = rl.num_threads()
    ks = 8
    while True:
        t0 = time.perf_counter()
        p = rl.compressed_product(variant, None, AT[:ks], B[:ks], d, b, seed)
        ts = time.perf_counter() - t0
        if ts > budget_s * 0.25 or ks >= n:
            break
        ks = min(n, ks * max(2, int(budget_s * 0.3 / max(ts, 1e-3))))
    rows = 8
    while True:
        Cbuf = np.empty((rows, n))  # rows [0, rows) of C
        t0 = time.perf_counter()
        rl.decompress_rows(variant, None, p, d, b, seed, n, 0, rows, Cbuf)
        tdec = time.perf_counter() - t0
        if tdec > budget_s * 0.15 or rows >= n:
            break
        rows = min(n, rows * max(2, int(budget_s * 0.2 / max(tdec, 1e-3))))
    per_product = ts * (n / ks) + tdec * (n / rows)
    sample = (f"reference CPU path ({variant}) on the first {ks} of {n} inner indices "
              f"({ts:.2f} s) and the first {rows} of {n} rows of the dense decompression "
              f"({tdec:.2f} s), scaled linearly to one product")
    return per_product, thr, sample


# ------------------------------------------------- batched products (config 4)
def product_flops(s):
    f = fft_flops if s["variant"] == "fft" else fwht_ops
    return f(s["m"], s["n"], s["p"], s["d"], s["b"])


def bench_batch(args, world, rank, local):
    """Config 4: 256 uneven planted products (FP32 inputs) as one batch plan:
    one persistent sketch launch over a work queue, the whole batch replayed
    from a CUDA graph; a step is one run of all products (sketches + dense
    median estimates).  Compared with the plain FP64 path on the same
    inputs, both batched and as one cmm_dev_matmul call per product."""
    from compmatmul_b200.planted import batch_shapes, planted_problem_device
    count = args.batch_count
    shapes = batch_shapes(count=count, seed=4004 + 1000 * rank)
    if args.batch_variant != "both":  # one variant only (component timing)
        shapes = [dict(s, variant=args.batch_variant) for s in shapes]
    config = {"workload": f"config4: {count} planted products m x n x p, each dimension log-uniform in "
                          f"[256, 4096], FP32 noise N(0,0.01^2) + K=max(8,m/64) planted +10/+10, "
                          f"b = next pow2 >= 256 K, d in {{5,7,9}}, FFT/FWHT 50/50; sketch + dense median "
                          f"estimate per product",
              "products": count, "l2": "inputs (sum 4 n (m+p) bytes) larger than L2, no flush"}
    flops_total = sum(product_flops(s) for s in shapes)
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle.oracle import RefLib
        from compmatmul_b200.planted import planted_problem
        rl = RefLib()
        t_used, f_used, done = 0.0, 0.0, 0
        for s in shapes:
            AT, B, _ = planted_problem(s["m"], s["n"], s["p"], s["K"], s["gen_seed"], dtype=np.float32)
            t0 = time.perf_counter()
            rl.matmul(s["variant"], None, AT.astype(np.float64), B.astype(np.float64), s["d"], s["b"], s["seed"])
            t_used += time.perf_counter() - t0
            f_used += product_flops(s)
            done += 1
            if t_used > args.cpu_seconds:
                break
        sec = t_used * flops_total / f_used  # one batch, scaled by modelled work
        val = count / sec
        sample = (f"reference CPU path (headers compiled with shims, {rl.num_threads()} threads, FP64 on the "
                  f"FP32-valued inputs) on the first {done} of {count} products ({t_used:.1f} s), scaled to the "
                  f"batch by the modelled flops")
        print(json.dumps({"metric": METRIC, "value": val, "unit": "products/s", "impl": "reference",
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                          "cpu_baseline": {"value": val, "unit": "products/s", "cores": rl.num_threads(),
                                           "kind": "reference", "sample": sample},
                          "e2e": {"value": val, "unit": "products/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return

    import ctypes as C
    import torch
    import compmatmul_b200 as cmb
    from compmatmul_b200 import device as dev
    from compmatmul_b200.batch import BatchPlan
    from compmatmul_b200.replicas import Replicas
    reps = Replicas()
    L = cmb.lib()
    prods, planted = [], []
    for s in shapes:
        AT, B, pl = planted_problem_device(s["m"], s["n"], s["p"], s["K"], s["gen_seed"], "float32")
        prods.append(dict(AT=AT, B=B, d=s["d"], b=s["b"], seed=s["seed"], variant=s["variant"]))
        planted.append(pl)
    t0 = time.perf_counter()
    plan = BatchPlan(prods, f32=True, tune=bool(args.batch_tune), dense=True)
    plan_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        plan.run()
    torch.cuda.synchronize()

    barrier = reps.barrier
    clocks = ClockSampler(torch.cuda.current_device())
    L.cmm_profile_reset()
    L.cmm_profile_enable(1)
    launches0 = L.cmm_launch_count()
    barrier()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        plan.run()
    ev1.record()
    barrier()
    clk = clocks.stop()
    launches = L.cmm_launch_count() - launches0
    L.cmm_profile_enable(0)
    total_ms = ev0.elapsed_time(ev1)
    value = reps.throughput(count * args.steps, total_ms / 1e3)
    total_ms = reps.max(total_ms)
    ms_per_step = total_ms / args.steps
    info = plan.info()

    # the persistent sketch kernel alone (its own run, events on the same stream)
    ek0 = torch.cuda.Event(enable_timing=True)
    ek1 = torch.cuda.Event(enable_timing=True)
    L.cmm_profile_reset()
    L.cmm_profile_enable(1)
    ek0.record()
    plan.run()
    ek1.record()
    torch.cuda.synchronize()
    L.cmm_profile_enable(0)
    batch_ms = cmb.profile_read("batch")[0]

    # recovery: planted entries among each product's top-K estimates
    rec = tot = 0
    for q, (is_, ks, js), s in zip(plan.products, planted, shapes):
        ti, tj, _ = dev.topk(q["C"], s["K"])
        rec += len(set(zip(ti.tolist(), tj.tolist())) & set(zip(is_.tolist(), js.tolist())))
        tot += s["K"]

    # plain FP64 on the same inputs: batched, and one cmm_dev_matmul per product
    fp64 = None
    if args.compare_fp64:
        prods64 = [dict(q, AT=q["AT"].double(), B=q["B"].double()) for q in prods]
        plan64 = BatchPlan(prods64, f32=False, tune=True, dense=True)
        for _ in range(2):
            plan64.run()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.compare_fp64):
            plan64.run()
        e1.record()
        torch.cuda.synchronize()
        b64 = e0.elapsed_time(e1) / args.compare_fp64
        outs = [torch.empty((q["AT"].shape[1], q["B"].shape[1]), dtype=torch.float64, device="cuda")
                for q in prods64]
        for q, o in zip(prods64, outs):  # warm
            dev.matmul(q["AT"], q["B"], q["d"], q["b"], q["seed"], variant=q["variant"], out=o)
        torch.cuda.synchronize()
        e0.record()
        for q, o in zip(prods64, outs):
            dev.matmul(q["AT"], q["B"], q["d"], q["b"], q["seed"], variant=q["variant"], out=o)
        e1.record()
        torch.cuda.synchronize()
        single64 = e0.elapsed_time(e1)
        maxrel = {"fft": 0.0, "fwht": 0.0}
        same_sets = 0
        for q, q64, s in zip(plan.products, plan64.products, shapes):
            ti, tj, tv = dev.topk(q64["C"], s["K"])
            mi, mj, _ = dev.topk(q["C"], s["K"])
            same_sets += set(zip(ti.tolist(), tj.tolist())) == set(zip(mi.tolist(), mj.tolist()))
            got = q["C"][torch.as_tensor(ti, device="cuda"), torch.as_tensor(tj, device="cuda")].cpu().numpy()
            err = float(np.max(np.abs(got - tv) / np.maximum(np.abs(tv), 1e-300)))
            maxrel[s["variant"]] = max(maxrel[s["variant"]], err)
        fp64 = {"batched_ms_per_step": b64, "single_product_calls_ms_per_step": single64,
                "speedup_vs_batched_fp64": b64 / ms_per_step, "speedup_vs_single_fp64": single64 / ms_per_step,
                "max_rel_err_recovered_vs_fp64": maxrel,
                "same_recovered_sets_as_fp64": f"{same_sets}/{count}"}
        plan64.close()
        del prods64, outs

    # end to end with host buffers: pinned inputs in, dense estimates out
    hin = [(torch.empty_like(q["AT"], device="cpu").pin_memory(), torch.empty_like(q["B"], device="cpu").pin_memory())
           for q in prods]
    hout = [torch.empty_like(q["C"], device="cpu").pin_memory() for q in plan.products]
    for (ha, hb), q in zip(hin, prods):
        ha.copy_(q["AT"])
        hb.copy_(q["B"])
    h2d = sum(ha.numel() * 4 + hb.numel() * 4 for ha, hb in hin)
    d2h = sum(o.numel() * 8 for o in hout)
    e2e_steps = max(1, args.e2e_steps)
    barrier()
    te0 = time.perf_counter()
    for _ in range(e2e_steps):
        for (ha, hb), q in zip(hin, prods):
            q["AT"].copy_(ha, non_blocking=True)
            q["B"].copy_(hb, non_blocking=True)
        plan.run()
        for o, q in zip(hout, plan.products):
            o.copy_(q["C"], non_blocking=True)
        torch.cuda.synchronize()
    barrier()
    e2e_s = (time.perf_counter() - te0) / e2e_steps
    e2e_value = reps.throughput(count, e2e_s)

    fma = C.c_double(0.0)
    fma_peak = fma.value if L.cmm_probe_fma_tflops(0, C.byref(fma)) == 0 else None
    alg_bytes = sum(4.0 * s["d"] * s["n"] * (s["m"] + s["p"]) for s in shapes)
    peak, peak_kind = measured_peaks()
    if rank != 0:
        plan.close()
        reps.close()
        return
    line = {
        "metric": METRIC, "value": value, "unit": "products/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (mixed: FP32 transforms, FP64 reduction)", "data": "synthetic",
        "config": config,
        "roofline": {"bound": "hbm", "achieved": alg_bytes / (batch_ms / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": alg_bytes / (batch_ms / 1e3) / 1e9 / peak, "traffic": None,
                     "kernel": "batch graph (persistent k_batch_sketch + per-product finalize/decompress)",
                     "peak_source": peak_kind, "launch_ms": batch_ms, "algorithmic_bytes_per_launch": alg_bytes,
                     "binding": {"bound": "fp32", "achieved": flops_total / (batch_ms / 1e3) / 1e12,
                                 "peak": fma_peak, "unit": "TFLOP/s",
                                 "frac": (flops_total / (batch_ms / 1e3) / 1e12 / fma_peak) if fma_peak else None,
                                 "peak_source": "measured FMA loop (cmm_probe_fma_tflops)",
                                 "flops_per_launch": flops_total}},
        "e2e": {"value": e2e_value, "unit": "products/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clk,
        "recovered_planted": f"{rec}/{tot}",
        "batch": {"items": info["items"], "ctas": info["ctas"], "launches_per_run": info["launches"],
                  "plan_and_tune_s": plan_s},
        "cpu_baseline": None,
    }
    if fp64 is not None:
        line["plain_fp64_same_inputs"] = fp64
    print(json.dumps(line), flush=True)
    plan.close()
    reps.close()


# ------------------------------------------------------------ serving (config 5)
def serve_stream(srv, pool, arrivals, poll_every=64):
    """Submits pool[i % len(pool)] at arrivals[i] (seconds from start) and
    collects completions as they come; returns (latencies, span_s)."""
    from collections import deque
    out = deque()
    lat = []
    t0 = time.perf_counter()
    for i, ta in enumerate(arrivals):
        while True:
            dt = ta - (time.perf_counter() - t0)
            if dt <= 0:
                break
            if dt > 0.002:
                time.sleep(dt - 0.001)
        q = pool[i % len(pool)]
        out.append(srv.submit(q["AT"], q["B"], q["d"], q["b"], q["seed"], q["variant"]))
        if i % poll_every == 0:
            while out:
                done, l = srv.wait(out[0], 0.0)
                if not done:
                    break
                lat.append(l)
                srv._live.pop(out.popleft(), None)
    while out:
        rid = out.popleft()
        done, l = srv.wait(rid, None)
        lat.append(l)
        srv._live.pop(rid, None)
    span = time.perf_counter() - t0
    return np.array(lat), span


def bench_serve(args, world, rank, local):
    """Config 5: Poisson arrivals (rate, duration) of requests sized as the
    batched config, served with continuous batching under a device-memory
    admission cap; latency p50/p99 and products/s, against the plain FP64
    path on the same stream."""
    import torch
    import compmatmul_b200 as cmb
    from compmatmul_b200.batch import BatchPlan
    from compmatmul_b200.planted import batch_shapes, planted_problem_device
    from compmatmul_b200.serve import Server
    rate, secs, cap = args.serve_rate, args.serve_seconds, int(args.serve_cap_gb * (1 << 30))
    config = {"workload": f"config5: Poisson arrivals at {rate:g} req/s for {secs:g} s; each request one compressed "
                          f"product sized as config4 (m, n, p log-uniform in [256, 4096], FP32, planted, "
                          f"b = next pow2 >= 256 K, d in {{5,7,9}}, FFT/FWHT 50/50) from a pool of "
                          f"{args.batch_count} inputs; admission cap {args.serve_cap_gb:g} GB; resident hash codes + plans "
                          f"{args.serve_cache_gb:g} GB; result = sketch p",
              "rate_per_s": rate, "seconds": secs, "cap_bytes": cap}
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving loop; its per-product "
                              "CPU cost is the config4 reference line"}), flush=True)
        return
    torch.cuda.set_device(local if world > 1 else 0)
    shapes = batch_shapes(count=args.batch_count, seed=5005 + 1000 * rank)
    pool = []
    for sh in shapes:
        AT, B, _ = planted_problem_device(sh["m"], sh["n"], sh["p"], sh["K"], sh["gen_seed"], "float32")
        pool.append(dict(AT=AT, B=B, d=sh["d"], b=sh["b"], seed=sh["seed"], variant=sh["variant"]))
    # the autotuner's cache covers the request classes before the stream starts
    BatchPlan(pool, f32=True, tune=True, dense=False).close()
    rng = np.random.default_rng(77 + rank)
    n_req = int(rate * secs)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    L = cmb.lib()

    def run(pool_, f32, arr, streams=args.serve_streams, cache=int(args.serve_cache_gb * (1 << 30))):
        srv = Server(mem_cap_bytes=cap, f32=f32, streams=streams, max_wave=args.serve_max_wave, cache_bytes=cache)
        # warm-up: one burst of the whole pool fills the pinned staging and
        # device pools (and, when enabled, the code/plan residency)
        warm = [srv.submit(q["AT"], q["B"], q["d"], q["b"], q["seed"], q["variant"]) for q in pool_]
        for w in warm:
            srv.result(w)
        serve_stream(srv, pool_, arr[arr < 1.0])  # one untimed second of the same stream
        st0 = srv.stats()
        l0 = L.cmm_launch_count()
        clocks = ClockSampler(torch.cuda.current_device())
        clocks.start()
        lat, span = serve_stream(srv, pool_, arr)
        clk = clocks.stop()
        st = srv.stats()
        srv.close()
        return {"products_per_s": len(lat) / span, "cache_bytes": cache,
                "cache_hits": int(st["cache_hits"] - st0["cache_hits"]),
                "cache_misses": int(st["cache_misses"] - st0["cache_misses"]), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
                "requests": int(len(lat)), "span_s": span, "waves": int(st["waves"] - st0["waves"]),
                "max_waves_in_flight": int(st["max_waves_in_flight"]),
                "max_mem_in_use_bytes": int(st["max_mem_in_use"]), "launches": int(L.cmm_launch_count() - l0),
                "clocks": clk}

    main_run = run(pool, True, arrivals)
    # the same stream with every request hashing and planning for itself
    no_cache = run(pool, True, arrivals, cache=0) if args.serve_cache_gb > 0 else None
    # latency without queueing: half the measured capacity, 10 s
    light_rate = 0.5 * main_run["products_per_s"]
    light = run(pool, True, np.cumsum(rng.exponential(1.0 / light_rate, size=int(light_rate * 10))))
    light["rate_per_s"] = light_rate
    # host payloads (pinned), H2D inside each request
    hpool = [dict(q, AT=q["AT"].cpu().pin_memory(), B=q["B"].cpu().pin_memory()) for q in pool[:64]]
    host = run(hpool, True, np.cumsum(rng.exponential(1.0 / light_rate, size=int(light_rate * 10))))
    host["rate_per_s"] = light_rate
    h2d = float(np.mean([q["AT"].numel() * 4 + q["B"].numel() * 4 for q in hpool]))
    d2h = float(np.mean([q["d"] * q["b"] * 8 for q in hpool]))
    del hpool
    fp64 = None
    if args.compare_fp64:
        pool64 = [dict(q, AT=q["AT"].double(), B=q["B"].double()) for q in pool]
        fp64 = run(pool64, False, arrivals)
        del pool64
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": main_run["products_per_s"], "unit": "products/s", "n_gpus": world,
        "steps": main_run["requests"], "warmup": len(pool), "ms_per_step": 1e3 / main_run["products_per_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (mixed: FP32 transforms, FP64 reduction)", "data": "synthetic", "config": config,
        "latency_ms": {"p50": main_run["p50_ms"], "p99": main_run["p99_ms"], "mean": main_run["mean_ms"]},
        "serving": main_run, "serving_without_code_cache": no_cache, "unsaturated": light, "host_payload": host,
        "e2e": {"value": host["products_per_s"], "unit": "products/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": main_run["launches"], "clocks": main_run["clocks"], "roofline": None, "cpu_baseline": None,
    }
    if fp64 is not None:
        line["plain_fp64_same_stream"] = fp64
        line["plain_fp64_same_stream"]["speedup"] = main_run["products_per_s"] / fp64["products_per_s"]
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- main
def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "config4":
        bench_batch(args, world, rank, local)
        return
    if args.workload == "config5":
        bench_serve(args, world, rank, local)
        return
    from compmatmul_b200.planted import WORKLOADS, planted_problem
    w = dict(WORKLOADS[args.workload])
    if args.n:
        w["n"] = args.n
    n, K, d, b = w["n"], w["K"], w["d"], w["b"]
    variant = args.variant
    mixed = args.precision == "mixed" or (args.precision == "auto" and w.get("dtype") == "float32")
    config = {"workload": f"{args.workload}: planted-entry A,B {n}x{n} {'FP32' if mixed else 'FP64'} (noise N(0,0.01^2), "
                          f"K={K} planted +10/+10), {variant.upper()}, b={b}, d={d}, "
                          f"hash=multiply-add-shift; dense median decompression + top-{K}",
              "n": n, "b": b, "d": d, "K": K, "variant": variant,
              "l2": "inputs (2x8n^2 bytes) larger than L2, no flush"}

    if args.impl == "reference":
        if rank != 0:
            return
        AT, B, _ = planted_problem(n, n, n, K, w["gen_seed"])
        steps = []
        thr, sample = 0, ""
        for _ in range(max(1, args.steps)):
            sec, thr, sample = cpu_reference_sample(AT, B, n, d, b, variant, w["seed"],
                                                    args.cpu_seconds / max(1, args.steps) + 2)
            steps.append(sec)
        sec = float(np.median(steps))
        val = 1.0 / sec
        line = {"metric": METRIC, "value": val, "unit": "products/s", "impl": "reference",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                "cpu_baseline": {"value": val, "unit": "products/s", "cores": thr,
                                 "kind": "reference", "sample": sample},
                "e2e": {"value": val, "unit": "products/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import compmatmul_b200 as cmb
    from compmatmul_b200 import device as dev
    from compmatmul_b200.replicas import Replicas

    reps = Replicas()
    L = cmb.lib()
    dv = torch.device("cuda", torch.cuda.current_device())

    # inputs: per-rank seeds (independent products), pinned host + HBM copies
    AT, B, planted = planted_problem(n, n, n, K, w["gen_seed"] + 1000 * rank,
                                     dtype=np.float32 if mixed else np.float64)
    hAT = torch.from_numpy(AT).pin_memory()
    hB = torch.from_numpy(B).pin_memory()
    dAT = hAT.to(dv)
    dB = hB.to(dv)
    dC = torch.empty((n, n), dtype=torch.float64, device=dv)
    seed = w["seed"] + rank

    def step():
        dev.matmul(dAT, dB, d, b, seed, variant=variant, out=dC)
        return dev.topk(dC, K, as_numpy=False)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    barrier = reps.barrier
    clocks = ClockSampler(torch.cuda.current_device())
    L.cmm_profile_reset()
    L.cmm_profile_enable(1)
    launches0 = L.cmm_launch_count()
    barrier()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        out = step()
    ev1.record()
    barrier()
    clk = clocks.stop()
    launches = L.cmm_launch_count() - launches0
    L.cmm_profile_enable(0)
    total_ms = ev0.elapsed_time(ev1)
    fam = {f: cmb.profile_read(f) for f in ("hash", "scale", "plan", "materialize", "sketch",
                                             "finalize", "decompress", "topk")}
    sketch_kernel = L.cmm_last_sketch_kernel().decode()
    value = reps.throughput(args.steps, total_ms / 1e3)  # products of all ranks / slowest rank
    total_ms = reps.max(total_ms)
    ms_per_step = total_ms / args.steps

    # recovery check on this rank's last step (planted entries should be the top-K)
    ti, tj, tv = [x.cpu().numpy() for x in out]
    rec = len(set(zip(ti.tolist(), tj.tolist())) & set(zip(planted[0].tolist(), planted[2].tolist())))

    # end to end through the C ABI with host (pinned) buffers
    hC = torch.empty((n, n), dtype=torch.float64).pin_memory()
    e2e_steps = max(1, args.e2e_steps)
    import ctypes as C
    for i in range(e2e_steps + 1):
        if i == 1:
            barrier()
            te0 = time.perf_counter()
        fn = L.cmm_matmul_f32 if mixed else L.cmm_matmul
        st = fn(0 if variant == "fft" else 1, 1, n, n, n, C.c_void_p(hC.data_ptr()),
                C.c_void_p(hAT.data_ptr()), C.c_void_p(hB.data_ptr()), d, b, 1, seed)
        cmb.check(st)
    barrier()
    e2e_s = (time.perf_counter() - te0) / e2e_steps
    e2e_value = reps.throughput(1, e2e_s)

    # the plain FP64 path on the same (FP32-valued) inputs, for the mixed speed-up
    fp64_ms = None
    if mixed and args.compare_fp64:
        dAT64 = dAT.double()
        dB64 = dB.double()
        for i in range(args.compare_fp64 + 1):
            if i == 1:
                torch.cuda.synchronize()
                tf0 = time.perf_counter()
            dev.matmul(dAT64, dB64, d, b, seed, variant=variant, out=dC)
            dev.topk(dC, K, as_numpy=False)
        torch.cuda.synchronize()
        fp64_ms = (time.perf_counter() - tf0) / args.compare_fp64 * 1e3
        del dAT64, dB64

    # roofline of the dominant kernel (the sketch kernel): one launch covers a
    # chunk of the inner indices; per launch it must read the chunk's row
    # pairs once per repetition (d * k_chunk * (n_a + n_b) elements) and does
    # the chunk's share of the transform arithmetic
    sk_ms, sk_n = fam["sketch"]
    sk_launch_ms = sk_ms / max(1, sk_n)
    chunks = max(1, sk_n // max(1, args.steps))  # launches per product
    esz = 4.0 if mixed else 8.0
    alg_bytes = esz * d * n * (n + n) / chunks
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (sk_launch_ms / 1e3) / 1e9
    flops = (fft_flops(n, n, n, d, b) if variant == "fft" else fwht_ops(n, n, n, d, b)) / chunks
    ratio = TRAFFIC_RATIO.get((sketch_kernel, variant, "f32" if mixed else "f64"))
    import ctypes as C
    fma_peak = None
    tf = C.c_double(0.0)
    if L.cmm_probe_fma_tflops(0 if mixed else 1, C.byref(tf)) == 0:
        fma_peak = tf.value

    if rank != 0:
        reps.close()
        return

    cpu = None
    if world == 1 and not args.no_cpu_baseline and not mixed:
        try:
            sec, thr, sample = cpu_reference_sample(AT, B, n, d, b, variant, seed, args.cpu_seconds)
            cpu = {"value": 1.0 / sec, "unit": "products/s", "cores": thr, "kind": "reference",
                   "sample": sample}
        except Exception as e:  # the checker binary may be absent
            cpu = {"value": None, "unit": "products/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    line = {
        "metric": METRIC, "value": value, "unit": "products/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (mixed: FP32 transforms, FP64 reduction)" if mixed else "f64",
        "data": "synthetic", "config": config,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": ratio * alg_bytes if ratio else None,
                     "traffic_source": "ncu small case scaled by units" if ratio else None,
                     "kernel": f"sketch ({sketch_kernel})", "peak_source": peak_kind,
                     "launch_ms": sk_launch_ms, "launches_per_product": chunks,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "binding": {"bound": "fp32" if mixed else "fp64",
                                 "achieved": flops / (sk_launch_ms / 1e3) / 1e12,
                                 "peak": fma_peak, "unit": "TFLOP/s",
                                 "frac": (flops / (sk_launch_ms / 1e3) / 1e12 / fma_peak) if fma_peak else None,
                                 "peak_source": "measured FMA loop (cmm_probe_fma_tflops)",
                                 "flops_per_launch": flops}},
        "kernel_ms_per_step": {k: v[0] / max(1, args.steps) for k, v in fam.items()},
        "e2e": {"value": e2e_value, "unit": "products/s", "h2d_bytes_per_step": int(2 * esz * n * n),
                "d2h_bytes_per_step": int(8 * n * n)},
        "gpu_launches": int(launches),
        "clocks": clk,
        "recovered_planted": f"{rec}/{K}",
        "cpu_baseline": cpu,
    }
    if fp64_ms is not None:
        line["plain_fp64_same_inputs"] = {"ms_per_step": fp64_ms, "speedup": fp64_ms / ms_per_step}
    print(json.dumps(line), flush=True)
    reps.close()


if __name__ == "__main__":
    main()
