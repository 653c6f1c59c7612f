"""Benchmark of the compressed product on B200.

One step = one compressed product of a planted-entry workload: hash codes,
per-k balancing, fused sketch/transform/accumulate, inverse, dense median
decompression of all n_a x n_b entries into HBM, and device top-K recovery
(K = planted count).  Default workload: n = 16384 square FP64, b = 2^16,
d = 9, FFT variant, K = 256 (inputs 4.3 GB > L2, so no flush is needed).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--variant fft|fwht]
                  [--workload config2_n16384|config2_n4096|config1|config3|config4|config5|wht_rows]
                  [--impl reference] [--no-legs] [--inner K]

The default single-GPU run also measures the other workloads as short legs,
reported as extra keys of the same JSON line ("legs"): config 2 FWHT at
n = 16384, config 1 (n = 512, FFT), config 2 at n = 4096 (both variants),
config 3 (mixed precision, FFT and FWHT, against the FP64 path on the same
inputs), the FP32 FWHT with its Hadamard-16 stages on the tensor cores
(tcgen05) against CUDA cores on the same rows, config 4 (256 uneven
products in one batch plan) and a bounded config 5 serving run.
Each leg states its steps, its clocks and its result check.

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
GOLDEN = os.path.join(ROOT, "tests", "golden")


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config2_n16384")
    ap.add_argument("--variant", default="fft", choices=["fft", "fwht"])
    ap.add_argument("--e2e-steps", type=int, default=2, help="0 skips the end-to-end legs")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-legs", action="store_true", help="headline workload only")
    ap.add_argument("--ref-fraction", type=float, default=0.125,
                    help="share of one product (inner indices and decompressed rows) per CPU reference step")
    ap.add_argument("--n", type=int, default=0, help="override the workload size")
    ap.add_argument("--inner", type=int, default=0,
                    help="override the inner dimension (a small case of the same kernels, for profiler captures)")
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
    ap.add_argument("--serve-pool", type=int, default=256, help="config5: distinct request inputs")
    ap.add_argument("--serve-cache-gb", type=float, default=4.0,
                    help="config5: resident hash codes + plans across requests (0: off)")
    ap.add_argument("--serve-extra", type=int, default=1,
                    help="config5: also run without the code cache, unsaturated, and with host payloads")
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed"],
                    help="fp64 = plain path; mixed = FP32 inputs (default for config3)")
    return ap.parse_args(argv)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            m = json.load(f)
        return float(m.get("hbm_gbs", HBM_PEAK_FALLBACK)), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return HBM_PEAK_FALLBACK, "fallback (6.65 TB/s, earlier copy measurement on this GPU type)"


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
        return self

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


def fma_peak(L, fp64):
    """FMA throughput of this GPU (TFLOP/s, 2 flops per FMA), measured now by
    the library's register-resident FMA loop (cmm_probe_fma_tflops)."""
    import ctypes as C
    tf = C.c_double(0.0)
    return tf.value if L.cmm_probe_fma_tflops(1 if fp64 else 0, C.byref(tf)) == 0 else None


def time_events(fn, warm, steps):
    """(ms per call, clocks) of fn() with CUDA events on the current stream,
    after `warm` untimed calls; nvidia-smi samples the clocks meanwhile."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device()).start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, clocks.stop()


def golden_sets(workload, variant):
    """(i, j, v) top-K of the reference's own dense estimate for a named
    workload (tests/golden/<workload>.npz, made by the reference), or None."""
    path = os.path.join(GOLDEN, f"{workload}.npz")
    if not os.path.exists(path):
        return None
    z = np.load(path)
    if f"{variant}_top_i" not in z.files:
        return None
    return z[f"{variant}_top_i"], z[f"{variant}_top_j"], z[f"{variant}_top_v"]


def set_check(ours, ref):
    """Recovered (i, j) set equal to the reference's, and the max relative
    difference of the recovered values."""
    oi, oj, ov = (np.asarray(x) for x in ours)
    ri, rj, rv = (np.asarray(x) for x in ref)
    same = set(zip(oi.tolist(), oj.tolist())) == set(zip(ri.tolist(), rj.tolist()))
    mine = {(int(i), int(j)): float(v) for i, j, v in zip(oi, oj, ov)}
    rel = 0.0
    for i, j, v in zip(ri, rj, rv):
        got = mine.get((int(i), int(j)))
        rel = max(rel, float("inf") if got is None else abs(got - float(v)) / max(abs(float(v)), 1e-300))
    return {"same_set_as_reference": bool(same), "max_rel_diff_vs_reference": float(rel)}


# ------------------------------------------------------------- CPU legs
def cpu_reference_sample(AT, B, n, d, b, variant, seed, fraction):
    """The reference's own CPU path (its headers and binding compiled with
    the project shims, oracle/_ref) on a fixed share of one product: the
    compressed product over the first `fraction` of the inner indices and
    the dense decompression of the first `fraction` of the rows.  Both
    phases are linear in those counts, so one such sample is `fraction` of
    a product.  Returns (seconds, fraction actually used, threads, sample)."""
    from oracle.oracle import RefLib
    rl = RefLib()
    thr = rl.num_threads()
    ks = max(8, int(round(n * fraction)))
    rows = max(8, int(round(n * fraction)))
    t0 = time.perf_counter()
    p = rl.compressed_product(variant, None, AT[:ks], B[:ks], d, b, seed)
    ts = time.perf_counter() - t0
    Cbuf = np.empty((rows, n))
    t0 = time.perf_counter()
    rl.decompress_rows(variant, None, p, d, b, seed, n, 0, rows, Cbuf)
    tdec = time.perf_counter() - t0
    frac = ks / n  # == rows / n
    sample = (f"reference CPU path ({variant}, {thr} threads) on a {frac:.4g} share of one product: the "
              f"compressed product over the first {ks} of {n} inner indices ({ts:.2f} s) and the dense "
              f"decompression of the first {rows} of {n} rows ({tdec:.2f} s)")
    return ts + tdec, frac, thr, sample


# ------------------------------------------------- batched products (config 4)
def product_flops(s):
    f = fft_flops if s["variant"] == "fft" else fwht_ops
    return f(s["m"], s["n"], s["p"], s["d"], s["b"])


def batch_config(count):
    return {"workload": f"config4: {count} planted products m x n x p, each dimension log-uniform in "
                        f"[256, 4096], FP32 noise N(0,0.01^2) + K=max(8,m/64) planted +10/+10, "
                        f"b = next pow2 >= 256 K, d in {{5,7,9}}, FFT/FWHT 50/50; sketch + dense median "
                        f"estimate per product",
            "products": count, "l2": "inputs (sum 4 n (m+p) bytes) larger than L2, no flush"}


def batch_reference(args):
    from oracle.oracle import RefLib
    from compmatmul_b200.planted import batch_shapes, planted_problem
    count = args.batch_count
    shapes = batch_shapes(count=count, seed=4004)
    flops_total = sum(product_flops(s) for s in shapes)
    rl = RefLib()
    t_used, f_used, done = 0.0, 0.0, 0
    for s in shapes:
        AT, B, _ = planted_problem(s["m"], s["n"], s["p"], s["K"], s["gen_seed"], dtype=np.float32)
        t0 = time.perf_counter()
        rl.matmul(s["variant"], None, AT.astype(np.float64), B.astype(np.float64), s["d"], s["b"], s["seed"])
        t_used += time.perf_counter() - t0
        f_used += product_flops(s)
        done += 1
        if t_used > 12.0:
            break
    frac = f_used / flops_total
    val = count * frac / t_used
    sample = (f"reference CPU path (headers compiled with shims, {rl.num_threads()} threads, FP64 on the "
              f"FP32-valued inputs) on the first {done} of {count} products ({t_used:.1f} s, {frac:.3f} of "
              f"the batch's modelled flops)")
    return {"metric": METRIC, "value": val, "unit": "products/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": t_used * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": batch_config(count),
            "cpu_baseline": {"value": val, "unit": "products/s", "cores": rl.num_threads(),
                             "kind": "reference", "sample": sample},
            "e2e": {"value": val, "unit": "products/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_batch(args, reps, warm, steps, compare_fp64, e2e_steps):
    """Config 4: `batch_count` uneven planted products (FP32 inputs) as one
    batch plan -- one persistent sketch launch over a work queue, the whole
    batch replayed from a CUDA graph.  A step is one run of all products
    (sketches + dense median estimates).  With compare_fp64 the plain FP64
    path runs on the same inputs, batched and as one call per product.
    Returns the fields of a bench line."""
    import torch
    import compmatmul_b200 as cmb
    from compmatmul_b200 import device as dev
    from compmatmul_b200.batch import BatchPlan
    from compmatmul_b200.planted import batch_shapes, planted_problem_device
    L = cmb.lib()
    rank = reps.rank
    count = args.batch_count
    shapes = batch_shapes(count=count, seed=4004 + 1000 * rank)
    if args.batch_variant != "both":  # one variant only (component timing)
        shapes = [dict(s, variant=args.batch_variant) for s in shapes]
    flops_total = sum(product_flops(s) for s in shapes)
    prods, planted = [], []
    for s in shapes:
        AT, B, pl = planted_problem_device(s["m"], s["n"], s["p"], s["K"], s["gen_seed"], "float32")
        prods.append(dict(AT=AT, B=B, d=s["d"], b=s["b"], seed=s["seed"], variant=s["variant"]))
        planted.append(pl)
    t0 = time.perf_counter()
    plan = BatchPlan(prods, f32=True, tune=bool(args.batch_tune), dense=True)
    plan_s = time.perf_counter() - t0
    for _ in range(warm):
        plan.run()
    torch.cuda.synchronize()

    clocks = ClockSampler(torch.cuda.current_device())
    L.cmm_profile_reset()
    L.cmm_profile_enable(1)
    launches0 = L.cmm_launch_count()
    reps.barrier()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(steps):
        plan.run()
    ev1.record()
    reps.barrier()
    clk = clocks.stop()
    launches = L.cmm_launch_count() - launches0
    L.cmm_profile_enable(0)
    total_ms = ev0.elapsed_time(ev1)
    value = reps.throughput(count * steps, total_ms / 1e3)
    ms_per_step = reps.max(total_ms) / steps
    info = plan.info()

    # the persistent sketch kernel alone, event-timed on its stream
    L.cmm_profile_reset()
    L.cmm_profile_enable(1)
    plan.run()
    torch.cuda.synchronize()
    L.cmm_profile_enable(0)
    batch_ms = cmb.profile_read("batch")[0]

    rec = tot = 0
    for q, (is_, ks, js), s in zip(plan.products, planted, shapes):
        ti, tj, _ = dev.topk(q["C"], s["K"])
        rec += len(set(zip(ti.tolist(), tj.tolist())) & set(zip(is_.tolist(), js.tolist())))
        tot += s["K"]

    fp64 = None
    if compare_fp64:
        prods64 = [dict(q, AT=q["AT"].double(), B=q["B"].double()) for q in prods]
        plan64 = BatchPlan(prods64, f32=False, tune=bool(args.batch_tune), dense=True)
        b64, _ = time_events(plan64.run, 2, compare_fp64)
        outs = [torch.empty((q["AT"].shape[1], q["B"].shape[1]), dtype=torch.float64, device="cuda")
                for q in prods64]

        def singles():
            for q, o in zip(prods64, outs):
                dev.matmul(q["AT"], q["B"], q["d"], q["b"], q["seed"], variant=q["variant"], out=o)
        single64, _ = time_events(singles, 1, 1)
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

    e2e = None
    if e2e_steps > 0:
        hin = [(torch.empty_like(q["AT"], device="cpu").pin_memory(),
                torch.empty_like(q["B"], device="cpu").pin_memory()) for q in prods]
        hout = [torch.empty_like(q["C"], device="cpu").pin_memory() for q in plan.products]
        for (ha, hb), q in zip(hin, prods):
            ha.copy_(q["AT"])
            hb.copy_(q["B"])
        h2d = sum(ha.numel() * 4 + hb.numel() * 4 for ha, hb in hin)
        d2h = sum(o.numel() * 8 for o in hout)
        reps.barrier()
        te0 = time.perf_counter()
        for _ in range(e2e_steps):
            for (ha, hb), q in zip(hin, prods):
                q["AT"].copy_(ha, non_blocking=True)
                q["B"].copy_(hb, non_blocking=True)
            plan.run()
            for o, q in zip(hout, plan.products):
                o.copy_(q["C"], non_blocking=True)
            torch.cuda.synchronize()
        reps.barrier()
        e2e = {"value": reps.throughput(count, (time.perf_counter() - te0) / e2e_steps), "unit": "products/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "api": "BatchPlan.run with pinned host inputs copied in and dense estimates copied out"}
        del hin, hout

    peak_tf = fma_peak(L, fp64=False)
    alg_bytes = sum(4.0 * s["n"] * (s["m"] + s["p"]) for s in shapes)
    peak, peak_kind = measured_peaks()
    achieved_tf = flops_total / (batch_ms / 1e3) / 1e12
    out = {
        "value": value, "ms_per_step": ms_per_step, "steps": steps, "warmup": warm,
        "roofline": {"bound": "fp32", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": achieved_tf / peak_tf if peak_tf else None, "traffic": None,
                     "peak_source": "measured now on this GPU by the library's FMA loop (cmm_probe_fma_tflops)",
                     "kernel": "batch graph (persistent k_batch_sketch + finalize + dense decompress)",
                     "launch_ms": batch_ms, "flops_per_launch": flops_total,
                     "hbm": {"achieved": alg_bytes / (batch_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                             "frac": alg_bytes / (batch_ms / 1e3) / 1e9 / peak, "peak_source": peak_kind,
                             "algorithmic_bytes_per_launch": alg_bytes}},
        "e2e": e2e, "gpu_launches": int(launches), "clocks": clk, "recovered_planted": f"{rec}/{tot}",
        "batch": {"items": info["items"], "ctas": info["ctas"], "launches_per_run": info["launches"],
                  "plan_and_tune_s": plan_s},
    }
    if fp64 is not None:
        out["plain_fp64_same_inputs"] = fp64
    plan.close()
    return out


def bench_batch(args, world, rank, local):
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(batch_reference(args)), flush=True)
        return
    from compmatmul_b200.replicas import Replicas
    reps = Replicas()
    r = run_batch(args, reps, args.warmup, args.steps, args.compare_fp64, args.e2e_steps)
    if rank == 0:
        line = {"metric": METRIC, "value": r.pop("value"), "unit": "products/s", "n_gpus": world,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (mixed: FP32 transforms, FP64 reduction)", "data": "synthetic",
                "config": batch_config(args.batch_count), "cpu_baseline": None}
        line.update(r)
        print(json.dumps(line), flush=True)
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


def serve_config(args):
    rate, secs = args.serve_rate, args.serve_seconds
    return {"workload": f"config5: Poisson arrivals at {rate:g} req/s for {secs:g} s; each request one compressed "
                        f"product sized as config4 (m, n, p log-uniform in [256, 4096], FP32, planted, "
                        f"b = next pow2 >= 256 K, d in {{5,7,9}}, FFT/FWHT 50/50) from a pool of "
                        f"{args.serve_pool} inputs; admission cap {args.serve_cap_gb:g} GB; resident hash codes + "
                        f"plans {args.serve_cache_gb:g} GB; result = sketch p",
            "rate_per_s": rate, "seconds": secs, "cap_bytes": int(args.serve_cap_gb * (1 << 30))}


def run_serve(args, rank, extra, compare_fp64, compare_fp64_window=1e9):
    """Config 5: Poisson arrivals of requests sized as the batched config,
    served with continuous batching under a device-memory admission cap.
    Returns the fields of a bench line."""
    import torch
    import compmatmul_b200 as cmb
    from compmatmul_b200.batch import BatchPlan
    from compmatmul_b200.planted import batch_shapes, planted_problem_device
    from compmatmul_b200.serve import Server
    rate, secs, cap = args.serve_rate, args.serve_seconds, int(args.serve_cap_gb * (1 << 30))
    shapes = batch_shapes(count=args.serve_pool, seed=5005 + 1000 * rank)
    pool = []
    for sh in shapes:
        AT, B, _ = planted_problem_device(sh["m"], sh["n"], sh["p"], sh["K"], sh["gen_seed"], "float32")
        pool.append(dict(AT=AT, B=B, d=sh["d"], b=sh["b"], seed=sh["seed"], variant=sh["variant"]))
    # the autotuner's cache covers the request classes before the stream starts
    BatchPlan(pool, f32=True, tune=True, dense=False).close()
    rng = np.random.default_rng(77 + rank)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * secs)))
    L = cmb.lib()

    def run(pool_, f32, arr, cache=int(args.serve_cache_gb * (1 << 30))):
        srv = Server(mem_cap_bytes=cap, f32=f32, streams=args.serve_streams, max_wave=args.serve_max_wave,
                     cache_bytes=cache)
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
        return {"products_per_s": len(lat) / span, "offered_per_s": len(arr) / float(arr[-1]),
                "cache_bytes": cache, "cache_hits": int(st["cache_hits"] - st0["cache_hits"]),
                "cache_misses": int(st["cache_misses"] - st0["cache_misses"]),
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3), "requests": int(len(lat)), "span_s": span,
                "waves": int(st["waves"] - st0["waves"]), "max_waves_in_flight": int(st["max_waves_in_flight"]),
                "max_mem_in_use_bytes": int(st["max_mem_in_use"]), "launches": int(L.cmm_launch_count() - l0),
                "clocks": clk}

    main_run = run(pool, True, arrivals)
    # steady state: the server completed requests as fast as they arrived
    # (over the whole run, drain included)
    main_run["kept_up"] = bool(main_run["products_per_s"] >= 0.97 * main_run["offered_per_s"])
    out = {"value": main_run["products_per_s"], "steps": main_run["requests"], "warmup": len(pool),
           "ms_per_step": 1e3 / main_run["products_per_s"],
           "latency_ms": {"p50": main_run["p50_ms"], "p99": main_run["p99_ms"], "mean": main_run["mean_ms"]},
           "serving": main_run, "gpu_launches": main_run["launches"], "clocks": main_run["clocks"]}
    if extra:
        if args.serve_cache_gb > 0:  # every request hashing and planning for itself
            out["serving_without_code_cache"] = run(pool, True, arrivals, cache=0)
        light_rate = 0.5 * main_run["products_per_s"]  # latency without queueing
        light = run(pool, True, np.cumsum(rng.exponential(1.0 / light_rate, size=int(light_rate * 10))))
        light["rate_per_s"] = light_rate
        out["unsaturated"] = light
    # host payloads (pinned), H2D inside each request
    hpool = [dict(q, AT=q["AT"].cpu().pin_memory(), B=q["B"].cpu().pin_memory()) for q in pool[:64]]
    host_rate = min(rate, 0.5 * main_run["products_per_s"])
    host = run(hpool, True, np.cumsum(rng.exponential(1.0 / host_rate, size=int(host_rate * min(secs, 10)))))
    host["rate_per_s"] = host_rate
    out["host_payload"] = host
    out["e2e"] = {"value": host["products_per_s"], "unit": "products/s",
                  "h2d_bytes_per_step": int(np.mean([q["AT"].numel() * 4 + q["B"].numel() * 4 for q in hpool])),
                  "d2h_bytes_per_step": int(np.mean([q["d"] * q["b"] * 8 for q in hpool])),
                  "api": "Server.submit with pinned host inputs; p copied back per request"}
    del hpool
    if compare_fp64:
        # the plain FP64 server on the same inputs and the same arrivals (the
        # first `window_s` seconds of the stream, which bounds the run's
        # length when FP64 falls behind); a failure here is reported beside
        # the mixed result instead of replacing it
        pool64 = None
        try:
            pool64 = [dict(q, AT=q["AT"].double(), B=q["B"].double()) for q in pool]
            win = min(secs, float(compare_fp64_window))
            fp64 = run(pool64, False, arrivals[arrivals < win])
            fp64["window_s"] = win
            fp64["mixed_products_per_s"] = main_run["products_per_s"]
            fp64["mixed_speedup"] = main_run["products_per_s"] / fp64["products_per_s"]
            out["plain_fp64_same_stream"] = fp64
        except Exception as e:
            out["plain_fp64_same_stream"] = {"error": f"{type(e).__name__}: {e}"}
        del pool64
        torch.cuda.empty_cache()
    return out


def bench_serve(args, world, rank, local):
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving loop; its per-product "
                              "CPU cost is the config4 reference line"}), flush=True)
        return
    import torch
    torch.cuda.set_device(local if world > 1 else 0)
    r = run_serve(args, rank, bool(args.serve_extra), args.compare_fp64)
    if rank == 0:
        line = {"metric": METRIC, "value": r.pop("value"), "unit": "products/s", "n_gpus": world,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (mixed: FP32 transforms, FP64 reduction)", "data": "synthetic",
                "config": serve_config(args), "roofline": None, "cpu_baseline": None}
        line.update(r)
        print(json.dumps(line), flush=True)


# ------------------------------------------------------- single products
def single_config(workload, n, n_inner, K, d, b, variant, mixed):
    return {"workload": f"{workload}: planted-entry A,B {n}x{n_inner} / {n_inner}x{n} "
                        f"{'FP32' if mixed else 'FP64'} (noise N(0,0.01^2), K={K} planted +10/+10), "
                        f"{variant.upper()}, b={b}, d={d}, hash=multiply-add-shift; dense median "
                        f"decompression + top-{K}",
            "n": n, "n_inner": n_inner, "b": b, "d": d, "K": K, "variant": variant,
            "l2": "inputs (2 x e n^2 bytes) larger than L2, no flush"}


def leg_product(name, AT, B, d, b, seed, variant, K, warm, steps, golden=None, planted=None, out=None):
    """One named single-product leg on device inputs: event-timed dense
    product + top-K, with the recovered set checked against the reference's
    (golden) when given, and recall of the planted entries."""
    import torch
    from compmatmul_b200 import device as dev
    n_a, n_b = AT.shape[1], B.shape[1]
    dC = out if out is not None else torch.empty((n_a, n_b), dtype=torch.float64, device=AT.device)
    res = {}

    def step():
        dev.matmul(AT, B, d, b, seed, variant=variant, out=dC)
        res["top"] = dev.topk(dC, K, as_numpy=False)
    ms, clk = time_events(step, warm, steps)
    top = [x.cpu().numpy() for x in res["top"]]
    leg = {"workload": name, "variant": variant, "dtype": "f64" if AT.dtype == torch.float64 else "f32 (mixed)",
           "n_a": n_a, "n_inner": AT.shape[0], "n_b": n_b, "b": b, "d": d, "K": K, "warmup": warm, "steps": steps,
           "ms_per_step": ms, "products_per_s": 1e3 / ms, "clocks": clk}
    if golden is not None:
        leg.update(set_check(top, golden))
    if planted is not None:
        leg["recovered_planted"] = (f"{len(set(zip(top[0].tolist(), top[1].tolist())) & set(zip(planted[0].tolist(), planted[2].tolist())))}/{K}")
    return leg, top, dC


def leg_mixed_vs_fp64(workload, variant, warm=2, steps=3, warm64=1, steps64=2):
    """Config 3: the mixed-precision path on FP32 planted inputs against the
    plain FP64 path on the same (FP32-valued) inputs: both times, the
    speed-up, recovered-set equality and the max relative error of the
    recovered values against FP64."""
    import torch
    from compmatmul_b200.planted import WORKLOADS, planted_problem_device
    w = WORKLOADS[workload]
    n, K, d, b = w["n"], w["K"], w["d"], w["b"]
    AT, B, planted = planted_problem_device(n, n, n, K, w["gen_seed"], "float32")
    C32 = torch.empty((n, n), dtype=torch.float64, device=AT.device)
    mixed, top32, _ = leg_product(workload, AT, B, d, b, w["seed"], variant, K, warm, steps, planted=planted, out=C32)
    AT64, B64 = AT.double(), B.double()
    del AT, B
    fp64, top64, C64 = leg_product(workload, AT64, B64, d, b, w["seed"], variant, K, warm64, steps64,
                                   planted=planted)
    del AT64, B64
    i64 = torch.as_tensor(top64[0].astype(np.int64), device=C32.device)
    j64 = torch.as_tensor(top64[1].astype(np.int64), device=C32.device)
    got = C32[i64, j64].cpu().numpy()
    want = C64[i64, j64].cpu().numpy()
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    dense_diff = float((C32 - C64).abs().max())
    mixed.update({"fp64_same_inputs": {"ms_per_step": fp64["ms_per_step"], "clocks": fp64["clocks"],
                                       "recovered_planted": fp64["recovered_planted"]},
                  "speedup_vs_fp64": fp64["ms_per_step"] / mixed["ms_per_step"],
                  "same_set_as_fp64": set(zip(top32[0].tolist(), top32[1].tolist()))
                  == set(zip(top64[0].tolist(), top64[1].tolist())),
                  "max_rel_err_recovered_vs_fp64": float(rel.max()),
                  "max_abs_diff_dense_vs_fp64": dense_diff})
    del C32, C64
    torch.cuda.empty_cache()
    return mixed


def leg_wht_rows(rows=16384, log2n=13, warm=3, steps=1000):
    """The FWHT's Hadamard-16 stages on the tensor cores (tcgen05 MMAs on
    BF16 hi/mid/lo splits, FP32 accumulators in tensor memory) against the
    same batched transform on CUDA cores: rows of 2^13 FP32 values (the
    mixed FWHT's slab length), 512 MB in and out per call (over L2).  Each
    call is synchronous; the time includes one host round trip per call.
    1000 calls per form keep the timed region long enough for the clock
    samples."""
    import torch
    from compmatmul_b200 import device
    g = torch.Generator(device="cuda").manual_seed(11)
    x = torch.randn((rows, 1 << log2n), device="cuda", generator=g, dtype=torch.float32)
    y = torch.empty_like(x)
    out = {"rows": rows, "row_length": 1 << log2n}
    bytes_per_call = 2 * 4 * rows * (1 << log2n)
    peak, _ = measured_peaks()
    results = {}
    for method in ("cuda", "tensor"):
        ms, clocks = time_events(lambda: device.wht_rows(x, method, out=y), warm, steps)
        results[method] = y.clone()
        out[method] = {"ms_per_call": ms, "clocks": clocks, "hbm_gbs": bytes_per_call / ms / 1e6,
                       "hbm_frac": bytes_per_call / ms / 1e6 / peak}
    # tensor work of the two Hadamard-16 stages: 3 MMAs of 128 x 16 x 16 per 128-row tile
    tflop = 2 * 3 * 2 * 16 * (rows * (1 << log2n)) / 1e12
    out["tensor"]["tensor_tflops"] = tflop / (out["tensor"]["ms_per_call"] * 1e-3)
    out["tensor_vs_cuda"] = out["cuda"]["ms_per_call"] / out["tensor"]["ms_per_call"]
    ref = results["cuda"]
    out["max_abs_diff_tensor_vs_cuda_rel"] = float((results["tensor"] - ref).abs().max() / ref.abs().max())
    del x, y, results, ref
    torch.cuda.empty_cache()
    return out


def run_legs(args, reps, dAT, dB, dC, L):
    """Short legs of the other configurations (single GPU, after the
    headline): every one reports its own steps, clocks and result check."""
    import torch
    from compmatmul_b200.planted import WORKLOADS, planted_problem
    legs = {}

    def guard(name, fn):
        t0 = time.perf_counter()
        try:
            legs[name] = fn()
        except Exception as e:  # a failing leg is reported, not hidden
            legs[name] = {"error": f"{type(e).__name__}: {e}"}
        legs[name]["leg_wall_s"] = time.perf_counter() - t0
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    w = WORKLOADS["config2_n16384"]
    if dAT is not None:  # the headline's device inputs (config 2, n = 16384)
        other = "fwht" if args.variant == "fft" else "fft"
        guard(f"config2_n16384_{other}",
              lambda: leg_product("config2_n16384", dAT, dB, w["d"], w["b"], w["seed"], other, w["K"], 3, 5,
                                  golden=golden_sets("config2_n16384", other), out=dC)[0])
    w1 = WORKLOADS["config1"]

    def config1():
        AT, B, pl = planted_problem(w1["n"], w1["n"], w1["n"], w1["K"], w1["gen_seed"])
        A_d, B_d = torch.from_numpy(AT).cuda(), torch.from_numpy(B).cuda()
        return leg_product("config1", A_d, B_d, w1["d"], w1["b"], w1["seed"], "fft", w1["K"], 3, 20,
                           golden=golden_sets("config1", "fft"), planted=pl)[0]
    guard("config1", config1)
    w4 = WORKLOADS["config2_n4096"]

    def n4096():
        AT, B, pl = planted_problem(w4["n"], w4["n"], w4["n"], w4["K"], w4["gen_seed"])
        A_d, B_d = torch.from_numpy(AT).cuda(), torch.from_numpy(B).cuda()
        out = {}
        for v in ("fft", "fwht"):
            out[v] = leg_product("config2_n4096", A_d, B_d, w4["d"], w4["b"], w4["seed"], v, w4["K"], 3, 10,
                                 golden=golden_sets("config2_n4096", v), planted=pl)[0]
        return out
    guard("config2_n4096", n4096)
    for v in ("fft", "fwht"):
        guard(f"config3_{v}", lambda v=v: leg_mixed_vs_fp64("config3", v))
    guard("wht_rows_tensor_vs_cuda", leg_wht_rows)
    bargs = argparse.Namespace(**vars(args))
    bargs.batch_variant = "both"
    guard("config4", lambda: run_batch(bargs, reps, 2, 3, compare_fp64=2, e2e_steps=1))
    sargs = argparse.Namespace(**vars(args))
    sargs.serve_seconds, sargs.serve_pool = 5.0, 64
    guard("config5", lambda: dict(run_serve(sargs, reps.rank, extra=False, compare_fp64=1,
                                            compare_fp64_window=2.0),
                                  config=serve_config(sargs)))
    return legs


def reference_single(args, w, n, variant, config):
    """--impl reference on a single-product workload: the reference's CPU
    path, each step a fixed share (--ref-fraction) of one product."""
    from compmatmul_b200.planted import planted_problem
    AT, B, _ = planted_problem(n, n, n, w["K"], w["gen_seed"])
    for _ in range(args.warmup):
        cpu_reference_sample(AT, B, n, w["d"], w["b"], variant, w["seed"], args.ref_fraction)
    secs, fracs = [], []
    thr, sample = 0, ""
    for _ in range(max(1, args.steps)):
        s, frac, thr, sample = cpu_reference_sample(AT, B, n, w["d"], w["b"], variant, w["seed"],
                                                    args.ref_fraction)
        secs.append(s)
        fracs.append(frac)
    per = np.array(secs) / np.array(fracs)  # seconds per product, per step
    val = float(np.sum(fracs) / np.sum(secs))
    line = {"metric": METRIC, "value": val, "unit": "products/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": float(np.mean(secs) * 1e3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
            "product_fraction_per_step": float(np.mean(fracs)),
            "step_spread": {"seconds_per_product_min": float(per.min()), "max": float(per.max()),
                            "cv": float(per.std() / per.mean()) if len(per) > 1 else None},
            "cpu_baseline": {"value": val, "unit": "products/s", "cores": thr, "kind": "reference",
                             "sample": sample + f"; each of the {args.steps} timed steps runs one such share"},
            "e2e": {"value": val, "unit": "products/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    if args.workload == "wht_rows":  # the FWHT-of-rows leg alone (--n rows of 2^13)
        if rank == 0:
            print(json.dumps({"workload": "wht_rows",
                              **leg_wht_rows(rows=args.n or 16384, warm=args.warmup, steps=args.steps)}))
        return
    from compmatmul_b200.planted import WORKLOADS, aligned_empty, planted_problem
    w = dict(WORKLOADS[args.workload])
    if args.n:
        w["n"] = args.n
    n, K, d, b = w["n"], w["K"], w["d"], w["b"]
    n_inner = args.inner or n
    K = min(K, n_inner)
    variant = args.variant
    mixed = args.precision == "mixed" or (args.precision == "auto" and w.get("dtype") == "float32")
    config = single_config(args.workload, n, n_inner, K, d, b, variant, mixed)

    if args.impl == "reference":
        if rank == 0:
            reference_single(args, w, n, variant, config)
        return

    import torch
    import compmatmul_b200 as cmb
    from compmatmul_b200 import device as dev
    from compmatmul_b200.replicas import Replicas

    reps = Replicas()
    L = cmb.lib()
    dv = torch.device("cuda", torch.cuda.current_device())

    # inputs: per-rank seeds (independent products); host (64-byte aligned,
    # pageable, as a reference caller holds them) and HBM copies
    AT, B, planted = planted_problem(n, n_inner, n, K, w["gen_seed"] + 1000 * rank,
                                     dtype=np.float32 if mixed else np.float64)
    dAT = torch.from_numpy(AT).to(dv)
    dB = torch.from_numpy(B).to(dv)
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
    import ctypes as C
    phase_cyc, phase_steps = (C.c_double * 6)(), C.c_double(0.0)
    phases_on = L.cmm_cluster_phase_cycles(phase_cyc, C.byref(phase_steps)) == 0  # clears (instrumented builds)
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
    phases = None
    if phases_on and L.cmm_cluster_phase_cycles(phase_cyc, C.byref(phase_steps)) == 0 and phase_steps.value:
        names = ["radix_passes", "wait_staged_row", "scatter", "group_barrier_wait", "combine", "unused"]
        phases = {"cycles_per_cta_step": {nm: phase_cyc[i] / phase_steps.value for i, nm in enumerate(names)},
                  "cta_steps": phase_steps.value,
                  "note": "thread 0 of each CTA, clock64 between phase marks; instrumented build (CMM_PHASE_CLOCKS)"}
    value = reps.throughput(args.steps, total_ms / 1e3)  # products of all ranks / slowest rank
    total_ms = reps.max(total_ms)
    ms_per_step = total_ms / args.steps

    # recovery on this rank's last step: planted entries, and (rank 0, the
    # named workload's own inputs) the reference's recovered set
    ti, tj, tv = [x.cpu().numpy() for x in out]
    rec = len(set(zip(ti.tolist(), tj.tolist())) & set(zip(planted[0].tolist(), planted[2].tolist())))
    ref_check = None
    gold = golden_sets(args.workload, variant) if (rank == 0 and not mixed and not args.n and not args.inner) else None
    if gold is not None:
        ref_check = set_check((ti, tj, tv), gold)

    # end to end through the public APIs, with the inputs on the host and the
    # dense estimate returned to the host inside the timed region:
    #  * the drop-in module (compmatmul.matmul_fft / matmul_fwht) on the
    #    pageable, 64-byte aligned numpy arrays a reference caller passes;
    #  * the C ABI host entry (cmm_matmul) on pinned buffers.
    e2e = e2e_pinned = None
    esz = 4 if mixed else 8
    if args.e2e_steps > 0:
        import ctypes as C
        if not mixed:
            cm = cmb.load_dropin()
            fn = cm.matmul_fft if variant == "fft" else cm.matmul_fwht
            hC = aligned_empty((n, n))
            fn(hC, AT, B, d, b, seed)  # warm (first touch of hC)
            barrier()
            te0 = time.perf_counter()
            for _ in range(args.e2e_steps):
                fn(hC, AT, B, d, b, seed)
            barrier()
            e2e = {"value": reps.throughput(1, (time.perf_counter() - te0) / args.e2e_steps), "unit": "products/s",
                   "h2d_bytes_per_step": int(esz * n_inner * 2 * n), "d2h_bytes_per_step": int(8 * n * n),
                   "api": f"compmatmul.matmul_{variant} (pybind drop-in) on pageable 64-byte aligned numpy arrays"}
            del hC
        hAT = torch.from_numpy(AT).pin_memory()
        hB = torch.from_numpy(B).pin_memory()
        hCp = torch.empty((n, n), dtype=torch.float64).pin_memory()
        cfn = L.cmm_matmul_f32 if mixed else L.cmm_matmul
        for i in range(args.e2e_steps + 1):
            if i == 1:
                barrier()
                te0 = time.perf_counter()
            cmb.check(cfn(0 if variant == "fft" else 1, 1, n, n_inner, n, C.c_void_p(hCp.data_ptr()),
                          C.c_void_p(hAT.data_ptr()), C.c_void_p(hB.data_ptr()), d, b, 1, seed))
        barrier()
        e2e_pinned = {"value": reps.throughput(1, (time.perf_counter() - te0) / args.e2e_steps),
                      "unit": "products/s", "h2d_bytes_per_step": int(esz * n_inner * 2 * n),
                      "d2h_bytes_per_step": int(8 * n * n),
                      "api": "cmm_matmul" + ("_f32" if mixed else "") + " (C ABI host entry) on pinned buffers"}
        del hAT, hB, hCp
        if e2e is None:
            e2e = e2e_pinned

    # the plain FP64 path on the same (FP32-valued) inputs, for the mixed speed-up
    fp64_ms = None
    if mixed and args.compare_fp64:
        dAT64 = dAT.double()
        dB64 = dB.double()

        def step64():
            dev.matmul(dAT64, dB64, d, b, seed, variant=variant, out=dC)
            dev.topk(dC, K, as_numpy=False)
        fp64_ms, _ = time_events(step64, 1, args.compare_fp64)
        del dAT64, dB64

    # Roofline of the dominant kernel (the sketch kernel).  Its binding bound
    # is arithmetic (FP64 for the plain path, FP32 for the mixed one): the
    # transform work of the launch's share of the product, over its event
    # time, against this GPU's FMA peak measured now.  The HBM view counts
    # the algorithmic bytes of the inputs read once (8 n_inner (n_a + n_b)
    # per product, split evenly over the product's sketch launches).
    sk_ms, sk_n = fam["sketch"]
    sk_launch_ms = sk_ms / max(1, sk_n)
    launches_per_product = max(1, sk_n // max(1, args.steps))
    flops = (fft_flops(n, n_inner, n, d, b) if variant == "fft" else fwht_ops(n, n_inner, n, d, b))
    flops /= launches_per_product
    alg_bytes = esz * n_inner * (n + n) / launches_per_product
    peak_tf = fma_peak(L, fp64=not mixed)
    hbm_peak, hbm_kind = measured_peaks()
    achieved_tf = flops / (sk_launch_ms / 1e3) / 1e12
    achieved_gb = alg_bytes / (sk_launch_ms / 1e3) / 1e9
    roofline = {"bound": "fp32" if mixed else "fp64", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
                "frac": achieved_tf / peak_tf if peak_tf else None, "traffic": None,
                "peak_source": "measured now on this GPU by the library's FMA loop (cmm_probe_fma_tflops); "
                               "MEASURED_PEAKS.json has no FP64/FP32 CUDA-core entry",
                "kernel": f"sketch ({sketch_kernel})", "launch_ms": sk_launch_ms,
                "launches_per_product": launches_per_product, "flops_per_launch": flops,
                "hbm": {"achieved": achieved_gb, "peak": hbm_peak, "unit": "GB/s", "frac": achieved_gb / hbm_peak,
                        "peak_source": hbm_kind, "algorithmic_bytes_per_launch": alg_bytes}}

    legs = None
    if world == 1 and not args.no_legs and args.workload == "config2_n16384" and not args.n and not args.inner:
        legs = run_legs(args, reps, dAT if not mixed else None, dB, dC, L)

    if rank != 0:
        reps.close()
        return

    cpu = None
    if world == 1 and not args.no_cpu_baseline and not mixed and not args.inner:
        try:
            sec, frac, thr, sample = cpu_reference_sample(AT, B, n, d, b, variant, seed, args.ref_fraction)
            cpu = {"value": frac / sec, "unit": "products/s", "cores": thr, "kind": "reference",
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
        "roofline": roofline,
        "kernel_ms_per_step": {k: v[0] / max(1, args.steps) for k, v in fam.items()},
        "e2e": e2e, "e2e_capi_pinned": e2e_pinned,
        "gpu_launches": int(launches),
        "clocks": clk,
        "recovered_planted": f"{rec}/{K}",
        "reference_set_check": ref_check,
        "cpu_baseline": cpu,
    }
    if fp64_ms is not None:
        line["plain_fp64_same_inputs"] = {"ms_per_step": fp64_ms, "speedup": fp64_ms / ms_per_step}
    if phases is not None:
        line["cluster_phase_cycles"] = phases
    if legs is not None:
        line["legs"] = legs
    print(json.dumps(line), flush=True)
    reps.close()


if __name__ == "__main__":
    main()
