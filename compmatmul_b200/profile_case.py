"""One compressed product on synthetic device data, for profiler captures.

    python -m compmatmul_b200.profile_case [--variant fft|fwht] [--precision fp64|mixed]
        [--n N] [--k K] [--b B] [--d D] [--reps R]

Runs R compressed products (sketch only: hash codes, plan, sketch kernel,
finalize) of an n x k by k x n problem with inputs N(0, 0.01^2) generated
on the device, then prints one line.  Small shapes keep a profiler capture
of the sketch kernel short (a few hundred MB on the device).
"""
from __future__ import annotations

import argparse


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--variant", default="fft", choices=["fft", "fwht"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--k", type=int, default=512)
    ap.add_argument("--b", type=int, default=1 << 16)
    ap.add_argument("--d", type=int, default=9)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--seed", type=int, default=7)
    a = ap.parse_args()

    import torch

    from . import device, lib
    dt = torch.float32 if a.precision == "mixed" else torch.float64
    g = torch.Generator(device="cuda").manual_seed(1)
    AT = torch.randn((a.k, a.n), generator=g, device="cuda", dtype=dt) * 0.01
    B = torch.randn((a.k, a.n), generator=g, device="cuda", dtype=dt) * 0.01
    p = None
    for _ in range(a.reps):
        p = device.compressed_product(AT, B, a.d, a.b, a.seed, a.variant)
    torch.cuda.synchronize()
    print(f"ok variant={a.variant} precision={a.precision} n={a.n} k={a.k} b={a.b} d={a.d} "
          f"kernel={lib().cmm_last_sketch_kernel().decode()} max|p|={float(p.abs().max()):.6g}")


if __name__ == "__main__":
    main()
