"""Throughput of the surrogate's kernels, for measurement and profilers.

    python -m mercury_b200.profile_surrogate [--n 4096] [--batch 1024]
        [--mma-sync] [--train] [--reps 8]

Predicts n random genomes (chunks of `batch`) `reps` times after a warm-up,
or runs `reps` x 50 training steps of `batch` genomes with --train, and
prints genomes/s and the achieved dense FLOP rate.  FLOPs per genome
forward: conv 8->32 (K padded to 27*8), two conv 32->32, 6912->128, 128->128,
128->1; training = 3x the forward.  With ncu, profile one GEMM kernel, e.g.
-k regex:gemm_tc_kernel -s 5 -c 3.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from .surrogate import Surrogate

FWD_FLOP = 2 * 216 * 32 * (27 * 8) + 2 * 2 * 216 * 32 * (27 * 32) + 2 * 6912 * 128 + 2 * 128 * 128 + 2 * 128


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--reps", type=int, default=8)
    ap.add_argument("--mma-sync", action="store_true")
    ap.add_argument("--train", action="store_true")
    args = ap.parse_args()
    rng = np.random.default_rng(0)
    s = Surrogate(0, max_batch=args.batch, seed=0)
    s.use_tcgen05(not args.mma_sync)
    path = "mma.sync" if args.mma_sync else "tcgen05"
    if args.train:
        g = rng.integers(0, 5, (args.batch, 216)).astype(np.uint8)
        t = rng.normal(size=args.batch).astype(np.float32)
        s.train_step(g, t, 1e-4)
        t0 = time.perf_counter()
        for _ in range(args.reps * 50):
            s.train_step(g, t, 1e-4)
        el = time.perf_counter() - t0
        n = args.reps * 50 * args.batch
        print(f"train ({path} forward and input gradients; weight gradients on mma.sync): {n / el:.3e} genomes/s, "
              f"{3 * FWD_FLOP * n / el / 1e12:.1f} TFLOP/s, {el / (args.reps * 50) * 1e3:.3f} ms per step")
        return
    g = rng.integers(0, 5, (args.n, 216)).astype(np.uint8)
    s.predict(g)
    t0 = time.perf_counter()
    for _ in range(args.reps):
        s.predict(g)
    el = time.perf_counter() - t0
    n = args.reps * args.n
    print(f"predict ({path}): {n / el:.3e} genomes/s, {FWD_FLOP * n / el / 1e12:.1f} TFLOP/s "
          f"(host wall, H2D and D2H included), {el / args.reps * 1e3:.3f} ms per {args.n}")


if __name__ == "__main__":
    main()
