"""A small, self-contained case of the batched kernel for profilers.

    python -m spin_systems_b200.profile_case [--realizations N] [--blocks B]
        [--nspins L] [--precision mixed|fp64] [--repeat K]

Runs the XY-8 finite-pulse workload (the benchmark's shape with fewer
realisations and XY-8 blocks) through the batched engine: one upload, then
`repeat` executions, so a profiler can skip the first launch and capture a
warm one.  Prints one line with the wall time per execution.
"""
from __future__ import annotations

import argparse
import time

import spin_systems_b200 as ss
from spin_systems_b200 import abi, workloads


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--realizations", type=int, default=296)
    ap.add_argument("--blocks", type=int, default=2)
    ap.add_argument("--nspins", type=int, default=12)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--repeat", type=int, default=2)
    args = ap.parse_args()
    spec = workloads.xy8_finite(nspins=args.nspins, realizations=args.realizations,
                                blocks=args.blocks)
    prec = abi.MIXED if args.precision == "mixed" else abi.FP64
    with ss.Engine(0) as eng:
        batch = ss.Batch(eng, spec.config(), 0, args.realizations, prec)
        batch.upload()
        for _ in range(args.repeat):
            t0 = time.perf_counter()
            batch.execute()
            eng.synchronize()
            dt = time.perf_counter() - t0
        stats = batch.stats()
        print(f"profile_case L={args.nspins} n={args.realizations} blocks={args.blocks} "
              f"{args.precision}: {dt * 1e3:.2f} ms/execute, "
              f"{stats['amplitude_orders']:.3e} amplitude-orders")
        del batch


if __name__ == "__main__":
    main()
