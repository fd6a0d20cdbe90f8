"""Small, self-contained cases of the engine's kernels for profilers.

    python -m spin_systems_b200.profile_case [--realizations N] [--blocks B]
        [--nspins L] [--precision mixed|fp64] [--repeat K]
    python -m spin_systems_b200.profile_case --mlp [--batch B] [--steps S]

Runs the XY-8 finite-pulse workload (the benchmark's shape with fewer
realisations and XY-8 blocks) through the batched engine: one upload, then
`repeat` executions, so a profiler can skip the first launch and capture a
warm one.  Prints one line with the wall time per execution.  With --mlp it
instead trains the surrogate network for `steps` Adam steps on random data
(batches of `batch` rows), so every tcgen05 GEMM shape of a training step
launches `steps` times.
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
    ap.add_argument("--variant", default="",
                    help="force this schedule for the size (see spin_systems_b200.variants())")
    ap.add_argument("--mlp", action="store_true")
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--steps", type=int, default=4)
    args = ap.parse_args()
    if args.mlp:
        import numpy as np
        rng = np.random.default_rng(0)
        x = rng.uniform(-1, 1, size=(4 * args.batch, 6)).astype(np.float32)
        y = np.sin(x @ rng.normal(size=(6, 128))).astype(np.float32)
        with ss.Engine(0) as eng:
            net = ss.Mlp(eng, batch=args.batch, seed=1)
            net.set_data(x, y)
            t0 = time.perf_counter()
            losses = net.train(args.steps, 1e-3, 1e-3, seed=1)
            dt = time.perf_counter() - t0
            print(f"profile_case mlp batch={args.batch} steps={args.steps}: "
                  f"{dt * 1e3 / max(args.steps, 1):.3f} ms/step, loss {losses[-1]:.4g}")
            net._destroy()
        return
    spec = workloads.xy8_finite(nspins=args.nspins, realizations=args.realizations,
                                blocks=args.blocks)
    prec = abi.MIXED if args.precision == "mixed" else abi.FP64
    if args.variant:
        import tempfile
        import torch
        dev = torch.cuda.get_device_name(0)
        with tempfile.NamedTemporaryFile("w", suffix=".tsv", delete=False) as f:
            f.write(f"{dev}\t{args.nspins}\t{args.precision}\t{args.variant}\t1.0\n")
        ss.load_schedule(f.name)
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
              f"{args.precision} {args.variant or 'default'}: {dt * 1e3:.2f} ms/execute, "
              f"{stats['amplitude_orders']:.3e} amplitude-orders")
        del batch


if __name__ == "__main__":
    main()
