#!/usr/bin/env python
"""Benchmark: echo curves/s, batched mixed precision vs plain FP64, on B200.

Workload (one "step" = one batch): XY-8 x16 with finite pulses (evolution for
pi/50 under a transverse field of amplitude 50), tau = 0.25, L = 12 spins,
2D dipolar disorder sigma = 0.5, 1024 realisations per GPU, the S^x echo
correlator at 128 times, state and reference propagated together.  Inputs are
seeded synthetic realisations (seed 20240726, streams per (seed, index)).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --workload cpmg10      the reference's own CPU-runnable case:
      L = 10 ideal-pulse CPMG (pi/2_x, then 8 x (0.5, pi_y, 0.5, measure)),
      sigma = 0.5, 20 realisations, complex128 -- batched FP64 and mixed,
      the plain FP64 path and the reference's CPU build on the same 20

One JSON line on stdout from rank 0.  Multi-GPU: one process per GPU (torchrun),
each rank runs its own 1024 realisations (disjoint index ranges, no device
collective); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "echo curves/s, batched mixed vs plain FP64 on 1 B200 at <=1e-6 echo error"
UNIT = "curves/s"
REALIZATIONS = 1024
L = 12
MIXED_BYTES_PER_AMP_ORDER = 56.0   # FP32 T_{n-1}, T_{n-2}, T_n + FP64 psi read+write
FP64_BYTES_PER_AMP_ORDER = 80.0    # FP64 T_{n-1}, T_{n-2}, T_n + FP64 psi read+write
SMEM_BYTES_PER_AMP_ORDER = 168.0   # shared-memory traffic of the L=12, R=4 FP32 schedule
# DRAM bytes per amplitude-order of k_batch<12,4,float>: ncu capture of
# profile_case (296 realisations, 2 XY-8 blocks): 48.2 MB for 6.149e9.
DRAM_BYTES_PER_AMP_ORDER_MEASURED = 48.215296e6 / 6.149e9
FLOPS_PER_AMP_ORDER = L * (L - 1) * 2 + 20


def workload():
    from spin_systems_b200 import workloads
    return workloads.xy8_finite(nspins=L, realizations=REALIZATIONS)


def config_block(n_gpus):
    return {
        "workload": "XY-8x16 finite pulses (amp 50, width pi/50), tau=0.25, L=12, sigma=0.5, "
                    "2D dipolar, 128 S^x echo points, state+reference",
        "realizations_per_gpu": REALIZATIONS,
        "global_batch": REALIZATIONS * n_gpus,
        "precision": "FP32 recursion, FP64 series sum and reductions; realisations past 40000 "
                     "orders per state vector run in FP64 in the same graph",
        "parallelism": f"realisations sharded over {n_gpus} GPU(s), no device collective",
        "l2": "inputs larger than L2: 128 MB state pool + 64 MB psi0 pool + tables per step",
    }


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    return rank, world, local


def barrier_max(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_sample(spec, steps, warmup, per_step=None):
    """The reference's own CPU implementation (oracle/_ref when built here,
    else the C restatement) on the host cores, a bounded sample per step."""
    from oracle.oracle import Port, Ref
    threads = cpu_threads()
    if Ref.available():
        lib, kind = Ref(), "reference"
    else:
        lib, kind = Port(), "port"
    cfg = spec.config()
    n = per_step or threads
    for _ in range(warmup):
        lib.run_range(cfg, 0, min(n, threads), threads)
    total = 0.0
    for s in range(steps):
        _, _, secs = lib.run_range(cfg, (s * n) % REALIZATIONS, n, threads)
        total += secs
    return {"value": steps * n / total, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{n} realisations of the L=12 XY-8 workload per step on {threads} threads "
                      f"(LocalRunner-equivalent thread pool over runRealization)",
            "seconds": total}


def run_reference_arm(args):
    # CPU work on rank 0 alone: no process group, the other ranks exit at once
    if int(os.environ.get("RANK", "0")) != 0:
        return
    spec = workload()
    cb = reference_sample(spec, args.steps, args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * cb["seconds"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_block(1),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def kernel_desc(tuned):
    """The schedules the timed graph ran: the tuner's choice, else the defaults."""
    chosen = {r["precision"]: r["variant"] for r in tuned if r["L"] == L}
    mixed = chosen.get("mixed", "L12.R4.f32.smem.c1")
    fp64 = chosen.get("fp64", "L12.R3.f64.global.c1")
    return (f"{mixed} (mixed bucket) with the routed realisations in {fp64} (FP64 bucket) of "
            "the same graph; the recursion is resident in shared memory")

def run_ours(args):
    import torch
    rank, world, local = dist_setup(args.gpus)
    import spin_systems_b200 as ss
    from spin_systems_b200 import abi

    spec = workload()
    cfg = spec.config()
    eng = ss.Engine(local)
    stream = torch.cuda.ExternalStream(eng.stream, device=torch.device("cuda", local))
    first = rank * REALIZATIONS
    tuned = []
    if args.tune:
        # The autotuner picks each kernel's schedule (mixed and the FP64
        # routing target) on a sample of this rank's own realisations.
        t0 = time.perf_counter()
        tuned = ss.tune(eng, cfg, first, args.tune_sample, abi.MIXED)
        tune_s = time.perf_counter() - t0
    batch = ss.Batch(eng, cfg, first, REALIZATIONS, abi.MIXED)
    stats = batch.stats()
    prec, amp_each = batch.work()
    routed = prec == abi.FP64
    batch.upload()

    # Warm-up, then K device-resident steps: inputs already in HBM.
    for _ in range(args.warmup):
        batch.execute()
    eng.synchronize()
    barrier(world)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = eng.launches
    with Clocks(local) as clocks:
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            batch.execute()
        end.record(stream)
        end.synchronize()
    launches = eng.launches - launches0
    eng.synchronize()
    dev_ms = start.elapsed_time(end)
    dev_ms = barrier_max(world, dev_ms)
    barrier(world)

    # End to end through the C ABI with host buffers: upload of every input,
    # the run, download of the rows, all inside the timed region.
    t0 = time.perf_counter()
    for _ in range(args.steps):
        times, mixed = batch.run()
    e2e_s = time.perf_counter() - t0
    e2e_s = barrier_max(world, e2e_s)

    if rank != 0:
        barrier(world)
        return

    # Accuracy: FP64 batch on the same realisations (untimed), every curve.
    check = REALIZATIONS
    b64 = ss.Batch(eng, cfg, first, check, abi.FP64)
    _, fp64 = b64.run()
    corr0 = []
    for i in range(first, first + check):
        s = ss.realization_setup(cfg, i, L)
        psi = s["psi0"][0::2] + 1j * s["psi0"][1::2]
        k = np.arange(1 << L)
        ref = sum(psi[k ^ (1 << q)] for q in range(L))
        corr0.append(np.vdot(ref, ref).real)
    err = np.abs(mixed[:check, :, 0] - fp64[:, :, 0]).max(axis=1) / np.array(corr0)
    del b64

    # Plain FP64 path: one realisation at a time through runRealization.
    plain_n = 3
    ss.run_realization(eng, cfg, first, batch.points, batch.width)
    t0 = time.perf_counter()
    for i in range(plain_n):
        ss.run_realization(eng, cfg, first + i, batch.points, batch.width)
    plain_rate = plain_n / (time.perf_counter() - t0)

    value = world * REALIZATIONS * args.steps / (dev_ms / 1e3)
    ms_step = dev_ms / args.steps
    amp_orders = stats["amplitude_orders"]
    amp_fp64 = float(amp_each[routed].sum())
    amp_mixed = amp_orders - amp_fp64
    alg_bytes = MIXED_BYTES_PER_AMP_ORDER * amp_mixed + FP64_BYTES_PER_AMP_ORDER * amp_fp64
    achieved = alg_bytes / (ms_step / 1e3) / 1e9
    hbm, src = peaks()
    clk = clocks.summary()
    smem_peak = 128.0 * eng_sms() * (clk["sm_mhz"] or 1965.0) * 1e6 / 1e9
    smem_ach = SMEM_BYTES_PER_AMP_ORDER * amp_mixed / (ms_step / 1e3) / 1e9
    cb = reference_sample(spec, 1, 0, per_step=max(2, cpu_threads()))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_block(world),
        "e2e": {"value": world * REALIZATIONS * args.steps / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": stats["h2d_bytes"], "d2h_bytes_per_step": stats["d2h_bytes"]},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm,
                     "traffic": DRAM_BYTES_PER_AMP_ORDER_MEASURED * amp_mixed,
                     "traffic_note": "DRAM bytes of the mixed kernel per launch, scaled from "
                                     "an ncu capture of a smaller case by amplitude-orders",
                     "peak_source": src,
                     "kernel": kernel_desc(tuned),
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "note": "effective bandwidth of a shared-memory-resident kernel pair; the "
                             "binding limit is shared-memory bandwidth and issue (see smem)"},
        "smem": {"achieved_gbs": smem_ach, "peak_gbs": smem_peak, "frac": smem_ach / smem_peak,
                 "bytes_per_amp_order": SMEM_BYTES_PER_AMP_ORDER,
                 "note": "FP32 kernel's share only"},
        "routing": {"fp64_realizations": int(routed.sum()), "realizations": int(len(prec)),
                    "fp64_amplitude_order_share": amp_fp64 / amp_orders,
                    "rule": "more than 40000 Chebyshev orders per state vector -> FP64 kernel"},
        "fp32_tflops": FLOPS_PER_AMP_ORDER * amp_mixed / (ms_step / 1e3) / 1e12,
        "clocks": clk,
        "echo_error": {"max": float(err.max()), "mean": float(err.mean()), "curves": check,
                       "above_1e-6": int((err > 1e-6).sum()),
                       "max_mixed_only": float(err[~routed].max()) if (~routed).any() else 0.0,
                       "reference": "batched FP64 on the same realisations"},
        "plain_fp64": {"value": plain_rate, "unit": UNIT, "curves": plain_n,
                       "speedup_of_batched_mixed": value / world / plain_rate},
        "work": {"amplitude_orders_per_step": amp_orders, "orders_per_step": stats["orders"]},
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "schedule": ({"tuned": [{k: r[k] for k in ("L", "precision", "variant", "ns")} for r in tuned],
                      "tuning_seconds": tune_s, "sample": args.tune_sample}
                     if args.tune else {"tuned": [], "note": "default schedules (--no-tune)"}),
    }
    print(json.dumps(line), flush=True)
    barrier(world)
    del batch
    eng.close()



def run_cpmg10(args):
    """The L = 10 CPMG of the reference's demo config: every path on the same
    20 realisations, device time with CUDA events, the reference's CPU build
    on all host threads (wall clock around its experiment)."""
    import torch
    import spin_systems_b200 as ss
    from spin_systems_b200 import abi, workloads
    from oracle.oracle import Port, Ref
    spec = workloads.cpmg_ideal()
    cfg = spec.config()
    n = spec.realizations
    eng = ss.Engine(0)
    stream = torch.cuda.ExternalStream(eng.stream, device=torch.device("cuda", 0))
    out = {}
    tuned = []
    if args.tune:  # schedules for L = 10 in both precisions (mixed run includes FP64)
        tuned = ss.tune(eng, cfg, 0, n, abi.MIXED)
    for name, prec in (("batched_fp64", abi.FP64), ("batched_mixed", abi.MIXED)):
        b = ss.Batch(eng, cfg, 0, n, prec)
        b.upload()
        for _ in range(max(args.warmup, 3)):
            b.execute()
        eng.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            b.execute()
        e1.record(stream)
        e1.synchronize()
        sec = e0.elapsed_time(e1) / 1e3 / args.steps
        t0 = time.perf_counter()
        _, rows = b.run()
        e2e = time.perf_counter() - t0
        out[name] = {"curves_per_s": n / sec, "e2e_curves_per_s": n / e2e, "rows": rows}
        del b
    ss.run_realization(eng, cfg, 0, spec.measurement_count(), spec.width())
    t0 = time.perf_counter()
    plain = [ss.run_realization(eng, cfg, i, spec.measurement_count(), spec.width())[1]
             for i in range(n)]
    out["plain_fp64"] = {"curves_per_s": n / (time.perf_counter() - t0)}
    threads = cpu_threads()
    lib, kind = (Ref(), "reference") if Ref.available() else (Port(), "port")
    _, want, secs = lib.run_range(cfg, 0, n, threads)
    want = np.asarray(want).reshape(out["batched_fp64"]["rows"].shape)
    scale = np.abs(want[:, :, 0]).max()
    line = {"metric": "echo curves/s, L=10 CPMG (20 realisations)", "unit": UNIT,
            "value": out["batched_fp64"]["curves_per_s"], "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "higher_is_better": True, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "L=10 CPMG pi/2_x + 8x(0.5, pi_y, 0.5), "
                                             "sigma=0.5, 20 realisations, corr:x + norm"},
            "batched_fp64": {k: v for k, v in out["batched_fp64"].items() if k != "rows"},
            "batched_mixed": {k: v for k, v in out["batched_mixed"].items() if k != "rows"},
            "plain_fp64": out["plain_fp64"],
            "parity_vs_cpu_reference": {
                "batched_fp64_max_abs": float(np.abs(out["batched_fp64"]["rows"] - want).max()),
                "plain_fp64_max_abs": float(np.abs(np.stack(plain) - want).max()),
                "batched_mixed_echo_error": float(np.abs(out["batched_mixed"]["rows"][:, :, 0]
                                                         - want[:, :, 0]).max() / scale)},
            "cpu_baseline": {"value": n / secs, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"all {n} realisations on {threads} threads"},
            "schedule": [{k: r[k] for k in ("L", "precision", "variant", "ns")} for r in tuned]}
    print(json.dumps(line), flush=True)
    eng.close()

_SMS = [148]


def eng_sms():
    try:
        import torch
        return torch.cuda.get_device_properties(0).multi_processor_count
    except Exception:
        return _SMS[0]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--tune", dest="tune", action="store_true", default=True,
                    help="run the autotuner before timing (default)")
    ap.add_argument("--no-tune", dest="tune", action="store_false")
    ap.add_argument("--tune-sample", type=int, default=296)
    ap.add_argument("--workload", choices=["xy8", "cpmg10"], default="xy8",
                    help="xy8: the headline batch (default); cpmg10: the L=10 demo case")
    args = ap.parse_args()
    if args.workload == "cpmg10" and args.impl == "ours":
        run_cpmg10(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
