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
# FP32 flops per amplitude-order: two FMAs for each of the ~L(L-1)/4
# anti-aligned coupling terms, plus the fields and the recurrence.
FLOPS_PER_AMP_ORDER = L * (L - 1) + 20
CPU_SAMPLE_SEED = 0x5EED_C0DE


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


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def seeded_subset(count, total, seed):
    """`count` realisation indices from [0, total), drawn without
    replacement (then again, if more are asked for than exist) from a seeded
    stream: a sample spread over the whole batch, the same on every run."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        out.extend(rng.permutation(total)[: count - len(out)].tolist())
    return np.asarray(out, dtype=np.uint64)


def cpu_impl():
    from oracle.oracle import Port, Ref
    return (Ref(), "reference") if Ref.available() else (Port(), "port")


def reference_sample(spec, count, threads, seed):
    """The reference's own CPU implementation (oracle/_ref when built here,
    else the C restatement) over a seeded subset of the batch's realisations
    in one pool of `threads` host threads that take the next realisation as
    they finish (the reference's LocalRunner schedule), so every thread is
    busy until the sample runs out."""
    lib, kind = cpu_impl()
    idx = seeded_subset(count, REALIZATIONS, seed)
    _, _, secs = lib.run_indices(spec.config(), idx, threads)
    return {"value": len(idx) / secs, "unit": UNIT, "cores": threads, "kind": kind,
            "seconds": secs, "realizations": int(len(idx)),
            "sample": f"{len(idx)} realisations drawn at random (seeded) from the batch's "
                      f"{REALIZATIONS}, one runRealization pool on {threads} threads",
            "model": cpu_model()}


def run_reference_arm(args):
    # CPU work on rank 0 alone: no process group, the other ranks exit at once
    if int(os.environ.get("RANK", "0")) != 0:
        return
    spec = workload()
    threads = cpu_threads()
    lib, kind = cpu_impl()
    per_step = threads
    for w in range(args.warmup):  # untimed: a quarter step each
        lib.run_indices(spec.config(), seeded_subset(max(1, threads // 4), REALIZATIONS, w),
                        threads)
    # The K steps' samples (K x threads realisations across the batch) run as
    # one pool, so no thread idles at a step boundary waiting for the
    # slowest realisation of its step.
    cb = reference_sample(spec, args.steps * per_step, threads, CPU_SAMPLE_SEED)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * cb["seconds"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_block(1),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                "model")},
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

    # End to end through the C ABI from the config, as the reference arm
    # runs: every step assembles the realisations on the host (random
    # streams, geometry, disorder, initial states, expansions), uploads them
    # from host buffers, runs, and downloads the rows.
    e2e_steps = min(args.steps, 5)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        b = ss.Batch(eng, cfg, first, REALIZATIONS, abi.MIXED)
        times, mixed = b.run()
        b._destroy()
    e2e_s = barrier_max(world, time.perf_counter() - t0)
    # The same with the assembled tables kept: upload, run, download.
    res_steps = min(args.steps, 3)
    t0 = time.perf_counter()
    for _ in range(res_steps):
        times, mixed = batch.run()
    res_s = barrier_max(world, time.perf_counter() - t0)

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

    # Plain FP64 path: one realisation at a time through runRealization, on a
    # seeded sample spread over the batch (its realisations differ ~10x in work).
    plain = plain_sample(eng, cfg, first, batch, amp_each, PLAIN_SAMPLE, CPU_SAMPLE_SEED + 1)

    value = world * REALIZATIONS * args.steps / (dev_ms / 1e3)
    ms_step = dev_ms / args.steps
    amp_orders = stats["amplitude_orders"]
    amp_fp64 = float(amp_each[routed].sum())
    amp_mixed = amp_orders - amp_fp64
    alg_bytes = MIXED_BYTES_PER_AMP_ORDER * amp_mixed + FP64_BYTES_PER_AMP_ORDER * amp_fp64
    achieved = alg_bytes / (ms_step / 1e3) / 1e9
    hbm, src = peaks()
    clk = clocks.summary()
    mhz = clk["sm_mhz"] or 1965.0
    smem_peak = 128.0 * eng_sms() * mhz * 1e6 / 1e9
    smem_ach = SMEM_BYTES_PER_AMP_ORDER * amp_mixed / (ms_step / 1e3) / 1e9
    fma_peak = 2.0 * 128.0 * eng_sms() * mhz * 1e6 / 1e12
    fma_ach = FLOPS_PER_AMP_ORDER * amp_mixed / (ms_step / 1e3) / 1e12
    threads = cpu_threads()
    cb = reference_sample(spec, 3 * threads, threads, CPU_SAMPLE_SEED + 2)
    cb1 = reference_sample(spec, 2, 1, CPU_SAMPLE_SEED + 3)
    # Realisations differ ~10x in work: the CPU's seconds per amplitude-order
    # on its sample, times the batch's amplitude-orders, is the rate the
    # whole batch would run at.
    amp_all = np.asarray(amp_each, dtype=np.float64)
    for c, seed, count in ((cb, CPU_SAMPLE_SEED + 2, 3 * threads), (cb1, CPU_SAMPLE_SEED + 3, 2)):
        pick = [int(i) for i in seeded_subset(count, REALIZATIONS, seed)]
        c["amplitude_order_scaled"] = (len(amp_all) / (c["seconds"] / amp_all[pick].sum()
                                                         * amp_all.sum()))
    sizes = per_size_ratios(eng, args) if args.per_size else {}
    kern = plain_order_kernels(eng, hbm) if args.plain_kernels else {}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_block(world),
        "e2e": {"value": world * REALIZATIONS * e2e_steps / e2e_s, "unit": UNIT, "steps": e2e_steps,
                "h2d_bytes_per_step": stats["h2d_bytes"], "d2h_bytes_per_step": stats["d2h_bytes"],
                "includes": "host assembly of every realisation (ss_batch_create), upload from "
                            "host buffers, run, download of the rows"},
        "e2e_tables_resident": {"value": world * REALIZATIONS * res_steps / res_s, "unit": UNIT,
                                "steps": res_steps,
                                "includes": "upload from host buffers, run, download (tables "
                                            "assembled once before timing)"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "smem", "achieved": smem_ach, "peak": smem_peak, "unit": "GB/s",
                     "frac": smem_ach / smem_peak,
                     "traffic": DRAM_BYTES_PER_AMP_ORDER_MEASURED * amp_mixed,
                     "traffic_note": "DRAM bytes of the mixed kernel per launch, scaled from "
                                     "an ncu capture of a smaller case by amplitude-orders",
                     "peak_source": "architectural: 128 B/clk/SM x SMs x the median SM clock "
                                    "sampled under load (no measured shared-memory peak)",
                     "bytes_per_amp_order": SMEM_BYTES_PER_AMP_ORDER,
                     "kernel": kernel_desc(tuned),
                     "binding": "on-chip: the recursion lives in shared memory; shared-memory "
                                "bandwidth and instruction issue bind, not HBM",
                     "hbm_effective": {"achieved": achieved, "peak": hbm, "unit": "GB/s",
                                       "frac": achieved / hbm, "peak_source": src,
                                       "algorithmic_bytes_per_launch": alg_bytes,
                                       "note": "algorithmic bytes / time of an on-chip kernel: "
                                               "an effective bandwidth, not an HBM fraction"},
                     "fp32_fma": {"achieved_tflops": fma_ach, "peak_tflops": fma_peak,
                                  "frac": fma_ach / fma_peak,
                                  "peak_source": "architectural: 128 FP32 FMA/clk/SM x 2 flops "
                                                 "x SMs x the median SM clock under load"}},
        "plain_order_kernel_hbm": kern,
        "routing": {"fp64_realizations": int(routed.sum()), "realizations": int(len(prec)),
                    "fp64_amplitude_order_share": amp_fp64 / amp_orders,
                    "rule": "more than the size's order limit per state vector (38600 at "
                            "L = 12) -> FP64 kernel of the same graph"},
        "clocks": clk,
        "echo_error": {"max": float(err.max()), "mean": float(err.mean()), "curves": check,
                       "above_1e-6": int((err > 1e-6).sum()),
                       "max_mixed_only": float(err[~routed].max()) if (~routed).any() else 0.0,
                       "reference": "batched FP64 on the same realisations"},
        "plain_fp64": dict(plain, speedup_of_batched_mixed=value / world / plain["value"]),
        "per_size_cpmg32": sizes,
        "work": {"amplitude_orders_per_step": amp_orders, "orders_per_step": stats["orders"]},
        "cpu_baseline": dict({k: cb[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                 "model", "amplitude_order_scaled")},
                             one_thread={k: cb1[k] for k in ("value", "unit", "sample",
                                                             "amplitude_order_scaled")}),
        "schedule": ({"tuned": [{k: r[k] for k in ("L", "precision", "variant", "ns")} for r in tuned],
                      "tuning_seconds": tune_s, "sample": args.tune_sample}
                     if args.tune else {"tuned": [], "note": "default schedules (--no-tune)"}),
    }
    print(json.dumps(line), flush=True)
    barrier(world)
    del batch
    eng.close()


PLAIN_SAMPLE = 16


def plain_sample(eng, cfg, first, batch, amp_each, n, seed):
    """The plain FP64 path (ss_run_realization, one realisation at a time)
    on a seeded sample of the batch: its curves/s, and the rate its seconds
    per amplitude-order give for the whole batch."""
    import spin_systems_b200 as ss
    idx = [int(i) for i in seeded_subset(n, REALIZATIONS, seed)]
    ss.run_realization(eng, cfg, first + idx[0], batch.points, batch.width)  # warm-up
    secs = 0.0
    for i in idx:
        t0 = time.perf_counter()
        ss.run_realization(eng, cfg, first + i, batch.points, batch.width)
        secs += time.perf_counter() - t0
    amp = np.asarray(amp_each, dtype=np.float64)
    batch_secs = secs * amp.sum() / amp[idx].sum()
    return {"value": n / secs, "unit": UNIT, "curves": n,
            "sample": f"{n} realisations drawn at random (seeded) from the batch",
            "amplitude_order_scaled": len(amp) / batch_secs}


def per_size_ratios(eng, args):
    """The uneven batch's CPMG-32 program (sigma, tau ~ U[0.1, 1]) at one L
    at a time: the batched mixed engine (tuned for the size) against the
    plain FP64 path on a seeded sample of the same realisations."""
    import torch
    import spin_systems_b200 as ss
    from spin_systems_b200 import abi, workloads
    from spin_systems_b200.experiments import corr0
    out = {}
    stream = torch.cuda.ExternalStream(eng.stream, device=torch.device("cuda", 0))
    for Lx, n in ((14, 296), (16, 120)):
        spec = workloads.cpmg_uneven(realizations=n)
        spec.spin_choices = (Lx,)
        cfg = spec.config()
        ss.tune(eng, cfg, 0, 32, abi.MIXED)
        b = ss.Batch(eng, cfg, 0, n, abi.MIXED)
        b.upload()
        b.execute()
        eng.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.execute()
        e1.record(stream)
        e1.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        _, mixed = b.download()
        _, amp = b.work()
        amp = np.asarray(amp, dtype=np.float64)
        rng = np.random.default_rng(CPU_SAMPLE_SEED + Lx)
        idx = [int(i) for i in rng.permutation(n)[:8]]
        scale = corr0(cfg, idx, Lx)  # <ref|ref> = corr_x(0), the echo error's scale
        psec, errs = 0.0, []
        ss.run_realization(eng, cfg, idx[0], b.points, b.width)
        for i, sc in zip(idx, scale):
            t0 = time.perf_counter()
            _, rows = ss.run_realization(eng, cfg, i, b.points, b.width)
            psec += time.perf_counter() - t0
            errs.append(float(np.abs(mixed[i, :, 0] - rows[:, 0]).max() / sc))
        plain_rate = n / (psec * amp.sum() / amp[idx].sum())
        out[int(Lx)] = {"realizations": n, "batched_mixed_curves_per_s": n / sec,
                        "plain_fp64_curves_per_s": plain_rate, "ratio": n / sec / plain_rate,
                        "plain_sample": len(idx),
                        "plain_scaling": "seconds per amplitude-order of the seeded sample x "
                                         "the batch's amplitude-orders",
                        "echo_error_max": max(errs),
                        "schedule": {r["precision"]: r["variant"] for r in ss.schedule()
                                     if r["L"] == Lx}}
        b._destroy()
    return out


def plain_order_kernels(eng, hbm):
    """The plain path's order kernel on single vectors larger than L2 (the
    long-propagation realisation at L = 22 and 24): device time per order,
    effective bandwidth at the algorithmic 80 B (FP64) / 56 B (mixed) per
    amplitude-order as a fraction of measured HBM, and the bytes the tiled
    kernel's passes move by construction."""
    import torch
    import spin_systems_b200 as ss
    from spin_systems_b200 import abi, workloads
    stream = torch.cuda.ExternalStream(eng.stream, device=torch.device("cuda", 0))
    out = {}
    for Lx, prec, name in ((22, abi.FP64, "fp64"), (24, abi.FP64, "fp64"), (24, abi.MIXED, "mixed")):
        spec = workloads.long_propagation(nspins=Lx, steps=1, every=1, epsilon=1e-7)
        s = ss.realization_setup(spec.config(), 0, Lx)
        ham = ss.Hamiltonian(eng, Lx, s["fields"], s["pairs"], s["J"])
        psi = ss.StateVector(eng, Lx, s["psi0"])
        prop = ss.Propagator(Lx, 1e-7, prec, abi.KERNEL_TILED)
        prop.evolve(ham, abi.REAL, psi, 0.1, 1)
        eng.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        prop.evolve(ham, abi.REAL, psi, 0.1, 1)
        e1.record(stream)
        e1.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        orders = prop.last_order
        alg = 80.0 if prec == abi.FP64 else 56.0
        P = len(ss.tiled_plan(Lx, prec))
        pbytes = 48.0 * P + 24.0 if prec == abi.FP64 else 24.0 * P + 24.0
        amps = float(1 << Lx)
        eff = alg * amps * orders / sec / 1e9
        out[f"L{Lx}_{name}"] = {"ms_per_order": 1e3 * sec / orders, "effective_gbs": eff,
                                "frac_of_hbm": eff / hbm, "algorithmic_bytes": alg,
                                "passes": P, "pass_bytes": pbytes,
                                "pass_gbs": pbytes * amps * orders / sec / 1e9,
                                "pair_terms_per_s": 0.5 * len(s["J"]) / 3 * amps * orders / sec}
        del psi, ham
    return out


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
    ap.add_argument("--no-per-size", dest="per_size", action="store_false", default=True,
                    help="skip the per-size L = 14 / 16 CPMG-32 ratios")
    ap.add_argument("--no-plain-kernels", dest="plain_kernels", action="store_false",
                    default=True, help="skip the plain order kernel at L = 22 / 24")
    ap.add_argument("--workload", choices=["xy8", "cpmg10"], default="xy8",
                    help="xy8: the headline batch (default); cpmg10: the L=10 demo case")
    args = ap.parse_args()
    if args.workload == "cpmg10" and args.impl == "ours":
        run_cpmg10(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)
    # Under torchrun every rank leaves the process group it joined (no CUDA
    # graph holds a collective, so nothing is left in flight).
    if "torch.distributed" in sys.modules:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
