"""Measurement runs for the workloads beside the headline benchmark.

  uneven  4096 realisations with L drawn from {8, 10, 12, 14, 16}, sigma and
          tau drawn from U[0.1, 1] per realisation, CPMG with 32 ideal pi_y
          pulses: the batched mixed engine (all sizes in one graph, schedules
          from the autotuner) against the plain FP64 path run one realisation
          at a time (timed on a sample of each size and scaled to the batch).
  long    Single-realisation long propagation from a random product state,
          autonormalisation off, 10^4 steps of dt = 0.1 (sigma = 1): norm and
          energy drift of the plain FP64 path and of the mixed engine (batch of
          one) and the echo error of mixed against FP64.

  python -m spin_systems_b200.experiments uneven [--realizations N] [--out F]
  python -m spin_systems_b200.experiments long --nspins 16 [--steps S] [--out F]
  python -m spin_systems_b200.experiments plain [--sizes 16 20 22 24] [--out F]
  python -m spin_systems_b200.experiments per_size [--sizes 12 14 16] [--out F]

Inputs are seeded synthetic realisations (seed 20240726, streams per
(seed, index)); device time with CUDA events on the engine's stream.
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import Batch, Engine, abi, realization_setup, run_realization, schedule, tune
from . import workloads


def _events(eng):
    import torch
    s = torch.cuda.ExternalStream(eng.stream, device=torch.device("cuda", 0))
    return s, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def corr0(cfg, idx, lmax):
    out = []
    for i in idx:
        s = realization_setup(cfg, int(i), lmax)
        psi = s["psi0"][0::2] + 1j * s["psi0"][1::2]
        k = np.arange(1 << s["L"])
        ref = sum(psi[k ^ (1 << q)] for q in range(s["L"]))
        out.append(np.vdot(ref, ref).real)
    return np.array(out)


def plain_time_model(raw: dict, amps: dict) -> dict:
    """The plain path's time for every realisation of each size from a timed
    sample: least squares seconds = fixed + rate x amplitude-orders over the
    size's sample (both clamped at zero), summed over the size's
    realisations.  A per-realisation fixed cost (host set-up, graph capture
    of each new expansion) makes seconds per amplitude-order fall with the
    work, so scaling the sample's mean rate by the size's amplitude-orders
    would overstate the heavy realisations that carry most of them."""
    per, total = {}, 0.0
    for L, r in raw.items():
        x = np.asarray(r["amplitude_orders"], dtype=np.float64)
        y = np.asarray(r["seconds"], dtype=np.float64)
        if len(x) >= 2 and np.ptp(x) > 0:
            rate, fixed = np.polyfit(x, y, 1)
        else:
            rate, fixed = float(y.mean() / x.mean()), 0.0
        if fixed < 0.0:
            fixed, rate = 0.0, float((x * y).sum() / (x * x).sum())
        if rate < 0.0:
            fixed, rate = float(y.mean()), 0.0
        a = np.asarray(amps[L], dtype=np.float64)
        sec = float(len(a) * fixed + rate * a.sum())
        per[int(L)] = {"fixed_seconds": float(fixed), "ns_per_amp_order": float(rate * 1e9),
                       "seconds": sec, "realizations": int(len(a))}
        total += sec
    return {"seconds": total, "per_size": per}


def uneven(args) -> dict:
    eng = Engine(0)
    spec = workloads.cpmg_uneven(realizations=args.realizations)
    cfg = spec.config()
    n = args.realizations
    t0 = time.perf_counter()
    table = tune(eng, cfg, 0, args.tune_sample, abi.MIXED)
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    b = Batch(eng, cfg, 0, n, abi.MIXED)
    create_s = time.perf_counter() - t0
    stats = b.stats()
    prec, amp = b.work()
    sizes = np.array([realization_setup(cfg, i, 16)["L"] for i in range(n)])
    b.upload()
    for _ in range(args.warmup):
        b.execute()
    eng.synchronize()
    stream, e0, e1 = _events(eng)
    e0.record(stream)
    for _ in range(args.steps):
        b.execute()
    e1.record(stream)
    e1.synchronize()
    dev_s = e0.elapsed_time(e1) / 1e3 / args.steps
    if args.e2e:
        t0 = time.perf_counter()
        _, mixed = b.run()
        e2e_s = time.perf_counter() - t0
    else:
        _, mixed = b.download()
        e2e_s = float("nan")
    rep = {"workload": "uneven CPMG-32, L in {8,10,12,14,16}, sigma, tau ~ U[0.1,1]",
           "realizations": n, "per_size": {int(L): int((sizes == L).sum()) for L in np.unique(sizes)},
           "batched_mixed": {"seconds_per_batch": dev_s, "curves_per_s": n / dev_s,
                             "e2e_curves_per_s": n / e2e_s if args.e2e else None,
                             "amplitude_orders": stats["amplitude_orders"],
                             "fp64_routed": int((prec == abi.FP64).sum()),
                             "create_seconds": create_s},
           "schedule": [{k: r[k] for k in ("L", "precision", "variant", "ns")} for r in table],
           "tuning_seconds": tune_s}
    # The FP64 reference: the plain path on a sample of each size, which also
    # gives the echo error of those curves.  The sample of each size is
    # spread over its work distribution: the size's realisations sorted by
    # amplitude-orders, one taken at evenly spaced ranks (lightest to
    # heaviest).
    errs, samples, raw = {}, {}, {}
    for L in np.unique(sizes):
        members = np.flatnonzero(sizes == L)
        order = members[np.argsort(amp[members], kind="stable")]
        k = min(args.plain_sample, len(order))
        idx = order[np.unique(np.round(np.linspace(0, len(order) - 1, k)).astype(int))]
        ts, es = [], []
        scale = corr0(cfg, idx, 16)
        # untimed first call of the size: one-time set-up (module loading,
        # the size's first graphs) would otherwise land on its lightest
        # realisation and inflate its seconds per amplitude-order
        run_realization(eng, cfg, int(idx[0]), b.points, b.width)
        for j, i in enumerate(idx):
            t0 = time.perf_counter()
            _, ref = run_realization(eng, cfg, int(i), b.points, b.width)
            ts.append(time.perf_counter() - t0)
            es.append(float(np.abs(mixed[i, :, 0] - ref[:, 0]).max() / scale[j]))
        raw[int(L)] = {"index": [int(i) for i in idx], "amplitude_orders": amp[idx].tolist(),
                       "seconds": ts}
        samples[int(L)] = int(len(idx))
        errs[int(L)] = {"max": max(es), "mean": float(np.mean(es))}
    amps = {int(L): amp[sizes == L] for L in np.unique(sizes)}
    model = plain_time_model(raw, amps)
    plain_total = model["seconds"]
    rng = np.random.default_rng(20240726)
    boots = []
    for _ in range(2000):
        pick = {}
        for L, r in raw.items():
            j = rng.integers(0, len(r["seconds"]), len(r["seconds"]))
            pick[L] = {"amplitude_orders": np.asarray(r["amplitude_orders"])[j],
                       "seconds": np.asarray(r["seconds"])[j]}
        boots.append(plain_time_model(pick, amps)["seconds"])
    lo, hi = np.percentile([t / dev_s for t in boots], [2.5, 97.5])
    rep["plain_fp64"] = {"curves_per_s": n / plain_total, "seconds_per_batch": plain_total,
                         "per_size": model["per_size"], "sampled": samples, "samples": raw,
                         "note": "one realisation at a time through ss_run_realization on a "
                                 "sample of each size spread over its amplitude-orders; each "
                                 "size's time from a least-squares fit of seconds = fixed + "
                                 "rate x amplitude-orders over its sample, applied to every "
                                 "realisation of the size"}
    rep["speedup_batched_mixed_over_plain_fp64"] = plain_total / dev_s
    rep["speedup_95pct_bootstrap"] = [float(lo), float(hi)]
    rep["echo_error_vs_plain_fp64"] = errs
    b._destroy()
    eng.close()
    return rep


def routing(args) -> dict:
    """Mixed precision with no FP64 routing against batched FP64 on the same
    realisations: per curve, the echo error (max over time of |corr_x
    mixed - FP64| / <ref|ref>), the batch's error estimate (orders x the FP32
    rounding residuals the kernel leaves uncorrected) and the orders per
    state vector (the order-count rule's input)."""
    eng = Engine(0)
    rep = {}
    for L, n in zip(args.sizes, args.counts):
        if args.program == "xy8":
            spec = workloads.xy8_finite(nspins=L, realizations=n)
        else:
            spec = workloads.cpmg_uneven(realizations=n)
            spec.spin_choices = (L,)
        spec.mixed_order_limit = -1
        if args.norm:
            spec.observables = ["corr:x", "norm"]
        cfg = spec.config()
        bm = Batch(eng, cfg, 0, n, abi.MIXED)
        _, mixed = bm.run()
        est = bm.error_estimates()
        _, amp = bm.work()
        bm._destroy()
        b64 = Batch(eng, cfg, 0, n, abi.FP64)
        _, fp64 = b64.run()
        b64._destroy()
        scale = corr0(cfg, range(n), 16)
        err = np.abs(mixed[:, :, 0] - fp64[:, :, 0]).max(axis=1) / scale
        orders = amp / float(2 << L)
        if args.norm:
            # columns: corr re, corr im, |psi|, |ref|; drift against FP64
            drift = np.maximum(np.abs(mixed[:, :, 2] - fp64[:, :, 2]).max(axis=1),
                               np.abs(mixed[:, :, 3] - fp64[:, :, 3]).max(axis=1)
                               / np.sqrt(scale))
            # against the exact initial norms: |psi0| = 1, |ref0| = sqrt(<ref|ref>)
            self_drift = np.maximum(np.abs(mixed[:, :, 2] - 1.0).max(axis=1),
                                    np.abs(mixed[:, :, 3] - np.sqrt(scale)[:, None]).max(axis=1)
                                    / np.sqrt(scale))
        rep[int(L)] = {"program": args.program, "realizations": n,
                       "norm_drift": [float(x) for x in self_drift] if args.norm else None,
                       "echo_error": [float(x) for x in err],
                       "estimate": [float(x) for x in est],
                       "orders_per_state": [float(x) for x in orders],
                       "amplitude_orders": [float(x) for x in amp],
                       "max_error": float(err.max())}
        print(json.dumps({int(L): {"max_error": float(err.max()),
                                   "corr_log_est": float(np.corrcoef(np.log(err + 1e-300),
                                                                     np.log(est + 1e-300))[0, 1]),
                                   "corr_log_orders": float(np.corrcoef(np.log(err + 1e-300),
                                                                        np.log(orders))[0, 1])}}),
              flush=True)
    eng.close()
    return rep


def long_run(args) -> dict:
    """The long-propagation workload (random product state, sigma = 1,
    dt = 0.1, autonormalisation off) for one realisation: the plain FP64 path
    and the plain mixed path (FP32 Chebyshev vectors, FP64 psi), both with
    the size's default kernel family (tiled from 18 spins), device time with
    CUDA events, and the mixed run's deviation from FP64 in every observable;
    at L <= 16 also the batched mixed engine on a batch of one."""
    eng = Engine(0)
    L = args.nspins
    every = args.every
    spec = workloads.long_propagation(nspins=L, steps=args.steps, dt=0.1, every=every,
                                      epsilon=args.epsilon)
    spec.mixed_order_limit = -1  # the batched mixed run stays mixed at every order count
    cfg = spec.config()
    points = spec.measurement_count()
    width = spec.width()
    rep = {"workload": f"long propagation L={L}, {args.steps} steps of dt=0.1, sigma=1, "
                       "random product state, autonormalise off",
           "nspins": L, "steps": args.steps, "epsilon": args.epsilon}
    stream, e0, e1 = _events(eng)
    runs = {}
    for name, prec in (("fp64_plain", abi.FP64), ("mixed_plain", abi.MIXED)):
        e0.record(stream)
        times, rows = run_realization(eng, cfg, 0, points, width, prec)
        e1.record(stream)
        e1.synchronize()
        runs[name] = rows
        norm, energy = rows[:, 0], rows[:, 2]
        rep[name] = {"seconds": e0.elapsed_time(e1) / 1e3,
                     "norm_drift": float(np.abs(norm - norm[0]).max()),
                     "energy_drift": float(np.abs(energy - energy[0]).max()),
                     "energy0": float(energy[0])}
        print(json.dumps({name: rep[name]}), flush=True)
    fp64, mixed = runs["fp64_plain"], runs["mixed_plain"]
    scale = abs(fp64[0, 3]) if abs(fp64[0, 3]) > 0 else 1.0
    rep["mixed_plain"].update({
        "norm_vs_fp64": float(np.abs(mixed[:, 0] - fp64[:, 0]).max()),
        "energy_vs_fp64": float(np.abs(mixed[:, 2] - fp64[:, 2]).max()),
        "energy_vs_fp64_relative": float(np.abs(mixed[:, 2] - fp64[:, 2]).max()
                                         / max(abs(fp64[0, 2]), 1e-300)),
        "corr_z_error_vs_fp64": float(np.abs(mixed[:, 3:5] - fp64[:, 3:5]).max() / scale),
        "corr_z_error_curve": [float(x) for x in
                               np.abs(mixed[:, 3] - fp64[:, 3]) / scale]})
    if L <= 16:
        b = Batch(eng, cfg, 0, 1, abi.MIXED)
        b.upload()
        b.execute()
        eng.synchronize()
        e0.record(stream)
        b.execute()
        e1.record(stream)
        e1.synchronize()
        _, bm = b.download()
        bm = bm[0]
        rep["mixed_batch_of_one"] = {
            "seconds": e0.elapsed_time(e1) / 1e3,
            "norm_vs_fp64": float(np.abs(bm[:, 0] - fp64[:, 0]).max()),
            "energy_vs_fp64": float(np.abs(bm[:, 2] - fp64[:, 2]).max()),
            "corr_z_error_vs_fp64": float(np.abs(bm[:, 3] - fp64[:, 3]).max() / scale)}
        b._destroy()
    eng.close()
    return rep


def plain(args) -> dict:
    """The plain path's kernels on single large vectors.  For each L and each
    (precision, kernel family): milliseconds per Chebyshev order, the
    effective bandwidth at the algorithmic bytes per amplitude-order (80 B
    FP64, 56 B mixed: T_{n-1}, T_{n-2}, T_n, psi read and write; +8 B for the
    streamed diagonal is not counted), the DRAM bytes the tiled kernel's
    passes move by construction (48 P + 40 / 24 P + 40 B), anti-aligned pair
    terms applied per second, and the mixed result's deviation from FP64 after
    the timed steps.  Then the streaming StateVector kernels at L = 26 (1 GiB
    vectors), which have no partner gathers."""
    from . import Hamiltonian, Propagator, StateVector, tiled_plan, tiled_select
    eng = Engine(0)
    stream, e0, e1 = _events(eng)
    rep = {"order_kernel": {}, "streaming": {}}
    combos = [("fp64", abi.FP64, "gather", abi.KERNEL_GATHER, 0),
              ("mixed", abi.MIXED, "gather", abi.KERNEL_GATHER, 0)]
    combos += [("fp64", abi.FP64, "tiled", abi.KERNEL_TILED, r) for r in args.fp64_bits]
    combos += [("mixed", abi.MIXED, "tiled", abi.KERNEL_TILED, r) for r in args.mixed_bits]
    default_fp64 = f"tiled_r{args.fp64_bits[0]}" if args.fp64_bits else "tiled_r3"
    for L in args.sizes:
        spec = workloads.long_propagation(nspins=L, steps=1, every=1, epsilon=1e-7)
        cfg = spec.config()
        s = realization_setup(cfg, 0, L)
        ham = Hamiltonian(eng, L, s["fields"], s["pairs"], s["J"])
        amps = float(1 << L)
        npairs = len(s["pairs"]) // 2
        out = {"pairs": npairs}
        final = {}
        for pname, prec, kname, kern, bits in combos:
            if kname in args.skip or (kname == "gather" and L > args.gather_max):
                continue
            if kname == "tiled":
                tiled_select(prec, bits)
                kname = f"tiled_r{bits}"
            psi = StateVector(eng, L, s["psi0"])
            prop = Propagator(L, 1e-7, prec, kern)
            prop.evolve(ham, abi.REAL, psi, 0.1, 1)          # warm-up, builds the tables
            eng.synchronize()
            e0.record(stream)
            prop.evolve(ham, abi.REAL, psi, 0.1, args.steps)
            e1.record(stream)
            e1.synchronize()
            sec = e0.elapsed_time(e1) / 1e3
            orders = prop.last_order * args.steps
            alg = 80.0 if prec == abi.FP64 else 56.0
            r = {"orders": int(orders), "ms_per_order": 1e3 * sec / orders,
                 "effective_gbs": alg * amps * orders / sec / 1e9, "algorithmic_bytes": alg,
                 "pair_terms_per_s": 0.5 * npairs * amps * orders / sec}
            if kname.startswith("tiled"):
                P = len(tiled_plan(L, prec))
                r["passes"] = P
                r["pass_bytes"] = (48.0 * P + 24.0) if prec == abi.FP64 else (24.0 * P + 24.0)
                r["pass_gbs"] = r["pass_bytes"] * amps * orders / sec / 1e9
            final[(pname, kname)] = psi.download()
            out[f"{pname}_{kname}"] = r
            del psi
        ref = final.get(("fp64", "gather"), final.get(("fp64", default_fp64)))
        for key, v in final.items():
            if ref is not None and key != ("fp64", "gather"):
                out[f"{key[0]}_{key[1]}"]["max_dev_vs_fp64"] = float(np.abs(v - ref).max())
        rep["order_kernel"][int(L)] = out
        del ham
        tiled_select(abi.FP64, 0)
        tiled_select(abi.MIXED, 0)
        print(json.dumps({int(L): out}), flush=True)
    L = 26
    a = StateVector(eng, L)
    b = StateVector(eng, L)
    a.set_basis_state(0)
    b.set_basis_state(1)
    n = float(1 << L)
    for name, fn, nbytes in (("add_scaled", lambda: a.add_scaled(0.5, 0.25, b), 48.0),
                             ("scale", lambda: a.scale(1.0), 32.0),
                             ("norm", lambda: a.norm(), 16.0)):
        fn()
        eng.synchronize()
        reps = 20
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        sec = e0.elapsed_time(e1) / 1e3 / reps
        rep["streaming"][name] = {"bytes_per_amp": nbytes, "gbs": nbytes * n / sec / 1e9}
    eng.close()
    return rep


def per_size(args) -> dict:
    """The uneven batch's program (CPMG-32, sigma and tau ~ U[0.1, 1]) at one
    L at a time: the batched mixed engine (tuned) on enough realisations to
    fill the device, against the plain FP64 path on a sample of the same
    realisations, one at a time."""
    eng = Engine(0)
    rep = {}
    for L, n in zip(args.sizes, args.counts):
        spec = workloads.cpmg_uneven(realizations=n)
        spec.spin_choices = (L,)
        cfg = spec.config()
        tune(eng, cfg, 0, min(n, 64), abi.MIXED)
        b = Batch(eng, cfg, 0, n, abi.MIXED)
        b.upload()
        b.execute()
        eng.synchronize()
        stream, e0, e1 = _events(eng)
        e0.record(stream)
        b.execute()
        e1.record(stream)
        e1.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        _, mixed = b.download()
        _, amp = b.work()
        ts, es = [], []
        scale = corr0(cfg, range(args.plain_sample), 16)
        for i in range(args.plain_sample):
            t0 = time.perf_counter()
            _, ref = run_realization(eng, cfg, i, b.points, b.width)
            ts.append(time.perf_counter() - t0)
            es.append(float(np.abs(mixed[i, :, 0] - ref[:, 0]).max() / scale[i]))
        # Realisations differ ~10x in work: the plain path's time for the whole
        # batch is its measured seconds per amplitude-order times the batch's.
        plain_s = sum(ts) * float(amp.sum()) / float(amp[: args.plain_sample].sum())
        rate_b, rate_p = n / sec, n / plain_s
        rep[int(L)] = {"realizations": n, "batched_mixed_curves_per_s": rate_b,
                       "plain_fp64_curves_per_s": rate_p, "ratio": rate_b / rate_p,
                       "plain_sample": args.plain_sample,
                       "plain_scaling": "seconds per amplitude-order of the sample x the "
                                        "batch's amplitude-orders",
                       "echo_error_max": max(es),
                       "fp64_routed": int((b.precisions() == abi.FP64).sum()),
                       "schedule": {r["precision"]: r["variant"] for r in schedule()
                                    if r["L"] == L}}
        b._destroy()
    eng.close()
    return rep

def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description="measurement runs beside the headline benchmark")
    sub = ap.add_subparsers(dest="cmd", required=True)
    u = sub.add_parser("uneven")
    u.add_argument("--realizations", type=int, default=4096)
    u.add_argument("--steps", type=int, default=1)
    u.add_argument("--warmup", type=int, default=0,
                   help="untimed runs first (the graph is instantiated at creation)")
    u.add_argument("--tune-sample", type=int, default=64)
    u.add_argument("--plain-sample", type=int, default=16)
    u.add_argument("--no-e2e", dest="e2e", action="store_false", default=True,
                   help="skip the end-to-end run through ss_batch_run")
    u.add_argument("--out", default="")
    lo = sub.add_parser("long")
    lo.add_argument("--nspins", type=int, default=16)
    lo.add_argument("--steps", type=int, default=10000)
    lo.add_argument("--every", type=int, default=100)
    lo.add_argument("--epsilon", type=float, default=1e-12)
    lo.add_argument("--out", default="")
    pl = sub.add_parser("plain")
    pl.add_argument("--sizes", type=int, nargs="+", default=[16, 20, 22, 24])
    pl.add_argument("--steps", type=int, default=2)
    pl.add_argument("--skip", nargs="*", default=[], help="kernel families to leave out")
    pl.add_argument("--fp64-bits", type=int, nargs="+", default=[3, 4],
                    help="register bits of the FP64 tiled schedules to time (the first is "
                         "the reference for the deviations when the gather kernel is skipped)")
    pl.add_argument("--mixed-bits", type=int, nargs="+", default=[4, 5],
                    help="register bits of the mixed tiled schedules to time")
    pl.add_argument("--gather-max", type=int, default=30,
                    help="largest L timed with the gather kernel")
    pl.add_argument("--out", default="")
    ro = sub.add_parser("routing")
    ro.add_argument("--program", choices=["xy8", "cpmg"], default="xy8")
    ro.add_argument("--sizes", type=int, nargs="+", default=[12, 14, 16])
    ro.add_argument("--counts", type=int, nargs="+", default=[1024, 296, 72])
    ro.add_argument("--norm", action="store_true",
                    help="also measure the state and reference norms (drift per curve)")
    ro.add_argument("--out", default="")
    ps = sub.add_parser("per_size")
    ps.add_argument("--sizes", type=int, nargs="+", default=[12, 14, 16])
    ps.add_argument("--counts", type=int, nargs="+", default=[1184, 592, 112])
    ps.add_argument("--plain-sample", type=int, default=4)
    ps.add_argument("--out", default="")
    args = ap.parse_args(argv)
    rep = {"uneven": uneven, "long": long_run, "plain": plain,
           "per_size": per_size, "routing": routing}[args.cmd](args)
    text = json.dumps(rep, indent=1)
    print(text)
    if args.out:
        Path(args.out).write_text(text + "\n")


if __name__ == "__main__":
    main()
