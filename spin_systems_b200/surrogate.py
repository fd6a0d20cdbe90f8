"""Learned echo surrogate: a network from sweep parameters to the
disorder-averaged S^x echo, trained on curves the batched engine generates,
judged by the exact propagator, which is also its fallback.

Parameter space (one point = one experiment, averaged over realisations):
  areal density rho in [0.5, 2]   -> dipolar_scale = rho^(3/2) (lengths scale
                                     as rho^(-1/2), couplings as r^-3)
  field sigma in [0, 1.5]         -> Gaussian Hz disorder
  tau in [0.05, 1]                -> pulse spacing
  pulse-angle error e in [-0.05, 0.05] -> every pulse angle times (1 + e)
  sequence in {CPMG, XY-8}        -> pi/2_x, then 128 echoes:
                                     CPMG (tau, pi_y, tau, measure) x 128,
                                     XY-8 (tau/2, pi_a, tau/2, measure) for
                                     a in X Y X Y Y X Y X, x 16
  L in {10, 12, 14}
The target is the realisation average of Re corr_x(t) / ||ref||^2 at the 128
measurement times, with every point seeing the same realisations (seed
20240726, indices 0 .. R-1), so the average is a smooth function of the
continuous parameters.

Network: 6 -> 256 -> 256 -> 256 -> 128 GELU (ss_mlp_*), BF16 weights and
activations, FP32 accumulation, trained with Adam by the library's tcgen05
kernels.  The error model for the fallback is empirical: the error of a
query is estimated as the largest error of its nearest held-out calibration
points (same sequence and L), times a safety factor; a query whose estimate
exceeds the tolerance (1e-3 by default) is answered by the exact propagator.

The reference has no learned component and no sweep driver; its parameter
sweeps are separate runs of io/Experiment.cpp:57-72.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from pathlib import Path
from typing import Callable, Optional

import numpy as np

from . import Batch, ConvergenceError, Engine, Mlp, abi
from .abi import AXES3, Evolve, Measure, Pulse, Repeat, RunSpec

SEED = 20240726
RANGES = {"density": (0.5, 2.0), "sigma": (0.0, 1.5), "tau": (0.05, 1.0),
          "angle_error": (-0.05, 0.05)}
SEQUENCES = ("cpmg", "xy8")
SIZES = (10, 12, 14)
POINTS = 128
PARAMS = np.dtype([("density", "f8"), ("sigma", "f8"), ("tau", "f8"), ("angle_error", "f8"),
                   ("sequence", "i4"), ("nspins", "i4")])


def sample(n: int, seed: int, sizes=SIZES, sequences=(0, 1), ranges=None) -> np.ndarray:
    """n points drawn uniformly from the parameter space."""
    rng = np.random.default_rng(seed)
    r = dict(RANGES, **(ranges or {}))
    p = np.zeros(n, dtype=PARAMS)
    for k in ("density", "sigma", "tau", "angle_error"):
        lo, hi = r[k]
        p[k] = rng.uniform(lo, hi, n)
    p["sequence"] = rng.choice(np.asarray(sequences), n)
    p["nspins"] = rng.choice(np.asarray(sizes), n)
    return p


def features(p: np.ndarray) -> np.ndarray:
    """Network inputs in [-1, 1]: the four continuous parameters over their
    full ranges, the sequence as -1 / +1 and L as (L - 12) / 2."""
    x = np.zeros((len(p), 6), dtype=np.float32)
    for i, k in enumerate(("density", "sigma", "tau", "angle_error")):
        lo, hi = RANGES[k]
        x[:, i] = 2.0 * (p[k] - lo) / (hi - lo) - 1.0
    x[:, 4] = 2.0 * p["sequence"] - 1.0
    x[:, 5] = (p["nspins"] - 12) / 2.0
    return x


def program(sequence: int, points: int = POINTS, substeps: int = 1):
    """The pulse program; every free evolution is split into `substeps`
    equal propagation steps (the same evolution: a realisation with a very
    close pair needs shorter steps for the Chebyshev series to converge)."""
    def free(fraction):
        return Evolve(fraction / substeps, steps=substeps, tau_from_draw=True)
    if sequence == 0:
        body = [free(1.0), Pulse(math.pi, AXES3["y"]), free(1.0), Measure()]
        return [Pulse(0.5 * math.pi, AXES3["x"]), Repeat(points, body)]
    body = []
    for a in "XYXYYXYX":
        body += [free(0.5), Pulse(math.pi, AXES3[a.lower()]), free(0.5), Measure()]
    return [Pulse(0.5 * math.pi, AXES3["x"]), Repeat(points // 8, body)]


def sweep_spec(sequence: int, nspins: int, rows, realizations: int,
               mixed_order_limit: int = 0, substeps: int = 1) -> RunSpec:
    return RunSpec(nspins=nspins, steps=program(sequence, substeps=substeps),
                   observables=["corr:x", "norm"], realizations=realizations, seed=SEED,
                   reference_axis="x", sweep=rows, mixed_order_limit=mixed_order_limit)


def exact(engine: Engine, p: np.ndarray, realizations: int, precision: int = abi.MIXED,
          max_batch: int = 32768, mixed_order_limit: int = 0) -> np.ndarray:
    """The exact propagator's disorder-averaged echo [n][128] for each point,
    run as batched sweeps (one batch per sequence and L, chunked).  A chunk
    whose strongest realisation's series does not converge within the order
    limit at one step per free evolution is set up again with 2, 4, ... 64
    steps per evolution."""
    out = np.zeros((len(p), POINTS))
    per_batch = max(1, max_batch // realizations)
    for seq in np.unique(p["sequence"]):
        for L in np.unique(p["nspins"]):
            idx = np.flatnonzero((p["sequence"] == seq) & (p["nspins"] == L))
            for at in range(0, len(idx), per_batch):
                sel = idx[at:at + per_batch]
                rows = [(float(q["density"]) ** 1.5, float(q["sigma"]), float(q["tau"]),
                         1.0 + float(q["angle_error"])) for q in p[sel]]
                substeps = 1
                while True:
                    spec = sweep_spec(int(seq), int(L), rows, realizations, mixed_order_limit,
                                      substeps)
                    cfg = spec.config()
                    try:
                        b = Batch(engine, cfg, 0, len(sel) * realizations, precision)
                        break
                    except ConvergenceError:
                        if substeps >= 64:
                            raise
                        substeps *= 2
                _, r = b.run()
                b._destroy()
                echo = r[:, :, 0] / (r[:, :, 3] ** 2)
                out[sel] = echo.reshape(len(sel), realizations, POINTS).mean(axis=1)
    return out


def _groups(p: np.ndarray):
    """Indices of each (sequence, L) group."""
    key = p["sequence"].astype(np.int64) * 64 + p["nspins"].astype(np.int64)
    for k in np.unique(key):
        yield k, np.flatnonzero(key == k)


def _nearest(ref_x: np.ndarray, q_x: np.ndarray, k: int, chunk: int = 4096) -> np.ndarray:
    """Indices of the k nearest rows of ref_x for every row of q_x (squared
    Euclidean distance on the continuous features), in chunks of queries."""
    out = np.zeros((len(q_x), k), dtype=np.int64)
    rn = (ref_x ** 2).sum(axis=1)
    for at in range(0, len(q_x), chunk):
        q = q_x[at:at + chunk]
        d = (q ** 2).sum(axis=1)[:, None] + rn[None, :] - 2.0 * q @ ref_x.T
        if k >= ref_x.shape[0]:
            idx = np.argsort(d, axis=1)[:, :k]
        else:
            idx = np.argpartition(d, k - 1, axis=1)[:, :k]
        out[at:at + chunk, :idx.shape[1]] = idx
        if idx.shape[1] < k:
            out[at:at + chunk, idx.shape[1]:] = idx[:, -1:]
    return out


def nearest_neighbour(train_p: np.ndarray, train_y: np.ndarray, query: np.ndarray) -> np.ndarray:
    """The method without a network: the closest precomputed curve (feature
    distance, same sequence and L; any curve if the group has none)."""
    fx, fq = features(train_p).astype(np.float64), features(query).astype(np.float64)
    out = np.zeros((len(query), POINTS))
    tkey = train_p["sequence"].astype(np.int64) * 64 + train_p["nspins"].astype(np.int64)
    for key, qi in _groups(query):
        cand = np.flatnonzero(tkey == key)
        if len(cand) == 0:
            cand = np.arange(len(train_p))
        near = _nearest(fx[cand, :4], fq[qi, :4], 1)[:, 0]
        out[qi] = train_y[cand[near]]
    return out


class Surrogate:
    """The trained network plus its empirical error model.  With
    `standardize`, the network learns each echo point centred and scaled by
    the training curves' mean and spread at that time, and its outputs are
    mapped back."""

    def __init__(self, engine: Engine, batch: int = 1024, seed: int = 0,
                 standardize: bool = False):
        self.engine = engine
        self.net = Mlp(engine, batch=batch, seed=seed)
        self.standardize = standardize
        self.y_mean = np.zeros(POINTS)
        self.y_scale = np.ones(POINTS)
        self.cal_x: Optional[np.ndarray] = None
        self.cal_p: Optional[np.ndarray] = None
        self.cal_err: Optional[np.ndarray] = None

    def fit(self, p: np.ndarray, y: np.ndarray, steps: int, lr_start: float = 2e-3,
            lr_end: float = 1e-5, seed: int = 0) -> np.ndarray:
        y = np.asarray(y, dtype=np.float64)
        if self.standardize:
            self.y_mean = y.mean(axis=0)
            self.y_scale = np.maximum(y.std(axis=0), 1e-6)
        t = (y - self.y_mean) / self.y_scale
        self.net.set_data(features(p), t.astype(np.float32))
        return self.net.train(steps, lr_start, lr_end, seed)

    def raw(self, p: np.ndarray) -> np.ndarray:
        out = self.net.forward(features(p)).astype(np.float64)
        return out * self.y_scale + self.y_mean

    def calibrate(self, p: np.ndarray, y: np.ndarray) -> np.ndarray:
        err = np.abs(self.raw(p) - y).max(axis=1)
        self.cal_p, self.cal_x, self.cal_err = p.copy(), features(p), err
        return err

    def estimate_error(self, p: np.ndarray, k: int = 8, safety: float = 1.5) -> np.ndarray:
        """Largest calibration error among the k nearest calibration points
        (same sequence and L) times `safety`; +inf without calibration data."""
        est = np.full(len(p), np.inf)
        if self.cal_x is None:
            return est
        fq = features(p).astype(np.float64)
        cx = self.cal_x.astype(np.float64)
        ckey = self.cal_p["sequence"].astype(np.int64) * 64 + self.cal_p["nspins"].astype(np.int64)
        for key, qi in _groups(p):
            same = np.flatnonzero(ckey == key)
            if len(same) == 0:
                continue
            near = _nearest(cx[same, :4], fq[qi, :4], min(k, len(same)))
            est[qi] = safety * self.cal_err[same[near]].max(axis=1)
        return est

    def predict(self, p: np.ndarray, fallback: Callable[[np.ndarray], np.ndarray],
                tol: float = 1e-3):
        """Curves for every point: the network where its estimated error is
        within `tol`, the exact propagator (`fallback`) elsewhere.
        Returns (curves, answered_by_network, estimated_error)."""
        est = self.estimate_error(p)
        use = est <= tol
        out = np.zeros((len(p), POINTS))
        if use.any():
            out[use] = self.raw(p[use])
        if (~use).any():
            out[~use] = fallback(p[~use])
        return out, use, est


def split_counts(counts, test_points: int, cal_frac: float = 0.1):
    """(train, cal, test) points per size: `test_points` held-out points in
    all, shared in proportion to each size's points (10 % each when 0), and
    `cal_frac` of every size for calibration."""
    counts = [int(c) for c in counts]
    total = sum(counts)
    if test_points <= 0:
        test = [int(0.1 * c) for c in counts]
    else:
        if test_points >= total:
            raise SystemExit("--test-points must be below the total number of points")
        test = [int(round(test_points * c / total)) for c in counts]
        test[int(np.argmax(counts))] += test_points - sum(test)
    cal = [int(cal_frac * c) for c in counts]
    train = [c - a - b for c, a, b in zip(counts, cal, test)]
    if min(train) <= 0:
        raise SystemExit("no training points left for a size")
    return train, cal, test


def _max_err(pred: np.ndarray, y: np.ndarray) -> np.ndarray:
    return np.abs(pred - y).max(axis=1)


def _error_summary(pred: np.ndarray, y: np.ndarray) -> dict:
    err = _max_err(pred, y)
    return {"rms": float(np.sqrt(((pred - y) ** 2).mean())),
            "max_err_median": float(np.median(err)),
            "max_err_p90": float(np.quantile(err, 0.9)),
            "max_err_max": float(err.max())}


def generate(eng: Engine, sizes, counts, realizations: int, seed: int, ranges,
             save: str = "") -> dict:
    """Points and exact curves per size (all mixed precision, no routing);
    with `save`, the curves so far are written after every size."""
    data, gen = {}, {}
    for k, (L, n) in enumerate(zip(sizes, counts)):
        p = sample(n, seed + 7919 * k, sizes=(L,), ranges=ranges)
        t0 = time.perf_counter()
        y = exact(eng, p, realizations, mixed_order_limit=-1)
        dt = time.perf_counter() - t0
        gen[int(L)] = {"points": n, "seconds": dt, "curves_per_s": n * realizations / dt}
        data[int(L)] = (p, y)
        print(f"L = {L}: {n} points x {realizations} realisations in {dt:.0f} s",
              file=sys.stderr, flush=True)
        if save:
            save_data(save, data, realizations)
    return {"data": data, "generation": gen}


def save_data(path: str, data: dict, realizations: int) -> None:
    arrays = {"realizations": np.asarray(realizations)}
    for L, (p, y) in data.items():
        arrays[f"p{L}"] = p
        arrays[f"y{L}"] = y.astype(np.float32)
    np.savez_compressed(path, **arrays)


def load_data(path: str):
    z = np.load(path)
    data = {}
    for key in z.files:
        if key.startswith("p"):
            L = int(key[1:])
            data[L] = (z[key], z[f"y{L}"].astype(np.float64))
    return data, int(z["realizations"])


def run(args) -> dict:
    """Generate (or load), train, calibrate and evaluate; returns the report.
    Each size gets its own number of points (larger L costs more per curve);
    the held-out test set is `--test-points` points across the sizes, judged
    by the exact engine's curves."""
    eng = Engine(0)
    ranges = {"tau": (args.tau_min, args.tau_max)}
    if args.load_data:
        data, realizations = load_data(args.load_data)
        sizes = tuple(sorted(data))
        counts = [len(data[L][0]) for L in sizes]
        gen = None
    else:
        sizes = tuple(args.sizes)
        counts = list(args.points) if args.points else [args.train + args.cal + args.test] * len(sizes)
        if len(counts) != len(sizes):
            raise SystemExit("--points needs one count per size")
        realizations = args.realizations
        g = generate(eng, sizes, counts, realizations, args.seed, ranges, args.save_data)
        data, gen = g["data"], g["generation"]
    ntr, ncal, nte = split_counts(counts, args.test_points)
    rep: dict = {"realizations": realizations, "sizes": list(sizes), "points": counts,
                 "train_points": ntr, "cal_points": ncal, "test_points": nte,
                 "steps": args.steps, "standardize": bool(args.standardize),
                 "tau_range": list(ranges["tau"])}
    if gen is not None:
        rep["generation"] = gen
    parts = {"train": [], "cal": [], "test": []}
    for L, a, b in zip(sizes, ntr, ncal):
        p, y = data[int(L)]
        parts["train"].append((p[:a], y[:a]))
        parts["cal"].append((p[a:a + b], y[a:a + b]))
        parts["test"].append((p[a + b:], y[a + b:]))
    cat = {k: (np.concatenate([q for q, _ in v]), np.concatenate([z for _, z in v]))
           for k, v in parts.items()}
    ptr, ytr = cat["train"]
    pcal, ycal = cat["cal"]
    pte, yte = cat["test"]
    sur = Surrogate(eng, batch=args.batch, seed=args.seed, standardize=args.standardize)
    t0 = time.perf_counter()
    losses = sur.fit(ptr, ytr, args.steps, args.lr, args.lr_end, seed=args.seed)
    rep["training"] = {"points": int(len(ptr)), "seconds": time.perf_counter() - t0,
                       "loss_first": float(losses[:10].mean()),
                       "loss_last": float(losses[-50:].mean())}
    sur.calibrate(pcal, ycal)
    t0 = time.perf_counter()
    pred = sur.raw(pte)
    inf_s = time.perf_counter() - t0
    nn = nearest_neighbour(ptr, ytr, pte)
    rep["inference_curves_per_s"] = len(pte) / inf_s
    per = {}
    for L in sizes:
        m = pte["nspins"] == L
        per[int(L)] = {"test_points": int(m.sum()),
                       "surrogate": _error_summary(pred[m], yte[m]),
                       "nearest_neighbour": _error_summary(nn[m], yte[m])}
    rep["test"] = per
    rep["test_all"] = {"test_points": int(len(pte)),
                       "surrogate": _error_summary(pred, yte),
                       "nearest_neighbour": _error_summary(nn, yte)}
    # The exact engine's own cost on a sample of the test points (the same
    # realisations), for the speed comparison.
    rng = np.random.default_rng(args.seed)
    timing = np.sort(rng.choice(len(pte), min(len(pte), args.exact_timing_points),
                                replace=False))
    t0 = time.perf_counter()
    again = exact(eng, pte[timing], realizations, mixed_order_limit=-1)
    ex_s = time.perf_counter() - t0
    rep["exact_points_per_s"] = len(timing) / ex_s
    rep["exact_timing_points"] = int(len(timing))
    rep["exact_rerun_max_diff"] = float(np.abs(again - yte[timing]).max())
    rep["surrogate_speedup"] = (len(pte) / inf_s) / rep["exact_points_per_s"]
    err = _max_err(pred, yte)
    est = sur.estimate_error(pte)
    for tol in (1e-3, 1e-2, 3e-2, 1e-1):
        use = est <= tol
        rep[f"hybrid_tol_{tol:g}"] = {"answered_by_network": float(use.mean()),
                                      "violations": int(((err > tol) & use).sum()),
                                      "within_tol_at_all": float((err <= tol).mean())}
    sur.net._destroy()
    eng.close()
    return rep


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--cal", type=int, default=512)
    ap.add_argument("--test", type=int, default=512)
    ap.add_argument("--realizations", type=int, default=16)
    ap.add_argument("--sizes", type=int, nargs="+", default=[10])
    ap.add_argument("--points", type=int, nargs="+", default=None,
                    help="points per size (default: train + cal + test each)")
    ap.add_argument("--tau-min", type=float, default=RANGES["tau"][0])
    ap.add_argument("--tau-max", type=float, default=RANGES["tau"][1])
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--lr-end", type=float, default=1e-5)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--test-points", type=int, default=0,
                    help="held-out points across all sizes (default: 10 %% of each size)")
    ap.add_argument("--exact-timing-points", type=int, default=256,
                    help="test points the exact engine is re-timed on")
    ap.add_argument("--standardize", action="store_true",
                    help="train on curves centred and scaled per echo point")
    ap.add_argument("--save-data", type=str, default="", help="write the generated curves (.npz)")
    ap.add_argument("--load-data", type=str, default="",
                    help="train on curves written by --save-data instead of generating")
    ap.add_argument("--out", type=str, default="")
    args = ap.parse_args(argv)
    rep = run(args)
    text = json.dumps(rep, indent=1)
    print(text)
    if args.out:
        Path(args.out).write_text(text + "\n")


if __name__ == "__main__":
    main()
