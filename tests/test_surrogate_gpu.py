"""The learned echo surrogate end to end on the device: batched sweeps equal
the plain batches they stand for, and a network trained on engine-generated
curves beats the method without it (reusing the nearest precomputed curve)
at a fraction of the exact propagator's cost, with the exact propagator as
the fallback.  Small case: L = 10, short tau, 4 realisations per point."""
import math
import time

import numpy as np
import pytest

import spin_systems_b200 as ss
from spin_systems_b200 import abi, surrogate as sg
from spin_systems_b200.abi import AXES3, Evolve, Measure, Pulse, Repeat, RunSpec

pytestmark = pytest.mark.gpu


def _plain_spec(seq, L, scale, sigma, tau, angle, R):
    steps = sg.program(seq, points=16)

    def fix(nodes):
        out = []
        for n in nodes:
            if isinstance(n, Evolve):
                out.append(Evolve(n.tau * tau))
            elif isinstance(n, Pulse):
                out.append(Pulse(n.angle * angle, n.axis))
            elif isinstance(n, Repeat):
                out.append(Repeat(n.count, fix(n.body)))
            else:
                out.append(n)
        return out
    return RunSpec(nspins=L, steps=fix(steps), observables=["corr:x", "norm"], realizations=R,
                   seed=sg.SEED, reference_axis="x", dipolar_scale=scale, field_disorder=sigma)


def test_sweep_equals_the_batches_it_stands_for(engine):
    rows = [(0.7, 0.4, 0.15, 1.02), (1.9, 1.1, 0.08, 0.97)]
    R = 3
    spec = RunSpec(nspins=10, steps=sg.program(1, points=16), observables=["corr:x", "norm"],
                   realizations=R, seed=sg.SEED, reference_axis="x", sweep=rows)
    _, got = ss.Batch(engine, spec.config(), 0, 2 * R, abi.FP64).run()
    for p, (scale, sigma, tau, angle) in enumerate(rows):
        ps = _plain_spec(1, 10, scale, sigma, tau, angle, R)
        _, want = ss.Batch(engine, ps.config(), 0, R, abi.FP64).run()
        assert np.abs(got[p * R:(p + 1) * R] - want).max() <= 1e-13


def test_surrogate_gains_over_the_method_without_it(engine):
    ranges = {"tau": (0.05, 0.2)}
    p = sg.sample(768, 5, sizes=(10,), ranges=ranges)
    y = sg.exact(engine, p, 4, mixed_order_limit=-1)
    ptr, ytr = p[:512], y[:512]
    pcal, ycal = p[512:640], y[512:640]
    pte, yte = p[640:], y[640:]
    sur = sg.Surrogate(engine, batch=256, seed=2)
    losses = sur.fit(ptr, ytr, 1500, 2e-3, 1e-5, seed=2)
    assert losses[-50:].mean() < 0.2 * losses[:10].mean()
    sur.calibrate(pcal, ycal)
    t0 = time.perf_counter()
    pred = sur.raw(pte)
    t_net = time.perf_counter() - t0
    t0 = time.perf_counter()
    exact = sg.exact(engine, pte, 4, mixed_order_limit=-1)
    t_exact = time.perf_counter() - t0
    assert np.array_equal(exact, yte)           # the exact engine is deterministic
    rms = math.sqrt(((pred - yte) ** 2).mean())
    nn = sg.nearest_neighbour(ptr, ytr, pte)
    rms_nn = math.sqrt(((nn - yte) ** 2).mean())
    print(f"surrogate rms {rms:.3g}, nearest-neighbour rms {rms_nn:.3g}, "
          f"network {t_net * 1e3:.2f} ms vs exact {t_exact * 1e3:.1f} ms")
    assert rms < 0.8 * rms_nn
    assert t_net * 20 < t_exact
    # the hybrid: network where its estimate allows, the exact engine
    # elsewhere; the tolerance here is the median estimate, so that both
    # branches are exercised at this small training size
    est = sur.estimate_error(pte)
    tol = float(np.median(est))
    calls = []

    def fallback(q):
        calls.append(len(q))
        return sg.exact(engine, q, 4, mixed_order_limit=-1)
    out, use, est = sur.predict(pte, fallback, tol=tol)
    assert np.array_equal(out[~use], yte[~use])
    err = np.abs(out - yte).max(axis=1)
    assert 0.3 <= use.mean() <= 0.7
    assert (err[use] > tol).mean() <= 0.1
    assert sum(calls) == int((~use).sum())
    sur.net._destroy()
