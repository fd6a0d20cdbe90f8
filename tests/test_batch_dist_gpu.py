"""Batched sizes whose vectors are spread over a thread-block cluster
(k_batch_dist: L = 13..16 in FP64, 14..16 mixed), against the C port of the
reference on fresh realisations.  Same bars as the one-CTA sizes: FP64 to
1e-10, mixed precision to 1e-6 in echo error.  The short program puts
transverse fields, ideal pulses, every observable (a magnetisation on a
spin held across CTAs included) and both time modes on the cross-CTA paths.
"""
import math

import numpy as np
import pytest

import spin_systems_b200 as ss
from spin_systems_b200 import abi, workloads
from spin_systems_b200.abi import AXES3, Evolve, Measure, Pulse, RunSpec

pytestmark = pytest.mark.gpu

ECHO_TOL = 1e-6


def short_spec(L, realizations, sigma=0.5):
    spec = RunSpec(nspins=L, steps=[], observables=["corr:x", "corr:y", "norm", "energy",
                                                   "mag:1:x", f"mag:{L}:z"],
                   realizations=realizations, seed=20240726, field_disorder=sigma,
                   reference_axis="x")
    hx = spec.fields_for(hx=50.0)
    hy = spec.fields_for(hy=50.0)
    spec.steps = [Pulse(0.5 * math.pi, AXES3["x"]), Evolve(0.1), Measure(),
                  Evolve(math.pi / 50, fields=hx), Evolve(0.1), Measure(),
                  Pulse(math.pi, AXES3["y"]), Evolve(math.pi / 100, fields=hy), Measure()]
    return spec


def corr0(cfg, count, L):
    out = []
    for i in range(count):
        s = ss.realization_setup(cfg, i, L)
        psi = s["psi0"][0::2] + 1j * s["psi0"][1::2]
        k = np.arange(1 << s["L"])
        ref = sum(psi[k ^ (1 << q)] for q in range(s["L"]))
        out.append(np.vdot(ref, ref).real)
    return np.array(out)


@pytest.mark.parametrize("L", [13, 14, 15, 16])
def test_fp64_cluster_sizes_match_the_oracle(engine, port, L):
    # L = 16 runs on split clusters of 16 CTAs (its only FP64 schedule)
    n = 2 if L < 16 else 1
    spec = short_spec(L, n)
    cfg = spec.config()
    want = np.stack([port.run_realization(cfg, i)[1] for i in range(n)])
    b = ss.Batch(engine, cfg, 0, n, abi.FP64)
    assert (b.precisions() == abi.FP64).all()
    _, rows = b.run()
    assert np.abs(rows - want).max() < 1e-10


@pytest.mark.parametrize("L", [14, 15, 16])
def test_mixed_cluster_sizes_echo_error(engine, port, L):
    n = 2 if L < 16 else 1
    spec = short_spec(L, n)
    cfg = spec.config()
    want = np.stack([port.run_realization(cfg, i)[1] for i in range(n)])
    _, rows = ss.Batch(engine, cfg, 0, n, abi.MIXED).run()
    err = np.abs(rows[:, :, 0] - want[:, :, 0]).max(axis=1) / corr0(cfg, n, L)
    assert err.max() < ECHO_TOL, err
    assert np.abs(rows[:, :, 4:6] - want[:, :, 4:6]).max() < 1e-6  # norms


def test_cluster_imaginary_time_and_autonormalise(engine, port):
    steps = [Measure(), abi.Repeat(2, [Evolve(0.05, steps=2, mode=abi.IMAGINARY,
                                              autonormalize=True), Measure()])]
    spec = RunSpec(nspins=14, steps=steps, observables=["norm", "energy", "corr:z"],
                   realizations=2, seed=11, field_disorder=0.7, dipolar_scale=0.01,
                   base_fields=[(0.3, 0.0, 0.0)] * 14)
    cfg = spec.config()
    want = np.stack([port.run_realization(cfg, i)[1] for i in range(2)])
    _, rows = ss.Batch(engine, cfg, 0, 2, abi.FP64).run()
    assert np.abs(rows - want).max() < 1e-10


def test_uneven_batch_up_to_l16_in_one_launch(engine, port):
    spec = workloads.cpmg_uneven(realizations=10, pulses=2)
    spec.spin_choices = (8, 12, 14, 16)
    spec.tau_range = (0.05, 0.15)
    cfg = spec.config()
    want = [port.run_realization(cfg, i)[1] for i in range(10)]
    b = ss.Batch(engine, cfg, 0, 10, abi.MIXED)
    _, rows = b.run()
    Ls = [ss.realization_setup(cfg, i, 16)["L"] for i in range(10)]
    assert {14, 16} <= set(Ls)
    scale = corr0(cfg, 10, 16)
    for i in range(10):
        err = np.abs(rows[i, :, 0] - want[i][:, 0]).max() / scale[i]
        assert err < ECHO_TOL, (i, Ls[i], err)


def test_cluster_sizes_cap_the_observable_count(engine):
    # The cluster kernel's measurement holds at most eight observables; the
    # batch refuses more when it is built, before any launch.
    spec = short_spec(14, 1)
    spec.observables = ["corr:x", "corr:y", "corr:z", "norm", "energy"] + \
        [f"mag:{s}:x" for s in range(1, 6)]
    with pytest.raises(ss.SpinsimError) as e:
        ss.Batch(engine, spec.config(), 0, 1, abi.MIXED)
    assert e.value.kind == "config"
