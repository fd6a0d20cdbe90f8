"""The benchmark workloads, as pulse programs.

Each function returns a RunSpec with the shapes the engine is measured on:
seeded synthetic realisations (seed 20240726, streams per (seed, index)),
2D dipolar geometry at unit areal density and Gaussian Hz disorder, exactly as
the reference's ensemble code draws them (src/ensemble/Ensemble.cpp:60-112).
"""
from __future__ import annotations

import math

from .abi import Evolve, Measure, Pulse, Repeat, RunSpec, AXES3

SEED = 20240726


def cpmg_ideal(nspins: int = 10, realizations: int = 20, sigma: float = 0.5,
               tau: float = 0.5, echoes: int = 8) -> RunSpec:
    """Plain CPMG echo: ideal pi/2_x, then echoes x (tau, pi_y, tau, measure);
    total S^x correlator against an x-prepared reference (L=10, 20 realisations)."""
    steps = [
        Pulse(0.5 * math.pi, AXES3["x"]),
        Repeat(echoes, [Evolve(tau), Pulse(math.pi, AXES3["y"]), Evolve(tau), Measure()]),
    ]
    return RunSpec(nspins=nspins, steps=steps, observables=["corr:x", "norm"],
                   realizations=realizations, seed=SEED, field_disorder=sigma,
                   reference_axis="x")


def xy8_finite(nspins: int = 12, realizations: int = 1024, sigma: float = 0.5,
               tau: float = 0.25, blocks: int = 16, amplitude: float = 50.0) -> RunSpec:
    """XY-8 (X Y X Y Y X Y X) repeated `blocks` times with realistic pulses:
    each pi pulse is evolution for pi/amplitude under a transverse field of
    `amplitude` along x or y.  Pulses are centred in intervals of `tau`
    (tau/2, pulse, tau/2) and S^x is measured after every interval, giving
    8 * blocks = 128 points."""
    spec = RunSpec(nspins=nspins, steps=[], observables=["corr:x"],
                   realizations=realizations, seed=SEED, field_disorder=sigma,
                   reference_axis="x")
    width = math.pi / amplitude
    px = Evolve(width, fields=spec.fields_for(hx=amplitude))
    py = Evolve(width, fields=spec.fields_for(hy=amplitude))
    body = []
    for p in "XYXYYXYX":
        body += [Evolve(0.5 * tau), px if p == "X" else py, Evolve(0.5 * tau), Measure()]
    spec.steps = [Repeat(blocks, body)]
    return spec


def cpmg_uneven(realizations: int = 4096, pulses: int = 32) -> RunSpec:
    """Uneven batch: L drawn from {8,10,12,14,16}, sigma ~ U[0.1,1] and
    tau ~ U[0.1,1] per realisation from a harness stream that leaves the
    (seed, index) geometry stream untouched; CPMG with `pulses` ideal pi_y,
    each echo (tau, pi_y, tau, measure) as in the L=10 CPMG."""
    steps = [
        Pulse(0.5 * math.pi, AXES3["x"]),
        Repeat(pulses, [Evolve(1.0, tau_from_draw=True), Pulse(math.pi, AXES3["y"]),
                        Evolve(1.0, tau_from_draw=True), Measure()]),
    ]
    return RunSpec(nspins=16, steps=steps, observables=["corr:x"],
                   realizations=realizations, seed=SEED, reference_axis="x",
                   field_disorder=0.5, draw_seed=SEED ^ 0x5EED,
                   disorder_range=(0.1, 1.0), tau_range=(0.1, 1.0),
                   spin_choices=(8, 10, 12, 14, 16))


def long_propagation(nspins: int = 16, steps: int = 10000, dt: float = 0.1,
                     every: int = 100, epsilon: float = 1e-12) -> RunSpec:
    """Single-realisation long propagation from a random product state,
    autonormalisation off, norm and energy every `every` steps.  The
    coefficient cutoff defaults to 1e-12, the reference's own choice for its
    exactness and conservation tests (tests/test_Propagator.cpp); at its
    run default of 1e-7 the truncated tail alone moves the norm by ~1e-8
    per step."""
    prog = [Measure(), Repeat(steps // every, [Evolve(dt, steps=every), Measure()])]
    return RunSpec(nspins=nspins, steps=prog, observables=["norm", "energy", "corr:z"],
                   realizations=1, seed=SEED, field_disorder=1.0,
                   initial_state="random_product", reference_axis="z", epsilon=epsilon)
