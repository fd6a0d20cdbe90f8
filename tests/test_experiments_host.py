"""Host logic of the measurement runs (no GPU): the plain path's time model
for the uneven batch, which extrapolates a timed sample of each size to all
of the size's realisations."""
import numpy as np

from spin_systems_b200.experiments import plain_time_model


def test_plain_time_model_recovers_fixed_cost_and_rate():
    amps = {16: np.linspace(1e8, 2e9, 862), 8: np.linspace(1e5, 1e6, 835)}
    raw = {}
    for L, a in amps.items():
        idx = np.unique(np.round(np.linspace(0, len(a) - 1, 16)).astype(int))
        x = a[idx]
        raw[L] = {"amplitude_orders": x.tolist(), "seconds": (0.2 + 0.3e-9 * x).tolist()}
    m = plain_time_model(raw, amps)
    p = m["per_size"][16]
    assert abs(p["fixed_seconds"] - 0.2) < 1e-9 and abs(p["ns_per_amp_order"] - 0.3) < 1e-9
    want = sum(len(a) * 0.2 + 0.3e-9 * a.sum() for a in amps.values())
    assert abs(m["seconds"] - want) < 1e-6 * want


def test_plain_time_model_clamps_to_non_negative_terms():
    amps = {12: np.array([1.0, 2.0, 3.0, 4.0])}
    # a negative intercept falls back to a line through the origin
    m = plain_time_model({12: {"amplitude_orders": [1, 2, 3, 4], "seconds": [0.5, 1.6, 2.8, 4.1]}},
                         amps)
    assert m["per_size"][12]["fixed_seconds"] == 0.0 and m["per_size"][12]["ns_per_amp_order"] > 0
    # a falling trend keeps the mean as a fixed cost
    m = plain_time_model({12: {"amplitude_orders": [1, 2, 3, 4], "seconds": [4.0, 3.0, 2.0, 1.0]}},
                         amps)
    assert m["per_size"][12]["ns_per_amp_order"] == 0.0
    assert abs(m["seconds"] - 4 * 2.5) < 1e-12
