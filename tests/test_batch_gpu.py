"""Batched engine against the oracles, through the C ABI.

FP64 batches must agree with the reference (golden curves, and the C port on
fresh inputs) to 1e-10, as the plain path does.  Mixed-precision batches
(FP32 recursion, FP64 series sum and reductions) must stay within 1e-6 of
FP64 in echo error: max_t |corr_mixed(t) - corr_fp64(t)| / |corr(0)|, per
curve, where corr(0) = <A psi0|A psi0> = ||ref0||^2 (about L) is the
correlator at t = 0 for a reference prepared on the measured axis.
"""
import numpy as np
import pytest

import spin_systems_b200 as ss
from spin_systems_b200 import abi, workloads

pytestmark = pytest.mark.gpu

ECHO_TOL = 1e-6


def run(engine, spec, count, precision, first=0):
    b = ss.Batch(engine, spec.config(), first, count, precision)
    return b.run()


def corr0(spec, count, first=0):
    """corr(t=0) = ||ref0||^2 of each realisation, from the host assembly."""
    cfg = spec.config()
    out = []
    for i in range(first, first + count):
        s = ss.realization_setup(cfg, i, spec.max_spins())
        L = s["L"]
        psi = s["psi0"][0::2] + 1j * s["psi0"][1::2]
        ref = np.zeros_like(psi)
        k = np.arange(1 << L)
        for q in range(L):
            ref += psi[k ^ (1 << q)]  # A = sum sigma_x on an x-prepared reference
        out.append(np.vdot(ref, ref).real)
    return np.array(out)


def echo_error(mixed, fp64, scale):
    """Per-curve echo error on the first correlator column."""
    return np.abs(mixed[:, :, 0] - fp64[:, :, 0]).max(axis=1) / scale


def test_fp64_batch_reproduces_reference_cpmg(engine, golden):
    spec = workloads.cpmg_ideal()
    times, rows = run(engine, spec, 20, abi.FP64)
    assert np.array_equal(times, golden["curves_cpmg_times"])
    assert np.abs(rows - golden["curves_cpmg_rows"]).max() < 1e-10


def test_fp64_batch_reproduces_reference_xy8(engine, golden):
    spec = workloads.xy8_finite(nspins=8, realizations=4, blocks=2)
    spec.observables = ["corr:x", "norm", "energy", "mag:2:z"]
    times, rows = run(engine, spec, 4, abi.FP64)
    assert np.array_equal(times, golden["curves_xy8_l8_times"])
    assert np.abs(rows - golden["curves_xy8_l8_rows"]).max() < 1e-10
    spec = workloads.xy8_finite(realizations=2)
    _, rows = run(engine, spec, 2, abi.FP64)
    assert np.abs(rows - golden["curves_xy8_l12_rows"]).max() < 1e-10


@pytest.mark.parametrize("L", [6, 7, 8, 9, 10, 11, 12])
def test_fp64_batch_matches_the_oracle_at_every_size(engine, port, L):
    spec = workloads.xy8_finite(nspins=L, realizations=3, blocks=1)
    spec.observables = ["corr:x", "corr:y", "norm", "energy", "mag:1:x"]
    cfg = spec.config()
    want = np.stack([port.run_realization(cfg, i)[1] for i in range(3)])
    _, rows = run(engine, spec, 3, abi.FP64)
    assert np.abs(rows - want).max() < 1e-10


@pytest.mark.parametrize("L", [6, 7, 8, 9, 10, 11, 12, 13])
def test_mixed_batch_echo_error(engine, port, L):
    spec = workloads.xy8_finite(nspins=L, realizations=4, blocks=2)
    spec.observables = ["corr:x", "norm"]
    cfg = spec.config()
    want = np.stack([port.run_realization(cfg, i)[1] for i in range(4)])
    _, rows = run(engine, spec, 4, abi.MIXED)
    assert echo_error(rows, want, corr0(spec, 4)).max() < ECHO_TOL
    assert np.abs(rows[:, :, 2:] - want[:, :, 2:]).max() < 1e-6  # norms


def test_mixed_batch_full_xy8_against_reference(engine, golden):
    spec = workloads.xy8_finite(realizations=2)
    _, rows = run(engine, spec, 2, abi.MIXED)
    err = echo_error(rows, golden["curves_xy8_l12_rows"], corr0(spec, 2))
    assert err.max() < ECHO_TOL, err


def test_mixed_against_fp64_batch_many_realisations(engine):
    spec = workloads.xy8_finite(realizations=64, blocks=4)
    _, mixed = run(engine, spec, 64, abi.MIXED)
    _, fp64 = run(engine, spec, 64, abi.FP64)
    err = echo_error(mixed, fp64, corr0(spec, 64))
    assert err.max() < ECHO_TOL, err.max()


def orders_per_state(port, spec, count):
    """Chebyshev orders per state vector of each XY-8 realisation."""
    cfg, L = spec.config(), spec.nspins
    fx = np.array(spec.fields_for(hx=50.0)).ravel()
    fy = np.array(spec.fields_for(hy=50.0)).ravel()
    blocks = spec.steps[0].count
    out = []
    for i in range(count):
        s = port.setup(cfg, i, L)
        total = 0
        # per XY-8 block: 16 half-intervals, 4 x pulses, 4 y pulses
        for f, tau, n in ((s["fields"], 0.125, 16 * blocks), (fx, np.pi / 50, 4 * blocks),
                          (fy, np.pi / 50, 4 * blocks)):
            a, _ = port.chebyshev(0, port.spectral_bound(L, f, s["J"]), tau, spec.epsilon)
            total += (len(a) - 1) * n
        out.append(total)
    return np.array(out)


def test_mixed_routes_long_realisations_to_fp64(engine, port):
    # Full XY-8 x 16 at L = 12: realisations past the size's default limit
    # (38600 orders per state) run in the FP64 kernel of the same batch,
    # bit-identical to an FP64 batch.
    n = 192
    spec = workloads.xy8_finite(realizations=n)
    orders = orders_per_state(port, spec, n)
    b = ss.Batch(engine, spec.config(), 0, n, abi.MIXED)
    prec = b.precisions()
    assert np.array_equal(prec == abi.FP64, orders > 38600)
    assert (prec == abi.FP64).any() and (prec == abi.MIXED).any()
    _, mixed = b.run()
    _, fp64 = run(engine, spec, n, abi.FP64)
    routed = prec == abi.FP64
    assert np.array_equal(mixed[routed], fp64[routed])
    err = echo_error(mixed, fp64, corr0(spec, n))
    assert err.max() < ECHO_TOL, (err.max(), int(err.argmax()))


def test_mixed_order_limit_switches(engine):
    spec = workloads.xy8_finite(nspins=10, realizations=6, blocks=2)
    spec.mixed_order_limit = 1
    b = ss.Batch(engine, spec.config(), 0, 6, abi.MIXED)
    assert (b.precisions() == abi.FP64).all()
    _, every = b.run()
    _, fp64 = run(engine, spec, 6, abi.FP64)
    assert np.array_equal(every, fp64)
    spec.mixed_order_limit = -1
    assert (ss.Batch(engine, spec.config(), 0, 6, abi.MIXED).precisions() == abi.MIXED).all()
    spec16 = workloads.xy8_finite(nspins=16, realizations=2, blocks=1)
    spec16.mixed_order_limit = 1  # an explicit limit routes L = 16 to its FP64 kernel
    assert (ss.Batch(engine, spec16.config(), 0, 2, abi.MIXED).precisions() == abi.FP64).all()
    spec16.mixed_order_limit = 0  # the default keeps L = 16 mixed
    assert (ss.Batch(engine, spec16.config(), 0, 2, abi.MIXED).precisions() == abi.MIXED).all()
    assert (ss.Batch(engine, spec.config(), 0, 6, abi.FP64).precisions() == abi.FP64).all()


def test_uneven_sizes_share_one_launch(engine, port):
    spec = workloads.cpmg_uneven(realizations=12, pulses=4)
    spec.spin_choices = (8, 10, 12)
    spec.nspins = 12
    cfg = spec.config()
    want = np.stack([port.run_realization(cfg, i)[1] for i in range(12)])
    _, rows = run(engine, spec, 12, abi.FP64)
    assert np.abs(rows - want).max() < 1e-10
    _, rows = run(engine, spec, 12, abi.MIXED)
    assert echo_error(rows, want, corr0(spec, 12)).max() < ECHO_TOL


def test_imaginary_time_and_autonormalise(engine, port):
    # Imaginary time sums series terms of size up to I_0(alpha) ~ e^alpha to a
    # result of size ~1, so rounding differences grow like e^alpha: the case
    # keeps alpha = bound * tau below 1 (weak couplings, dipolar_scale 0.01).
    steps = [abi.Measure(), abi.Repeat(3, [abi.Evolve(0.05, steps=2, mode=abi.IMAGINARY,
                                                      autonormalize=True), abi.Measure()])]
    spec = abi.RunSpec(nspins=8, steps=steps, observables=["norm", "energy", "corr:z"],
                       realizations=3, seed=11, field_disorder=0.7, dipolar_scale=0.01,
                       base_fields=[(0.3, 0.0, 0.0)] * 8)
    cfg = spec.config()
    want = np.stack([port.run_realization(cfg, i)[1] for i in range(3)])
    _, rows = run(engine, spec, 3, abi.FP64)
    assert np.abs(rows - want).max() < 1e-10


def test_batch_offset_and_determinism(engine, golden):
    spec = workloads.cpmg_ideal()
    b = ss.Batch(engine, spec.config(), 5, 10, abi.MIXED)
    _, a = b.run()
    _, c = b.run()
    assert np.array_equal(a, c)
    assert echo_error(a, golden["curves_cpmg_rows"][5:15], corr0(spec, 10, 5)).max() < ECHO_TOL


def test_batch_rejects_unsupported_sizes(engine):
    spec = workloads.cpmg_ideal(nspins=4, realizations=2)
    with pytest.raises(ss.InvalidArgumentError):
        ss.Batch(engine, spec.config(), 0, 2, abi.MIXED)
