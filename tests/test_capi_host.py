"""The C ABI library without a GPU: it loads, exports every symbol the public
header declares, and its host-side entry points (Bessel, Chebyshev order rule,
rotation matrices, realisation assembly) agree with the oracle bit for bit."""
import ctypes as C

import numpy as np
import pytest

import spin_systems_b200 as ss
from spin_systems_b200 import abi, workloads


def test_library_exports_every_declared_symbol():
    lib = ss.load()
    declared = ss.header_symbols()
    assert len(declared) >= 50
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, missing


def test_engine_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ss.NoDeviceError):
        ss.Engine(0)


@pytest.mark.parametrize("kind", [0, 1])
def test_bessel_is_bit_identical_to_the_oracle(port, kind):
    for x in (1e-6, 0.01, 0.5, 1.0, 7.3, 50.0, 350.0, 700.0):
        if kind == 1 and x > 709:
            continue
        a, na = ss.bessel(kind, x, 400)
        b, nb = port.bessel(kind, x, 400)
        assert np.array_equal(a, b) and na == nb


def test_bessel_matches_reference_tables(bessel_golden):
    for kind, x, vals in zip(bessel_golden["kinds"], bessel_golden["x"], bessel_golden["values"]):
        if kind == 1 and x > 709:
            continue
        got, _ = ss.bessel(int(kind), float(x), len(vals))
        tol = 1e-14 if kind == 0 else 1e-13
        assert np.all(np.abs(got - vals) < tol * np.abs(vals).max())


def test_bessel_errors():
    with pytest.raises(ss.InvalidArgumentError):
        ss.bessel(0, -1.0, 4)
    with pytest.raises(ss.SpinsimError) as e:
        ss.bessel(1, 1000.0, 4)
    assert e.value.kind == "overflow"


def test_chebyshev_order_rule_matches_the_oracle(port):
    for mode in (0, 1):
        for bound, tau, eps in ((3.0, 0.1, 1e-7), (365.0, 0.125, 1e-7), (2000.0, 0.5, 1e-7),
                                (10.0, -0.7, 1e-12), (1.0, 1e-12, 1e-7)):
            if mode == 1 and bound * abs(tau) > 700:
                continue
            a, ba = ss.chebyshev(mode, bound, tau, eps)
            b, bb = port.chebyshev(mode, bound, tau, eps)
            assert np.array_equal(a, b) and ba == bb


def test_chebyshev_identity_and_convergence_error():
    a, b = ss.chebyshev(0, 1.0, 1e-12, 1e-7)
    assert list(a) == [1.0] and b == 1.0
    with pytest.raises(ss.ConvergenceError) as e:
        ss.chebyshev(0, 1.0, 1e6, 1e-7, 100)
    assert "tau" in str(e.value)


def test_rotation_matrix_matches_the_oracle(port):
    for axis in ((1, 0, 0), (0, 1, 0), (0, 0, 1), (0.3, -0.5, 0.8)):
        for angle in (0.25 * np.pi, 0.5 * np.pi, np.pi, 1.7):
            assert np.array_equal(ss.rotation_matrix(axis, angle), port.rotation_matrix(axis, angle))
    with pytest.raises(ss.InvalidArgumentError):
        ss.rotation_matrix((0, 0, 0), 1.0)


@pytest.mark.parametrize("spec", [workloads.cpmg_ideal(), workloads.xy8_finite(realizations=8),
                                  workloads.long_propagation(nspins=8),
                                  workloads.cpmg_uneven(realizations=16)])
def test_realisation_assembly_is_bit_identical(port, spec):
    cfg = spec.config()
    lmax = spec.max_spins()
    for idx in range(min(8, spec.realizations)):
        a = ss.realization_setup(cfg, idx, lmax)
        b = port.setup(cfg, idx, lmax)
        assert a["L"] == b["L"]
        for k in ("fields", "pairs", "J", "psi0"):
            assert np.array_equal(a[k], b[k]), k


def test_uneven_draws_cover_every_size(port):
    spec = workloads.cpmg_uneven(realizations=200)
    cfg = spec.config()
    sizes = {ss.realization_setup(cfg, i, 16)["L"] for i in range(200)}
    assert sizes == {8, 10, 12, 14, 16}


def test_program_flattening_counts_measurements():
    spec = workloads.xy8_finite()
    assert spec.measurement_count() == 128
    cfg = spec.config()
    assert cfg.n_steps == 1 + 8 * 4
    assert cfg.steps[0].kind == abi.REPEAT and cfg.steps[0].body_len == 32

