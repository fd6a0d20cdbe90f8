"""Pins the CPU oracle before anything is checked against it.

The C restatement (oracle/spinsim_oracle.c) is compared with
  * the reference's own golden Bessel tables (tests/data/bessel_reference.txt
    of the reference, committed as tests/golden/bessel_reference.npz) at the
    reference's tolerances (test_Bessel.cpp:90-132);
  * outputs of the reference core compiled from its sources (committed as
    tests/golden/reference_outputs.npz, and live through oracle/_ref when it
    is built here);
  * an independent dense-matrix exponential, at the tolerances of the
    reference's [propagator][exact] tests (test_Propagator.cpp:36-186).
"""
import hashlib
import math

import numpy as np
import pytest

from oracle.oracle import (dense_exp_apply, dense_hamiltonian, dense_hamiltonian_kron,
                           dense_pauli, random_state,
                           sample_hamiltonian, to_complex, to_interleaved)
from spin_systems_b200 import abi, workloads


def test_bessel_j_matches_reference_tables(port, bessel_golden):
    checked = 0
    for kind, x, vals in zip(bessel_golden["kinds"], bessel_golden["x"], bessel_golden["values"]):
        if kind != 0:
            continue
        got, _ = port.bessel(0, float(x), len(vals))
        scale = np.abs(vals).max()
        assert np.all(np.abs(got - vals) < 1e-14 * scale), x
        checked += 1
    assert checked == 14


def test_bessel_i_matches_reference_tables(port, bessel_golden):
    checked = 0
    for kind, x, vals in zip(bessel_golden["kinds"], bessel_golden["x"], bessel_golden["values"]):
        if kind != 1 or x > 709.0:
            continue
        got, _ = port.bessel(1, float(x), len(vals))
        scale = np.abs(vals).max()
        assert np.all(np.abs(got - vals) < 1e-13 * scale), x
        checked += 1
    assert checked == 14


def test_bessel_edge_cases(port):
    j, nz = port.bessel(0, 0.0, 5)
    assert j[0] == 1.0 and nz == 1 and np.all(j[1:] == 0)
    j, nz = port.bessel(0, 1e-6, 400)
    assert 0 < nz < 400 and np.all(j[nz:] == 0.0)
    from oracle.oracle import OracleError
    with pytest.raises(OracleError):
        port.bessel(0, -1.0, 4)
    with pytest.raises(OracleError):
        port.bessel(1, 1000.0, 4)


def test_random_streams_are_the_reference_streams(port, golden):
    for idx in (0, 7, 179):
        assert np.array_equal(port.rng(20240726, idx, 0, 64), golden[f"rng_u_{idx}"])
        assert np.array_equal(port.rng(20240726, idx, 1, 65), golden[f"rng_g_{idx}"])


@pytest.mark.parametrize("name,spec,count", [("cpmg", workloads.cpmg_ideal(), 20),
                                             ("xy8", workloads.xy8_finite(realizations=4), 4)])
def test_realisation_setup_is_bit_identical(port, golden, name, spec, count):
    cfg = spec.config()
    for idx in range(count):
        s = port.setup(cfg, idx, spec.nspins)
        assert np.array_equal(s["fields"], golden[f"setup_{name}_{idx}_fields"])
        assert np.array_equal(s["J"], golden[f"setup_{name}_{idx}_J"])
        assert np.array_equal(s["pairs"], golden[f"setup_{name}_{idx}_pairs"])
        assert hashlib.sha256(s["psi0"].tobytes()).digest() == bytes(golden[f"setup_{name}_{idx}_psi0_sha"])
        assert hashlib.sha256(s["ref0"].tobytes()).digest() == bytes(golden[f"setup_{name}_{idx}_ref0_sha"])


def test_propagator_matches_reference_outputs(port, golden):
    for L in range(1, 7):
        f, p, J = sample_hamiltonian(L)
        psi0 = golden[f"prop_psi0_{L}"]
        for tau in (0.05, 0.3, 1.0):
            psi, order = port.evolve(L, f, p, J, psi0, 0, tau, 1, eps=1e-12)
            assert order == int(golden[f"prop_real_order_{L}_{tau}"][0])
            assert np.abs(psi - golden[f"prop_real_{L}_{tau}"]).max() < 1e-13
        for tau in (0.05, 0.4):
            psi, _ = port.evolve(L, f, p, J, psi0, 1, tau, 1, eps=1e-12)
            assert np.abs(psi - golden[f"prop_imag_{L}_{tau}"]).max() < 1e-12


def test_real_time_propagation_matches_dense_exponential(port):
    # test_Propagator.cpp:36-67: exp(+iH tau), eps 1e-12, tolerance 1e-10.
    for L in range(1, 7):
        f, p, J = sample_hamiltonian(L)
        psi0 = random_state(L, 0x9001 + L)
        H = dense_hamiltonian(L, f, p, J)
        for tau in (0.05, 0.3, 1.0):
            psi, _ = port.evolve(L, f, p, J, psi0, 0, tau, 1, eps=1e-12)
            want = dense_exp_apply(H, 1j * tau, psi0)
            assert np.abs(to_complex(psi) - to_complex(want)).max() < 1e-10


def test_imaginary_time_matches_dense_exponential(port):
    # test_Propagator.cpp:168-186: exp(+H tau).
    L = 4
    f, p, J = sample_hamiltonian(L)
    psi0 = random_state(L, 0x1618)
    H = dense_hamiltonian(L, f, p, J)
    for tau in (0.05, 0.4):
        psi, _ = port.evolve(L, f, p, J, psi0, 1, tau, 1, eps=1e-12)
        assert np.abs(to_complex(psi) - to_complex(dense_exp_apply(H, tau, psi0))).max() < 1e-10


def test_dense_hamiltonian_matches_the_kron_products():
    # The permutation assembly against explicit kron products of the
    # single-spin matrices, every axis on fields and pairs.
    for L in range(1, 7):
        f, p, J = sample_hamiltonian(L)
        assert np.array_equal(dense_hamiltonian(L, f, p, J), dense_hamiltonian_kron(L, f, p, J))


def test_dense_pauli_algebra():
    # sigma_x sigma_y = i sigma_z in the down/up basis (DenseReference.cpp:52-58).
    x, y, z = (dense_pauli(1, 0, a) for a in "xyz")
    assert np.allclose(x @ y, 1j * z)


def test_curves_match_reference_cpmg(port, golden):
    cfg = workloads.cpmg_ideal().config()
    times, rows, _ = port.run_range(cfg, 0, 20, 4)
    assert np.array_equal(times, golden["curves_cpmg_times"])
    assert np.abs(rows - golden["curves_cpmg_rows"]).max() < 1e-12


def test_curves_match_reference_xy8_small(port, golden):
    spec = workloads.xy8_finite(nspins=8, realizations=4, blocks=2)
    spec.observables = ["corr:x", "norm", "energy", "mag:2:z"]
    times, rows, _ = port.run_range(spec.config(), 0, 4, 4)
    assert np.array_equal(times, golden["curves_xy8_l8_times"])
    assert np.abs(rows - golden["curves_xy8_l8_rows"]).max() < 1e-12


def test_correlator_starts_near_the_spin_count(port):
    # test_Config.cpp:229-249: corr(t=0) = ||A psi||^2 ~ L.
    spec = abi.RunSpec(nspins=6, steps=[abi.Measure()], observables=["corr:z"], realizations=32,
                       seed=5150, dipolar_geometry=False, reference_axis="z")
    _, rows, _ = port.run_range(spec.config(), 0, 32, 4)
    assert abs(rows[:, 0, 0].mean() - 6.0) < 0.5


def test_accumulator_textbook_values(port):
    # test_Ensemble.cpp:46-58.
    rows = np.array([2.0, 4.0, 4.0, 4.0, 5.0, 5.0, 7.0, 9.0])[:, None]
    mean, sd, se = port.accumulate(rows)
    assert mean[0] == pytest.approx(5.0)
    assert sd[0] == pytest.approx(math.sqrt(32.0 / 7.0))
    assert se[0] == pytest.approx(math.sqrt(32.0 / 7.0) / math.sqrt(8.0))


def test_port_matches_live_reference(port, ref):
    """Where the reference is built here, compare live on fresh inputs."""
    spec = workloads.xy8_finite(nspins=6, realizations=3, blocks=1)
    spec.observables = ["corr:x", "corr:y", "norm", "energy", "mag:1:x"]
    cfg = spec.config()
    for idx in range(3):
        a = port.run_realization(cfg, idx)
        b = ref.run_realization(cfg, idx)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    f, p, J = sample_hamiltonian(5)
    psi = random_state(5, 3)
    for op, axis in ((0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2)):
        for spin in range(5):
            o = random_state(5, 4)
            assert np.array_equal(port.pauli(5, op, axis, 0.75, spin, 0, None, psi, o),
                                  ref.pauli(5, op, axis, 0.75, spin, 0, None, psi, o))
    o = random_state(5, 5)
    assert np.array_equal(port.pauli(5, 2, 0, 0, 1, 3, [0.3, -1.1, 0.7], psi, o),
                          ref.pauli(5, 2, 0, 0, 1, 3, [0.3, -1.1, 0.7], psi, o))
    m = np.random.default_rng(1).standard_normal(32)
    assert np.array_equal(port.two_spin_gate(5, psi, m, 3, 1), ref.two_spin_gate(5, psi, m, 3, 1))
    for axis in ((1, 0, 0), (0.3, -0.5, 0.8)):
        assert np.array_equal(port.rotate(5, psi, axis, 1.7, [0, 2, 4]),
                              ref.rotate(5, psi, axis, 1.7, [0, 2, 4]))
