"""Plain FP64 device path against the oracles, through the C ABI.

Tolerances are the reference's own: kernels and observables 1e-13
(test_SpinOperators.cpp, test_Observable.cpp), propagator against the exact
exponential 1e-10 (test_Propagator.cpp:36-67), conservation 1e-11 / 1e-10
(:100-124), whole echo curves 1e-10 against the reference's outputs.
"""
import math

import numpy as np
import pytest

import spin_systems_b200 as ss
from spin_systems_b200 import abi, workloads
from oracle.oracle import (dense_exp_apply, dense_hamiltonian, dense_pauli, random_state,
                           sample_hamiltonian, to_complex)

pytestmark = pytest.mark.gpu

TOL = 1e-13


def dev(engine, v):
    L = int(round(math.log2(len(v) // 2)))
    return ss.StateVector(engine, L, v)


def test_state_operations(engine):
    psi = random_state(5, 1)
    other = random_state(5, 2)
    a, b = dev(engine, psi), dev(engine, other)
    assert abs(a.norm() - np.linalg.norm(psi)) < TOL
    re, im = a.inner_product(b)
    want = np.vdot(to_complex(other), to_complex(psi))
    assert abs(re - want.real) < TOL and abs(im - want.imag) < TOL
    a.scale(2.5)
    a.add_scaled(0.3, -0.7, b)
    z = 2.5 * to_complex(psi) + (0.3 - 0.7j) * to_complex(other)
    assert np.abs(to_complex(a.download()) - z).max() < TOL
    a.negate()
    assert np.abs(to_complex(a.download()) + z).max() < TOL
    a.set_basis_state(5)
    v = a.download()
    assert v[10] == 1.0 and np.count_nonzero(v) == 1
    with pytest.raises(ss.OutOfRangeError):
        a.set_basis_state(32)
    n = b.normalize()
    assert abs(n - 1.0) < 1e-15 and abs(b.norm() - 1.0) < 1e-15
    zero = ss.StateVector(engine, 2)
    with pytest.raises(ss.DomainError):
        zero.normalize()


def test_pauli_kernels_match_the_oracle(engine, port):
    for L in range(1, 6):
        psi = random_state(L, 0x5EED + L)
        d = dev(engine, psi)
        for spin in range(L):
            for axis in range(3):
                base = random_state(L, 7)
                out = dev(engine, base)
                ss.axpy_sigma(0.75, d, spin, axis, out)
                want = port.pauli(L, 0, axis, 0.75, spin, 0, None, psi, base)
                assert np.abs(out.download() - want).max() < TOL
                ss.apply_sigma(d, spin, axis, out)
                want = port.pauli(L, 1, axis, 0.0, spin, 0, None, psi, base)
                assert np.abs(out.download() - want).max() < TOL
        for a in range(L):
            for b in range(a + 1, L):
                out = ss.StateVector(engine, L)
                ss.axpy_coupling(0.3, -1.1, 0.7, d, a, b, out)
                want = port.pauli(L, 2, 0, 0, a, b, [0.3, -1.1, 0.7], psi, np.zeros_like(psi))
                assert np.abs(out.download() - want).max() < TOL
    with pytest.raises(ss.InvalidArgumentError):
        ss.apply_sigma(d, 0, 0, d)


def test_reference_state_is_bit_identical(engine, port):
    spec = workloads.cpmg_ideal()
    cfg = spec.config()
    for idx in range(3):
        s = port.setup(cfg, idx, 10)
        psi = dev(engine, s["psi0"])
        ref = ss.StateVector(engine, 10)
        ss.apply_total_spin(abi.AXIS["x"], psi, ref)
        assert np.array_equal(ref.download(), s["ref0"])


def test_hamiltonian_matches_dense_and_oracle(engine, port):
    for L in range(1, 6):
        f, p, J = sample_hamiltonian(L)
        h = ss.Hamiltonian(engine, L, f, p, J)
        psi = random_state(L, 0x4242 + L)
        out = ss.StateVector(engine, L, random_state(L, 9))
        h.apply_physical(dev(engine, psi), out)
        got = out.download()
        assert np.abs(got - port.apply(L, f, p, J, 1.0, psi)).max() < TOL
        want = dense_hamiltonian(L, f, p, J) @ to_complex(psi)
        assert np.abs(to_complex(got) - want).max() < TOL
        bound = h.spectral_bound()
        assert bound == pytest.approx(port.spectral_bound(L, f, J), abs=0)
        h.apply_twice_normalized(bound, dev(engine, psi), out)
        assert np.abs(to_complex(out.download()) - (-2.0 / bound) * want).max() < TOL


def test_real_time_propagation_matches_exact_exponential(engine):
    # test_Propagator.cpp:36-67
    for L in range(1, 7):
        f, p, J = sample_hamiltonian(L)
        psi0 = random_state(L, 0x9001 + L)
        H = dense_hamiltonian(L, f, p, J)
        h = ss.Hamiltonian(engine, L, f, p, J)
        for tau in (0.05, 0.3, 1.0):
            psi = dev(engine, psi0)
            prop = ss.Propagator(L, 1e-12)
            prop.evolve(h, abi.REAL, psi, tau, 1)
            want = dense_exp_apply(H, 1j * tau, psi0)
            assert np.abs(to_complex(psi.download()) - to_complex(want)).max() < 1e-10


def test_propagator_matches_reference_outputs(engine, golden):
    for L in range(1, 7):
        f, p, J = sample_hamiltonian(L)
        h = ss.Hamiltonian(engine, L, f, p, J)
        for tau in (0.05, 0.3, 1.0):
            psi = dev(engine, golden[f"prop_psi0_{L}"])
            prop = ss.Propagator(L, 1e-12)
            prop.evolve(h, abi.REAL, psi, tau, 1)
            assert prop.last_order == int(golden[f"prop_real_order_{L}_{tau}"][0])
            assert np.abs(psi.download() - golden[f"prop_real_{L}_{tau}"]).max() < 1e-12


def test_many_small_steps_and_reversal(engine):
    L = 4
    f, p, J = sample_hamiltonian(L)
    h = ss.Hamiltonian(engine, L, f, p, J)
    psi0 = random_state(L, 0x5150)
    psi = dev(engine, psi0)
    ss.Propagator(L, 1e-12).evolve(h, abi.REAL, psi, 0.01, 200)
    want = dense_exp_apply(dense_hamiltonian(L, f, p, J), 2.0j, psi0)
    assert np.abs(to_complex(psi.download()) - to_complex(want)).max() < 1e-9
    psi = dev(engine, psi0)
    prop = ss.Propagator(L, 1e-12)
    prop.evolve(h, abi.REAL, psi, 0.7, 1)
    assert np.abs(psi.download() - psi0).max() > 1e-3
    prop.evolve(h, abi.REAL, psi, -0.7, 1)
    assert np.abs(to_complex(psi.download()) - to_complex(psi0)).max() < 1e-11


def test_norm_and_energy_are_conserved(engine, golden):
    # test_Propagator.cpp:100-124 replayed on the reference's own state: 10^4
    # steps of 0.02, autonormalise off.  That test's 1e-11 margin is loosened by
    # Catch::Approx's default relative epsilon (1.19e-5); the reference's
    # algorithm itself drifts 1.3e-10 in norm here.  The device must reproduce
    # the reference's final state, hence its drift, to 1e-12.
    L = 5
    f, p, J = sample_hamiltonian(L)
    h = ss.Hamiltonian(engine, L, f, p, J)
    psi0 = golden["ref_state_5_12609"]
    psi = dev(engine, psi0)
    n0, e0 = psi.norm(), ss.measure_energy(h, psi)
    prop = ss.Propagator(L, 1e-12)
    for _ in range(100):
        prop.evolve(h, abi.REAL, psi, 0.02, 100)
    final = psi.download()
    want = golden["conservation_final"]
    assert np.abs(final - want).max() < 1e-12
    assert abs(psi.norm() - np.linalg.norm(want)) < 1e-13
    assert abs(psi.norm() - n0) < 2e-10
    assert abs(ss.measure_energy(h, psi) - e0) < 1e-9


def test_single_spin_precession(engine):
    # test_Propagator.cpp:126-152: <sigma_z> = -cos(hx t).
    h = ss.Hamiltonian(engine, 1, [2.0, 0.0, 0.0])
    psi = ss.StateVector(engine, 1)
    psi.set_basis_state(0)
    prop = ss.Propagator(1, 1e-13)
    for step in range(1, 61):
        prop.evolve(h, abi.REAL, psi, 0.05, 1)
        assert abs(ss.measure_mag(psi, 0, 2) + math.cos(2.0 * 0.05 * step)) < 1e-9


def test_tiny_step_is_identity_and_imaginary_time(engine):
    L = 3
    f, p, J = sample_hamiltonian(L)
    h = ss.Hamiltonian(engine, L, f, p, J)
    psi0 = random_state(L, 0x606)
    psi = dev(engine, psi0)
    prop = ss.Propagator(L, 1e-7)
    prop.evolve(h, abi.REAL, psi, 1e-12, 1)
    assert prop.last_order == 0 and np.array_equal(psi.download(), psi0)
    L = 4
    f, p, J = sample_hamiltonian(L)
    h = ss.Hamiltonian(engine, L, f, p, J)
    psi0 = random_state(L, 0x1618)
    for tau in (0.05, 0.4):
        psi = dev(engine, psi0)
        ss.Propagator(L, 1e-12).evolve(h, abi.IMAGINARY, psi, tau, 1)
        want = dense_exp_apply(dense_hamiltonian(L, f, p, J), tau, psi0)
        assert np.abs(to_complex(psi.download()) - to_complex(want)).max() < 1e-10


def test_autonormalise_and_errors(engine):
    L = 3
    f, p, J = sample_hamiltonian(L)
    h = ss.Hamiltonian(engine, L, f, p, J)
    psi = dev(engine, 3.0 * random_state(L, 1))
    ss.Propagator(L).evolve(h, abi.IMAGINARY, psi, 0.2, 3, autonormalize=True)
    assert abs(psi.norm() - 1.0) < 1e-14
    with pytest.raises(ss.InvalidArgumentError):
        ss.Propagator(4).evolve(h, abi.REAL, ss.StateVector(engine, 4), 0.1, 1)
    with pytest.raises(ss.ConvergenceError):
        big = ss.Hamiltonian(engine, L, [1e7, 0, 0] * L)
        ss.Propagator(L).evolve(big, abi.REAL, psi, 1.0, 1)


def test_rotations_match_the_oracle(engine, port):
    L = 4
    psi0 = random_state(L, 0xB0A7)
    for angle in (0.25 * math.pi, 0.5 * math.pi, math.pi, 1.7):
        for axis in ((1, 0, 0), (0, 1, 0), (0, 0, 1), (0.3, -0.5, 0.8)):
            psi = dev(engine, psi0)
            ss.rotate(psi, axis, angle, list(range(L)))
            want = port.rotate(L, psi0, axis, angle, list(range(L)))
            assert np.abs(psi.download() - want).max() < TOL
            assert abs(psi.norm() - 1.0) < 1e-14
    # pi about x is -i sigma_x (test_Gate.cpp:37-56).
    psi = dev(engine, psi0)
    ss.rotate(psi, (1, 0, 0), math.pi, [1])
    want = -1j * (dense_pauli(L, 1, "x") @ to_complex(psi0))
    assert np.abs(to_complex(psi.download()) - want).max() < TOL
    with pytest.raises(ss.OutOfRangeError):
        ss.rotate(psi, (1, 0, 0), 1.0, [4])


def test_two_spin_gate_matches_the_oracle(engine, port):
    L = 5
    psi0 = random_state(L, 3)
    m = np.random.default_rng(1).standard_normal(32)
    for a, b in ((0, 1), (3, 1), (2, 4)):
        psi = dev(engine, psi0)
        ss.two_spin_gate(psi, m, a, b)
        assert np.abs(psi.download() - port.two_spin_gate(L, psi0, m, a, b)).max() < TOL


def test_observables_match_the_oracle(engine, port):
    L = 5
    f, p, J = sample_hamiltonian(L)
    psi0, ref0 = random_state(L, 0x1111), random_state(L, 0x2222)
    psi, ref = dev(engine, psi0), dev(engine, ref0)
    h = ss.Hamiltonian(engine, L, f, p, J)
    for axis in range(3):
        got = ss.measure_corr(psi, ref, axis)
        want = port.measure(L, abi.SsObservable(abi.OBS_CORR, axis, 0, 0), psi0, ref0, f, p, J)
        assert abs(got[0] - want[0]) < TOL and abs(got[1] - want[1]) < TOL
        for spin in range(L):
            got = ss.measure_mag(psi, spin, axis)
            want = port.measure(L, abi.SsObservable(abi.OBS_MAG, axis, spin, 0), psi0, ref0, f, p, J)
            assert abs(got - want[0]) < TOL
    e = ss.measure_energy(h, psi)
    want = port.measure(L, abi.SsObservable(abi.OBS_ENERGY, 0, 0, 0), psi0, ref0, f, p, J)
    assert abs(e - want[0]) < TOL


def test_plain_path_reproduces_reference_cpmg_curves(engine, golden):
    spec = workloads.cpmg_ideal()
    cfg = spec.config()
    rows = np.stack([ss.run_realization(engine, cfg, i, spec.measurement_count(), spec.width())[1]
                     for i in range(20)])
    times, _ = ss.run_realization(engine, cfg, 0, spec.measurement_count(), spec.width())
    assert np.array_equal(times, golden["curves_cpmg_times"])
    assert np.abs(rows - golden["curves_cpmg_rows"]).max() < 1e-10


def test_plain_path_reproduces_reference_xy8_curves(engine, golden):
    spec = workloads.xy8_finite(nspins=8, realizations=4, blocks=2)
    spec.observables = ["corr:x", "norm", "energy", "mag:2:z"]
    cfg = spec.config()
    for i in range(4):
        t, v = ss.run_realization(engine, cfg, i, spec.measurement_count(), spec.width())
        assert np.array_equal(t, golden["curves_xy8_l8_times"])
        assert np.abs(v - golden["curves_xy8_l8_rows"][i]).max() < 1e-10
    spec = workloads.xy8_finite(realizations=2)
    cfg = spec.config()
    for i in range(2):
        _, v = ss.run_realization(engine, cfg, i, 128, 2)
        assert np.abs(v - golden["curves_xy8_l12_rows"][i]).max() < 1e-10
