"""The plain propagator's kernel families on the device, through the C ABI.

The tiled order kernel (tiled.cu: shared-memory tiles, a few passes per
order) against the reference's propagator (the C restatement, bit-identical
to the reference's own build) at the reference's 1e-10 propagator bar
(test_Propagator.cpp:36-67), against the gather kernel at 1e-12, and against
the dense exponential of the long-propagation workload at L = 12.  Mixed
precision (FP32 T vectors and partial sums, FP64 psi, weights, diagonal and
T_n formation) against FP64 within 1e-6 of the state norm.
"""
import numpy as np
import pytest

import spin_systems_b200 as ss
from spin_systems_b200 import abi, workloads
from oracle.oracle import dense_hamiltonian, dense_pauli, random_state, sample_hamiltonian

pytestmark = pytest.mark.gpu

SMALL, TILED, GATHER = abi.KERNEL_TILED_SMALL, abi.KERNEL_TILED, abi.KERNEL_GATHER


def propagate(engine, L, f, p, J, psi0, kernel, precision=abi.FP64, mode=abi.REAL, tau=0.1,
              nsteps=2, autonorm=False, eps=1e-12):
    h = ss.Hamiltonian(engine, L, f, p, J)
    psi = ss.StateVector(engine, L, psi0)
    prop = ss.Propagator(L, eps, precision, kernel)
    prop.evolve(h, mode, psi, tau, nsteps, autonorm)
    return psi.download(), prop.last_order


@pytest.mark.parametrize("kernel,sizes", [(SMALL, [8, 9, 10, 11, 12, 13, 14, 16]),
                                          (TILED, [12, 13, 14, 16])])
def test_tiled_fp64_matches_the_reference_propagator(engine, port, kernel, sizes):
    for L in sizes:
        f, p, J = sample_hamiltonian(L)  # transverse fields and jx != jy on every pair
        psi0 = random_state(L, 0x7117 + L)
        want, order = port.evolve(L, f, p, J, psi0, abi.REAL, 0.1, 2, eps=1e-12)
        got, got_order = propagate(engine, L, f, p, J, psi0, kernel)
        assert got_order == order
        assert np.abs(got - want).max() < 1e-10, (L, np.abs(got - want).max())
        gather, _ = propagate(engine, L, f, p, J, psi0, GATHER)
        assert np.abs(got - gather).max() < 1e-12, (L, np.abs(got - gather).max())


@pytest.mark.parametrize("precision,bits", [(abi.FP64, 3), (abi.FP64, 4), (abi.MIXED, 4),
                                           (abi.MIXED, 5)])
def test_every_tiled_schedule_matches(engine, port, precision, bits):
    # Every schedule (register bits per thread) against the reference
    # propagator, on a Hamiltonian with transverse fields and flip-both
    # terms, at sizes of one to eight tiles.
    tol = 1e-10 if precision == abi.FP64 else 1e-6
    ss.tiled_select(precision, bits)
    try:
        for L in (13, 15):
            f, p, J = sample_hamiltonian(L)
            psi0 = random_state(L, 0x5C4E + L)
            got, _ = propagate(engine, L, f, p, J, psi0, TILED, precision)
            want, _ = port.evolve(L, f, p, J, psi0, abi.REAL, 0.1, 2, eps=1e-12)
            assert np.abs(got - want).max() < tol, (L, np.abs(got - want).max())
    finally:
        ss.tiled_select(precision, 0)
    with pytest.raises(ss.InvalidArgumentError):
        ss.tiled_select(abi.FP64, 5)


def test_tiled_imaginary_time_with_autonormalisation(engine, port):
    for L, kernel in ((11, SMALL), (13, TILED)):
        f, p, J = sample_hamiltonian(L)
        psi0 = random_state(L, 0xA11 + L)
        want, _ = port.evolve(L, f, p, J, psi0, abi.IMAGINARY, 0.05, 3, autonorm=True, eps=1e-12)
        got, _ = propagate(engine, L, f, p, J, psi0, kernel, mode=abi.IMAGINARY, tau=0.05,
                           nsteps=3, autonorm=True)
        assert np.abs(got - want).max() < 1e-10


def test_tiled_tables_follow_field_changes(engine, port):
    # A pulse program swaps fields between steps: the per-pass tables must
    # be rebuilt when the Hamiltonian changes (Sequence.cpp:18-33).
    L = 12
    f, p, J = sample_hamiltonian(L)
    psi0 = random_state(L, 0xF1E1D)
    h = ss.Hamiltonian(engine, L, f, p, J)
    psi = ss.StateVector(engine, L, psi0)
    prop = ss.Propagator(L, 1e-12, abi.FP64, SMALL)
    prop.evolve(h, abi.REAL, psi, 0.1, 1)
    f2 = f.copy()
    f2[0::3] *= -1.5
    h.set_fields(f2)
    prop.evolve(h, abi.REAL, psi, 0.1, 1)
    want, _ = port.evolve(L, f, p, J, psi0, abi.REAL, 0.1, 1, eps=1e-12)
    want, _ = port.evolve(L, f2, p, J, want, abi.REAL, 0.1, 1, eps=1e-12)
    assert np.abs(psi.download() - want).max() < 1e-10


def test_mixed_precision_tracks_fp64(engine):
    for L, kernel in ((10, GATHER), (12, SMALL), (14, TILED), (16, TILED)):
        f, p, J = sample_hamiltonian(L)
        psi0 = random_state(L, 0xB0B + L)
        fp64, _ = propagate(engine, L, f, p, J, psi0, GATHER, nsteps=3, eps=1e-7)
        mixed, _ = propagate(engine, L, f, p, J, psi0, kernel, abi.MIXED, nsteps=3, eps=1e-7)
        assert np.abs(mixed - fp64).max() < 1e-6, (L, kernel, np.abs(mixed - fp64).max())


def test_tiled_kernel_needs_a_full_tile(engine):
    f, p, J = sample_hamiltonian(10)
    psi0 = random_state(10, 1)
    with pytest.raises(ss.InvalidArgumentError):
        propagate(engine, 10, f, p, J, psi0, TILED)
    with pytest.raises(ss.InvalidArgumentError):
        propagate(engine, 7, *sample_hamiltonian(7), random_state(7, 1), SMALL)


def _dense_reference(cfg, L, times):
    s = ss.realization_setup(cfg, 0, L)
    H = dense_hamiltonian(L, s["fields"], s["pairs"], s["J"])
    w, V = np.linalg.eigh(H)
    psi0 = s["psi0"][0::2] + 1j * s["psi0"][1::2]
    Z = sum(dense_pauli(L, q, "z") for q in range(L))
    ref0 = Z @ psi0
    c_psi, c_ref = V.conj().T @ psi0, V.conj().T @ ref0
    out = []
    for t in times:
        ph = np.exp(1j * w * t)
        psi, ref = V @ (ph * c_psi), V @ (ph * c_ref)
        corr = np.vdot(ref, Z @ psi)
        out.append((np.linalg.norm(psi), np.vdot(psi, H @ psi).real, corr.real, corr.imag))
    return np.array(out), np.abs(w).max()


def test_long_propagation_at_12_matches_the_dense_exponential(engine):
    # The long-propagation workload (random product state, sigma = 1,
    # dt = 0.1, autonormalisation off) at L = 12 through the plain runner:
    # FP64 on the tiled kernel (three 8-spin passes per order) within the
    # reference's 1e-10 state bar carried to each observable by its operator
    # norm; mixed precision within 1e-6 of the same.
    L = 12
    spec = workloads.long_propagation(nspins=L, steps=100, dt=0.1, every=20)
    cfg = spec.config()
    n, w = spec.measurement_count(), spec.width()
    times, fp64 = ss.run_realization(engine, cfg, 0, n, w, abi.FP64, SMALL)
    want, hn = _dense_reference(cfg, L, times)
    assert np.abs(fp64[:, 0] - want[:, 0]).max() < 1e-10
    assert np.abs(fp64[:, 2] - want[:, 1]).max() < 1e-10 * hn
    assert np.abs(fp64[:, 3:5] - want[:, 2:4]).max() < 1e-10 * L * L
    _, mixed = ss.run_realization(engine, cfg, 0, n, w, abi.MIXED, SMALL)
    assert np.abs(mixed[:, 0] - want[:, 0]).max() < 1e-6
    assert np.abs(mixed[:, 2] - want[:, 1]).max() < 1e-6 * hn
    assert np.abs(mixed[:, 3:5] - want[:, 2:4]).max() < 1e-6 * L
