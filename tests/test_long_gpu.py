"""The long-propagation workload (random product state, sigma = 1,
autonormalisation off, dt = 0.1, cutoff 1e-12) on the device: the plain FP64 path against
the dense eigendecomposition of the realisation's H at L = 10 (the
reference's DenseReference recipe, exp(+iHt)), and the mixed engine on a
batch of one against FP64 at L = 14 (cluster kernel)."""
import numpy as np
import pytest

import spin_systems_b200 as ss
from spin_systems_b200 import abi, workloads
from oracle.oracle import dense_hamiltonian, dense_pauli

pytestmark = pytest.mark.gpu


def test_fp64_long_propagation_matches_the_dense_exponential(engine):
    L = 10
    spec = workloads.long_propagation(nspins=L, steps=200, dt=0.1, every=20)
    cfg = spec.config()
    times, rows = ss.run_realization(engine, cfg, 0, spec.measurement_count(), spec.width())
    s = ss.realization_setup(cfg, 0, L)
    H = dense_hamiltonian(L, s["fields"], s["pairs"], s["J"])
    w, V = np.linalg.eigh(H)
    psi0 = s["psi0"][0::2] + 1j * s["psi0"][1::2]
    Z = sum(dense_pauli(L, q, "z") for q in range(L))
    ref0 = Z @ psi0
    c_psi, c_ref = V.conj().T @ psi0, V.conj().T @ ref0
    # the reference's 1e-10 state bar, carried to each observable by its
    # operator norm: ||H|| for the energy, ||sum sigma_z||^2 = L^2 for corr
    hn = np.abs(w).max()
    for t, row in zip(times, rows):
        ph = np.exp(1j * w * t)
        psi, ref = V @ (ph * c_psi), V @ (ph * c_ref)
        assert abs(row[0] - np.linalg.norm(psi)) < 1e-10
        assert abs(row[2] - np.vdot(psi, H @ psi).real) < 1e-10 * hn
        corr = np.vdot(ref, Z @ psi)
        assert abs(row[3] - corr.real) < 1e-10 * L * L and abs(row[4] - corr.imag) < 1e-10 * L * L


def test_mixed_batch_of_one_tracks_fp64_over_long_propagation(engine):
    L = 14
    spec = workloads.long_propagation(nspins=L, steps=300, dt=0.1, every=30, epsilon=1e-7)
    cfg = spec.config()
    _, fp64 = ss.run_realization(engine, cfg, 0, spec.measurement_count(), spec.width())
    b = ss.Batch(engine, cfg, 0, 1, abi.MIXED)
    _, mixed = b.run()
    mixed = mixed[0]
    assert np.abs(mixed[:, 0] - fp64[:, 0]).max() < 1e-6          # norm
    assert np.abs(mixed[:, 2] - fp64[:, 2]).max() < 1e-5 * max(1.0, abs(fp64[0, 2]))  # energy
    assert np.abs(mixed[:, 3:] - fp64[:, 3:]).max() < 1e-6 * L    # corr:z
