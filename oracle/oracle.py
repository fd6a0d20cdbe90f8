"""Test infrastructure: Python access to the CPU oracles.

Three checkers, none of them part of the product:

* ``Port``  -- liboracle_port.so, the C restatement in spinsim_oracle.c;
* ``Ref``   -- oracle/_ref/libspinsim_ref.so, the reference's own core compiled
  from its sources (present only where the reference source tree was);
* ``dense_*`` -- an independent dense-matrix oracle (Kronecker-product Pauli
  matrices, numpy ``eigh``), mirroring the reference's
  tests/DenseReference.cpp:28-192: it shares no bit arithmetic with either.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from spin_systems_b200.abi import SsObservable, SsRunConfig

HERE = Path(__file__).resolve().parent
PORT_SO = HERE / "_build" / "liboracle_port.so"
REF_SO = HERE / "_ref" / "libspinsim_ref.so"
REFERENCE_TREE = Path(os.environ.get("SPINSIM_REFERENCE", "/root/reference"))

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


def build(ref: bool = True) -> None:
    """Builds the port (always) and the reference (when its sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)
    if ref and (REFERENCE_TREE / "src" / "core").is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", "-j8",
                        f"REFERENCE={REFERENCE_TREE}"], check=True)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class OracleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class _Lib:
    prefix = ""

    def __init__(self, path: Path):
        self.lib = C.CDLL(str(path))
        self._last_error = getattr(self.lib, self.prefix + "last_error")
        self._last_error.restype = C.c_char_p

    def _check(self, rc: int) -> None:
        if rc:
            raise OracleError(rc, self._last_error().decode())


class Port(_Lib):
    """The C restatement (spinsim_oracle.c)."""
    prefix = "orc_"

    def __init__(self, path: Path = PORT_SO):
        if not path.exists():
            build(ref=False)
        super().__init__(path)
        L = self.lib
        L.orc_rng_uniform.restype = C.c_double
        L.orc_rng_gaussian.restype = C.c_double
        L.orc_spectral_bound.restype = C.c_double
        L.orc_norm.restype = C.c_double

    def rng(self, seed, index, kind, n):
        out = np.zeros(n)
        self.lib.orc_rng_draws(C.c_uint64(seed), C.c_uint64(index), kind, C.c_int64(n), _d(out))
        return out

    def bessel(self, kind, x, count):
        out = np.zeros(count)
        nz = C.c_int64()
        self._check(self.lib.orc_bessel(kind, C.c_double(x), C.c_int64(count), _d(out), C.byref(nz)))
        return out, nz.value

    def chebyshev(self, mode, bound, tau, eps, max_order=6000):
        cap = max_order + 8
        out = np.zeros(cap)
        order = C.c_int64()
        eb = C.c_double()
        self._check(self.lib.orc_chebyshev(mode, C.c_double(bound), C.c_double(tau), C.c_double(eps),
                                           C.c_int64(max_order), _d(out), C.c_int64(cap),
                                           C.byref(order), C.byref(eb)))
        return out[: order.value + 1].copy(), eb.value

    def apply(self, L, fields, pairs, J, scale, psi, out=None, accumulate=False):
        out = np.zeros_like(psi) if out is None else out.copy()
        self.lib.orc_ham_apply(L, _d(fields), len(J) // 3, _i(pairs), _d(J), C.c_double(scale),
                               _d(psi), _d(out), int(accumulate))
        return out

    def spectral_bound(self, L, fields, J):
        return self.lib.orc_spectral_bound(L, _d(fields), len(J) // 3, _d(J))

    def evolve(self, L, fields, pairs, J, psi, mode, tau, nsteps, autonorm=False, eps=1e-7):
        psi = psi.copy()
        order = C.c_int64()
        self._check(self.lib.orc_evolve(L, _d(fields), len(J) // 3, _i(pairs), _d(J), _d(psi), mode,
                                        C.c_double(tau), C.c_int64(nsteps), int(autonorm),
                                        C.c_double(eps), C.byref(order)))
        return psi, order.value

    def rotate(self, L, psi, axis, angle, targets):
        psi = psi.copy()
        ax = np.asarray(axis, dtype=np.float64)
        t = np.asarray(targets, dtype=np.int32)
        self._check(self.lib.orc_rotate(L, _d(psi), _d(ax), C.c_double(angle), _i(t), len(t)))
        return psi

    def rotation_matrix(self, axis, angle):
        u = np.zeros(8)
        ax = np.asarray(axis, dtype=np.float64)
        self.lib.orc_rotation_matrix(_d(ax), C.c_double(angle), _d(u))
        return u

    def two_spin_gate(self, L, psi, m, a, b):
        psi = psi.copy()
        mm = np.ascontiguousarray(m, dtype=np.float64)
        self._check(self.lib.orc_two_spin_gate(L, _d(psi), _d(mm), a, b))
        return psi

    def pauli(self, L, op, axis, c, spin, spin_b, jxyz, psi, out):
        out = out.copy()
        j = np.asarray(jxyz if jxyz is not None else [0, 0, 0], dtype=np.float64)
        self.lib.orc_pauli(L, op, axis, C.c_double(c), spin, spin_b, _d(j), _d(psi), _d(out))
        return out

    def norm(self, L, psi):
        return self.lib.orc_norm(L, _d(psi))

    def measure(self, L, obs: SsObservable, psi, ref, fields, pairs, J):
        out = np.zeros(2)
        self._check(self.lib.orc_measure(L, C.byref(obs), _d(psi), _d(ref), _d(fields), len(J) // 3,
                                         _i(pairs), _d(J), _d(out)))
        return out

    def shape(self, cfg: SsRunConfig):
        p, w = C.c_int64(), C.c_int64()
        self.lib.orc_shape(C.byref(cfg), C.byref(p), C.byref(w))
        return p.value, w.value

    def setup(self, cfg: SsRunConfig, index: int, lmax: int):
        n = 1 << lmax
        fields = np.zeros(3 * lmax)
        pairs = np.zeros(lmax * (lmax - 1) + 2, dtype=np.int32)
        J = np.zeros(3 * (lmax * (lmax - 1) // 2) + 3)
        psi0 = np.zeros(2 * n)
        ref0 = np.zeros(2 * n)
        L, P = C.c_int32(), C.c_int32()
        self._check(self.lib.orc_setup(C.byref(cfg), C.c_uint64(index), C.byref(L), _d(fields), _i(pairs),
                                       _d(J), C.byref(P), _d(psi0), _d(ref0)))
        L, P = L.value, P.value
        m = 1 << L
        return dict(L=L, fields=fields[: 3 * L].copy(), pairs=pairs[: 2 * P].copy(),
                    J=J[: 3 * P].copy(), psi0=psi0[: 2 * m].copy(), ref0=ref0[: 2 * m].copy())

    def run_realization(self, cfg: SsRunConfig, index: int):
        p, w = self.shape(cfg)
        times = np.zeros(max(p, 1))
        values = np.zeros(max(p * w, 1))
        self._check(self.lib.orc_run_realization(C.byref(cfg), C.c_uint64(index), _d(times), _d(values)))
        return times[:p], values[: p * w].reshape(p, w)

    def run_range(self, cfg: SsRunConfig, first: int, count: int, threads: int):
        p, w = self.shape(cfg)
        times = np.zeros(max(p, 1))
        values = np.zeros(max(count * p * w, 1))
        secs = C.c_double()
        self._check(self.lib.orc_run_range(C.byref(cfg), C.c_uint64(first), C.c_int64(count), threads,
                                           _d(times), _d(values), C.byref(secs)))
        return times[:p], values[: count * p * w].reshape(count, p, w), secs.value

    def run_indices(self, cfg: SsRunConfig, indices, threads: int):
        """runRealization for each index of `indices` on a thread pool taking
        the next index as it finishes; rows in list order, wall seconds."""
        idx = np.ascontiguousarray(indices, dtype=np.uint64)
        count = len(idx)
        p, w = self.shape(cfg)
        times = np.zeros(max(p, 1))
        values = np.zeros(max(count * p * w, 1))
        secs = C.c_double()
        self._check(self.lib.orc_run_indices(C.byref(cfg), idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                 C.c_int64(count), threads, _d(times), _d(values),
                                                 C.byref(secs)))
        return times[:p], values[: count * p * w].reshape(count, p, w), secs.value

    def accumulate(self, rows):
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        n, w = rows.shape
        mean, sd, se = np.zeros(w), np.zeros(w), np.zeros(w)
        self.lib.orc_accumulate(C.c_int64(n), C.c_int64(w), _d(rows), _d(mean), _d(sd), _d(se))
        return mean, sd, se


class Ref(_Lib):
    """The reference core, compiled from its own sources (oracle/Makefile)."""
    prefix = "refd_"

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def __init__(self, path: Path = REF_SO):
        super().__init__(path)

    def rng(self, seed, index, kind, n):
        out = np.zeros(n)
        self._check(self.lib.refd_rng(C.c_uint64(seed), C.c_uint64(index), kind, C.c_int64(n), _d(out)))
        return out

    def bessel(self, kind, x, count):
        out = np.zeros(count)
        nz = C.c_int64()
        self._check(self.lib.refd_bessel(kind, C.c_double(x), C.c_int64(count), _d(out), C.byref(nz)))
        return out, nz.value

    def chebyshev(self, mode, bound, tau, eps, max_order=6000):
        cap = max_order + 8
        out = np.zeros(cap)
        order = C.c_int64()
        eb = C.c_double()
        self._check(self.lib.refd_chebyshev(mode, C.c_double(bound), C.c_double(tau), C.c_double(eps),
                                            C.c_int64(max_order), _d(out), C.c_int64(cap),
                                            C.byref(order), C.byref(eb)))
        return out[: order.value + 1].copy(), eb.value

    def geometry(self, L, seed, index, scale):
        P = L * (L - 1) // 2
        pairs = np.zeros(2 * P + 2, dtype=np.int32)
        J = np.zeros(3 * P + 3)
        self._check(self.lib.refd_geometry(L, C.c_uint64(seed), C.c_uint64(index), C.c_double(scale),
                                           _i(pairs), _d(J)))
        return pairs[: 2 * P], J[: 3 * P]

    def setup(self, cfg: SsRunConfig, index: int):
        L = cfg.nspins
        n = 1 << L
        fields = np.zeros(3 * L)
        pairs = np.zeros(L * (L - 1) + 2, dtype=np.int32)
        J = np.zeros(3 * (L * (L - 1) // 2) + 3)
        psi0, ref0 = np.zeros(2 * n), np.zeros(2 * n)
        P = C.c_int32()
        self._check(self.lib.refd_setup(C.byref(cfg), C.c_uint64(index), _d(fields), _i(pairs), _d(J),
                                        C.byref(P), _d(psi0), _d(ref0)))
        P = P.value
        return dict(L=L, fields=fields, pairs=pairs[: 2 * P].copy(), J=J[: 3 * P].copy(),
                    psi0=psi0, ref0=ref0)

    def apply(self, L, fields, pairs, J, psi, out=None, variant=0, bound=1.0):
        out = np.zeros_like(psi) if out is None else out.copy()
        self._check(self.lib.refd_apply(L, _d(fields), len(J) // 3, _i(pairs), _d(J), _d(psi), _d(out),
                                        variant, C.c_double(bound)))
        return out

    def spectral_bound(self, L, fields, pairs, J):
        out = C.c_double()
        self._check(self.lib.refd_spectral_bound(L, _d(fields), len(J) // 3, _i(pairs), _d(J), C.byref(out)))
        return out.value

    def evolve(self, L, fields, pairs, J, psi, mode, tau, nsteps, autonorm=False, eps=1e-7):
        psi = psi.copy()
        order = C.c_int64()
        self._check(self.lib.refd_evolve(L, _d(fields), len(J) // 3, _i(pairs), _d(J), _d(psi), mode,
                                         C.c_double(tau), C.c_int64(nsteps), int(autonorm),
                                         C.c_double(eps), C.byref(order)))
        return psi, order.value

    def rotate(self, L, psi, axis, angle, targets):
        psi = psi.copy()
        ax = np.asarray(axis, dtype=np.float64)
        t = np.asarray(targets, dtype=np.int32)
        self._check(self.lib.refd_rotate(L, _d(psi), _d(ax), C.c_double(angle), _i(t), len(t)))
        return psi

    def two_spin_gate(self, L, psi, m, a, b):
        psi = psi.copy()
        mm = np.ascontiguousarray(m, dtype=np.float64)
        self._check(self.lib.refd_two_spin_gate(L, _d(psi), _d(mm), a, b))
        return psi

    def pauli(self, L, op, axis, c, spin, spin_b, jxyz, psi, out):
        out = out.copy()
        j = np.asarray(jxyz if jxyz is not None else [0, 0, 0], dtype=np.float64)
        self._check(self.lib.refd_pauli(L, op, axis, C.c_double(c), spin, spin_b, _d(j), _d(psi), _d(out)))
        return out

    def measure(self, L, obs: SsObservable, psi, ref, fields, pairs, J):
        out = np.zeros(2)
        self._check(self.lib.refd_measure(L, C.byref(obs), _d(psi), _d(ref), _d(fields), len(J) // 3,
                                          _i(pairs), _d(J), _d(out)))
        return out

    def shape(self, cfg: SsRunConfig):
        p, w = C.c_int64(), C.c_int64()
        self._check(self.lib.refd_measurement_count(C.byref(cfg), C.byref(p), C.byref(w)))
        return p.value, w.value

    def run_realization(self, cfg: SsRunConfig, index: int):
        p, w = self.shape(cfg)
        times = np.zeros(max(p, 1))
        values = np.zeros(max(p * w, 1))
        self._check(self.lib.refd_run_realization(C.byref(cfg), C.c_uint64(index), _d(times), _d(values)))
        return times[:p], values[: p * w].reshape(p, w)

    def run_range(self, cfg: SsRunConfig, first: int, count: int, threads: int):
        p, w = self.shape(cfg)
        times = np.zeros(max(p, 1))
        values = np.zeros(max(count * p * w, 1))
        secs = C.c_double()
        self._check(self.lib.refd_run_range(C.byref(cfg), C.c_uint64(first), C.c_int64(count), threads,
                                            _d(times), _d(values), C.byref(secs)))
        return times[:p], values[: count * p * w].reshape(count, p, w), secs.value

    def run_indices(self, cfg: SsRunConfig, indices, threads: int):
        """runRealization for each index of `indices` on a thread pool taking
        the next index as it finishes; rows in list order, wall seconds."""
        idx = np.ascontiguousarray(indices, dtype=np.uint64)
        count = len(idx)
        p, w = self.shape(cfg)
        times = np.zeros(max(p, 1))
        values = np.zeros(max(count * p * w, 1))
        secs = C.c_double()
        self._check(self.lib.refd_run_indices(C.byref(cfg), idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                 C.c_int64(count), threads, _d(times), _d(values),
                                                 C.byref(secs)))
        return times[:p], values[: count * p * w].reshape(count, p, w), secs.value

    def random_state(self, L: int, seed: int):
        """The reference tests' randomState (DenseReference.cpp:204-214)."""
        out = np.zeros(2 << L)
        self._check(self.lib.refd_random_state(L, C.c_uint64(seed), _d(out)))
        return out

    def experiment_csv(self, cfg: SsRunConfig, threads: int) -> str:
        """The reference's runExperiment written by its own writeCsv."""
        need = C.c_size_t()
        self._check(self.lib.refd_experiment_csv(C.byref(cfg), threads, None, C.c_size_t(0),
                                                 C.byref(need)))
        buf = C.create_string_buffer(need.value + 1)
        self._check(self.lib.refd_experiment_csv(C.byref(cfg), threads, buf,
                                                 C.c_size_t(need.value + 1), C.byref(need)))
        return buf.raw[: need.value].decode()

    def run_experiment(self, cfg: SsRunConfig, threads: int):
        p, w = self.shape(cfg)
        times = np.zeros(max(p, 1))
        mean, sd, se = (np.zeros(max(p * w, 1)) for _ in range(3))
        secs = C.c_double()
        self._check(self.lib.refd_run_experiment(C.byref(cfg), threads, _d(times), _d(mean), _d(sd),
                                                 _d(se), C.byref(secs)))
        return times[:p], mean[: p * w], sd[: p * w], se[: p * w], secs.value


# ------------------------------------------------------------- dense oracle
# tests/DenseReference.cpp:43-67 (basis index 0 = down), :69-78 (spin s at
# Kronecker position nspins-1-s), :113-131 (physical H with S = sigma/2).
_PAULI = {
    "x": np.array([[0, 1], [1, 0]], dtype=complex),
    "y": np.array([[0, 1j], [-1j, 0]], dtype=complex),
    "z": np.array([[-1, 0], [0, 1]], dtype=complex),
}


def dense_pauli(L: int, spin: int, axis: str) -> np.ndarray:
    out = np.eye(1, dtype=complex)
    for pos in range(L - 1, -1, -1):
        out = np.kron(out, _PAULI[axis] if pos == spin else np.eye(2))
    return out


def _pauli_string(L: int, ops) -> tuple:
    """Row index and value of each column k of a product of single-spin
    Paulis on distinct spins, ops = [(spin, axis), ...]: the product maps
    basis state k to one basis state with a phase, so it is a column
    permutation with a factor (the same matrix as the kron product of
    dense_pauli, without forming it)."""
    k = np.arange(1 << L)
    row = k.copy()
    val = np.ones(1 << L, dtype=complex)
    for spin, axis in ops:
        b = (k >> spin) & 1
        m = _PAULI[axis]
        nb = b ^ 1 if axis in "xy" else b
        val = val * m[nb, b]
        if axis in "xy":
            row = row ^ (1 << spin)
    return row, val


def dense_hamiltonian(L: int, fields, pairs, J) -> np.ndarray:
    """The dense matrix of Hamiltonian.cpp:95-127's H: sum of h_a / 2 sigma_a
    per spin and J_a / 4 sigma_a sigma_a per pair, assembled term by term as
    phased permutations (tests.test_oracle_pins checks it against the kron
    construction)."""
    H = np.zeros((1 << L, 1 << L), dtype=complex)
    cols = np.arange(1 << L)
    f = np.asarray(fields).reshape(L, 3)
    for s in range(L):
        for a, ax in enumerate("xyz"):
            if f[s, a] != 0.0:
                row, val = _pauli_string(L, [(s, ax)])
                H[row, cols] += 0.5 * f[s, a] * val
    pr = np.asarray(pairs).reshape(-1, 2)
    jj = np.asarray(J).reshape(-1, 3)
    for (lo, hi), j in zip(pr, jj):
        for a, ax in enumerate("xyz"):
            if j[a] != 0.0:
                row, val = _pauli_string(L, [(int(lo), ax), (int(hi), ax)])
                H[row, cols] += 0.25 * j[a] * val
    return H


def dense_hamiltonian_kron(L: int, fields, pairs, J) -> np.ndarray:
    """dense_hamiltonian by explicit kron products (small L only)."""
    H = np.zeros((1 << L, 1 << L), dtype=complex)
    f = np.asarray(fields).reshape(L, 3)
    for s in range(L):
        for a, ax in enumerate("xyz"):
            if f[s, a] != 0.0:
                H += 0.5 * f[s, a] * dense_pauli(L, s, ax)
    pr = np.asarray(pairs).reshape(-1, 2)
    jj = np.asarray(J).reshape(-1, 3)
    for (lo, hi), j in zip(pr, jj):
        for a, ax in enumerate("xyz"):
            if j[a] != 0.0:
                H += 0.25 * j[a] * dense_pauli(L, int(lo), ax) @ dense_pauli(L, int(hi), ax)
    return H


def dense_exp_apply(H: np.ndarray, factor: complex, psi_interleaved: np.ndarray) -> np.ndarray:
    """exp(factor * H) psi via eigendecomposition (DenseReference.cpp:151-192)."""
    w, V = np.linalg.eigh(H)
    psi = psi_interleaved[0::2] + 1j * psi_interleaved[1::2]
    out = V @ (np.exp(factor * w) * (V.conj().T @ psi))
    res = np.empty(2 * len(out))
    res[0::2], res[1::2] = out.real, out.imag
    return res


def to_complex(v: np.ndarray) -> np.ndarray:
    return v[0::2] + 1j * v[1::2]


def to_interleaved(z: np.ndarray) -> np.ndarray:
    out = np.empty(2 * len(z))
    out[0::2], out[1::2] = z.real, z.imag
    return out


def random_state(L: int, seed: int) -> np.ndarray:
    """A normalised random state (numpy generator; tests only need variety)."""
    g = np.random.default_rng(seed)
    v = g.standard_normal(2 << L)
    return v / np.linalg.norm(v)


def sample_hamiltonian(L: int):
    """test_Propagator.cpp:19-34 sampleHamiltonian."""
    fields = []
    for s in range(L):
        k = s + 1.0
        fields += [0.4 * k, -0.3 / k, 0.9]
    pairs, J = [], []
    for a in range(L):
        for b in range(a + 1, L):
            r = float(b - a)
            pairs += [a, b]
            J += [0.5 / r, -0.2 / r, 0.8 / (r * r)]
    return (np.array(fields), np.array(pairs, dtype=np.int32), np.array(J))
