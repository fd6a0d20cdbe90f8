"""spin_systems_b200 -- Python access to the B200 Chebyshev echo engine.

The engine itself is native: CUDA kernels for sm_100a and C++ host code in
``lib/libspinsim_b200.so``, behind the C ABI of ``include/spinsim_b200.h``.
This module binds that ABI with ctypes and mirrors the reference's objects
(spinsim's StateVector, Hamiltonian, Propagator, SpinRotation, observables)
so tests and benchmarks read like the reference's own.  There is no Python or
CPU fallback: without the built library every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from . import abi
from .abi import SsRunConfig, SsObservable

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libspinsim_b200.so"
HEADER = PKG.parent / "include" / "spinsim_b200.h"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lib: Optional[C.CDLL] = None


class SpinsimError(RuntimeError):
    """A failed C ABI call: `.code` is the ss_status, `.kind` its name."""

    def __init__(self, code: int, msg: str):
        self.code = code
        self.kind = abi.STATUS_NAMES.get(code, "unknown")
        super().__init__(f"{self.kind}: {msg}")


class ConvergenceError(SpinsimError):
    pass


class DomainError(SpinsimError):
    pass


class OutOfRangeError(SpinsimError):
    pass


class InvalidArgumentError(SpinsimError):
    pass


class NoDeviceError(SpinsimError):
    pass


_ERRORS = {1: InvalidArgumentError, 2: OutOfRangeError, 3: DomainError, 4: ConvergenceError,
           9: NoDeviceError}


def load(path: Path = LIB_PATH) -> C.CDLL:
    """Loads the engine library (built in-tree by __graft_entry__.build())."""
    global _lib
    if _lib is not None:
        return _lib
    if not path.exists():
        raise FileNotFoundError(
            f"{path} is missing: build the CUDA extension first (python -c "
            "'import __graft_entry__ as g; g.build()')")
    lib = C.CDLL(str(path))
    lib.ss_last_error.restype = C.c_char_p
    lib.ss_engine_stream.restype = C.c_void_p
    lib.ss_engine_stream.argtypes = [C.c_void_p]
    lib.ss_engine_launch_count.restype = C.c_int64
    lib.ss_engine_launch_count.argtypes = [C.c_void_p]
    for name in ("ss_state_scale",):
        getattr(lib, name).argtypes = [C.c_void_p, C.c_double]
    lib.ss_state_add_scaled.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_void_p]
    lib.ss_axpy_sigma.argtypes = [C.c_double, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    lib.ss_axpy_coupling.argtypes = [C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_int,
                                     C.c_int, C.c_void_p]
    lib.ss_ham_apply.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
    lib.ss_evolve.argtypes = [C.c_void_p, C.c_void_p, _dp, C.c_int64, C.c_double, C.c_int,
                              C.c_int64, C.c_int]
    lib.ss_propagate.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int64, C.c_int,
                                 C.c_double, C.POINTER(C.c_int64)]
    lib.ss_evolve_ex.argtypes = [C.c_void_p, C.c_void_p, _dp, C.c_int64, C.c_double, C.c_int,
                                 C.c_int64, C.c_int, C.c_int, C.c_int]
    lib.ss_propagate_ex.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int64,
                                    C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int64)]
    lib.ss_tile_plan.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int32),
                                 C.POINTER(C.c_uint32), C.c_int32]
    lib.ss_bessel.argtypes = [C.c_int, C.c_double, C.c_int64, _dp, C.POINTER(C.c_int64)]
    lib.ss_chebyshev_build.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int64, _dp,
                                       C.c_int64, C.POINTER(C.c_int64), _dp]
    lib.ss_rotation_matrix.argtypes = [_dp, C.c_double, _dp]
    lib.ss_state_set_basis.argtypes = [C.c_void_p, C.c_uint64]
    lib.ss_realization_setup.argtypes = [C.POINTER(SsRunConfig), C.c_uint64, _ip, _dp, _ip, _dp,
                                         _ip, _dp]
    lib.ss_batch_create.argtypes = [C.c_void_p, C.POINTER(SsRunConfig), C.c_uint64, C.c_int64,
                                    C.c_int, C.POINTER(C.c_void_p)]
    lib.ss_run_realization.argtypes = [C.c_void_p, C.POINTER(SsRunConfig), C.c_uint64, _dp, _dp]
    lib.ss_run_realization_ex.argtypes = [C.c_void_p, C.POINTER(SsRunConfig), C.c_uint64, C.c_int,
                                          C.c_int, _dp, _dp]
    lib.ss_measure_corr_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                            _dp]
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc:
        msg = load().ss_last_error().decode()
        raise _ERRORS.get(rc, SpinsimError)(rc, msg)


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def header_symbols() -> list:
    """Every function the public header declares."""
    import re
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*|void\*|int64_t)\s+(ss_\w+)\(", text, re.M)))


# ------------------------------------------------------------------ engine
class Engine:
    """One device and its stream (ss_engine_create)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.ss_engine_create(device, C.byref(h)))
        self.handle = h
        self._children = weakref.WeakSet()

    def _adopt(self, child) -> None:
        self._children.add(child)

    def close(self) -> None:
        """Destroys every object still alive on this engine, then the engine
        (the C ABI requires states, Hamiltonians and batches to go first)."""
        if self.handle:
            for child in list(self._children):
                child._destroy()
            check(self.lib.ss_engine_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self) -> None:
        check(self.lib.ss_engine_synchronize(self.handle))

    @property
    def stream(self) -> int:
        return self.lib.ss_engine_stream(self.handle)

    @property
    def launches(self) -> int:
        return self.lib.ss_engine_launch_count(self.handle)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class StateVector:
    """2^L complex amplitudes on the device (core/StateVector.hpp:82-140)."""

    def __init__(self, engine: Engine, nspins: int, data: Optional[np.ndarray] = None):
        self.engine, self.lib, self.nspins = engine, engine.lib, nspins
        h = C.c_void_p()
        check(self.lib.ss_state_create(engine.handle, nspins, C.byref(h)))
        self.handle = h
        engine._adopt(self)
        if data is not None:
            self.upload(data)

    def _destroy(self) -> None:
        if getattr(self, "handle", None):
            self.lib.ss_state_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass

    @property
    def size(self) -> int:
        return 1 << self.nspins

    def upload(self, data: np.ndarray) -> None:
        a = np.ascontiguousarray(data, dtype=np.float64)
        assert a.size == 2 * self.size
        check(self.lib.ss_state_upload(self.handle, _d(a)))

    def download(self) -> np.ndarray:
        out = np.empty(2 * self.size)
        check(self.lib.ss_state_download(self.handle, _d(out)))
        return out

    def copy_from(self, other: "StateVector") -> None:
        check(self.lib.ss_state_copy(self.handle, other.handle))

    def set_zero(self) -> None:
        check(self.lib.ss_state_set_zero(self.handle))

    def scale(self, f: float) -> None:
        check(self.lib.ss_state_scale(self.handle, f))

    def negate(self) -> None:
        check(self.lib.ss_state_negate(self.handle))

    def add_scaled(self, cr: float, ci: float, other: "StateVector") -> None:
        check(self.lib.ss_state_add_scaled(self.handle, cr, ci, other.handle))

    def set_basis_state(self, index: int) -> None:
        check(self.lib.ss_state_set_basis(self.handle, index))

    def norm(self) -> float:
        out = C.c_double()
        check(self.lib.ss_state_norm(self.handle, C.byref(out)))
        return out.value

    def normalize(self) -> float:
        out = C.c_double()
        check(self.lib.ss_state_normalize(self.handle, C.byref(out)))
        return out.value

    def inner_product(self, other: "StateVector"):
        out = (C.c_double * 2)()
        check(self.lib.ss_state_inner_product(self.handle, other.handle, out))
        return out[0], out[1]

    def swap(self, other: "StateVector") -> None:
        check(self.lib.ss_state_swap(self.handle, other.handle))


# Pauli kernels (core/SpinOperators.hpp:22-58)
def axpy_sigma(c: float, src: StateVector, spin: int, axis: int, dst: StateVector) -> None:
    check(src.lib.ss_axpy_sigma(c, src.handle, spin, axis, dst.handle))


def apply_sigma(src: StateVector, spin: int, axis: int, dst: StateVector) -> None:
    check(src.lib.ss_apply_sigma(src.handle, spin, axis, dst.handle))


def axpy_coupling(jx, jy, jz, src: StateVector, a: int, b: int, dst: StateVector) -> None:
    check(src.lib.ss_axpy_coupling(jx, jy, jz, src.handle, a, b, dst.handle))


def apply_total_spin(axis: int, src: StateVector, dst: StateVector) -> None:
    check(src.lib.ss_apply_total_spin(axis, src.handle, dst.handle))


class Hamiltonian:
    """Fields and couplings on the device (core/Hamiltonian.hpp:32-110)."""

    def __init__(self, engine: Engine, nspins: int, fields=None, pairs=None, couplings=None):
        self.engine, self.lib, self.nspins = engine, engine.lib, nspins
        h = C.c_void_p()
        check(self.lib.ss_ham_create(engine.handle, nspins, C.byref(h)))
        self.handle = h
        engine._adopt(self)
        self.set_terms(np.zeros(3 * nspins) if fields is None else fields,
                       np.zeros(0, dtype=np.int32) if pairs is None else pairs,
                       np.zeros(0) if couplings is None else couplings)

    def _destroy(self) -> None:
        if getattr(self, "handle", None):
            self.lib.ss_ham_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass

    def set_terms(self, fields, pairs, couplings) -> None:
        f = np.ascontiguousarray(fields, dtype=np.float64)
        p = np.ascontiguousarray(pairs, dtype=np.int32)
        j = np.ascontiguousarray(couplings, dtype=np.float64)
        check(self.lib.ss_ham_set_terms(self.handle, _d(f), len(p) // 2, _i(p), _d(j)))

    def set_fields(self, fields) -> None:
        f = np.ascontiguousarray(fields, dtype=np.float64)
        check(self.lib.ss_ham_set_fields(self.handle, _d(f)))

    def spectral_bound(self) -> float:
        out = C.c_double()
        check(self.lib.ss_ham_spectral_bound(self.handle, C.byref(out)))
        return out.value

    def apply(self, scale: float, src: StateVector, dst: StateVector, accumulate: bool) -> None:
        check(self.lib.ss_ham_apply(self.handle, scale, src.handle, dst.handle, int(accumulate)))

    def apply_physical(self, src: StateVector, dst: StateVector) -> None:
        self.apply(1.0, src, dst, False)

    def apply_twice_normalized(self, bound: float, src: StateVector, dst: StateVector) -> None:
        if not bound > 0:
            raise DomainError(3, "spectral bound must be positive")
        self.apply(-2.0 / bound, src, dst, False)


def bessel(kind: int, x: float, count: int):
    lib = load()
    out = np.zeros(count)
    nz = C.c_int64()
    check(lib.ss_bessel(kind, x, count, _d(out), C.byref(nz)))
    return out, nz.value


def chebyshev(mode: int, bound: float, tau: float, epsilon: float, max_order: int = 6000):
    lib = load()
    cap = max_order + 8
    out = np.zeros(cap)
    order = C.c_int64()
    eb = C.c_double()
    check(lib.ss_chebyshev_build(mode, bound, tau, epsilon, max_order, _d(out), cap,
                                 C.byref(order), C.byref(eb)))
    return out[: order.value + 1].copy(), eb.value


class Propagator:
    """Propagator::evolve (src/core/Propagator.cpp:75-100) on the device.

    ``precision`` (abi.FP64 / abi.MIXED) and ``kernel`` (abi.KERNEL_*) choose
    the arithmetic and the order kernel; the defaults are the reference's FP64
    and the faster kernel family for the size."""

    def __init__(self, nspins: int, epsilon: float = 1e-7, precision: int = 0, kernel: int = 0):
        if not epsilon > 0:
            raise InvalidArgumentError(1, "epsilon must be positive")
        self.nspins, self.epsilon, self.last_order = nspins, epsilon, 0
        self.precision, self.kernel = precision, kernel

    def evolve(self, ham: Hamiltonian, mode: int, psi: StateVector, tau: float, nsteps: int,
               autonormalize: bool = False) -> None:
        if psi.nspins != ham.nspins:
            raise InvalidArgumentError(1, "state and Hamiltonian disagree on spin count")
        if psi.nspins != self.nspins:
            raise InvalidArgumentError(1, "state does not match the propagator's size")
        order = C.c_int64(0)
        check(ham.lib.ss_propagate_ex(ham.handle, psi.handle, mode, tau, nsteps,
                                      int(autonormalize), self.epsilon, self.precision,
                                      self.kernel, C.byref(order)))
        if nsteps:
            self.last_order = order.value


def tiled_select(precision: int, register_bits: int = 0) -> None:
    """The tiled kernel's schedule for a precision: register bits per thread
    (FP64 3 or 4, mixed 4 or 5, 0 = default)."""
    check(load().ss_tiled_select(precision, register_bits))


def tile_plan(nspins: int, tile_bits: int, line_bits: int = 0) -> list:
    """Tile patterns (bit masks, one per pass; the last forms T_n) for an
    nspins-spin vector and tiles of tile_bits spins that all hold spins
    0 .. line_bits-1."""
    lib = load()
    n = C.c_int32()
    check(lib.ss_tile_plan(nspins, tile_bits, line_bits, C.byref(n), None, 0))
    masks = (C.c_uint32 * max(1, n.value))()
    check(lib.ss_tile_plan(nspins, tile_bits, line_bits, C.byref(n), masks, n.value))
    return [int(m) for m in masks[: n.value]]


def tiled_plan(nspins: int, precision: int) -> list:
    """The patterns SS_KERNEL_TILED runs for a precision (12-spin tiles with
    8-amplitude runs in FP64, 13-spin tiles with 16-amplitude runs mixed)."""
    return tile_plan(nspins, 12, 3) if precision == abi.FP64 else tile_plan(nspins, 13, 4)


def rotation_matrix(axis: Sequence[float], angle: float) -> np.ndarray:
    u = np.zeros(8)
    ax = np.asarray(axis, dtype=np.float64)
    check(load().ss_rotation_matrix(_d(ax), angle, _d(u)))
    return u


def rotate(psi: StateVector, axis, angle: float, targets) -> None:
    """SpinRotation::apply (src/core/Gate.cpp:60-85)."""
    u = rotation_matrix(axis, angle)
    t = np.ascontiguousarray(targets, dtype=np.int32)
    check(psi.lib.ss_rotate(psi.handle, _d(u), _i(t), len(t)))


def two_spin_gate(psi: StateVector, m, a: int, b: int) -> None:
    mm = np.ascontiguousarray(m, dtype=np.float64)
    check(psi.lib.ss_two_spin_gate(psi.handle, _d(mm), a, b))


def measure_corr(psi: StateVector, ref: StateVector, axis: int):
    out = (C.c_double * 2)()
    check(psi.lib.ss_measure_corr(psi.handle, ref.handle, axis, out))
    return out[0], out[1]


def measure_corr_noalloc(psi_ptr: int, ref_ptr: int, nspins: int, axis: int,
                         stream: Optional[int] = None):
    """ss_measure_corr over caller-owned device vectors (device addresses of
    2*2^nspins doubles each), with no allocation; waits for `stream`."""
    out = np.zeros(2)
    check(load().ss_measure_corr_noalloc(psi_ptr, ref_ptr, nspins, axis, stream, _d(out)))
    return out[0], out[1]


def measure_mag(psi: StateVector, spin: int, axis: int) -> float:
    out = C.c_double()
    check(psi.lib.ss_measure_mag(psi.handle, spin, axis, C.byref(out)))
    return out.value


def measure_energy(ham: Hamiltonian, psi: StateVector) -> float:
    out = C.c_double()
    check(psi.lib.ss_measure_energy(ham.handle, psi.handle, C.byref(out)))
    return out.value


def realization_setup(cfg: SsRunConfig, index: int, lmax: int):
    """ss_realization_setup: the realisation's fields, couplings and psi0."""
    lib = load()
    n = 1 << lmax
    fields = np.zeros(3 * lmax)
    pairs = np.zeros(lmax * (lmax - 1) + 2, dtype=np.int32)
    J = np.zeros(3 * (lmax * (lmax - 1) // 2) + 3)
    psi0 = np.zeros(2 * n)
    L, P = C.c_int32(), C.c_int32()
    check(lib.ss_realization_setup(C.byref(cfg), index, C.byref(L), _d(fields), _i(pairs), _d(J),
                                   C.byref(P), _d(psi0)))
    L, P = L.value, P.value
    return dict(L=L, fields=fields[: 3 * L].copy(), pairs=pairs[: 2 * P].copy(),
                J=J[: 3 * P].copy(), psi0=psi0[: 2 << L].copy())


def run_realization(engine: Engine, cfg: SsRunConfig, index: int, points: int, width: int,
                    precision: int = abi.FP64, kernel: int = abi.KERNEL_AUTO):
    """The plain path for one realisation (ss_run_realization_ex): FP64 by
    default, or mixed precision, with the propagator's kernel family."""
    times = np.zeros(max(points, 1))
    values = np.zeros(max(points * width, 1))
    check(engine.lib.ss_run_realization_ex(engine.handle, C.byref(cfg), index, precision, kernel,
                                           _d(times), _d(values)))
    return times[:points], values[: points * width].reshape(points, width)


class Batch:
    """The batched engine (ss_batch_*): many realisations of one program."""

    def __init__(self, engine: Engine, cfg: SsRunConfig, first: int, count: int,
                 precision: int = abi.MIXED):
        self.engine, self.lib = engine, engine.lib
        self._cfg = cfg
        h = C.c_void_p()
        check(self.lib.ss_batch_create(engine.handle, C.byref(cfg), first, count, precision,
                                       C.byref(h)))
        self.handle = h
        engine._adopt(self)
        p, w = C.c_int64(), C.c_int64()
        check(self.lib.ss_batch_shape(self.handle, C.byref(p), C.byref(w)))
        self.points, self.width, self.count = p.value, w.value, count

    def _destroy(self) -> None:
        if getattr(self, "handle", None):
            self.lib.ss_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass

    def run(self):
        rows = np.zeros(max(self.count * self.points * self.width, 1))
        times = np.zeros(max(self.points, 1))
        check(self.lib.ss_batch_run(self.handle, _d(rows), _d(times)))
        return times[: self.points], rows[: self.count * self.points * self.width].reshape(
            self.count, self.points, self.width)

    def upload(self) -> None:
        check(self.lib.ss_batch_upload(self.handle))

    def execute(self) -> None:
        check(self.lib.ss_batch_execute(self.handle))

    def download(self):
        rows = np.zeros(max(self.count * self.points * self.width, 1))
        times = np.zeros(max(self.points, 1))
        check(self.lib.ss_batch_download(self.handle, _d(rows), _d(times)))
        return times[: self.points], rows[: self.count * self.points * self.width].reshape(
            self.count, self.points, self.width)

    def stats(self):
        orders, amp, launches = C.c_int64(), C.c_double(), C.c_int64()
        check(self.lib.ss_batch_stats(self.handle, C.byref(orders), C.byref(amp),
                                      C.byref(launches)))
        h2d, d2h = C.c_int64(), C.c_int64()
        check(self.lib.ss_batch_io_bytes(self.handle, C.byref(h2d), C.byref(d2h)))
        return dict(orders=orders.value, amplitude_orders=amp.value, launches=launches.value,
                    h2d_bytes=h2d.value, d2h_bytes=d2h.value)

    def precisions(self) -> np.ndarray:
        """The precision (abi.FP64 / abi.MIXED) each realisation runs in."""
        return self.work()[0]

    def error_estimates(self):
        """Per realisation: orders x the FP32 rounding residuals mixed
        precision leaves uncorrected (ss_batch_error_estimates)."""
        out = np.zeros(max(self.count, 1))
        check(self.lib.ss_batch_error_estimates(self.handle, _d(out)))
        return out[: self.count]

    def work(self):
        """(precision, amplitude-orders per run) of each realisation."""
        prec = np.zeros(max(self.count, 1), dtype=np.int32)
        amp = np.zeros(max(self.count, 1))
        check(self.lib.ss_batch_precisions(self.handle, _i(prec), _d(amp)))
        return prec[: self.count], amp[: self.count]


# ------------------------------------------------------------ echo surrogate
_fp = C.POINTER(C.c_float)


def _f(a: np.ndarray):
    return a.ctypes.data_as(_fp)


class Mlp:
    """The surrogate network on the device (ss_mlp_*): 6 -> 256 -> 256 ->
    256 -> 128 GELU MLP, BF16 weights/activations, FP32 accumulation, trained
    with Adam by the library's own tensor-core kernels."""

    def __init__(self, engine: Engine, batch: int = 1024, seed: int = 0):
        self.engine, self.lib = engine, engine.lib
        self.lib.ss_mlp_param_count.restype = C.c_int64
        self.lib.ss_mlp_create.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]
        self.lib.ss_mlp_forward.argtypes = [C.c_void_p, _fp, C.c_int64, _fp]
        self.lib.ss_mlp_gradients.argtypes = [C.c_void_p, _fp, _fp, C.c_int64, _fp,
                                              C.POINTER(C.c_double)]
        self.lib.ss_mlp_set_data.argtypes = [C.c_void_p, _fp, _fp, C.c_int64]
        self.lib.ss_mlp_train.argtypes = [C.c_void_p, C.c_int64, C.c_float, C.c_float, C.c_uint64,
                                          _dp]
        self.lib.ss_mlp_get_params.argtypes = [C.c_void_p, _fp]
        self.lib.ss_mlp_set_params.argtypes = [C.c_void_p, _fp]
        h = C.c_void_p()
        check(self.lib.ss_mlp_create(engine.handle, batch, seed, C.byref(h)))
        self.handle, self.batch = h, batch
        self.nparams = int(self.lib.ss_mlp_param_count())
        engine._adopt(self)

    def _destroy(self) -> None:
        if getattr(self, "handle", None):
            self.lib.ss_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.zeros(self.nparams, dtype=np.float32)
        check(self.lib.ss_mlp_get_params(self.handle, _f(p)))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.nparams
        check(self.lib.ss_mlp_set_params(self.handle, _f(p)))

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 6)
        y = np.zeros((max(len(x), 1), 128), dtype=np.float32)
        check(self.lib.ss_mlp_forward(self.handle, _f(x), len(x), _f(y)))
        return y[: len(x)]

    def gradients(self, x, target):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 6)
        t = np.ascontiguousarray(target, dtype=np.float32).reshape(-1, 128)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = C.c_double()
        check(self.lib.ss_mlp_gradients(self.handle, _f(x), _f(t), len(x), _f(g), C.byref(loss)))
        return loss.value, g

    def set_data(self, x, y) -> None:
        self._x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 6)
        self._y = np.ascontiguousarray(y, dtype=np.float32).reshape(-1, 128)
        check(self.lib.ss_mlp_set_data(self.handle, _f(self._x), _f(self._y), len(self._x)))

    def train(self, steps: int, lr_start: float = 1e-3, lr_end: float = 1e-5,
              seed: int = 0) -> np.ndarray:
        losses = np.zeros(max(steps, 1))
        check(self.lib.ss_mlp_train(self.handle, steps, lr_start, lr_end, seed, _d(losses)))
        return losses[:steps]


def mlp_gemm_test(engine: Engine, a_bits: np.ndarray, b_bits: np.ndarray) -> np.ndarray:
    """c = a b^T on the surrogate's tensor-core GEMM (BF16 bit patterns in)."""
    a = np.ascontiguousarray(a_bits, dtype=np.uint16)
    b = np.ascontiguousarray(b_bits, dtype=np.uint16)
    M, K = a.shape
    N = b.shape[0]
    c = np.zeros((M, N), dtype=np.float32)
    u16 = C.POINTER(C.c_uint16)
    engine.lib.ss_mlp_gemm_test.argtypes = [C.c_void_p, u16, u16, C.c_int, C.c_int, C.c_int, _fp]
    check(engine.lib.ss_mlp_gemm_test(engine.handle, a.ctypes.data_as(u16), b.ctypes.data_as(u16),
                                      M, N, K, _f(c)))
    return c


# ----------------------------------------------------------------- autotuner
def _text(fn) -> str:
    need = C.c_size_t()
    check(fn(None, 0, C.byref(need)))
    buf = C.create_string_buffer(max(need.value, 1))
    check(fn(buf, need.value, C.byref(need)))
    return buf.value.decode()


def _rows(text: str):
    out = []
    for line in text.splitlines():
        dev, L, prec, var, ns = line.split("\t")
        out.append(dict(device=dev, L=int(L), precision=prec, variant=var, ns=float(ns)))
    return out


def variants():
    """Every compiled batched schedule: (name, threads, shared bytes)."""
    lib = load()
    lib.ss_batch_variants.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    rows = []
    for line in _text(lib.ss_batch_variants).splitlines():
        name, threads, smem = line.split("\t")
        rows.append((name, int(threads), int(smem)))
    return rows


def schedule():
    """The process-wide schedule table (ss_schedule_describe)."""
    lib = load()
    lib.ss_schedule_describe.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    return _rows(_text(lib.ss_schedule_describe))


def load_schedule(path) -> None:
    lib = load()
    lib.ss_schedule_load.argtypes = [C.c_char_p]
    check(lib.ss_schedule_load(str(path).encode()))


def clear_schedule() -> None:
    check(load().ss_schedule_clear())


def set_snapshot_budget(nbytes: int) -> None:
    """ss_set_snapshot_budget: device memory one launch of a split-cluster
    schedule may hold in measurement snapshots (default 16 GiB)."""
    lib = load()
    lib.ss_set_snapshot_budget.argtypes = [C.c_int64]
    check(lib.ss_set_snapshot_budget(int(nbytes)))


def tune(engine: Engine, cfg: SsRunConfig, first: int = 0, sample: int = 64,
         precision: int = abi.MIXED, cache=None):
    """ss_batch_tune: time every candidate schedule of the config's sizes and
    install the fastest; returns the schedule table."""
    lib = engine.lib
    lib.ss_batch_tune.argtypes = [C.c_void_p, C.POINTER(SsRunConfig), C.c_uint64, C.c_int64,
                                  C.c_int, C.c_char_p]
    check(lib.ss_batch_tune(engine.handle, C.byref(cfg), first, sample, precision,
                            None if cache is None else str(cache).encode()))
    return schedule()
