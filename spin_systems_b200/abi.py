"""ctypes mirror of include/spinsim_b200.h and a builder for pulse programs.

The structures here are the C ABI's own (``ss_step``, ``ss_observable``,
``ss_run_config``); ``RunSpec`` owns the arrays a config points into, so a
caller can build a run programmatically the way a TOML file describes it
(io/Config.hpp:32-58 in the reference) and hand it to the library.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

# ---------------------------------------------------------------- constants
SS_OK = 0
STATUS_NAMES = {
    1: "invalid_argument", 2: "out_of_range", 3: "domain_error", 4: "convergence",
    5: "config", 6: "runtime", 7: "overflow", 8: "cuda", 9: "no_device", 10: "timeout",
    11: "numeric",
}
AXIS = {"x": 0, "y": 1, "z": 2}
REAL, IMAGINARY = 0, 1
FP64, MIXED = 0, 1
KERNEL_AUTO, KERNEL_GATHER, KERNEL_TILED, KERNEL_TILED_SMALL = 0, 1, 2, 3
INIT = {"random": 0, "up": 1, "down": 2, "basis": 3, "random_product": 4}
EVOLVE, PULSE, MEASURE, REPEAT = 0, 1, 2, 3
OBS_CORR, OBS_MAG, OBS_NORM, OBS_ENERGY = 0, 1, 2, 3


class SsStep(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("mode", C.c_int32), ("autonormalize", C.c_int32),
        ("field_table", C.c_int32), ("count", C.c_int64), ("body_len", C.c_int32),
        ("target", C.c_int32), ("tau", C.c_double), ("angle", C.c_double),
        ("axis", C.c_double * 3), ("tau_from_draw", C.c_int32), ("reserved", C.c_int32),
    ]


class SsObservable(C.Structure):
    _fields_ = [("kind", C.c_int32), ("axis", C.c_int32), ("spin", C.c_int32),
                ("reserved", C.c_int32)]


class SsRunConfig(C.Structure):
    _fields_ = [
        ("nspins", C.c_int32), ("initial_state", C.c_int32), ("basis_index", C.c_uint64),
        ("realizations", C.c_uint64), ("seed", C.c_uint64),
        ("generate_geometry", C.c_int32), ("reference_axis", C.c_int32),
        ("dipolar_scale", C.c_double), ("field_disorder", C.c_double),
        ("epsilon", C.c_double), ("base_fields", C.POINTER(C.c_double)),
        ("n_observables", C.c_int32), ("n_steps", C.c_int32),
        ("observables", C.POINTER(SsObservable)), ("steps", C.POINTER(SsStep)),
        ("n_step_fields", C.c_int32), ("reserved0", C.c_int32),
        ("step_fields", C.POINTER(C.c_double)), ("draw_seed", C.c_uint64),
        ("disorder_range", C.c_double * 2), ("tau_range", C.c_double * 2),
        ("n_spin_choices", C.c_int32), ("spin_choices", C.c_int32 * 8),
        ("mixed_order_limit", C.c_int64),
        ("sweep_points", C.c_int32), ("reserved1", C.c_int32),
        ("sweep_params", C.POINTER(C.c_double)),
    ]


# ------------------------------------------------------------ program nodes
@dataclass
class Evolve:
    """sequence/Sequence.hpp:28-34.  `fields` overrides (hx, hy, hz) per spin
    for this step; None keeps the system's fields."""
    tau: float
    steps: int = 1
    mode: int = REAL
    autonormalize: bool = False
    fields: Optional[Sequence[Sequence[float]]] = None
    tau_from_draw: bool = False


@dataclass
class Pulse:
    """An ideal rotation exp(-i angle/2 n.sigma) on `target` (None = all)."""
    angle: float
    axis: Sequence[float]
    target: Optional[int] = None


@dataclass
class Measure:
    pass


@dataclass
class Repeat:
    count: int
    body: List[object] = field(default_factory=list)


AXES3 = {"x": (1.0, 0.0, 0.0), "y": (0.0, 1.0, 0.0), "z": (0.0, 0.0, 1.0)}


def rotation(spec: str, nspins: int) -> Pulse:
    """makeRotation (src/core/Gate.cpp:173-195): "pi:x", "pi/2:y", "pi:x:3"."""
    parts = spec.split(":")
    if len(parts) not in (2, 3):
        raise ValueError(f"malformed pulse '{spec}'")
    angles = {"pi": math.pi, "pi/2": 0.5 * math.pi, "pi/4": 0.25 * math.pi}
    if parts[0] not in angles:
        raise ValueError(f"unknown pulse angle '{parts[0]}'; expected pi, pi/2 or pi/4")
    if parts[1] not in AXES3:
        raise ValueError(f"unknown rotation axis '{parts[1]}'; expected x, y or z")
    target = None
    if len(parts) == 3:
        idx = int(parts[2])
        if idx < 1 or idx > nspins:
            raise ValueError(f"pulse '{spec}': spin must be between 1 and {nspins}")
        target = idx - 1
    return Pulse(angles[parts[0]], AXES3[parts[1]], target)


def observable(spec: str) -> SsObservable:
    """makeObservable (src/core/Observable.cpp:149-176)."""
    p = spec.split(":")
    if p == ["norm"]:
        return SsObservable(OBS_NORM, 0, 0, 0)
    if p == ["energy"]:
        return SsObservable(OBS_ENERGY, 0, 0, 0)
    if len(p) == 2 and p[0] == "corr" and p[1].lower() in AXIS:
        return SsObservable(OBS_CORR, AXIS[p[1].lower()], 0, 0)
    if len(p) == 3 and p[0] == "mag" and p[1].isdigit() and int(p[1]) > 0 and p[2].lower() in AXIS:
        return SsObservable(OBS_MAG, AXIS[p[2].lower()], int(p[1]) - 1, 0)
    raise ValueError(f"unknown observable '{spec}'; expected one of corr:<axis>, "
                     "mag:<spin>:<axis>, norm, energy")


def observable_width(o: SsObservable) -> int:
    return 2 if o.kind in (OBS_CORR, OBS_NORM) else 1


@dataclass
class RunSpec:
    """Everything one experiment needs; `.config()` gives the C view."""
    nspins: int
    steps: List[object]
    observables: List[str]
    base_fields: Optional[Sequence[Sequence[float]]] = None
    initial_state: str = "random"
    basis_index: int = 0
    realizations: int = 1
    seed: int = 0
    dipolar_geometry: bool = True
    dipolar_scale: float = 1.0
    field_disorder: float = 0.0
    reference_axis: str = "z"
    epsilon: float = 1e-7
    draw_seed: int = 0
    disorder_range: Sequence[float] = (0.0, 0.0)
    tau_range: Sequence[float] = (0.0, 0.0)
    spin_choices: Sequence[int] = ()
    mixed_order_limit: int = 0
    # additive: a parameter sweep for the batched engine, one row per point
    # (dipolar_scale, field_disorder, tau of tau_from_draw steps, angle scale)
    sweep: Optional[Sequence[Sequence[float]]] = None

    def __post_init__(self) -> None:
        self._keep: list = []

    # -- flattening -------------------------------------------------------
    def _flatten(self, nodes, out: List[SsStep], tables: List[List[float]]) -> None:
        for n in nodes:
            s = SsStep()
            s.field_table = -1
            s.target = -1
            if isinstance(n, Evolve):
                s.kind, s.count, s.mode = EVOLVE, int(n.steps), int(n.mode)
                s.autonormalize, s.tau = int(bool(n.autonormalize)), float(n.tau)
                s.tau_from_draw = int(bool(n.tau_from_draw))
                if n.fields is not None:
                    flat = [float(v) for f in n.fields for v in f]
                    if len(flat) != 3 * self.nspins:
                        raise ValueError("step field table does not match the number of spins")
                    s.field_table = len(tables)
                    tables.append(flat)
                out.append(s)
            elif isinstance(n, Pulse):
                s.kind, s.angle = PULSE, float(n.angle)
                for i in range(3):
                    s.axis[i] = float(n.axis[i])
                s.target = -1 if n.target is None else int(n.target)
                out.append(s)
            elif isinstance(n, Measure):
                s.kind = MEASURE
                out.append(s)
            elif isinstance(n, Repeat):
                s.kind, s.count = REPEAT, int(n.count)
                at = len(out)
                out.append(s)
                self._flatten(n.body, out, tables)
                out[at].body_len = len(out) - at - 1
            else:
                raise TypeError(f"unknown step {n!r}")

    def measurement_count(self) -> int:
        def count(nodes) -> int:
            t = 0
            for n in nodes:
                if isinstance(n, Measure):
                    t += 1
                elif isinstance(n, Repeat):
                    t += n.count * count(n.body)
            return t
        return count(self.steps)

    def width(self) -> int:
        return sum(observable_width(observable(s)) for s in self.observables)

    def fields_for(self, hx=None, hy=None, hz=None):
        """A per-spin table overriding the named components only (the rule of
        src/io/Config.cpp:108-123)."""
        base = self.base_fields or [(0.0, 0.0, 0.0)] * self.nspins
        return [(hx if hx is not None else b[0], hy if hy is not None else b[1],
                 hz if hz is not None else b[2]) for b in base]

    def config(self) -> SsRunConfig:
        steps: List[SsStep] = []
        tables: List[List[float]] = []
        self._flatten(self.steps, steps, tables)
        base = self.base_fields or [(0.0, 0.0, 0.0)] * self.nspins
        bf = (C.c_double * (3 * self.nspins))(*[float(v) for f in base for v in f])
        st = (SsStep * max(1, len(steps)))(*steps)
        obs = [observable(o) for o in self.observables]
        ob = (SsObservable * max(1, len(obs)))(*obs)
        flat = [v for t in tables for v in t]
        tf = (C.c_double * max(1, len(flat)))(*flat)
        c = SsRunConfig()
        c.nspins = self.nspins
        c.initial_state = INIT[self.initial_state]
        c.basis_index = self.basis_index
        c.realizations = self.realizations
        c.seed = self.seed & 0xFFFFFFFFFFFFFFFF
        c.generate_geometry = int(self.dipolar_geometry)
        c.reference_axis = AXIS[self.reference_axis]
        c.dipolar_scale = self.dipolar_scale
        c.field_disorder = self.field_disorder
        c.epsilon = self.epsilon
        c.base_fields = C.cast(bf, C.POINTER(C.c_double))
        c.n_observables = len(obs)
        c.n_steps = len(steps)
        c.observables = C.cast(ob, C.POINTER(SsObservable))
        c.steps = C.cast(st, C.POINTER(SsStep))
        c.n_step_fields = len(tables)
        c.step_fields = C.cast(tf, C.POINTER(C.c_double))
        c.draw_seed = self.draw_seed & 0xFFFFFFFFFFFFFFFF
        c.disorder_range[0], c.disorder_range[1] = self.disorder_range
        c.tau_range[0], c.tau_range[1] = self.tau_range
        c.n_spin_choices = len(self.spin_choices)
        for i, v in enumerate(self.spin_choices):
            c.spin_choices[i] = v
        c.mixed_order_limit = int(self.mixed_order_limit)
        sw = None
        if self.sweep is not None and len(self.sweep) > 0:
            flat_sw = [float(v) for row in self.sweep for v in row]
            if len(flat_sw) != 4 * len(self.sweep):
                raise ValueError("a sweep row is (dipolar_scale, field_disorder, tau, angle_scale)")
            sw = (C.c_double * len(flat_sw))(*flat_sw)
            c.sweep_points = len(self.sweep)
            c.sweep_params = C.cast(sw, C.POINTER(C.c_double))
        self._keep = [bf, st, ob, tf, sw]
        return c

    def max_spins(self) -> int:
        return max([self.nspins, *self.spin_choices])
