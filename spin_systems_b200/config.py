"""TOML run configurations -> RunSpec, with the reference's schema
(src/io/Config.cpp:83-281) and the same additive keys as the C++ reader
(initial_state = "random_product"; [ensemble] draw_seed, disorder_range,
tau_range, spin_choices; evolve tau_from_draw; pulse angle)."""
from __future__ import annotations

import tomllib
from pathlib import Path
from typing import Optional

from .abi import Evolve, Measure, Pulse, Repeat, RunSpec, rotation, REAL, IMAGINARY


class ConfigError(ValueError):
    pass


def _component(node: dict, key: str, n: int):
    v = node.get(key)
    if v is None:
        return [0.0] * n
    if isinstance(v, (int, float)) and not isinstance(v, bool):
        return [float(v)] * n
    if not isinstance(v, list) or len(v) != n:
        raise ConfigError(f"'{key}' has the wrong shape")
    return [float(x) for x in v]


def _fields(node: dict, n: int):
    hx, hy, hz = (_component(node, k, n) for k in ("hx", "hy", "hz"))
    return list(zip(hx, hy, hz))


def _steps(items, n: int, base):
    out = []
    for t in items:
        kind = t["kind"]
        if kind == "measure":
            out.append(Measure())
        elif kind == "evolve":
            fields = None
            if any(k in t for k in ("hx", "hy", "hz")):
                hx, hy, hz = (_component(t, k, n) for k in ("hx", "hy", "hz"))
                fields = [(hx[s] if "hx" in t else base[s][0], hy[s] if "hy" in t else base[s][1],
                           hz[s] if "hz" in t else base[s][2]) for s in range(n)]
            mode = {"real": REAL, "imaginary": IMAGINARY}[t.get("mode", "real")]
            out.append(Evolve(float(t["tau"]), int(t.get("steps", 1)), mode,
                              bool(t.get("autonormalize", False)), fields,
                              bool(t.get("tau_from_draw", False))))
        elif kind == "pulse":
            p = rotation(t["rotation"], n)
            if "angle" in t:
                p = Pulse(float(t["angle"]), p.axis, p.target)
            out.append(p)
        elif kind == "repeat":
            out.append(Repeat(int(t["count"]), _steps(t["body"], n, base)))
        else:
            raise ConfigError(f"unknown step kind '{kind}'")
    return out


def load(path, realizations: Optional[int] = None) -> RunSpec:
    return from_document(tomllib.loads(Path(path).read_text()), realizations)


def from_document(doc: dict, realizations: Optional[int] = None) -> RunSpec:
    system = doc["system"]
    n = int(system["spins"])
    base = _fields(doc.get("field", {}), n)
    ens = doc.get("ensemble", {})
    meas = doc.get("measurement", {})
    spec = RunSpec(
        nspins=n, steps=_steps(doc["step"], n, base), observables=list(meas["observables"]),
        base_fields=base, initial_state=system.get("initial_state", "random"),
        basis_index=int(system.get("basis_index", 0)),
        realizations=int(realizations if realizations is not None else ens.get("realizations", 1)),
        seed=int(ens.get("seed", 0)), dipolar_geometry=bool(ens.get("dipolar_geometry", True)),
        dipolar_scale=float(ens.get("dipolar_scale", 1.0)),
        field_disorder=float(ens.get("field_disorder", 0.0)),
        reference_axis=meas.get("reference_axis", "z"),
        epsilon=float(doc.get("numerics", {}).get("epsilon", 1e-7)),
        draw_seed=int(ens.get("draw_seed", 0)),
        disorder_range=tuple(ens.get("disorder_range", (0.0, 0.0))),
        tau_range=tuple(ens.get("tau_range", (0.0, 0.0))),
        spin_choices=tuple(ens.get("spin_choices", ())),
    )
    return spec
