"""Regenerates the committed golden fixtures under tests/golden/.

Sources, both read here and never at test time on a machine without them:

* the reference's Bessel tables, tests/data/bessel_reference.txt (written by
  its gen_bessel_reference.f from Cody's rjbesl/ribesl), parsed into
  bessel_reference.npz;
* outputs of the reference core itself, compiled from its sources into
  oracle/_ref/libspinsim_ref.so by oracle/Makefile: realisation set-ups,
  propagator steps and whole echo curves, stored in reference_outputs.npz.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import REFERENCE_TREE, Ref, build, random_state, sample_hamiltonian  # noqa: E402
from spin_systems_b200 import workloads  # noqa: E402

OUT = Path(__file__).resolve().parent


def parse_bessel(path: Path):
    kinds, xs, ncalc, values = [], [], [], []
    lines = path.read_text().splitlines()
    i = 0
    while i < len(lines):
        head = lines[i].split()
        i += 1
        if len(head) != 4:
            continue
        kind, x, nb, nc = head[0], float(head[1]), int(head[2]), int(head[3])
        vals = [float(lines[i + k]) for k in range(nb)]
        i += nb
        kinds.append(0 if kind == "J" else 1)
        xs.append(x)
        ncalc.append(nc)
        values.append(vals)
    return (np.array(kinds, dtype=np.int32), np.array(xs), np.array(ncalc, dtype=np.int32),
            np.array(values))


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    build(ref=True)
    ref = Ref()

    kinds, xs, ncalc, values = parse_bessel(REFERENCE_TREE / "tests" / "data" / "bessel_reference.txt")
    np.savez_compressed(OUT / "bessel_reference.npz", kinds=kinds, x=xs, ncalc=ncalc, values=values)

    out = {}
    # Random streams of a few realisations (uniform and gaussian).
    for idx in (0, 7, 179):
        out[f"rng_u_{idx}"] = ref.rng(20240726, idx, 0, 64)
        out[f"rng_g_{idx}"] = ref.rng(20240726, idx, 1, 65)

    # Realisation set-ups: fields and couplings kept, states by digest.
    for name, spec, indices in (("cpmg", workloads.cpmg_ideal(), range(20)),
                                ("xy8", workloads.xy8_finite(realizations=4), range(4))):
        cfg = spec.config()
        for idx in indices:
            s = ref.setup(cfg, idx)
            out[f"setup_{name}_{idx}_fields"] = s["fields"]
            out[f"setup_{name}_{idx}_J"] = s["J"]
            out[f"setup_{name}_{idx}_pairs"] = s["pairs"]
            out[f"setup_{name}_{idx}_psi0_sha"] = np.frombuffer(bytes.fromhex(digest(s["psi0"])), dtype=np.uint8)
            out[f"setup_{name}_{idx}_ref0_sha"] = np.frombuffer(bytes.fromhex(digest(s["ref0"])), dtype=np.uint8)
            out[f"setup_{name}_{idx}_psi0_head"] = s["psi0"][:32]

    # The reference tests' own random states (DenseReference.cpp:204-214).
    for L, seed in [(L, 0x9001 + L) for L in range(1, 7)] + [(4, 0x5150), (4, 0x2718), (5, 0x3141),
                                                               (4, 0x1618), (3, 0x606), (3, 0x4004),
                                                               (4, 0x1111), (4, 0x2222), (4, 0x4444)]:
        out[f"ref_state_{L}_{seed}"] = ref.random_state(L, seed)
    # Conservation over 10^4 steps of 0.02 at L=5 (test_Propagator.cpp:100-124),
    # replayed on the reference's own state: final state, norm and energy drift.
    from oracle.oracle import dense_hamiltonian
    f, p, J = sample_hamiltonian(5)
    psi = out["ref_state_5_12609"].copy()
    for _ in range(100):
        psi, _ = ref.evolve(5, f, p, J, psi, 0, 0.02, 100, eps=1e-12)
    out["conservation_final"] = psi

    # Propagator steps on the reference's own sampleHamiltonian recipe.
    for L in range(1, 7):
        f, p, J = sample_hamiltonian(L)
        psi0 = random_state(L, 0x9001 + L)
        out[f"prop_psi0_{L}"] = psi0
        for tau in (0.05, 0.3, 1.0):
            psi, order = ref.evolve(L, f, p, J, psi0, 0, tau, 1, eps=1e-12)
            out[f"prop_real_{L}_{tau}"] = psi
            out[f"prop_real_order_{L}_{tau}"] = np.array([order])
        for tau in (0.05, 0.4):
            psi, order = ref.evolve(L, f, p, J, psi0, 1, tau, 1, eps=1e-12)
            out[f"prop_imag_{L}_{tau}"] = psi

    # Whole echo curves: the L=10 CPMG (20 realisations), an L=8 XY-8 with
    # finite pulses (4 realisations, 2 blocks), two full L=12 XY-8 curves.
    cfg = workloads.cpmg_ideal().config()
    t, v, _ = ref.run_range(cfg, 0, 20, 8)
    out["curves_cpmg_times"], out["curves_cpmg_rows"] = t, v
    spec = workloads.xy8_finite(nspins=8, realizations=4, blocks=2)
    spec.observables = ["corr:x", "norm", "energy", "mag:2:z"]
    cfg = spec.config()
    t, v, _ = ref.run_range(cfg, 0, 4, 4)
    out["curves_xy8_l8_times"], out["curves_xy8_l8_rows"] = t, v
    cfg = workloads.xy8_finite(realizations=2).config()
    t, v, _ = ref.run_range(cfg, 0, 2, 2)
    out["curves_xy8_l12_times"], out["curves_xy8_l12_rows"] = t, v

    # Whole experiments (runExperiment with LocalRunner): mean/sd/stderr per
    # (point, column) for the CLI's CSV, on this repository's L=10 CPMG config
    # and on the reference's own example configs with few realisations.
    from spin_systems_b200 import config as tomlcfg
    for name, path, count in (("cpmg_l10", ROOT / "configs" / "cpmg_ideal_l10.toml", None),
                              ("ref_cpmg8z", REFERENCE_TREE / "configs" / "cpmg8z.toml", 3),
                              ("ref_rabi", REFERENCE_TREE / "configs" / "rabi_szsz.toml", 3)):
        spec = tomlcfg.load(path, realizations=count)
        t, m, sd, se, _ = ref.run_experiment(spec.config(), 4)
        out[f"exp_{name}_times"], out[f"exp_{name}_mean"] = t, m
        out[f"exp_{name}_sd"], out[f"exp_{name}_se"] = sd, se

    # The same experiments as the reference's own CSV bytes (writeCsv), the
    # output `spinsim run` must reproduce.
    csv_text = {}
    for name, path, count in (("cpmg_l10", ROOT / "configs" / "cpmg_ideal_l10.toml", None),
                              ("ref_cpmg8z", REFERENCE_TREE / "configs" / "cpmg8z.toml", 3),
                              ("ref_rabi", REFERENCE_TREE / "configs" / "rabi_szsz.toml", 3)):
        csv_text[name] = ref.experiment_csv(tomlcfg.load(path, realizations=count).config(), 4)

    np.savez_compressed(OUT / "reference_outputs.npz", **out)
    # The reference's example configurations as parsed documents (JSON), so the
    # device runs can be checked against exp_ref_* where the reference tree
    # is absent.
    import json
    import tomllib
    docs = {name: tomllib.loads((REFERENCE_TREE / "configs" / f"{fname}.toml").read_text())
            for name, fname in (("ref_cpmg8z", "cpmg8z"), ("ref_rabi", "rabi_szsz"))}
    (OUT / "reference_configs.json").write_text(json.dumps(docs, indent=1, sort_keys=True))
    (OUT / "reference_csv.json").write_text(json.dumps(csv_text, indent=1, sort_keys=True))
    print("wrote", sorted(p.name for p in OUT.glob("*.npz")))


if __name__ == "__main__":
    main()
