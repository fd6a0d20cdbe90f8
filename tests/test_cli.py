"""The `spinsim` command line and its TOML reader against the reference's
behaviour (apps/spinsim/main.cpp, src/io/Config.cpp, tests/test_Config.cpp).

CPU: parsing, validation and error messages (no device needed).
GPU: `spinsim run` CSV output against the reference's runExperiment."""
import csv
import io
import json
import math
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from spin_systems_b200 import config as tomlcfg

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "spin_systems_b200" / "bin" / "spinsim"
CONFIGS = sorted((ROOT / "configs").glob("*.toml"))
# The reference's source tree, where present (the same variable the oracle's
# build reads); the tests that need it skip without it.
_REF_TREE = os.environ.get("SPINSIM_REFERENCE")
REFERENCE_CONFIGS = Path(_REF_TREE) / "configs" if _REF_TREE else None

MINIMAL = """
[system]
spins = 3

[field]
hz = 1.0

[measurement]
observables = ["corr:z"]

[[step]]
kind = "measure"

[[step]]
kind = "evolve"
tau = 0.1

[[step]]
kind = "measure"
"""


def cli(*args, check=False):
    if not CLI.exists():
        pytest.fail("spinsim binary missing: run __graft_entry__.build()")
    r = subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, timeout=600)
    if check and r.returncode != 0:
        raise AssertionError(r.stderr)
    return r


def write(tmp_path, text, name="c.toml"):
    p = tmp_path / name
    p.write_text(text)
    return p


def test_usage_and_exit_codes():
    r = cli()
    assert r.returncode == 2 and "Usage" in r.stdout
    assert cli("--help").returncode == 0


@pytest.mark.parametrize("path", CONFIGS, ids=[p.name for p in CONFIGS])
def test_configs_validate_and_describe(path):
    assert cli("validate", path).stdout.strip().endswith(": ok")
    d = cli("describe", path, check=True).stdout
    spec = tomlcfg.load(path)
    assert f"spins           {spec.nspins}" in d
    assert f"measurements    {spec.measurement_count()} per realization" in d


@pytest.mark.skipif(REFERENCE_CONFIGS is None or not REFERENCE_CONFIGS.is_dir(),
                    reason="SPINSIM_REFERENCE does not name the reference's source tree")
def test_reference_configs_parse():
    for p in sorted(REFERENCE_CONFIGS.glob("*.toml")):
        assert cli("validate", p).returncode == 0, p


def test_describe_text_is_the_references(tmp_path):
    # apps/spinsim/main.cpp:80-104: one line per field, names padded to 16
    # columns, {:g} for the floating-point values, observables each after a
    # space.  (The reference has no random_product state; this build prints
    # its name.)
    want = ("spins           10\n"
            "state space     1024 amplitudes\n"
            "initial state   random\n"
            "realizations    20\n"
            "seed            20240726\n"
            "geometry        dipolar 2D, per realization\n"
            "field disorder  0.5\n"
            "reference axis  x\n"
            "epsilon         1e-07\n"
            "measurements    8 per realization\n"
            "observables     corr:x norm\n")
    assert cli("describe", ROOT / "configs" / "cpmg_ideal_l10.toml", check=True).stdout == want
    d = cli("describe", ROOT / "configs" / "long_propagation_l16.toml", check=True).stdout
    assert "initial state   random_product\n" in d and "epsilon         1e-12\n" in d
    assert "field disorder  1\n" in d and "geometry        dipolar 2D, per realization\n" in d


def test_minimal_config_and_overrides(tmp_path):
    # test_Config.cpp:39-47, 116-138
    d = cli("describe", write(tmp_path, MINIMAL), check=True).stdout
    assert "measurements    2 per realization" in d
    text = MINIMAL + '\n[[step]]\nkind = "repeat"\ncount = 3\nbody = [ { kind = "repeat", count = 4, body = [ { kind = "measure" } ] } ]\n'
    d = cli("describe", write(tmp_path, text), check=True).stdout
    assert "measurements    14 per realization" in d


@pytest.mark.parametrize("text,needle", [
    ('[system]\nspins = 3\n[field]\nhx = [1.0, 2.0]\n[measurement]\nobservables = ["norm"]\n[[step]]\nkind = "measure"\n', "hx"),
    ('[system]\nspins = 2\n[measurement]\nobservables = ["norm"]\n[[step]]\nkind = "evolve"\ntau = 0.1\n', "'step'"),
    ('[system]\nspins = 2\n[measurement]\nobservables = ["corr:w"]\n[[step]]\nkind = "measure"\n', "observables"),
    ('[system]\nspins = 2\n[measurement]\nobservables = ["norm"]\n[[step]]\nkind = "teleport"\n', "teleport"),
    ('[system\nspins = 2', "<syntax>"),
    ('[system]\nspins = 99\n[measurement]\nobservables = ["norm"]\n[[step]]\nkind = "measure"\n', "system.spins"),
    ('[system]\nspins = 2\n[measurement]\nobservables = ["norm"]\n[[step]]\nkind = "evolve"\ntau = 0.1\nsteps = -1\n[[step]]\nkind = "measure"\n', "steps"),
    ('[system]\nspins = 2\n[measurement]\nobservables = ["norm"]\n[[step]]\nkind = "pulse"\nrotation = "pi:x:9"\n[[step]]\nkind = "measure"\n', "rotation"),
    ('[system]\nspins = 2\n[measurement]\nobservables = ["norm"]\n[[step]]\nkind = "repeat"\ncount = 2\n', "body"),
    ('[system]\nspins = 2\n[system]\nspins = 3\n', "<syntax>"),
])
def test_configuration_errors_name_the_key(tmp_path, text, needle):
    r = cli("validate", write(tmp_path, text))
    assert r.returncode == 1
    assert needle in r.stderr and "c.toml" in r.stderr, r.stderr
    if needle == "teleport":
        assert "evolve" in r.stderr


def test_unknown_option_and_bad_values(tmp_path):
    p = write(tmp_path, MINIMAL)
    assert cli("run", p, "--bogus").returncode == 1
    assert cli("run", p, "--threads", "x").returncode == 1
    assert cli("run", p, "--precision", "fp16").returncode == 1


def read_csv(text):
    rows = list(csv.reader(io.StringIO(text)))
    header, body = rows[0], np.array([[float(x) for x in r] for r in rows[1:]])
    return header, body


def check_against(header, body, golden, name, atol):
    times = golden[f"exp_{name}_times"]
    mean, sd, se = golden[f"exp_{name}_mean"], golden[f"exp_{name}_sd"], golden[f"exp_{name}_se"]
    ncols = (len(header) - 1) // 3
    assert np.allclose(body[:, 0], times, rtol=1e-9, atol=1e-12)
    got = body[:, 1:].reshape(len(times), ncols, 3)
    want = np.stack([mean, sd, se], axis=-1).reshape(len(times), ncols, 3)
    err = np.abs(got - want) - 1e-11 * np.abs(want)  # 12 significant digits in the CSV
    assert err.max() < atol, err.max()


def dump_toml(doc):
    """A TOML writer for the parsed reference documents (tables, one array of
    step tables, inline tables in arrays)."""
    def val(v):
        if isinstance(v, bool):
            return "true" if v else "false"
        if isinstance(v, (int, float)):
            return repr(v)
        if isinstance(v, str):
            return json.dumps(v)
        if isinstance(v, list):
            return "[" + ", ".join(val(x) for x in v) + "]"
        if isinstance(v, dict):
            return "{ " + ", ".join(f"{k} = {val(x)}" for k, x in v.items()) + " }"
        raise TypeError(v)
    out = []
    for k, v in doc.items():
        if k == "step":
            continue
        out.append(f"[{k}]")
        out += [f"{kk} = {val(vv)}" for kk, vv in v.items()]
    for st in doc["step"]:
        out.append("[[step]]")
        out += [f"{kk} = {val(vv)}" for kk, vv in st.items()]
    return "\n".join(out) + "\n"


@pytest.mark.gpu
@pytest.mark.parametrize("engine", ["batch", "plain"])
def test_run_matches_reference_experiment(golden, engine):
    r = cli("run", ROOT / "configs" / "cpmg_ideal_l10.toml", "--engine", engine, check=True)
    header, body = read_csv(r.stdout)
    assert header[:4] == ["time", "corr_x_re_mean", "corr_x_re_sd", "corr_x_re_stderr"]
    check_against(header, body, golden, "cpmg_l10", 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ref_cpmg8z", "ref_rabi"])
def test_reference_example_configs_run(golden, tmp_path, name):
    docs = json.loads((ROOT / "tests" / "golden" / "reference_configs.json").read_text())
    p = write(tmp_path, dump_toml(docs[name]), f"{name}.toml")
    r = cli("run", p, "--realizations", "3", check=True)
    header, body = read_csv(r.stdout)
    check_against(header, body, golden, name, 1e-9)


@pytest.mark.gpu
def test_run_mixed_precision_and_output_file(golden, tmp_path):
    out = tmp_path / "o" / "r.csv"
    r = cli("run", ROOT / "configs" / "cpmg_ideal_l10.toml", "--precision", "mixed", "--out", out,
            check=True)
    assert "realizations on batched mixed" in r.stderr
    header, body = read_csv(out.read_text())
    mean = golden["exp_cpmg_l10_mean"].reshape(len(body), -1)
    assert np.abs(body[:, 1] - mean[:, 0]).max() < 1e-5


def csv_diff(got: str, want: str):
    """(data fields, fields that differ, largest gap of those beyond the
    12-digit print rounding).  The header and the time column must match
    byte for byte."""
    g, w = got.splitlines(), want.splitlines()
    assert len(g) == len(w) and g[0] == w[0]
    fields, differ, gap = 0, 0, 0.0
    for a, b in zip(g[1:], w[1:]):
        fa, fb = a.split(","), b.split(",")
        assert len(fa) == len(fb) and fa[0] == fb[0]
        for x, y in zip(fa[1:], fb[1:]):
            fields += 1
            if x != y:
                differ += 1
                gap = max(gap, abs(float(x) - float(y)) - 1e-11 * abs(float(y)))
    return fields, differ, gap


@pytest.mark.gpu
@pytest.mark.parametrize("engine", ["batch", "plain"])
def test_run_csv_is_the_references_bytes(engine, tmp_path):
    # `spinsim run` against the reference's own runExperiment + writeCsv
    # (io/Experiment.cpp:57-97), byte for byte: the header and the time
    # column are identical.  The device adds the same FP64 terms in another
    # order, so a value's last printed digits may differ: every such field
    # stays within the repository's 1e-10 parity bar (absolute, beyond the
    # 12-significant-digit rounding of the print).
    want = json.loads((ROOT / "tests" / "golden" / "reference_csv.json").read_text())
    got = cli("run", ROOT / "configs" / "cpmg_ideal_l10.toml", "--engine", engine,
              check=True).stdout
    fields, differ, gap = csv_diff(got, want["cpmg_l10"])
    print(f"cpmg_l10 {engine}: {differ} of {fields} fields differ, largest gap {gap:.3g}")
    assert gap < 1e-10, (differ, gap)
    docs = json.loads((ROOT / "tests" / "golden" / "reference_configs.json").read_text())
    for name in ("ref_cpmg8z", "ref_rabi"):
        p = write(tmp_path, dump_toml(docs[name]), f"{name}.toml")
        got = cli("run", p, "--realizations", "3", "--engine", engine, check=True).stdout
        fields, differ, gap = csv_diff(got, want[name])
        print(f"{name} {engine}: {differ} of {fields} fields differ, largest gap {gap:.3g}")
        assert gap < 1e-9, (name, differ, gap)
