"""The engine's host layer built with AddressSanitizer and
UndefinedBehaviorSanitizer and run without a GPU (csrc/apps/host_check.cpp):
the TOML reader and config validation on every shipped config and on
malformed ones, then the realisation assembly (random streams, dipolar
placement, field disorder, every initial-state kind, the harness draws), the
Bessel sequences and the Chebyshev expansions at L = 2..16.  A sanitizer
finding (out-of-bounds access, use after free, leak, signed overflow, ...)
aborts the checker with its report, so the test fails on it."""
import os
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "spin_systems_b200" / "csrc"
EXE = ROOT / "spin_systems_b200" / "_build" / "host_check_asan"

MALFORMED = [
    '[system]\nspins = 3\n[field]\nhx = [1.0, 2.0]\n[measurement]\nobservables = ["norm"]\n'
    '[[step]]\nkind = "measure"\n',
    '[system\nspins = 2',
    '[system]\nspins = 99\n[measurement]\nobservables = ["norm"]\n[[step]]\nkind = "measure"\n',
    '[system]\nspins = 2\n[measurement]\nobservables = ["norm"]\n[[step]]\nkind = "repeat"\n'
    'count = 2\n',
    '[system]\nspins = 2\n[system]\nspins = 3\n',
    'title = "unterminated\n',
    '[system]\nspins = 2\n[measurement]\nobservables = ["corr:w"]\n[[step]]\nkind = "measure"\n',
    '[system]\nspins = 2\n[measurement]\nobservables = ["norm"]\n[[step]]\nkind = "pulse"\n'
    'rotation = "pi:x:9"\n[[step]]\nkind = "measure"\n',
]


def _run(args):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    return subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True, env=env,
                          timeout=600)


def test_host_layer_under_sanitizers(tmp_path):
    subprocess.run(["make", "-s", "-C", str(CSRC), "host-check"], check=True, timeout=900)
    good = sorted((ROOT / "configs").glob("*.toml"))
    ref = os.environ.get("SPINSIM_REFERENCE")
    if ref and (Path(ref) / "configs").is_dir():
        good += sorted((Path(ref) / "configs").glob("*.toml"))
    r = _run(good)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failure(s)" in r.stdout
    bad = []
    for i, text in enumerate(MALFORMED):
        p = tmp_path / f"bad{i}.toml"
        p.write_text(text)
        bad.append(p)
    r = _run(["--expect-errors", *bad])
    assert r.returncode == 0, r.stdout + r.stderr
    assert f"{len(bad)} config(s) rejected as expected" in r.stdout


def test_statistics_and_csv_are_the_references_bytes(tmp_path):
    # The C++ API's Accumulator and writeCsv (under the sanitizers), fed the
    # L = 10 CPMG rows of the C restatement, which are bit-identical to the
    # reference's curves, print the reference's own runExperiment + writeCsv
    # output byte for byte (tests/golden/reference_csv.json; Welford in index
    # order, {:.10g} times, {:.12g} statistics; io/Experiment.cpp:74-110).
    import json

    from oracle.oracle import Port
    from spin_systems_b200 import workloads

    subprocess.run(["make", "-s", "-C", str(CSRC), "host-check"], check=True, timeout=900)
    want = json.loads((ROOT / "tests" / "golden" / "reference_csv.json").read_text())["cpmg_l10"]
    spec = workloads.cpmg_ideal()
    times, rows, _ = Port().run_range(spec.config(), 0, spec.realizations, 4)
    header = want.splitlines()[0].split(",")[1:]
    columns = [h[: -len("_mean")] for h in header[0::3]]
    n, points, width = rows.shape
    assert width == len(columns) and points == len(times)
    lines = [f"{points} {width} {n}", " ".join(columns), " ".join(repr(float(t)) for t in times)]
    lines += [" ".join(repr(float(v)) for v in r.ravel()) for r in rows]
    src = tmp_path / "rows.txt"
    src.write_text("\n".join(lines) + "\n")
    r = _run(["--csv", src])
    assert r.returncode == 0, r.stderr
    assert r.stdout == want
