"""bench.py's reference arm on the host cores (no GPU): the reference's own
CPU build (or the C restatement) timed on a bounded sample, printed as one
JSON line with the headline metric's keys; under torchrun only rank 0 works."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run_arm(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                           "--warmup", "0"], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=900)


def test_reference_arm_prints_the_contract_line():
    out = run_arm({"RANK": "0", "WORLD_SIZE": "1"})
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "curves/s"
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["warmup"] == 0
    assert line["value"] > 0 and line["ms_per_step"] > 0
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert cb["model"] and "seeded" in cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"],
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "workload" in line["config"]


def test_reference_arm_other_ranks_exit_without_work():
    out = run_arm({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert out.returncode == 0 and out.stdout.strip() == ""


def test_cpu_sample_is_seeded_and_spread_over_the_batch():
    sys.path.insert(0, str(ROOT))
    import numpy as np
    import bench
    a = bench.seeded_subset(320, 1024, 7)
    assert np.array_equal(a, bench.seeded_subset(320, 1024, 7))
    assert len(set(a.tolist())) == 320 and a.max() < 1024 and a.max() > 900 and a.min() < 100
    b = bench.seeded_subset(1500, 1024, 7)  # more than exist: every index, then again
    assert len(b) == 1500 and len(set(b[:1024].tolist())) == 1024
