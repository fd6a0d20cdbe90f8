"""Split-cluster schedules (L = 14..16 mixed): the state and the reference of
a realisation run on clusters of their own, and the observables come from
snapshots taken at each measurement point.  Against the C port of the
reference on the short program of the cluster tests (every observable kind,
transverse fields, ideal pulses), against the paired schedule of the same
size, with more observables than the paired kernel holds, and in several
launches when the snapshot budget is smaller than the bucket."""
import numpy as np
import pytest
import torch

import spin_systems_b200 as ss
from spin_systems_b200 import abi

from test_batch_dist_gpu import ECHO_TOL, corr0, short_spec

pytestmark = pytest.mark.gpu

SPLIT = {14: "L14.R4.f32.global.c2.split", 15: "L15.R4.f32.global.c4.split",
         16: "L16.R4.f32.global.c8.split"}


def force(tmp_path, L, variant):
    ss.clear_schedule()
    p = tmp_path / "force.tsv"
    p.write_text(f"{torch.cuda.get_device_name(0)}\t{L}\tmixed\t{variant}\t1.0\n")
    ss.load_schedule(p)


def launches(batch):
    return batch.stats()["launches"]


@pytest.mark.parametrize("L", [14, 15, 16])
def test_split_schedules_match_the_oracle_and_the_paired_kernel(engine, port, tmp_path, L):
    n = 2 if L < 16 else 1
    cfg = short_spec(L, n).config()
    want = np.stack([port.run_realization(cfg, i)[1] for i in range(n)])
    ss.clear_schedule()
    _, paired = ss.Batch(engine, cfg, 0, n, abi.MIXED).run()
    force(tmp_path, L, SPLIT[L])
    b = ss.Batch(engine, cfg, 0, n, abi.MIXED)
    _, rows = b.run()
    assert launches(b) == 3  # prepare, the split kernel, the snapshot measurement
    ss.clear_schedule()
    err = np.abs(rows[:, :, 0] - want[:, :, 0]).max(axis=1) / corr0(cfg, n, L)
    assert err.max() < ECHO_TOL, err
    assert np.abs(rows[:, :, 4:6] - want[:, :, 4:6]).max() < 1e-6  # norms
    # the paired kernel's arithmetic on each vector; the measurement sums
    # run in another order (bar: the mixed path's own accuracy)
    assert np.abs(rows - paired).max() <= 1e-6 * max(1.0, np.abs(paired).max())


def test_split_schedule_measures_more_than_eight_observables(engine, port, tmp_path):
    # Ten observables (14 columns) in one split batch; the paired kernel
    # measures the same realisation in two batches of at most eight.
    first = ["corr:x", "corr:y", "corr:z", "norm", "energy"]
    mags = [f"mag:{s}:x" for s in range(1, 6)]
    spec = short_spec(14, 1)
    spec.observables = first + mags
    cfg = spec.config()
    force(tmp_path, 14, SPLIT[14])
    _, rows = ss.Batch(engine, cfg, 0, 1, abi.MIXED).run()
    ss.clear_schedule()
    parts = []
    for obs in (first, mags):
        spec.observables = obs
        parts.append(ss.Batch(engine, spec.config(), 0, 1, abi.MIXED).run()[1])
    paired = np.concatenate(parts, axis=2)
    assert rows.shape == paired.shape == (1, 3, 14)
    assert np.abs(rows - paired).max() <= 1e-6 * max(1.0, np.abs(paired).max())
    want = port.run_realization(cfg, 0)[1]
    assert np.abs(rows[0, :, 0] - want[:, 0]).max() / corr0(cfg, 1, 14)[0] < ECHO_TOL


def test_split_schedule_in_launches_of_the_snapshot_budget(engine, tmp_path):
    # 70 realisations at three measurement points: 1.5 MiB of snapshots
    # each, a budget of 64 -> launches of 64 and 6, bit for bit the rows of
    # one launch; a budget below 64 realisations -> the paired kernel.
    cfg = short_spec(14, 70).config()
    per = 3 * 2 * (1 << 14) * 16
    force(tmp_path, 14, SPLIT[14])
    try:
        one = ss.Batch(engine, cfg, 0, 70, abi.MIXED)
        _, rows_one = one.run()
        ss.set_snapshot_budget(64 * per)
        two = ss.Batch(engine, cfg, 0, 70, abi.MIXED)
        _, rows_two = two.run()
        ss.set_snapshot_budget(63 * per)
        paired = ss.Batch(engine, cfg, 0, 70, abi.MIXED)
        _, rows_paired = paired.run()
    finally:
        ss.set_snapshot_budget(16 << 30)
        ss.clear_schedule()
    assert launches(one) == 3 and launches(two) == 5 and launches(paired) == 2
    assert np.array_equal(rows_one, rows_two)
    assert np.abs(rows_paired - rows_one).max() <= 1e-6 * max(1.0, np.abs(rows_one).max())


def test_fp64_l16_has_only_split_clusters_and_runs_one_per_launch_when_tight(engine):
    # FP64 at L = 16 has no paired schedule: a budget below one realisation's
    # snapshots still runs, one realisation per launch, with the same rows.
    cfg = short_spec(16, 2).config()
    ss.clear_schedule()
    b = ss.Batch(engine, cfg, 0, 2, abi.FP64)
    _, rows = b.run()
    assert launches(b) == 3
    ss.set_snapshot_budget(1)
    try:
        tight = ss.Batch(engine, cfg, 0, 2, abi.FP64)
        _, rows_tight = tight.run()
    finally:
        ss.set_snapshot_budget(16 << 30)
    assert launches(tight) == 5  # prepare + two (kernel, measurement) pairs
    assert np.array_equal(rows, rows_tight)
