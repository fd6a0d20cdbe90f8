"""Realisation sharding over ranks and the host fold (CPU, gloo).

The fold must reproduce the reference's Accumulator bit for bit
(src/ensemble/Ensemble.cpp:114-166; LocalRunner adds rows in index order,
EnsembleRunner.cpp:66-88), whichever way the realisations were split."""
import multiprocessing as mp
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from spin_systems_b200 import workloads
from spin_systems_b200.ensemble import Accumulator, fold_rows, run_sharded, shard


@pytest.mark.parametrize("total,world", [(0, 1), (1, 2), (5, 2), (1024, 8), (7, 3), (3, 4)])
def test_shards_tile_the_index_range(total, world):
    got = [shard(total, world, r) for r in range(world)]
    assert sum(c for _, c in got) == total
    nxt = 0
    for first, count in got:
        assert first == nxt and count >= 0
        nxt = first + count
    assert max(c for _, c in got) - min(c for _, c in got) <= 1


def test_shard_rejects_bad_ranks():
    with pytest.raises(ValueError):
        shard(4, 2, 2)
    with pytest.raises(ValueError):
        shard(4, 0, 0)


@pytest.fixture(scope="module")
def cpmg_rows(port):
    spec = workloads.cpmg_ideal()
    times, rows, _ = port.run_range(spec.config(), 0, spec.realizations, os.cpu_count() or 1)
    return times, rows


def test_fold_is_the_reference_accumulator(cpmg_rows, golden):
    times, rows = cpmg_rows
    acc = fold_rows(rows)
    assert np.array_equal(times, golden["exp_cpmg_l10_times"])
    assert np.array_equal(acc.mean, golden["exp_cpmg_l10_mean"])
    assert np.array_equal(acc.standard_deviation(), golden["exp_cpmg_l10_sd"])
    assert np.array_equal(acc.standard_error(), golden["exp_cpmg_l10_se"])


def test_merge_of_shards_agrees_with_the_fold(cpmg_rows):
    _, rows = cpmg_rows
    whole = fold_rows(rows)
    merged = Accumulator(whole.width)
    for r in range(3):
        first, count = shard(len(rows), 3, r)
        merged.merge(fold_rows(rows[first:first + count]))
    assert merged.count == whole.count
    assert np.allclose(merged.mean, whole.mean, rtol=0, atol=1e-13)
    assert np.allclose(merged.standard_deviation(), whole.standard_deviation(), rtol=0, atol=1e-12)


def test_accumulator_rejects_wrong_widths():
    a = Accumulator(3)
    with pytest.raises(ValueError):
        a.add([1.0, 2.0])
    with pytest.raises(ValueError):
        a.merge(Accumulator(2))
    assert np.array_equal(a.standard_deviation(), np.zeros(3))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, data, total, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        d = np.load(data)
        times, rows = d["times"], d["rows"]

        def runner(first, count):
            return times, rows[first:first + count]

        res = run_sharded(runner, total)
        if rank == 0:
            t, acc = res
            np.savez(out, times=t, mean=acc.mean, sd=acc.standard_deviation(),
                     se=acc.standard_error(), count=acc.count)
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,total", [(2, 20), (2, 1), (3, 20)])
def test_gloo_ranks_fold_like_one_process(cpmg_rows, tmp_path, world, total):
    times, rows = cpmg_rows
    rows = rows[:total]
    data = tmp_path / "rows.npz"
    np.savez(data, times=times, rows=rows)
    out = tmp_path / "out.npz"
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(data), total, str(out)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0] * world, codes
    got = np.load(out)
    want = fold_rows(rows)
    assert int(got["count"]) == total
    assert np.array_equal(got["times"], times)
    assert np.array_equal(got["mean"], want.mean)
    assert np.array_equal(got["sd"], want.standard_deviation())
    assert np.array_equal(got["se"], want.standard_error())


def _subgroup_main(rank, world, port, data, total, out):
    # Ranks 1 and 2 form a group without global rank 0; the group's rank 0
    # (global rank 1) receives the fold.
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        sub = dist.new_group([1, 2])
        if rank != 0:
            d = np.load(data)
            times, rows = d["times"], d["rows"]
            res = run_sharded(lambda first, count: (times, rows[first:first + count]), total,
                              group=sub)
            if rank == 1:
                t, acc = res
                np.savez(out, times=t, mean=acc.mean, count=acc.count)
            else:
                assert res is None
        # Rank 0 hosts the rendezvous store that the subgroup still uses:
        # it leaves only after the other two are done.
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_subgroup_without_global_rank_zero(cpmg_rows, tmp_path):
    times, rows = cpmg_rows
    data = tmp_path / "rows.npz"
    np.savez(data, times=times, rows=rows)
    out = tmp_path / "out.npz"
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_subgroup_main, args=(r, 3, port, str(data), len(rows), str(out)))
             for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0, 0], codes
    got = np.load(out)
    assert int(got["count"]) == len(rows)
    assert np.array_equal(got["mean"], fold_rows(rows).mean)
