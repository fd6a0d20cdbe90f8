"""Ensemble statistics and realisation sharding across ranks.

Accumulator follows src/ensemble/Ensemble.cpp:114-166 (Welford add in index
order, Chan merge, sample standard deviation and standard error) with the
same operation order, so a fold here is bit-identical to the reference's
fold of the same rows.  Sharding follows the partitioning the reference's
LocalRunner admits (src/ensemble/EnsembleRunner.cpp:27-88): realisations
are independent, each rank runs a contiguous index range on its own GPU,
and rank 0 folds all rows in index order; there is no device collective.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np


class Accumulator:
    """Running mean and M2 over samples of a fixed width."""

    def __init__(self, width: int):
        self.count = 0
        self.mean = np.zeros(width)
        self.m2 = np.zeros(width)

    @property
    def width(self) -> int:
        return self.mean.size

    def add(self, sample) -> None:
        x = np.asarray(sample, dtype=np.float64).ravel()
        if x.size != self.mean.size:
            raise ValueError("sample width does not match the accumulator")
        self.count += 1
        n = float(self.count)
        delta = x - self.mean
        self.mean = self.mean + delta / n
        self.m2 = self.m2 + delta * (x - self.mean)

    def merge(self, other: "Accumulator") -> None:
        if other.mean.size != self.mean.size:
            raise ValueError("cannot merge accumulators of different width")
        if other.count == 0:
            return
        if self.count == 0:
            self.count, self.mean, self.m2 = other.count, other.mean.copy(), other.m2.copy()
            return
        na, nb = float(self.count), float(other.count)
        total = na + nb
        delta = other.mean - self.mean
        self.mean = self.mean + delta * nb / total
        self.m2 = self.m2 + other.m2 + delta * delta * na * nb / total
        self.count += other.count

    def standard_deviation(self) -> np.ndarray:
        if self.count < 2:
            return np.zeros_like(self.mean)
        return np.sqrt(self.m2 / float(self.count - 1))

    def standard_error(self) -> np.ndarray:
        sd = self.standard_deviation()
        if self.count < 2:
            return sd
        return sd * (1.0 / np.sqrt(float(self.count)))


def fold_rows(rows: np.ndarray) -> Accumulator:
    """Adds realisation rows (realisations x points x columns) in index order."""
    rows = np.asarray(rows, dtype=np.float64)
    acc = Accumulator(int(np.prod(rows.shape[1:])) if rows.ndim > 1 else 1)
    for r in rows:
        acc.add(r)
    return acc


def shard(total: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous index range [first, first + count) of `rank`; the first
    total % world ranks take one realisation more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    if total < 0:
        raise ValueError("negative realisation count")
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


Runner = Callable[[int, int], Tuple[np.ndarray, np.ndarray]]


def run_sharded(runner: Runner, total: int, group=None) -> Optional[Tuple[np.ndarray, Accumulator]]:
    """Runs this rank's shard through `runner(first, count) -> (times, rows)`
    and folds every rank's rows on the group's rank 0 in index order.

    Returns (times, accumulator) on the group's rank 0 and None elsewhere
    (`group` defaults to the whole world; only its members may call).  With no
    initialised process group it runs everything locally.  Every rank takes
    the same collective steps (one gather), also when its shard is empty."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        times, rows = runner(0, total)
        return np.asarray(times), fold_rows(rows)
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    if rank < 0:
        raise ValueError("this process is not a member of the group")
    first, count = shard(total, world, rank)
    times, rows = runner(first, count) if count else (None, None)
    gathered = [None] * world if rank == 0 else None
    # gather_object names its destination by global rank: the group's rank 0.
    dst = 0 if group is None else dist.get_global_rank(group, 0)
    dist.gather_object((first, times, rows), gathered, dst=dst, group=group)
    if rank != 0:
        return None
    parts = sorted((p for p in gathered if p[2] is not None), key=lambda p: p[0])
    if not parts:
        raise ValueError("an ensemble needs at least one realisation")
    times = np.asarray(parts[0][1])
    for p in parts[1:]:
        if not np.array_equal(np.asarray(p[1]), times):
            raise RuntimeError("ranks disagree on the measurement times")
    acc = None
    for p in parts:
        rows = np.asarray(p[2], dtype=np.float64)
        if acc is None:
            acc = Accumulator(int(np.prod(rows.shape[1:])))
        for r in rows:
            acc.add(r)
    return times, acc
