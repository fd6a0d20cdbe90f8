"""Tile patterns of the tiled order kernel (host logic, no GPU).

Every pair of spins must share a tile (so every coupling is applied on chip
exactly once), every tile must hold exactly the kernel's tile width, the
plan must be reproducible, and the last tile -- the one that forms T_n and
streams psi, T_{n-2} and the diagonal -- has the longest run of low bits.
"""
import itertools

import pytest

import spin_systems_b200 as ss


def low_run(m: int) -> int:
    r = 0
    while (m >> r) & 1:
        r += 1
    return r


@pytest.mark.parametrize("tile_bits,line_bits", [(8, 3), (8, 4), (12, 3), (13, 4)])
def test_plans_cover_every_pair_with_full_tiles(tile_bits, line_bits):
    for L in range(tile_bits, 31):
        plan = ss.tile_plan(L, tile_bits, line_bits)
        assert all(bin(m).count("1") == tile_bits for m in plan)
        # every tile's copies move runs of 2^line_bits consecutive amplitudes
        assert all(low_run(m) >= min(line_bits, tile_bits - 2) for m in plan)
        assert all(m < (1 << L) for m in plan)
        for i, j in itertools.combinations(range(L), 2):
            pair = (1 << i) | (1 << j)
            assert any(m & pair == pair for m in plan), (L, i, j)
        assert low_run(plan[-1]) == max(low_run(m) for m in plan)
        if L == tile_bits:
            assert plan == [(1 << L) - 1]


def test_plans_are_reproducible_and_small():
    first = {L: ss.tile_plan(L, 12, 3) for L in (18, 20, 22, 24)}
    again = {L: ss.tile_plan(L, 12, 3) for L in (18, 20, 22, 24)}
    assert first == again
    # pass counts at the sizes the propagation workloads use: whole 128-byte
    # runs in every tile cost L = 24 a seventh pass over the bare minimum
    assert len(first[18]) <= 4 and len(first[24]) == 7
    assert len(ss.tiled_plan(24, 1)) == 7 and ss.tiled_plan(24, 0) == first[24]


def test_plan_arguments_are_checked():
    with pytest.raises(ss.OutOfRangeError):
        ss.tile_plan(31, 12, 3)
    with pytest.raises(ss.InvalidArgumentError):
        ss.tile_plan(20, 14, 3)
    with pytest.raises(ss.InvalidArgumentError):
        ss.tile_plan(20, 1, 0)
    with pytest.raises(ss.InvalidArgumentError):
        ss.tile_plan(20, 12, 9)
