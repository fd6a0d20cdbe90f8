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


@pytest.mark.parametrize("tile_bits", [8, 12, 13])
def test_plans_cover_every_pair_with_full_tiles(tile_bits):
    for L in range(tile_bits, 31):
        plan = ss.tile_plan(L, tile_bits)
        assert all(bin(m).count("1") == tile_bits for m in plan)
        assert all(m < (1 << L) for m in plan)
        for i, j in itertools.combinations(range(L), 2):
            pair = (1 << i) | (1 << j)
            assert any(m & pair == pair for m in plan), (L, i, j)
        assert low_run(plan[-1]) == max(low_run(m) for m in plan)
        if L == tile_bits:
            assert plan == [(1 << L) - 1]


def test_plans_are_reproducible_and_small():
    first = {L: ss.tile_plan(L, 12) for L in (18, 20, 22, 24)}
    again = {L: ss.tile_plan(L, 12) for L in (18, 20, 22, 24)}
    assert first == again
    # pass counts at the sizes the propagation workloads use (6 passes at
    # L = 22-24 is the lower bound for 12-spin tiles that keep a low bit)
    assert len(first[18]) == 3 and len(first[24]) == 6
    assert len(ss.tile_plan(24, 13)) == 6


def test_plan_arguments_are_checked():
    with pytest.raises(ss.OutOfRangeError):
        ss.tile_plan(31, 12)
    with pytest.raises(ss.InvalidArgumentError):
        ss.tile_plan(20, 14)
    with pytest.raises(ss.InvalidArgumentError):
        ss.tile_plan(20, 1)
