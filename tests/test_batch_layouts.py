"""Host-side checks of the batched kernel's register-blocking schedule.

For every (L, R) schedule the kernel is compiled with, this simulates the
shared-memory addresses each warp instruction touches (own blocks, partner
blocks, partial sums, the recursion buffers) under the padded layout
phys(k) = k + (k >> R), and checks that

  * every coupling (i, j) and every field is applied exactly once, by the
    layout the kernel assigns it to;
  * the padded index of a thread's amplitude slot x is its base plus a
    constant of x (what lets the kernel use immediate offsets);
  * no access pattern has a bank conflict: for 8-byte elements each
    half-warp touches 16 distinct 8-byte bank slots, for 16-byte elements
    each quarter-warp touches 8 distinct 16-byte slots.  The one-warp
    schedules of L <= 8 are allowed 2-way conflicts (their whole state is
    256 amplitudes or fewer).
"""
import itertools

import pytest

MIXED = [(6, 1), (7, 2), (8, 3), (9, 4), (10, 4), (11, 4), (12, 4), (13, 4)]
FP64 = [(6, 1), (7, 2), (8, 3), (9, 3), (10, 3), (11, 3), (12, 3)]


def base(L, R, g):
    return g * R if (g + 1) * R <= L else L - R


def layouts(L, R):
    return (L + R - 1) // R


def holds(L, R, g, s):
    b = base(L, R, g)
    return b <= s < b + R


def first_layout(L, R, s):
    return next(g for g in range(layouts(L, R)) if holds(L, R, g, s))


def pair_layout(L, R, i, j):
    for g in range(layouts(L, R)):
        if holds(L, R, g, i) and holds(L, R, g, j):
            return g
    return first_layout(L, R, i)


def cross_mine(L, R, g, p):
    G = layouts(L, R)
    b = base(L, R, g)
    return first_layout(L, R, b + p) == g and not (g < G - 1 and b + p >= L - R)


def kbase(L, R, g, t):
    b = base(L, R, g)
    return ((t >> b) << (b + R)) | (t & ((1 << b) - 1))


def phys(k, R):
    return k + (k >> R)


@pytest.mark.parametrize("L,R", sorted(set(MIXED + FP64)))
def test_every_term_is_applied_once(L, R):
    G = layouts(L, R)
    applied = {}
    for g in range(G):
        b = base(L, R, g)
        for p in range(R):
            for q in range(p + 1, R):
                if pair_layout(L, R, b + p, b + q) == g:
                    applied[(b + p, b + q)] = applied.get((b + p, b + q), 0) + 1
            if cross_mine(L, R, g, p):
                for j in range(b + R, L):
                    applied[(b + p, j)] = applied.get((b + p, j), 0) + 1
    want = {(i, j): 1 for i in range(L) for j in range(i + 1, L)}
    assert applied == want
    fields = [first_layout(L, R, s) for s in range(L)]
    assert all(f is not None for f in fields)


@pytest.mark.parametrize("L,R", sorted(set(MIXED + FP64)))
def test_padded_index_is_additive_in_the_slot(L, R):
    NT = 1 << (L - R)
    for g in range(layouts(L, R)):
        b = base(L, R, g)
        for t in range(NT):
            kb = kbase(L, R, g, t)
            for x in range(1 << R):
                y = x << b
                assert phys(kb | y, R) == phys(kb, R) + phys(y, R)
                for j in range(b + R, L):
                    assert phys((kb ^ (1 << j)) | y, R) == phys(kb ^ (1 << j), R) + phys(y, R)


def conflicts(addresses, elem_bytes):
    """Largest number of distinct addresses sharing a bank slot within one
    wavefront group (16 lanes for 8-byte, 8 lanes for 16-byte elements)."""
    group = 16 if elem_bytes == 8 else 8
    slots = 16 if elem_bytes == 8 else 8
    worst = 1
    for g0 in range(0, len(addresses), group):
        by_slot = {}
        for a in addresses[g0:g0 + group]:
            by_slot.setdefault(a % slots, set()).add(a)
        worst = max(worst, max(len(v) for v in by_slot.values()))
    return worst


@pytest.mark.parametrize("L,R,elem", [(L, R, 8) for L, R in MIXED] + [(L, R, 16) for L, R in FP64])
def test_shared_accesses_are_conflict_free(L, R, elem):
    NT = 1 << (L - R)
    for g in range(layouts(L, R)):
        b = base(L, R, g)
        for w0 in range(0, NT, 32):
            lanes = range(w0, min(w0 + 32, NT))
            for x in range(1 << R):
                allowed = 1 if L >= 9 else 2
                own = [phys(kbase(L, R, g, t) | (x << b), R) for t in lanes]
                assert conflicts(own, elem) <= allowed, (g, x)
                for j in range(b + R, L):
                    part = [phys((kbase(L, R, g, t) ^ (1 << j)) | (x << b), R) for t in lanes]
                    assert conflicts(part, elem) <= allowed, (g, x, j)
