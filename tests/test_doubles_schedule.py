"""The synchronisation schedule of the two-warp doubles kernel
(k2d_doubles_duo, csrc/twodir.cu), checked on the CPU.

One Trotter sub-step of the doubles (propagate.c:956-1045) applies, for every
coupling (a, b) in lexicographic order, the rotation (|aa>,|ab>) at the
sqrt(2) angle and the rotations (|ac>,|bc>) for every c != a.  The kernel
shares a doubles vector between two warps, thread c owning column c
(warp c >> 5), and keeps row a (|ac>) in registers while a is unchanged.  It
runs the couplings in segments of one first site a and one owner warp
(b >> 5): a named barrier of the two warps starts each segment (with the
pivot row stored back and reloaded when a changes); the owner warp
synchronises per coupling (__syncwarp); the other warp does not synchronise
inside a segment.

This enumerates every shared-memory access of the schedule and checks that
every two accesses of one element by different threads, one of them a write,
are ordered: a barrier between them, or both in the owner warp in different
couplings.  Broken variants of the schedule must be caught."""
import random

import pytest


def segments(pairs):
    """(a, first, end, owner warp), as the host builds them (singles.cpp)."""
    segs, k = [], 0
    while k < len(pairs):
        a, w, k0 = pairs[k][0], pairs[k][1] >> 5, k
        while k < len(pairs) and pairs[k][0] == a and (pairs[k][1] >> 5) == w:
            k += 1
        segs.append((a, k0, k, w))
    return segs


def unordered_conflicts(n, pairs, es=False, owner_syncs=True, segment_barrier=True):
    """Number of conflicting access pairs the schedule leaves unordered."""
    def el(x, y):
        return (x, y) if x < y else (y, x)

    bad = 0
    open_acc = {}  # element -> accesses of the current barrier epoch: (coupling, thread, write, synced)
    epoch = 0

    def access(elem, k, t, write, synced):
        nonlocal bad
        lst = open_acc.setdefault(elem, [epoch, []])
        if lst[0] != epoch:
            lst[0], lst[1] = epoch, []
        for (k2, t2, w2, s2) in lst[1]:
            if t2 == t or not (write or w2):
                continue
            if (t2 >> 5) != (t >> 5) or k2 == k or not (synced and s2):
                bad += 1
        lst[1].append((k, t, write, synced))

    cur_a = -1
    for (a, k0, k1, w) in segments(pairs):
        if a != cur_a:
            if cur_a >= 0:
                for c in range(n):
                    if c != cur_a:
                        access(el(cur_a, c), k0 - 0.5, c, True, False)
            epoch += 1
            for c in range(n):
                if c != a:
                    access(el(a, c), k0 - 0.25, c, False, False)
            cur_a = a
        elif segment_barrier:
            epoch += 1
        for k in range(k0, k1):
            b = pairs[k][1]
            if not es:
                access(el(a, a), k, b, False, owner_syncs)
                access(el(a, a), k, b, True, owner_syncs)
            for c in range(n):
                if c == a or (es and c == b):
                    continue
                synced = owner_syncs and (c >> 5) == w
                access(el(b, c), k, c, False, synced)
                access(el(b, c), k, c, True, synced)
    return bad


def lexicographic(n, keep=1.0, seed=0):
    rng = random.Random(seed)
    return [(a, b) for a in range(n) for b in range(a + 1, n) if keep >= 1.0 or rng.random() < keep]


@pytest.mark.parametrize("n", [33, 40, 48, 64])
@pytest.mark.parametrize("es", [False, True])
def test_schedule_orders_every_conflict(n, es):
    assert unordered_conflicts(n, lexicographic(n), es) == 0
    for seed in range(2):
        assert unordered_conflicts(n, lexicographic(n, 0.3, seed), es) == 0


def test_broken_schedules_are_caught():
    pairs = lexicographic(64)
    assert unordered_conflicts(64, pairs, owner_syncs=False) > 0
    assert unordered_conflicts(64, pairs, segment_barrier=False) > 0
