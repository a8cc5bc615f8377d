"""Level order of the Trotter rotations, on the CPU.

The engine stores the coupling pairs in level order: rotation k gets level
1 + the highest level of the earlier rotations sharing one of its sites
(rotation_levels in csrc/absrun.cpp), and the GPU kernels apply the
rotations level by level, a level (split into chunks of at most 32) in
parallel.  That is only exact if every site sees the same float operations
as in the lexicographic order of propagate.c:876-888.  These tests apply
the reference's float32 rotation both ways on lattice and chain patterns and
require bitwise equality.
"""
import numpy as np

from nise_2017_b200 import synth


def lattice_pairs(n, seed):
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        files = synth.write(synth.c1_spec(n_sites=n, frames=2, seed=seed), td)
        rec = np.fromfile(files["coupling"], dtype=np.float32)[1:]
    pairs = []
    for a in range(n):
        for b in range(a + 1, n):
            if abs(rec[b + a * (2 * n - a - 1) // 2]) >= 2.0:
                pairs.append((a, b))
    return pairs


def levels(pairs, n):
    last = [0] * n
    lv = []
    for a, b in pairs:
        l = max(last[a], last[b]) + 1
        last[a] = last[b] = l
        lv.append(l - 1)
    return lv


def rotate(cr, ci, pairs, cs, order, flip=None):
    """propagate.c:876-888 in float32, rotations taken in `order` (flip[q]:
    rotation order[q] with its sites swapped)."""
    cr, ci = cr.copy(), ci.copy()
    for q, k in enumerate(order):
        a, b = pairs[k]
        if flip is not None and flip[q]:
            a, b = b, a
        co, si = cs[k]
        ra, ia, rb, ib = cr[a], ci[a], cr[b], ci[b]
        cr[a] = co * ra - si * ib
        ci[a] = co * ia + si * rb
        cr[b] = co * rb - si * ia
        ci[b] = co * ib + si * ra
    return cr, ci


def bank_cost(pairs, n, perm, flip, chk):
    """Conflicting shared-memory wavefronts of the warp kernels' site loads:
    lane l of a chunk loads its rotation's first and second site (idle lanes
    the spare n + ((start + l - K) & 31)); 8-byte sites in half-warps (site mod
    16), 16-byte sites in quarter-warps (site mod 8)."""
    K, tot = len(pairs), 0
    for c0, c1 in zip(chk[:-1], chk[1:]):
        sa, sb = [], []
        for l in range(32):
            if c0 + l < c1:
                a, b = pairs[perm[c0 + l]]
                if flip[c0 + l]:
                    a, b = b, a
            else:
                a = b = n + ((c0 + l - K) & 31)
            sa.append(a)
            sb.append(b)
        for w in (16, 8):
            for l0 in range(0, 32, w):
                for s in (sa, sb):
                    tot += max(np.bincount([x % w for x in s[l0:l0 + w]]))
    return tot


def engine_matches(pairs, n, lv, cr, ci, cs, r0):
    """The engine's schedule (nise_rotation_schedule, the code the kernels'
    tables come from): the levels of levels(), split into chunks of at most
    32; within a chunk the rotations of that chunk in the engine's bank order,
    some with their sites swapped.  Applied as the engine applies it, the
    schedule gives the lexicographic float32 result bitwise, and its bank
    order has no more conflicting wavefronts than the plain level order."""
    import nise_2017_b200 as nise
    perm, lvptr, chk, flip = nise.rotation_schedule(pairs, n)
    expect = sorted(range(len(pairs)), key=lambda k: (lv[k], k))
    widths = np.bincount(lv, minlength=1) if len(lv) else np.zeros(0, int)
    assert list(np.diff(lvptr)) == list(widths)
    bounds = [0] + [min(q + 32, e) for s, e in zip(lvptr[:-1], lvptr[1:]) for q in range(s, e, 32)]
    assert list(chk) == bounds
    for c0, c1 in zip(chk[:-1], chk[1:]):
        assert sorted(perm[c0:c1]) == expect[c0:c1]
    r = rotate(cr, ci, pairs, cs, perm, flip)
    assert np.array_equal(r0[0], r[0]) and np.array_equal(r0[1], r[1])
    plain = bank_cost(pairs, n, expect, np.zeros(len(pairs), int), chk)
    ours = bank_cost(pairs, n, perm, flip, chk)
    assert ours <= plain
    return plain, ours


def check(pairs, n, seed):
    rng = np.random.default_rng(seed)
    cr = rng.normal(size=n).astype(np.float32)
    ci = rng.normal(size=n).astype(np.float32)
    ang = rng.uniform(-0.3, 0.3, size=len(pairs)).astype(np.float32)
    cs = [(np.float32(np.cos(x)), np.float32(-np.sin(x))) for x in ang]
    lv = levels(pairs, n)
    by_level = sorted(range(len(pairs)), key=lambda k: (lv[k], k))
    # every level touches disjoint sites
    for l in set(lv):
        sites = [s for k in range(len(pairs)) if lv[k] == l for s in pairs[k]]
        assert len(sites) == len(set(sites))
    r0 = rotate(cr, ci, pairs, cs, range(len(pairs)))
    r1 = rotate(cr, ci, pairs, cs, by_level)
    assert np.array_equal(r0[0], r1[0]) and np.array_equal(r0[1], r1[1])
    # within a level any order (any lane assignment) gives the same bits
    shuffled = sorted(range(len(pairs)), key=lambda k: (lv[k], rng.random()))
    r2 = rotate(cr, ci, pairs, cs, shuffled)
    assert np.array_equal(r0[0], r2[0]) and np.array_equal(r0[1], r2[1])
    # and with either site of a rotation first
    flips = rng.integers(0, 2, len(pairs))
    r3 = rotate(cr, ci, pairs, cs, shuffled, flips)
    assert np.array_equal(r0[0], r3[0]) and np.array_equal(r0[1], r3[1])
    engine_matches(pairs, n, lv, cr, ci, cs, r0)
    return lv


def test_lattice_level_order_is_bitwise_lexicographic():
    n = 120
    pairs = lattice_pairs(n, seed=7)
    lv = check(pairs, n, seed=1)
    widths = np.bincount(lv)
    assert len(pairs) > 4 * len(widths)  # wide levels: the warp-per-vector case
    assert widths.max() <= 32


def test_chain_level_order_is_bitwise_lexicographic():
    n = 40
    pairs = [(a, a + 1) for a in range(n - 1)]
    lv = check(pairs, n, seed=2)
    assert len(set(lv)) == n - 1  # a chain: one rotation per level


def test_dimer_levels_wider_than_a_warp():
    """Levels of 40, 80 and 40 rotations, split into chunks of at most 32."""
    n = 160
    pairs = sorted([(2 * i, 2 * i + 1) for i in range(n // 2)] + [(i, i + n // 2) for i in range(n // 2)])
    lv = check(pairs, n, seed=3)
    widths = np.bincount(lv)
    assert list(widths) == [40, 80, 40]
    chunks = [min(32, w - q) for w in widths for q in range(0, w, 32)]
    assert chunks == [32, 8, 32, 32, 16, 32, 8]
    _, _, chk, _ = __import__("nise_2017_b200").rotation_schedule(pairs, n)
    assert list(np.diff(chk)) == chunks


def test_engine_schedule_rejects_bad_pairs():
    import pytest
    import nise_2017_b200 as nise
    with pytest.raises(nise.NiseError):
        nise.rotation_schedule([(0, 5)], 4)
    perm, lv, chk, flip = nise.rotation_schedule([], 4)
    assert len(perm) == 0 and list(lv) == [0] and list(chk) == [0] and len(flip) == 0


def test_bank_order_on_the_1024_site_lattice():
    """On the 1024-site benchmark lattice the engine's bank order cuts the
    conflicting wavefronts of the rotation loads by more than 10 %."""
    import nise_2017_b200 as nise
    n = 1024
    pairs = lattice_pairs(n, seed=20171)
    lv = levels(pairs, n)
    perm, lvptr, chk, flip = nise.rotation_schedule(pairs, n)
    expect = sorted(range(len(pairs)), key=lambda k: (lv[k], k))
    plain = bank_cost(pairs, n, expect, np.zeros(len(pairs), int), chk)
    ours = bank_cost(pairs, n, perm, flip, chk)
    print("rotation-load wavefronts per Trotter sub-step: level order %d, bank order %d" % (plain, ours))
    assert ours < 0.9 * plain
