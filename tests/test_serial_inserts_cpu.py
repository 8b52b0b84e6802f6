"""The oracle's serial inserts (oracle/kgoracle.cpp kgo_serial_inserts), the
reference point of the GPU merge test, against a direct Python
restatement of the reference's rules on small pools:

* Nhood::parallel_try_insert (kgraph.cpp:723-736): an offer beyond the stored
  radius returns pool.size() untouched; else the sorted insert, then L grows
  while L + 1 < pool.size(), and once it cannot, the radius becomes the
  distance of entry L - 1.
* UpdateKnnListHelper (kgraph.cpp:176-202): the insert position is after every
  entry of distance <= d; an entry with the same id inside the run of equal
  distances just before that position makes it a duplicate (return L + 1,
  nothing moves); otherwise entries [i, L) shift up by one (entry L is
  overwritten) and the offer lands at i, flagged new.

Every output is compared exactly: pool distances and ids with flag bits, L,
the radius bits and each offer's return value (the value the `found` rule
reads, kgraph.cpp:808-810).
"""
import numpy as np
import pytest

from oracle import kgoracle as ko

FLAG = 0x80000000
ID_MASK = 0x7FFFFFFF
UNSET_ID = 0x7FFFFFFF
FMAX = float(np.finfo(np.float32).max)


def restated(pool_d, pool_i, L, radius, cand, dist):
    """Serial parallel_try_insert calls on one pool, as plain Python lists."""
    d = [float(x) for x in pool_d]
    ids = [int(x) for x in pool_i]
    L, radius = int(L), float(radius)
    size = len(d)
    rets = []
    for c, x in zip(cand, dist):
        c, x = int(c), float(x)
        if x > radius:
            rets.append(size)
            continue
        i = L
        while i > 0 and not (d[i - 1] <= x):
            i -= 1
        dup = False
        k = i
        while k > 0 and not (d[k - 1] < x):
            if ids[k - 1] & ID_MASK == c:
                dup = True
                break
            k -= 1
        if dup:
            rets.append(L + 1)
            continue
        for j in range(L, i, -1):
            d[j], ids[j] = d[j - 1], ids[j - 1]
        d[i], ids[i] = x, c | FLAG
        if L + 1 < size:
            L += 1
        else:
            radius = d[L - 1]
        rets.append(i)
    return (np.array(d, np.float32), np.array(ids, np.uint32), L, np.float32(radius),
            np.array(rets, np.uint32))


def pool_case(rng, Lp, table):
    """A pool in a state the build can reach: a sorted prefix of L distinct ids
    at their distances in `table` (flags mixed), unset slots beyond it, and
    when the list is full either the radius an insert set or still FLT_MAX,
    with or without an evicted entry in the overflow slot."""
    ids, dmax = len(table), int(table.max()) + 1
    L = int(rng.integers(0, Lp))
    pool_d = np.full(Lp, FMAX, np.float32)
    pool_i = np.full(Lp, UNSET_ID, np.uint32)
    members = rng.choice(ids, L, replace=False)
    order = np.argsort(table[members], kind="stable")
    pool_d[:L] = table[members][order]
    pool_i[:L] = members[order].astype(np.uint32) | np.where(rng.random(L) < 0.5, FLAG, 0).astype(np.uint32)
    radius = np.float32(FMAX)
    if L == Lp - 1 and L > 0:
        if rng.random() < 0.5:
            radius = pool_d[L - 1]
        if rng.random() < 0.5:
            pool_d[L] = max(pool_d[L - 1], np.float32(rng.integers(0, dmax)))
            pool_i[L] = int(rng.integers(0, ids))
    return pool_d, pool_i, L, radius


@pytest.mark.parametrize("seed,Lp,dmax,ids,n_off", [(1, 9, 6, 40, 30), (2, 17, 20, 100, 60), (3, 5, 3, 12, 25),
                                                    (4, 41, 1000, 5000, 120), (5, 2, 4, 8, 10)])
def test_oracle_serial_inserts_follow_the_reference_rules(seed, Lp, dmax, ids, n_off):
    rng = np.random.default_rng(seed)
    for _ in range(60):
        # the build offers a pair at one distance every time: most offers take their id's
        # distance from a table (repeats of a listed or an earlier offer are duplicates while
        # that entry stays in the list); a fifth take another distance (not duplicates)
        table = rng.integers(0, dmax, ids).astype(np.float32)
        pool_d, pool_i, L, radius = pool_case(rng, Lp, table)
        m = int(rng.integers(0, n_off + 1))
        cand = rng.integers(0, ids, m).astype(np.uint32)
        listed = pool_i[:L] & ID_MASK
        rep = rng.random(m) < 0.3
        if L and rep.any():
            cand[rep] = rng.choice(listed, int(rep.sum()))
        dist = table[cand]
        other = rng.random(m) < 0.2
        dist[other] = rng.integers(0, dmax, int(other.sum())).astype(np.float32)
        got = ko.serial_inserts(pool_d, pool_i, L, radius, cand, dist)
        want = restated(pool_d, pool_i, L, radius, cand, dist)
        for name, g, w in zip(("pool distances", "pool ids", "L", "radius", "returns"), got, want):
            assert np.array_equal(norm(name, g), norm(name, w)), (name, seed, L, m)


def norm(name, x):
    """Distances and the radius as float32 bit patterns, the rest as integers."""
    if name in ("pool distances", "radius"):
        return np.atleast_1d(np.asarray(x, np.float32)).view(np.uint32)
    return np.atleast_1d(np.asarray(x)).astype(np.int64)
