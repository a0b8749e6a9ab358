"""The grouping of the direct remove (k_rx_find / k_rx_exec in
flash-map_b200/csrc/fm_remove.cu), checked on the CPU oracle.

A remove's probe reads only [home, E], E the first EMPTY slot at or after its
home, and writes at most one slot there; removes make no EMPTY slot.  So ops
with different E touch disjoint slots, and the device runs the groups of
equal E at the same time, each in index order.  The claim checked here:
applying the groups one after another in a shuffled order gives the same
counts and the same table, slot for slot, as the batch in index order --
with tombstones from earlier removes, in-batch duplicate keys, absent keys
and runs that go past the end of the table into slot 0."""
import numpy as np
import pytest

from fm_testutil import OracleAdapter


def remove_groups(flags, homes):
    st = flags & 0xF
    eidx = np.nonzero(st == 0)[0]
    if len(eidx) == 0:
        return None  # the device leaves such a call to the rounds
    pos = np.searchsorted(eidx, homes)
    E = eidx[np.where(pos < len(eidx), pos, 0)]
    groups = {}
    for j, e in enumerate(E):
        groups.setdefault(int(e), []).append(j)
    return [np.array(g) for g in groups.values()]


@pytest.mark.parametrize("load", [0.5, 0.8, 0.9, 0.97])
@pytest.mark.parametrize("seed", [0, 1])
def test_remove_groups_commute(load, seed):
    cap = 1 << 12
    rng = np.random.default_rng(70 + seed)
    a, b = OracleAdapter(cap, 8, 8), OracleAdapter(cap, 8, 8)
    pk = rng.integers(0, 256, (int(cap * load), 8), dtype=np.uint8)
    for m in (a, b):
        m.bulk_insert(pk, pk)
        m.bulk_remove(pk[: len(pk) // 10])  # earlier tombstones
    n = cap // 4
    k = np.concatenate([pk[rng.integers(0, len(pk), n - n // 4)], rng.integers(0, 256, (n // 4, 8), dtype=np.uint8)])
    k[rng.choice(n, n // 10)] = k[rng.integers(0, n, n // 10)]  # in-batch duplicates: the first removes
    k = k[rng.permutation(n)]
    homes = (k.view("<u8").reshape(-1) & np.uint64(cap - 1)).astype(np.int64)
    groups = remove_groups(a.snapshot()[0].astype(np.int64), homes)
    assert groups is not None and len(groups) > 10
    assert np.array_equal(np.sort(np.concatenate(groups)), np.arange(n))
    whole = a.bulk_remove(k)
    parts = sum(b.bulk_remove(k[groups[gi]]) for gi in rng.permutation(len(groups)))
    assert whole == parts
    for x, y in zip(a.snapshot(), b.snapshot()):
        assert np.array_equal(x, y)


def test_remove_groups_round_the_end_of_the_table():
    cap = 1 << 10
    rng = np.random.default_rng(5)
    a, b = OracleAdapter(cap, 8, 8), OracleAdapter(cap, 8, 8)
    homes = (cap - 60 + rng.integers(0, 60, 300)).astype(np.uint64)
    pk = ((np.arange(300, dtype=np.uint64) + 1) * np.uint64(cap) + homes).view(np.uint8).reshape(300, 8).copy()
    for m in (a, b):
        m.bulk_insert(pk, pk)
    k = pk[rng.permutation(300)[:200]]
    groups = remove_groups(a.snapshot()[0].astype(np.int64),
                           (k.view("<u8").reshape(-1) & np.uint64(cap - 1)).astype(np.int64))
    whole = a.bulk_remove(k)
    parts = sum(b.bulk_remove(k[g]) for g in groups[::-1])
    assert whole == parts
    for x, y in zip(a.snapshot(), b.snapshot()):
        assert np.array_equal(x, y)


def _look(flags, keys, cap, key, h):
    """The probe of one remove (rayon_cpu.rs:273-328) on raw arrays: (target
    slot or None, stop slot)."""
    mask = cap - 1
    for p in range(cap):
        s = (h + p) & mask
        f = int(flags[s])
        st, d = f & 0xF, f >> 4
        if st == 0 or (st == 1 and p > d):
            return None, s
        if st == 1 and d == p and bytes(keys[s]) == key:
            return s, s
    return None, None


def group_commit(flags, keys, cap, ops, E, chunk=32):
    """rx_group of flash-map_b200/csrc/fm_probe.cuh restated: the group's ops
    (key, home) in index order, chunk by chunk: probe all on the table as it
    is, then commit in order; an op whose [home, stop] holds a slot an earlier
    op of its chunk tombstoned probes again.  Returns the count removed."""
    mask = cap - 1
    removed = 0
    for c0 in range(0, len(ops), chunk):
        part = ops[c0:c0 + chunk]
        pre = [_look(flags, keys, cap, k, h) for k, h in part]
        done = []  # distances before E of this chunk's tombstones
        for (k, h), (tgt, stop) in zip(part, pre):
            dh, ds = (E - h) & mask, ((E - stop) & mask) if stop is not None else 0
            if any(ds <= dt <= dh for dt in done):
                tgt, _ = _look(flags, keys, cap, k, h)
            if tgt is not None:
                flags[tgt] = 2
                done.append((E - tgt) & mask)
                removed += 1
    return removed


@pytest.mark.parametrize("load", [0.7, 0.85, 0.95])
@pytest.mark.parametrize("chunk", [4, 32])
def test_group_commit_equals_sequential(load, chunk):
    """Duplicates, absent keys and removes of one another's exits inside
    groups: the commit rule gives the sequential result slot for slot."""
    cap = 1 << 10
    rng = np.random.default_rng(int(load * 100) + chunk)
    a, b = OracleAdapter(cap, 8, 8), OracleAdapter(cap, 8, 8)
    pk = rng.integers(0, 256, (int(cap * load), 8), dtype=np.uint8)
    for m in (a, b):
        m.bulk_insert(pk, pk)
        m.bulk_remove(pk[::9])
    n = cap // 3
    k = np.concatenate([pk[rng.integers(0, len(pk), n - n // 5)], rng.integers(0, 256, (n // 5, 8), dtype=np.uint8)])
    k[rng.choice(n, n // 8)] = k[rng.integers(0, n, n // 8)]
    homes = (k.view("<u8").reshape(-1) & np.uint64(cap - 1)).astype(np.int64)
    flags = b.m.flags()  # the oracle's own arrays, written in place
    keys = b.m.keys()
    st = flags & 0xF
    eidx = np.nonzero(st == 0)[0]
    pos = np.searchsorted(eidx, homes)
    E = eidx[np.where(pos < len(eidx), pos, 0)]
    whole = a.bulk_remove(k)
    parts = 0
    for e in np.unique(E):
        idx = np.nonzero(E == e)[0]  # index order
        parts += group_commit(flags, keys, cap, [(bytes(k[j]), int(homes[j])) for j in idx], int(e), chunk)
    b.m.set_len(len(b.m) - parts)
    assert whole == parts
    for x, y in zip(a.snapshot(), b.snapshot()):
        assert np.array_equal(x, y)
