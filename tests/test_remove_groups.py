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
