"""The component split of the one-at-a-time insert path, checked on the CPU
oracle.

When insert rounds stall, the pending ops are split into components by a
carry walk over the free slots (EMPTY or TOMBSTONE) in slot order: a free
slot s with d(s) ops whose first free slot is s passes on
max(0, c + d(s) - 1) of the c ops arriving at it; a free slot with demand
and no arriving carry starts a component, and every op belongs to the last
start at or before its first free slot (round the ring).  The device runs
the components at the same time, each in index order.  This restates the
split in numpy and checks its claim on the oracle: applying the components
one after another in reverse start order gives the same counts and the same
table, slot for slot, as the batch in index order.
"""
import numpy as np
import pytest

from fm_testutil import OracleAdapter


def component_of(flags, homes, cap):
    st = flags & 0xF
    fidx = np.nonzero((st == 0) | (st == 2))[0]
    pos = np.searchsorted(fidx, homes)
    F = fidx[np.where(pos < len(fidx), pos, 0)]  # first free slot at or after home, round the ring
    d = np.zeros(cap, np.int64)
    np.add.at(d, F, 1)
    assert d[fidx].sum() < len(fidx), "no free slot to spare: the device takes the plain order"
    # carry into every free slot; two turns settle the carry round the ring
    c = 0
    cin = np.zeros(len(fidx), np.int64)
    for _ in range(2):
        for i, s in enumerate(fidx):
            cin[i] = c
            c = max(0, c + d[s] - 1)
    demand = d[fidx] > 0
    starts = fidx[demand & (cin == 0)]
    assert len(starts)
    at = np.searchsorted(starts, F, side="right") - 1
    return starts[at]  # -1 wraps to the last start


@pytest.mark.parametrize("case", [(1 << 12, 0.8, 0.18, 0.0), (1 << 13, 0.85, 0.13, 0.0), (1 << 13, 0.9, 0.2, 0.3)])
@pytest.mark.parametrize("seed", [0, 1])
def test_components_commute(case, seed):
    cap, load0, frac, rm = case
    rng = np.random.default_rng(seed)
    a, b = OracleAdapter(cap, 8, 8), OracleAdapter(cap, 8, 8)
    pk = rng.integers(0, 256, (int(cap * load0), 8), dtype=np.uint8)
    for m in (a, b):
        m.bulk_insert(pk, pk)
    if rm:
        r = pk[rng.choice(len(pk), int(len(pk) * rm), replace=False)]
        assert a.bulk_remove(r) == b.bulk_remove(r)
    n = int(cap * frac)
    k = rng.integers(0, 256, (n, 8), dtype=np.uint8)
    k[rng.choice(n, n // 10)] = k[rng.integers(0, n, n // 10)]  # in-batch duplicates
    k[rng.choice(n, n // 10)] = pk[rng.integers(0, len(pk), n // 10)]  # updates
    v = rng.integers(0, 256, (n, 8), dtype=np.uint8)
    homes = (k.view("<u8").reshape(-1) & np.uint64(cap - 1)).astype(np.int64)  # identity hash
    comp = component_of(a.snapshot()[0].astype(np.int64), homes, cap)
    starts = np.unique(comp)
    assert len(starts) > 10  # a real split, not one component
    whole = a.bulk_insert(k, v)
    parts = 0
    for c in starts[::-1]:
        idx = np.nonzero(comp == c)[0]
        parts += b.bulk_insert(k[idx], v[idx])
    assert whole == parts
    for x, y in zip(a.snapshot(), b.snapshot()):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_components_commute_round_the_ring(seed):
    """The same claim when the crowded region runs past the end of the table
    into slot 0 (keys homed in the last 400 slots of a 0.85-load table)."""
    cap = 1 << 12
    rng = np.random.default_rng(100 + seed)
    a, b = OracleAdapter(cap, 8, 8), OracleAdapter(cap, 8, 8)
    pk = rng.integers(0, 256, (int(cap * 0.85), 8), dtype=np.uint8)
    for m in (a, b):
        m.bulk_insert(pk, pk)
    n = 500
    homes = (cap - 400 + rng.integers(0, 400, n)).astype(np.uint64)
    k = ((np.arange(n, dtype=np.uint64) + 1) * np.uint64(cap) + homes).view(np.uint8).reshape(n, 8).copy()
    v = rng.integers(0, 256, (n, 8), dtype=np.uint8)
    comp = component_of(a.snapshot()[0].astype(np.int64), homes.astype(np.int64), cap)
    starts = np.unique(comp)
    whole = a.bulk_insert(k, v)
    parts = 0
    for c in starts[::-1]:
        idx = np.nonzero(comp == c)[0]
        parts += b.bulk_insert(k[idx], v[idx])
    assert whole == parts
    for x, y in zip(a.snapshot(), b.snapshot()):
        assert np.array_equal(x, y)


def direct_groups(flags, homes, cap):
    """The grouping of the direct insert (k_dx_find / k_dx_flow / k_dx_exec /
    k_dx_warp in flash-map_b200/csrc/fm_insert.cu), restated: every op's
    first free slot F; the ops at each F; from every F holding c >= 2 ops a
    flow walk over the following free slots carrying c - 1, each slot taking
    one op and adding its own, which marks every later F it reaches; then an
    op alone at an unmarked F is its own group, and an unmarked F with c >= 2
    leads a group of the ops of every F its flow reaches.  Returns the groups
    (op indices in index order), or None where the device hands the whole call
    to the component path (an op with no free slot, a flow round the ring)."""
    st = flags & 0xF
    fidx = np.nonzero((st == 0) | (st == 2))[0]
    if len(fidx) == 0:
        return None
    pos = np.searchsorted(fidx, homes)
    F = fidx[np.where(pos < len(fidx), pos, 0)]
    ops_at = {}
    for j, f in enumerate(F):
        ops_at.setdefault(int(f), []).append(j)
    nxt = {int(fidx[i]): int(fidx[(i + 1) % len(fidx)]) for i in range(len(fidx))}

    def chain(f0):
        out, f, flow = [f0], f0, len(ops_at[f0]) - 1
        while flow > 0:
            f = nxt[f]
            if f == f0:
                return None  # the carry comes back round the ring
            out.append(f)
            flow += len(ops_at.get(f, [])) - 1
        return out

    marked = set()
    for f, ops in ops_at.items():
        if len(ops) >= 2:
            ch = chain(f)
            if ch is None:
                return None
            marked.update(x for x in ch[1:] if x in ops_at)
    groups = []
    for f, ops in ops_at.items():
        if f in marked:
            continue
        if len(ops) == 1:
            groups.append(np.array(ops))
        else:
            groups.append(np.array(sorted(j for x in chain(f) for j in ops_at.get(x, []))))
    return groups


@pytest.mark.parametrize("case", [(1 << 12, 0.5, 0.1, 0.0), (1 << 12, 0.8, 0.05, 0.0), (1 << 13, 0.85, 0.1, 0.0),
                                  (1 << 13, 0.8, 0.08, 0.3), (1 << 12, 0.9, 0.05, 0.2)])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_direct_groups_commute(case, seed):
    """Every op lands in exactly one group of the direct insert, and running
    the groups one after another in a shuffled order gives the same counts
    and the same table, slot for slot, as the batch in index order."""
    cap, load0, frac, rm = case
    rng = np.random.default_rng(50 + seed)
    a, b = OracleAdapter(cap, 8, 8), OracleAdapter(cap, 8, 8)
    pk = rng.integers(0, 256, (int(cap * load0), 8), dtype=np.uint8)
    for m in (a, b):
        m.bulk_insert(pk, pk)
    if rm:
        r = pk[rng.choice(len(pk), int(len(pk) * rm), replace=False)]
        assert a.bulk_remove(r) == b.bulk_remove(r)
    n = int(cap * frac)
    k = rng.integers(0, 256, (n, 8), dtype=np.uint8)
    k[rng.choice(n, n // 10)] = k[rng.integers(0, n, n // 10)]  # in-batch duplicates
    k[rng.choice(n, n // 10)] = pk[rng.integers(0, len(pk), n // 10)]  # updates
    v = rng.integers(0, 256, (n, 8), dtype=np.uint8)
    homes = (k.view("<u8").reshape(-1) & np.uint64(cap - 1)).astype(np.int64)
    groups = direct_groups(a.snapshot()[0].astype(np.int64), homes, cap)
    assert groups is not None
    allops = np.sort(np.concatenate(groups))
    assert np.array_equal(allops, np.arange(n))
    assert sum(len(g) == 1 for g in groups) > len(groups) // 2  # mostly lone ops
    whole = a.bulk_insert(k, v)
    parts = 0
    for gi in rng.permutation(len(groups)):
        parts += b.bulk_insert(k[groups[gi]], v[groups[gi]])
    assert whole == parts
    for x, y in zip(a.snapshot(), b.snapshot()):
        assert np.array_equal(x, y)


def test_direct_groups_hand_a_ring_flow_to_the_component_path():
    """A batch whose flow would come back round the whole ring: the direct
    insert leaves it to the component path (Ctl::serial[0])."""
    cap = 64
    flags = np.zeros(cap, np.int64)
    flags[:] = 1  # occupied, distance 0
    flags[[5, 40]] = 0  # two free slots
    homes = np.array([3, 4, 3], np.int64)  # three ops at slot 5: a carry of 2, one slot after it
    assert direct_groups(flags, homes, cap) is None
