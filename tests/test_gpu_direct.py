"""The direct insert (no rounds: lone ops at once, components per warp) and
its hand-offs, through the C ABI against the sequential oracle, bit for bit:
counts, len, gets and the whole table.

Cases: lone ops on the thread path and the warp path; components of a few
ops; a component larger than a warp gathers (its ops go to the component
path); a full table met by the direct path (the whole call goes to the
component path); flows running past the end of the table into slot 0;
tables too small for the thread path (fewer than 8 slots) or the tile walk
(fewer than 128)."""
import numpy as np
import pytest

from fm_testutil import OracleAdapter, gpu_map

pytestmark = pytest.mark.gpu

SHAPES = [(8, 8), (32, 128), (32, 64), (32, 32), (8, 32)]


def _same(g, o):
    assert g.len() == o.len()
    for x, y in zip(g.snapshot(), o.snapshot()):
        assert np.array_equal(x, y)


def _u64(x, ks):
    a = np.asarray(x, np.uint64).view(np.uint8).reshape(-1, 8)
    if ks == 8:
        return np.ascontiguousarray(a)
    out = np.zeros((len(a), ks), np.uint8)
    out[:, :8] = a
    return out


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("load", [0.3, 0.7, 0.85])
def test_direct_fill_with_updates_and_duplicates(shape, load):
    ks, vs = shape
    cap = 1 << 15
    rng = np.random.default_rng(int(load * 100) + ks + vs)
    g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
    n0 = int(cap * load)
    k0 = rng.integers(0, 256, (n0, ks), dtype=np.uint8)
    v0 = rng.integers(0, 256, (n0, vs), dtype=np.uint8)
    for b in range(0, n0, 3000):  # calls of 3000 up to the load
        assert g.bulk_insert(k0[b:b + 3000], v0[b:b + 3000]) == o.bulk_insert(k0[b:b + 3000], v0[b:b + 3000])
    _same(g, o)
    n = 2000
    k = rng.integers(0, 256, (n, ks), dtype=np.uint8)
    k[rng.choice(n, 200)] = k[rng.integers(0, n, 200)]  # in-batch duplicates: later wins
    k[rng.choice(n, 300)] = k0[rng.integers(0, n0, 300)]  # updates of stored keys
    v = rng.integers(0, 256, (n, vs), dtype=np.uint8)
    assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
    _same(g, o)
    gv, gf = g.bulk_get(np.concatenate([k, k0]))
    ov, of = o.bulk_get(np.concatenate([k, k0]))
    assert np.array_equal(gf, of) and np.array_equal(gv, ov)


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
def test_direct_after_removes_reuses_tombstones(shape):
    ks, vs = shape
    cap = 1 << 14
    rng = np.random.default_rng(9)
    g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
    for r in range(6):
        k = rng.integers(0, 256, (2500, ks), dtype=np.uint8)
        v = rng.integers(0, 256, (2500, vs), dtype=np.uint8)
        assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
        rm = k[rng.choice(2500, 1200, replace=False)]
        assert g.bulk_remove(rm) == o.bulk_remove(rm)
        _same(g, o)


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
@pytest.mark.parametrize("nkeys", [70, 200, 1000])
def test_direct_component_larger_than_a_warp_gathers(shape, nkeys):
    """nkeys ops homed on the same few slots of a half-full table: one
    component of more than 64 ops (handed to the component path) beside lone
    ops elsewhere."""
    ks, vs = shape
    cap = 1 << 14
    rng = np.random.default_rng(nkeys)
    g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
    k0 = rng.integers(0, 256, (cap // 2, ks), dtype=np.uint8)
    v0 = rng.integers(0, 256, (cap // 2, vs), dtype=np.uint8)
    assert g.bulk_insert(k0, v0) == o.bulk_insert(k0, v0)
    homes = 5000 + rng.integers(0, 4, nkeys).astype(np.uint64)
    crowd = _u64((np.arange(nkeys, dtype=np.uint64) + 1) * np.uint64(cap) + homes, ks)
    lone = rng.integers(0, 256, (3000, ks), dtype=np.uint8)
    k = np.concatenate([lone[:1500], crowd, lone[1500:]])
    v = rng.integers(0, 256, (len(k), vs), dtype=np.uint8)
    assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
    _same(g, o)


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
def test_direct_flow_round_the_end_of_the_table(shape):
    ks, vs = shape
    cap = 1 << 12
    rng = np.random.default_rng(31)
    g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
    k0 = rng.integers(0, 256, (int(cap * 0.8), ks), dtype=np.uint8)
    v0 = rng.integers(0, 256, (len(k0), vs), dtype=np.uint8)
    assert g.bulk_insert(k0, v0) == o.bulk_insert(k0, v0)
    n = 300
    homes = (cap - 200 + rng.integers(0, 200, n)).astype(np.uint64)
    k = _u64((np.arange(n, dtype=np.uint64) + 1) * np.uint64(cap) + homes, ks)
    v = rng.integers(0, 256, (n, vs), dtype=np.uint8)
    assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
    _same(g, o)


def _full_but_counted_low(g, o, ks, vs, cap, free, rng):
    """g and o hold the same table with `free` free slots; g's len is loaded
    as 0, so its next calls take the direct path (chosen by the counted load)
    although the table is all but full."""
    k = rng.integers(0, 256, (cap, ks), dtype=np.uint8)
    v = rng.integers(0, 256, (cap, vs), dtype=np.uint8)
    assert g.bulk_insert(k, v) == o.bulk_insert(k, v) == cap
    if free:
        rm = k[rng.choice(cap, free, replace=False)]
        assert g.bulk_remove(rm) == o.bulk_remove(rm) == free
    f, kk, vv = g.snapshot()
    g.load(f, kk, vv, 0)
    return k


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
@pytest.mark.parametrize("free", [0, 2])
def test_direct_call_hands_a_full_table_to_the_component_path(shape, free):
    """No free slot (free = 0: the find pass sees an op with none) or fewer
    free slots than new keys (free = 2: a flow comes back round the ring):
    the direct insert runs nothing and the component path takes the whole
    call, stopping each walk that finds no free slot at the 2*capacity+2 step
    limit and dropping its carried entry, like the oracle."""
    import torch

    import flash_map as F
    import oracle as O

    ks, vs = shape
    cap = 256
    rng = np.random.default_rng(4 + free)
    g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
    k = _full_but_counted_low(g, o, ks, vs, cap, free, rng)
    k2 = np.concatenate([k[:10], rng.integers(0, 256, (20, ks), dtype=np.uint8)])
    v2 = rng.integers(0, 256, (30, vs), dtype=np.uint8)
    with pytest.raises(O.ProbeLimit):
        o.bulk_insert_uncounted(k2, v2)
    dk, dv = torch.from_numpy(k2.copy()).cuda(), torch.from_numpy(v2.copy()).cuda()
    with pytest.raises(F.KernelLaunch, match="2\\*capacity"):
        g.bulk_insert_device_uncounted(dk, dv, len(k2))
    for x, y in zip(g.snapshot(), o.snapshot()):
        assert np.array_equal(x, y)
    assert g.recount() == o.recount() == cap


@pytest.mark.parametrize("cap", [2, 4, 8, 16, 64, 128, 256])
@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
def test_direct_small_tables(cap, shape):
    ks, vs = shape
    rng = np.random.default_rng(cap)
    g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
    for r in range(4):
        n = max(1, cap // 3)
        k = rng.integers(0, 256, (n, ks), dtype=np.uint8)
        if r % 2:
            k[: n // 2] = k[n - n // 2:][: n // 2]  # duplicates
        v = rng.integers(0, 256, (n, vs), dtype=np.uint8)
        if g.len() + n > cap:
            break
        assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
        _same(g, o)
        rm = k[: n // 3]
        assert g.bulk_remove(rm) == o.bulk_remove(rm)
        _same(g, o)


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
@pytest.mark.parametrize("ngroup", [300, 3000, 9000])
def test_direct_remove_group_sizes(shape, ngroup):
    """A remove whose ops share one run between EMPTY slots in groups too
    large for a warp: 300 and 3,000 ops (the block pass) and 9,000 ops (the
    rounds), with repeats of the same keys and absent keys among them, beside
    lone removes and small groups elsewhere."""
    ks, vs = shape
    cap = 1 << 15
    rng = np.random.default_rng(ngroup + ks)
    g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
    nclu = min(ngroup + ngroup // 4, 12000)
    homes = 2000 + (np.arange(nclu, dtype=np.uint64) % np.uint64(200))
    clu = _u64((np.arange(nclu, dtype=np.uint64) + 1) * np.uint64(cap) + homes, ks)
    k0 = np.concatenate([clu, rng.integers(0, 256, (cap // 3, ks), dtype=np.uint8)])
    v0 = rng.integers(0, 256, (len(k0), vs), dtype=np.uint8)
    assert g.bulk_insert(k0, v0) == o.bulk_insert(k0, v0)
    absent = _u64((np.arange(ngroup // 10, dtype=np.uint64) + 20000) * np.uint64(cap) + np.uint64(2050), ks)
    grp = np.concatenate([clu[rng.choice(nclu, ngroup - ngroup // 10 - ngroup // 20, replace=False)],
                          clu[rng.integers(0, nclu, ngroup // 20)], absent])
    rest = k0[nclu + rng.choice(len(k0) - nclu, 2000, replace=False)]
    rm = np.concatenate([grp, rest])
    rm = rm[rng.permutation(len(rm))]
    assert g.bulk_remove(rm) == o.bulk_remove(rm)
    _same(g, o)
    q = np.concatenate([clu, rest])
    gv, gf = g.bulk_get(q)
    ov, of = o.bulk_get(q)
    assert np.array_equal(gf, of) and np.array_equal(gv, ov)
