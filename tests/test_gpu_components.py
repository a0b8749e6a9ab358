"""Parity of the component path: the one-at-a-time insert order spread over
the GPU when rounds stall (a big batch into a near-full table).

The pending ops are split into components by a carry walk over the free
slots; components run at the same time, each in index order.  Every case
compares the returned count, len, the full table layout and get results
with the sequential oracle, bit for bit, and checks that the path ran.
"""
import numpy as np
import pytest

from fm_testutil import OracleAdapter, gpu_map, le

pytestmark = pytest.mark.gpu


def assert_same(g, o, probe=None):
    gf, gk, gv = g.snapshot()
    of_, ok, ov = o.snapshot()
    assert np.array_equal(gf, of_), f"flags differ at {np.nonzero(gf != of_)[0][:10]}"
    assert np.array_equal(gk, ok), "keys differ"
    assert np.array_equal(gv, ov), "values differ"
    assert g.len() == o.len()
    if probe is not None:
        a, fa = g.bulk_get(probe)
        b, fb = o.bulk_get(probe)
        assert np.array_equal(fa, fb) and np.array_equal(a, b)


def rand_keys(rng, n, ks):
    return rng.integers(0, 256, (n, ks), dtype=np.uint8)


def serial_ran(g):
    return g.kernel_times().get("k_ins_serial", (0.0, 0))[1] > 0


def insert_both(g, o, k, v):
    g.kernel_timing(True, reset=True)
    got = g.bulk_insert(k, v)
    ran = serial_ran(g)
    g.kernel_timing(False)
    assert got == o.bulk_insert(k, v)
    return ran


@pytest.mark.parametrize("shape", [(8, 8), (32, 128), (12, 20)])
@pytest.mark.parametrize("cap_bits", [12, 16])
def test_big_batch_into_near_full_table(shape, cap_bits):
    """Prefill to 0.80, then one batch of 0.185 x capacity holding in-batch
    duplicates and updates of present keys: rounds stall and the rest runs
    as components (final load about 0.98)."""
    ks, vs = shape
    cap = 1 << cap_bits
    rng = np.random.default_rng(cap_bits * 10 + ks)
    g = gpu_map(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    pk = rand_keys(rng, int(cap * 0.80), ks)
    pv = rand_keys(rng, len(pk), vs)
    assert g.bulk_insert(pk, pv) == o.bulk_insert(pk, pv)
    n = int(cap * 0.185)
    k = rand_keys(rng, n, ks)
    d = rng.choice(n, n // 10, replace=False)
    k[d] = k[rng.integers(0, n, len(d))]  # in-batch duplicates (later wins)
    u = rng.choice(n, n // 10, replace=False)
    k[u] = pk[rng.integers(0, len(pk), len(u))]  # updates of present keys
    v = rand_keys(rng, n, vs)
    ran = insert_both(g, o, k, v)
    assert_same(g, o, np.concatenate([k, pk[:2000], rand_keys(rng, 500, ks)]))
    if cap_bits >= 16:  # smaller batches finish inside the single-block tail
        assert ran, "the one-at-a-time path did not run"


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
def test_batch_that_fills_every_free_slot(shape):
    """New keys exactly as many as the free slots: the carry walk has no slot
    to spare round the ring, so every op goes to one block (the plain index
    order); the table ends completely full."""
    ks, vs = shape
    cap = 1 << 13
    rng = np.random.default_rng(7 + ks)
    g = gpu_map(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    pk = le(rng.permutation(int(cap * 0.9)).astype(np.uint64) * 3 + 1, ks)
    pv = np.ascontiguousarray(pk[:, :1].repeat(vs, 1))
    assert g.bulk_insert(pk, pv) == o.bulk_insert(pk, pv)
    free = cap - o.len()
    k = le(np.arange(free, dtype=np.uint64) * 3 + 2, ks)  # distinct from the prefill
    v = rand_keys(rng, free, vs)
    insert_both(g, o, k, v)
    assert g.len() == cap
    assert_same(g, o, k[:500])


def test_tombstones_count_as_free_slots():
    """Remove a third of a 0.9-load table (tombstones), then one batch that
    takes it to 0.99: inserts claim tombstones and EMPTY slots alike."""
    cap = 1 << 15
    rng = np.random.default_rng(11)
    g = gpu_map(cap, 32, 128)
    o = OracleAdapter(cap, 32, 128)
    pk = rand_keys(rng, int(cap * 0.9), 32)
    pv = rand_keys(rng, len(pk), 128)
    assert g.bulk_insert(pk, pv) == o.bulk_insert(pk, pv)
    rm = pk[rng.choice(len(pk), len(pk) // 3, replace=False)]
    assert g.bulk_remove(rm) == o.bulk_remove(rm)
    n = cap - o.len() - int(cap * 0.01)
    k = rand_keys(rng, n, 32)
    k[: n // 20] = rm[: n // 20]  # some removed keys come back
    v = rand_keys(rng, n, 128)
    ran = insert_both(g, o, k, v)
    assert_same(g, o, np.concatenate([k[:3000], pk[:3000]]))
    assert ran


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
def test_components_wrap_the_table_end(shape):
    """Identity hash with keys homed in the last slots of the table: the
    crowded region and its components run past the end into slot 0."""
    ks, vs = shape
    cap = 1 << 14
    rng = np.random.default_rng(5)
    g = gpu_map(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    bk = le(rng.integers(0, 1 << 62, int(cap * 0.7), dtype=np.uint64), ks)  # background load 0.7
    bv = np.ascontiguousarray(bk[:, :1].repeat(vs, 1))
    assert g.bulk_insert(bk, bv) == o.bulk_insert(bk, bv)
    homes = cap - 600 + rng.integers(0, 600, 2500).astype(np.uint64)  # 2500 keys homed in the last 600 slots
    k = le(homes + (np.arange(2500, dtype=np.uint64) + 1) * np.uint64(cap), ks)
    v = rand_keys(rng, len(k), vs)
    insert_both(g, o, k, v)
    assert_same(g, o, k)


def test_chunk_tail_and_small_tables():
    """Capacities below one chunk and below one thread's 32 slots."""
    for cap in (16, 64, 256, 2048):
        rng = np.random.default_rng(cap)
        g = gpu_map(cap, 8, 8)
        o = OracleAdapter(cap, 8, 8)
        pk = rand_keys(rng, int(cap * 0.5), 8)
        assert g.bulk_insert(pk, pk) == o.bulk_insert(pk, pk)
        n = cap - o.len() - 1
        k = rand_keys(rng, n, 8)
        insert_both(g, o, k, k)
        assert_same(g, o, k)


def test_large_table_many_components():
    """2^20 u64 slots at 0.85, then a batch to 0.985 (hundreds of chunks,
    components crossing chunk borders)."""
    cap = 1 << 20
    rng = np.random.default_rng(3)
    g = gpu_map(cap, 8, 8)
    o = OracleAdapter(cap, 8, 8)
    pk = le(rng.integers(0, 1 << 63, int(cap * 0.85), dtype=np.uint64))
    assert g.bulk_insert(pk, pk) == o.bulk_insert(pk, pk)
    n = int(cap * 0.135)
    k = le(rng.integers(0, 1 << 63, n, dtype=np.uint64))
    v = le(rng.integers(0, 1 << 63, n, dtype=np.uint64))
    ran = insert_both(g, o, k, v)
    assert_same(g, o, k[:20000])
    assert ran


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
def test_chain_longer_than_the_block_buffer(shape):
    """One cluster of 31,800 entries at their homes (identity hash), then an
    insert homed inside it: the call takes the table past load 0.97, so it
    runs as a component, and its chain of about 31,790 evictions is several
    times the block's 8K-entry buffer (moved chunk by chunk from the top)."""
    ks, vs = shape
    cap = 1 << 15
    g = gpu_map(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    homes = np.arange(31800, dtype=np.uint64)
    pk = le(homes, ks)
    pv = le(homes + np.uint64(7), vs)
    assert g.bulk_insert(pk, pv) == o.bulk_insert(pk, pv)
    k = le(np.array([5 + cap, 12 + 2 * cap], dtype=np.uint64), ks)  # homes 5 and 12
    v = le(np.array([1, 2], dtype=np.uint64), vs)
    ran = insert_both(g, o, k, v)
    assert_same(g, o, np.concatenate([k, pk[::97]]))
    assert ran
