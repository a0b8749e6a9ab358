"""Parity of the B200 backend (through the C ABI) with the CPU oracle.

Every comparison is bit-exact: returned counts, len, every get result
(found mask and value bytes, zeros for misses) and the full table layout
(metadata words of every slot, key and value bytes of every OCCUPIED slot).
"""
import numpy as np
import pytest

from fm_testutil import (OracleAdapter, churn_workload, expected_layout, gpu_map, le, load_json, mix64,
                         replay_layout_case, splitmix64, table_full_types)

pytestmark = pytest.mark.gpu


def assert_same_layout(g, o):
    gf, gk, gv = g.snapshot()
    of, ok, ov = o.snapshot()
    assert np.array_equal(gf, of), f"flags differ at {np.nonzero(gf != of)[0][:10]}"
    assert np.array_equal(gk, ok), "keys differ"
    assert np.array_equal(gv, ov), "values differ"


def assert_same_gets(g, o, keys):
    gv, gfnd = g.bulk_get(keys)
    ov, ofnd = o.bulk_get(keys)
    assert np.array_equal(gfnd, ofnd), f"found differs at {np.nonzero(gfnd != ofnd)[0][:10]}"
    assert np.array_equal(gv, ov), "values differ"


@pytest.mark.parametrize("case_id", range(7))
def test_golden_layouts(case_id):
    case = load_json("layouts.json")[case_id]
    g = gpu_map(case["capacity"], case["key_size"], case["value_size"], case["hash_mode"])
    f, k, v = replay_layout_case(case, g)
    ef, ek, ev = expected_layout(case)
    assert np.array_equal(f, ef) and np.array_equal(k, ek) and np.array_equal(v, ev)


@pytest.mark.parametrize("ksz", [1, 3, 5, 8, 12, 16, 31, 32, 33, 64])
@pytest.mark.parametrize("mode", [0, 1])
def test_device_hash_matches_golden(ksz, mode):
    """Home slot of every stored key = golden hash & mask (20 low bits)."""
    import oracle as O

    cap = 1 << 20
    rng = np.random.default_rng(ksz * 7 + mode)
    keys = rng.integers(0, 256, (2000, ksz), dtype=np.uint8)
    keys = np.unique(keys, axis=0)
    g = gpu_map(cap, ksz, 4, mode)
    g.bulk_insert(keys, np.zeros((len(keys), 4), np.uint8))
    f, k, _ = g.snapshot()
    occ = np.nonzero((f & 0xF) == 1)[0]
    assert len(occ) == len(keys)
    for s in occ[:400]:
        home = (int(s) - int(f[s] >> 4)) & (cap - 1)
        assert home == O.hash_key(bytes(k[s]), mode) & (cap - 1)


SHAPES = [(8, 8), (32, 128), (32, 64), (32, 32), (8, 32), (5, 3), (12, 20), (16, 16), (4, 0)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("mode", [0, 1])
def test_churn_parity(shape, mode):
    """Remove->insert churn with in-batch duplicates on crowded tables: the
    layout-sensitive regime (tombstone reuse, duplicate copies, false
    negatives of the reference) must match slot for slot."""
    ks, vs = shape
    rng = np.random.default_rng(hash((ks, vs, mode)) & 0xFFFF)
    cap = 512
    g = gpu_map(cap, ks, vs, mode)
    o = OracleAdapter(cap, ks, vs, mode)
    seen = []
    for op, keys, vals in churn_workload(rng, cap, ks, vs, rounds=40):
        if op == "insert":
            try:
                a = o.bulk_insert(keys, vals)
            except table_full_types():
                with pytest.raises(table_full_types()):
                    g.bulk_insert(keys, vals)
                continue
            b = g.bulk_insert(keys, vals)
        else:
            a, b = o.bulk_remove(keys), g.bulk_remove(keys)
        assert a == b, op
        assert g.len() == o.len()
        seen.append(keys)
    assert_same_layout(g, o)
    allk = np.concatenate(seen) if seen else np.zeros((0, ks), np.uint8)
    assert_same_gets(g, o, allk)
    assert_same_gets(g, o, rng.integers(0, 256, (300, ks), dtype=np.uint8))


@pytest.mark.parametrize("cap", [1, 2, 4, 8, 16])
def test_tiny_capacities(cap):
    g = gpu_map(cap, 8, 8)
    o = OracleAdapter(cap, 8, 8)
    assert g.capacity() == o.capacity() == cap
    rng = np.random.default_rng(cap)
    for r in range(12):
        n = int(rng.integers(1, cap + 1))
        keys = le(rng.integers(0, 3 * cap, n).astype(np.uint64))
        vals = le(rng.integers(0, 1 << 40, n).astype(np.uint64))
        if r % 3 == 2:
            assert g.bulk_remove(keys) == o.bulk_remove(keys)
        else:
            try:
                a = o.bulk_insert(keys, vals)
            except table_full_types():
                with pytest.raises(table_full_types()):
                    g.bulk_insert(keys, vals)
                continue
            assert g.bulk_insert(keys, vals) == a
        assert g.len() == o.len()
        assert_same_layout(g, o)
    assert_same_gets(g, o, le(np.arange(3 * cap, dtype=np.uint64)))


def test_in_batch_duplicates_later_wins():
    cap = 1 << 12
    g = gpu_map(cap, 8, 8)
    o = OracleAdapter(cap, 8, 8)
    rng = np.random.default_rng(11)
    base = rng.integers(0, 1 << 62, 200).astype(np.uint64)
    # Zipf-like multiplicities: some keys repeated many times in one batch.
    idx = np.minimum(rng.zipf(1.3, 2500) - 1, len(base) - 1)
    keys = le(base[idx])
    vals = le(np.arange(len(idx), dtype=np.uint64))
    assert g.bulk_insert(keys, vals) == o.bulk_insert(keys, vals)
    assert_same_layout(g, o)
    assert_same_gets(g, o, le(base))
    # later position wins
    v, f = g.bulk_get(le(base[idx[:50]]))
    last = {int(k): i for i, k in enumerate(base[idx])}
    for t in range(50):
        assert v[t].view(np.uint64)[0] == last[int(base[idx[t]])]
    # duplicate removes inside one batch: the first removes, the rest miss
    rk = le(np.concatenate([base[:20], base[:20], base[:5]]))
    assert g.bulk_remove(rk) == o.bulk_remove(rk)
    assert_same_layout(g, o)


def test_full_table_uncounted_drop_and_recount():
    """Past a full table (only reachable through the uncounted device insert,
    which skips the precheck) a walk whose probe passes the capacity drops
    its entry (rayon_cpu.rs:167-169); len counts it, recount does not."""
    import torch

    cap = 16
    g = gpu_map(cap, 8, 8)
    o = OracleAdapter(cap, 8, 8)
    k = le(np.arange(16, dtype=np.uint64) * 16)  # identity hash: all home 0
    assert g.bulk_insert(k, k) == o.bulk_insert(k, k) == 16
    extra = le([32 * 16])
    o.bulk_insert_uncounted(extra, extra)
    dk = torch.from_numpy(extra.copy()).cuda()
    g.bulk_insert_device_uncounted(dk, dk, 1)
    torch.cuda.synchronize()
    assert g.len() == o.len() == 17
    assert_same_layout(g, o)
    assert g.recount() == o.recount() == 16
    assert_same_gets(g, o, np.concatenate([k, extra]))


def test_full_table_walk_limit():
    """On a table with no free slot the reference's insert loop can cycle
    forever.  Both the oracle and the backend stop such a walk after
    2*capacity+2 slots, run the remaining ops, and report the limit."""
    import torch

    import flash_map as F
    import oracle as O

    cap = 16
    g = gpu_map(cap, 8, 8)
    o = OracleAdapter(cap, 8, 8)
    k = le(np.arange(14, dtype=np.uint64) * 16)
    assert g.bulk_insert(k, k) == o.bulk_insert(k, k)
    extra = le(np.arange(100, 108, dtype=np.uint64))
    with pytest.raises(O.ProbeLimit):
        o.bulk_insert_uncounted(extra, extra)
    dk = torch.from_numpy(extra.copy()).cuda()
    with pytest.raises(F.KernelLaunch, match="2\\*capacity"):
        g.bulk_insert_device_uncounted(dk, dk, len(extra))
    assert g.len() == o.len() == 22
    assert_same_layout(g, o)
    assert g.recount() == o.recount()
    assert_same_gets(g, o, np.concatenate([k, extra]))


def test_table_full_keeps_state():
    g = gpu_map(64, 8, 8)
    k = le(np.arange(60, dtype=np.uint64))
    g.bulk_insert(k, k)
    before = g.snapshot()
    with pytest.raises(table_full_types()) as ei:
        g.bulk_insert(le(np.arange(100, 105, dtype=np.uint64)), le(np.arange(5, dtype=np.uint64)))
    assert ei.value.occupied == 60 and ei.value.capacity == 64
    after = g.snapshot()
    for a, b in zip(before, after):
        assert np.array_equal(a, b)


def test_device_resident_api():
    import torch

    cap = 1 << 14
    g = gpu_map(cap, 32, 128)
    o = OracleAdapter(cap, 32, 128)
    rng = np.random.default_rng(5)
    keys = rng.integers(0, 256, (5000, 32), dtype=np.uint8)
    vals = rng.integers(0, 256, (5000, 128), dtype=np.uint8)
    dk = torch.from_numpy(keys).cuda()
    dv = torch.from_numpy(vals).cuda()
    assert g.bulk_insert_device(dk, dv, 5000) == o.bulk_insert(keys, vals)
    q = np.concatenate([keys[:3000], rng.integers(0, 256, (1000, 32), dtype=np.uint8)])
    dq = torch.from_numpy(q).cuda()
    out_v = torch.full((len(q), 128), 7, dtype=torch.uint8, device="cuda")
    out_f = torch.full((len(q),), 7, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream()
    g.bulk_get_device(dq, len(q), out_v, out_f, stream=s)
    torch.cuda.synchronize()
    ov, of = o.bulk_get(q)
    assert np.array_equal(out_f.cpu().numpy().astype(bool), of)
    assert np.array_equal(out_v.cpu().numpy(), ov)  # misses written as zeros
    out_v2 = torch.full((len(q), 128), 9, dtype=torch.uint8, device="cuda")
    g.bulk_get_values_device(dq, len(q), out_v2, stream=s)
    torch.cuda.synchronize()
    assert np.array_equal(out_v2.cpu().numpy(), ov)
    # misaligned (odd byte offset) device buffers take the run-time-size path
    raw = torch.zeros(len(q) * 32 + 1, dtype=torch.uint8, device="cuda")
    raw[1:] = dq.reshape(-1)
    outm = torch.zeros(len(q) * 128 + 3, dtype=torch.uint8, device="cuda")
    g.bulk_get_values_device(raw.data_ptr() + 1, len(q), outm.data_ptr() + 3, stream=s)
    torch.cuda.synchronize()
    assert np.array_equal(outm[3:].cpu().numpy().reshape(len(q), 128), ov)
    rm = dk[:1000]
    assert g.bulk_remove_device(rm, 1000) == o.bulk_remove(keys[:1000])
    assert_same_layout(g, o)


def test_baseline_small_config():
    """The small CPU-runnable workload: FlashMap<u64,u64>, with_capacity(2^20),
    700K splitmix64 keys, values = splitmix64 mix of the key; get 700K present +
    700K absent; remove the first 100K; get the 700K again."""
    n = 700_000
    keys = np.unique(splitmix64(1, n + 1000))[:n]
    rng = np.random.default_rng(1)
    keys = keys[rng.permutation(len(keys))]
    vals = mix64(keys)
    absent = splitmix64(2, n + 10000)
    absent = absent[~np.isin(absent, keys)][:n]
    g = gpu_map(1 << 20, 8, 8)
    o = OracleAdapter(1 << 20, 8, 8)
    assert g.bulk_insert(keys, vals) == o.bulk_insert(keys, vals) == n
    q = np.concatenate([keys, absent])
    gv, gf = g.bulk_get(q)
    assert gf[:n].all() and not gf[n:].any()
    assert np.array_equal(gv[:n].view(np.uint64).ravel(), vals)
    assert_same_gets(g, o, q)
    assert g.bulk_remove(keys[:100_000]) == o.bulk_remove(keys[:100_000]) == 100_000
    assert g.len() == o.len() == n - 100_000
    assert_same_gets(g, o, keys)
    assert_same_layout(g, o)


def test_account_shape_scaled():
    """[u8;32] -> [u8;128] at the account shape, scaled down: 10 insert calls
    to 80% of capacity, then gets with 50% hits and a 10% remove."""
    cap = 1 << 16
    n = int(cap * 0.8)
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    vals = rng.integers(0, 256, (n, 128), dtype=np.uint8)
    g = gpu_map(cap, 32, 128)
    o = OracleAdapter(cap, 32, 128)
    for c in np.array_split(np.arange(n), 10):
        assert g.bulk_insert(keys[c], vals[c]) == o.bulk_insert(keys[c], vals[c])
    assert_same_layout(g, o)
    q = np.concatenate([keys[rng.choice(n, n // 2, replace=False)], rng.integers(0, 256, (n // 2, 32), dtype=np.uint8)])
    q = q[rng.permutation(len(q))]
    assert_same_gets(g, o, q)
    rm = keys[rng.choice(n, n // 10, replace=False)]
    assert g.bulk_remove(rm) == o.bulk_remove(rm)
    assert_same_layout(g, o)
    assert_same_gets(g, o, keys)


def test_skewed_duplicate_heavy_scaled():
    """u64 keys (2-bit packed 32-mers), fill to 0.9 with batches holding 20%
    in-batch repeats (a later copy carries a new value), Zipf lookups and
    interleaved removes -- scaled down."""
    cap = 1 << 16
    target = int(cap * 0.9)
    rng = np.random.default_rng(4)
    g = gpu_map(cap, 8, 8)
    o = OracleAdapter(cap, 8, 8)
    present = []
    while o.len() < target:
        b = min(4096, target - o.len())
        fresh = rng.integers(0, 1 << 62, b - b // 5, dtype=np.uint64)  # 31 bases * 2 bits = 62 bits
        rep = fresh[rng.integers(0, len(fresh), b // 5)]
        batch = np.concatenate([fresh, rep])
        batch = batch[rng.permutation(len(batch))]
        vals = rng.integers(0, 1 << 63, len(batch), dtype=np.uint64)
        assert g.bulk_insert(batch, vals) == o.bulk_insert(batch, vals)
        present.append(batch)
    assert_same_layout(g, o)
    present = np.unique(np.concatenate(present))
    for r in range(4):
        z = np.minimum(rng.zipf(1.1, 20000) - 1, len(present) - 1)
        perm = rng.permutation(len(present))
        q = np.concatenate([present[perm[z]], rng.integers(0, 1 << 62, 2000, dtype=np.uint64)])
        assert_same_gets(g, o, q)
        rm = present[rng.integers(0, len(present), 3000)]
        assert g.bulk_remove(rm) == o.bulk_remove(rm)
    assert_same_layout(g, o)


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
@pytest.mark.parametrize("chain", [3, 4, 5, 30, 63, 64, 65, 70, 128, 129, 200])
def test_long_eviction_chains(shape, chain):
    """An insert whose Robin Hood walk evicts `chain` entries in a row (homes
    1..chain each at dist 0 behind a home-0 entry): exercises the thread
    path's eviction limit, chains spanning several metadata windows and
    chains longer than the tile's chain buffer (moved chunk by chunk)."""
    ks, vs = shape
    cap = 256 if chain < 200 else 512
    g = gpu_map(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    homes = np.arange(0, chain + 1, dtype=np.uint64)
    keys = le(homes, ks)
    vals = le(homes * 3 + 1, vs)
    assert g.bulk_insert(keys, vals) == o.bulk_insert(keys, vals)
    k2 = le([np.uint64(cap)], ks)  # home 0 again: evicts homes 1..chain
    v2 = le([np.uint64(999)], vs)
    assert g.bulk_insert(k2, v2) == o.bulk_insert(k2, v2) == 1
    assert_same_layout(g, o)
    # the same as several ops in one batch (segments merge as free slots fill)
    g2 = gpu_map(cap, ks, vs)
    o2 = OracleAdapter(cap, ks, vs)
    batch = np.concatenate([keys, le(np.arange(1, 6, dtype=np.uint64) * cap, ks)])
    bv = le(np.arange(len(batch), dtype=np.uint64), vs)
    assert g2.bulk_insert(batch, bv) == o2.bulk_insert(batch, bv)
    assert_same_layout(g2, o2)


@pytest.mark.parametrize("extra_n", [100, 300])
def test_overfull_table_serial_path(extra_n):
    """Uncounted inserts into a completely full table: every round finds no
    free slot, so the ops run one at a time in index order (inside the tail
    block for small counts, in the host-launched sequential kernel above the
    tail limit).  Layout, len and the limit report match the oracle."""
    import torch

    import flash_map as F
    import oracle as O

    cap = 512
    rng = np.random.default_rng(extra_n)
    g = gpu_map(cap, 8, 8)
    o = OracleAdapter(cap, 8, 8)
    k = le(rng.permutation(np.arange(cap, dtype=np.uint64) * 7 + 3))
    assert g.bulk_insert(k, k) == o.bulk_insert(k, k) == cap
    extra = le(rng.integers(0, 1 << 40, extra_n).astype(np.uint64))
    o_limit = False
    try:
        o.bulk_insert_uncounted(extra, extra)
    except O.ProbeLimit:
        o_limit = True
    dk = torch.from_numpy(extra.copy()).cuda()
    g_limit = False
    try:
        g.bulk_insert_device_uncounted(dk, dk, extra_n)
    except F.KernelLaunch as e:
        assert "2*capacity" in str(e)
        g_limit = True
    torch.cuda.synchronize()
    assert g_limit == o_limit
    assert g.len() == o.len() == cap + extra_n
    assert_same_layout(g, o)
    assert g.recount() == o.recount()


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
@pytest.mark.parametrize("run", [2, 3, 10, 33, 40, 100])
def test_many_possible_updates(shape, run):
    """`run` keys sharing one home sit at distances 0..run-1, so a walk from
    that home meets a possible update (stored distance == probe depth) at
    every slot: a fresh key compares all of them and claims the slot after;
    an existing key deep in the run updates in place (buffered compares
    flushed in walk order)."""
    ks, vs = shape
    cap = 256
    g = gpu_map(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    homes0 = np.arange(run, dtype=np.uint64) * cap + 5
    keys = le(homes0, ks)
    vals = le(homes0 + 1, vs)
    assert g.bulk_insert(keys, vals) == o.bulk_insert(keys, vals)
    # a fresh key and an update of the key at depth run-2, in one batch and alone
    fresh = le([np.uint64(run * cap + 5)], ks)
    upd = le([homes0[max(run - 2, 0)]], ks)
    for batch in (np.concatenate([fresh, upd]), upd, fresh):
        bv = le(np.arange(len(batch), dtype=np.uint64) + 777, vs)
        assert g.bulk_insert(batch, bv) == o.bulk_insert(batch, bv)
        assert_same_layout(g, o)


@pytest.mark.parametrize("load", [0.9, 0.97, 0.995])
def test_high_load_fill_and_churn(load):
    """u64 pairs filled to a high load in calls of 2% of the capacity (eviction
    chains of hundreds of entries, many possible updates per walk), then
    remove/insert churn that reuses tombstones; full layout after each call."""
    cap = 1 << 14
    rng = np.random.default_rng(int(load * 100))
    g = gpu_map(cap, 8, 8)
    o = OracleAdapter(cap, 8, 8)
    n = int(cap * load)
    keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
    call = cap // 50
    for b in range(0, n, call):
        k = le(keys[b:b + call])
        assert g.bulk_insert(k, k) == o.bulk_insert(k, k)
    assert_same_layout(g, o)
    for r in range(3):
        rm = le(keys[rng.choice(n, call, replace=False)])
        assert g.bulk_remove(rm) == o.bulk_remove(rm)
        fresh = le(rng.integers(0, 1 << 63, call, dtype=np.uint64))
        assert g.bulk_insert(fresh, fresh) == o.bulk_insert(fresh, fresh)
        assert_same_layout(g, o)
    assert_same_gets(g, o, le(keys))


def test_host_api_pieces_pinned_buffers():
    """Host-API calls larger than one transfer piece, from pinned host
    buffers: an insert of 150K account-shape pairs whose in-batch duplicates
    straddle piece boundaries (later wins), a get of 1.2M keys and a remove of
    100K, each split into overlapping upload/compute/download pieces."""
    import torch

    cap = 1 << 18
    rng = np.random.default_rng(11)
    n = 150_000
    keys = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    dup = rng.choice(n // 2, n // 10, replace=False)
    keys[n // 2 + dup] = keys[dup]  # repeats of first-half keys in the second half
    vals = rng.integers(0, 256, (n, 128), dtype=np.uint8)
    pk = torch.from_numpy(keys).pin_memory().numpy()
    pv = torch.from_numpy(vals).pin_memory().numpy()
    g = gpu_map(cap, 32, 128)
    o = OracleAdapter(cap, 32, 128)
    assert g.bulk_insert(pk, pv) == o.bulk_insert(keys, vals)
    assert_same_layout(g, o)
    q = np.concatenate([keys, rng.integers(0, 256, (1_200_000 - n, 32), dtype=np.uint8)])
    q = q[rng.permutation(len(q))]
    pq = torch.from_numpy(q).pin_memory().numpy()
    ov = torch.empty((len(q), 128), dtype=torch.uint8).pin_memory().numpy()
    of = torch.empty((len(q),), dtype=torch.uint8).pin_memory().numpy()
    gv, gf = g.bulk_get(pq, out_values=ov, out_found=of)
    ev, ef = o.bulk_get(q)
    assert np.array_equal(np.asarray(gf, bool), np.asarray(ef, bool))
    assert np.array_equal(gv, ev)
    rm = torch.from_numpy(keys[rng.choice(n, 100_000, replace=False)]).pin_memory().numpy()
    assert g.bulk_remove(rm) == o.bulk_remove(np.array(rm))
    assert_same_layout(g, o)


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
def test_remove_long_windows_chunk_summaries(shape):
    """Removes where the largest stored distance is in the hundreds (load
    0.97 after churn that reuses tombstones, so keys can have copies past a
    probe's exit): the remove windows run long and the kernels skip chunks by
    their summaries.  Big batches with in-batch duplicates and absent keys;
    counts, gets and the full layout after every call."""
    ks, vs = shape
    cap = 1 << 16
    rng = np.random.default_rng(97 + ks)
    g = gpu_map(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    keys = rng.integers(0, 256, (int(cap * 0.97), ks), dtype=np.uint8)
    vals = rng.integers(0, 256, (len(keys), vs), dtype=np.uint8)
    assert g.bulk_insert(keys, vals) == o.bulk_insert(keys, vals)
    for r in range(3):
        rm = keys[rng.choice(len(keys), len(keys) // 10, replace=False)]
        assert g.bulk_remove(rm) == o.bulk_remove(rm)
        back = np.concatenate([rm[: len(rm) // 2], rng.integers(0, 256, (len(rm) // 3, ks), dtype=np.uint8)])
        bv = rng.integers(0, 256, (len(back), vs), dtype=np.uint8)
        assert g.bulk_insert(back, bv) == o.bulk_insert(back, bv)
        assert_same_layout(g, o)
    big = keys[rng.integers(0, len(keys), len(keys) // 2)]  # repeats: in-batch duplicates
    big = np.concatenate([big, rng.integers(0, 256, (5000, ks), dtype=np.uint8)])
    big = big[rng.permutation(len(big))]
    assert g.bulk_remove(big) == o.bulk_remove(big)
    assert_same_layout(g, o)
    assert_same_gets(g, o, keys[:20000])
