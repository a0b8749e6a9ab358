"""Batched form: a queue of bulk ops over many tables, run as waves of grouped
kernels (eagerly and replayed from a CUDA graph), must equal the sequential
oracle replaying the same queue one op at a time in queue order: every get
output, every insert/remove count and status (TableFull for oversized
inserts), every table's final len and slot layout."""
import numpy as np
import pytest

from fm_testutil import OracleAdapter, gpu_map

pytestmark = pytest.mark.gpu

SHAPES = [(8, 8), (32, 128), (32, 32), (8, 32)]


@pytest.fixture(autouse=True, params=["queue", "lanes"])
def batch_mode(request, monkeypatch):
    """Every test under both queue-mode executions: the persistent kernel
    draining the ops (with device-driven steps for the large ones), and
    every op as device-driven kernels on its table's stream lane."""
    monkeypatch.setenv("FLASHMAP_BATCH_MODE", request.param)
    return request.param


def _keys(rng, n, ks):
    return rng.integers(0, 256, (n, ks), dtype=np.uint8)


def make_queue(seed, ntables=8, nops=70, cap_bits=(10, 14), sizes=(16, 6000)):
    import flash_map as F

    rng = np.random.default_rng(seed)
    tables = []
    for i in range(ntables):
        ks, vs = SHAPES[i % len(SHAPES)]
        cap = 1 << int(rng.integers(cap_bits[0], cap_bits[1] + 1))
        g = gpu_map(cap, ks, vs)
        o = OracleAdapter(cap, ks, vs)
        n = int(cap * rng.uniform(0.5, 0.85))
        k, v = _keys(rng, n, ks), _keys(rng, n, vs)
        assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
        tables.append({"g": g, "o": o, "ks": ks, "vs": vs, "known": [k]})
    queue = []
    for i in range(nops):
        ti = int(rng.integers(ntables))
        t = tables[ti]
        kind = int(rng.choice([F.batch.GET, F.batch.INSERT, F.batch.REMOVE], p=[0.4, 0.4, 0.2]))
        n = int(np.exp(rng.uniform(np.log(sizes[0]), np.log(sizes[1]))))
        if i == 5:
            n = 0  # an empty op
        known = np.concatenate(t["known"])
        if kind == F.batch.INSERT:
            k = _keys(rng, n, t["ks"])
            if n >= 10:
                d = rng.choice(n, n // 10, replace=False)
                k[d] = k[rng.integers(0, n, len(d))]  # in-batch duplicates
                e = rng.choice(n, n // 10, replace=False)
                k[e] = known[rng.integers(0, len(known), len(e))]  # updates of present keys
            v = _keys(rng, n, t["vs"])
            t["known"].append(k)
        else:
            npres = int(n * 0.8)
            k = np.concatenate([known[rng.integers(0, len(known), npres)], _keys(rng, n - npres, t["ks"])])
            k = k[rng.permutation(n)] if n else k
            v = None
        queue.append((ti, kind, k, v))
    return tables, queue


def run_batch(tables, queue, graph):
    import torch

    import flash_map as F

    ops, outs = [], []
    for ti, kind, k, v in queue:
        t = tables[ti]
        n = len(k)
        dk = torch.from_numpy(np.ascontiguousarray(k)).cuda() if n else torch.empty((1, t["ks"]), dtype=torch.uint8,
                                                                                      device="cuda")
        dv = torch.from_numpy(np.ascontiguousarray(v)).cuda() if v is not None and n else None
        ov = of = None
        if kind == F.batch.GET:
            ov = torch.full((max(n, 1), t["vs"]), 0xAB, dtype=torch.uint8, device="cuda")
            of = torch.full((max(n, 1),), 0xAB, dtype=torch.uint8, device="cuda")
        ops.append(F.BatchOp(kind, t["g"], n, dk, dv, ov, of))
        outs.append((ov, of))
    b = F.FlashMapBatch(ops)
    assert b.waves >= 1
    s = torch.cuda.Stream()
    if graph:
        b.capture(s)
    b.run(s)
    res = b.wait()
    b.close()
    torch.cuda.synchronize()
    return res, [(None if ov is None else ov.cpu().numpy(), None if of is None else of.cpu().numpy())
                 for ov, of in outs]


def oracle_replay(tables, queue):
    import oracle as O

    import flash_map as F

    res, outs = [], []
    for ti, kind, k, v in queue:
        o = tables[ti]["o"]
        if len(k) == 0:
            res.append((0, 0))
            outs.append(None)
            continue
        if kind == F.batch.GET:
            outs.append(o.bulk_get(k))
            res.append((0, 0))
        elif kind == F.batch.INSERT:
            outs.append(None)
            try:
                res.append((o.bulk_insert(k, v), 0))
            except O.TableFull:
                res.append((0, 5))
        else:
            outs.append(None)
            res.append((o.bulk_remove(k), 0))
    return res, outs


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("seed", [1, 2])
def test_batch_matches_sequential_replay(seed, graph):
    import flash_map as F

    tables, queue = make_queue(seed)
    g_res, g_out = run_batch(tables, queue, graph)
    o_res, o_out = oracle_replay(tables, queue)
    full = 0
    for i, ((ti, kind, k, v), gr, orr) in enumerate(zip(queue, g_res, o_res)):
        assert gr == orr, f"op {i} kind {kind} n {len(k)}: gpu {gr} oracle {orr}"
        full += orr[1] == 5
        if kind == F.batch.GET and len(k):
            ov, of = g_out[i]
            ev, ef = o_out[i]
            assert np.array_equal(of.astype(bool), ef), f"op {i}: found differs"
            assert np.array_equal(ov, ev), f"op {i}: values differ"
    assert full >= 1  # the mix holds oversized inserts
    for t in tables:
        assert t["g"].len() == t["o"].len()
        gf, gk, gv = t["g"].snapshot()
        of_, ok, ov = t["o"].snapshot()
        assert np.array_equal(gf, of_) and np.array_equal(gk, ok) and np.array_equal(gv, ov)


def test_batch_single_table_chain_of_dependent_ops():
    """Every op on one table: one wave per op (gets in a row share a wave),
    each insert seeing the previous ops' effects."""
    import flash_map as F

    rng = np.random.default_rng(7)
    cap = 1 << 12
    g = gpu_map(cap, 8, 8)
    o = OracleAdapter(cap, 8, 8)
    tables = [{"g": g, "o": o, "ks": 8, "vs": 8, "known": []}]
    queue = []
    pool = rng.integers(0, 256, (3000, 8), dtype=np.uint8)
    for i in range(20):
        kind = [F.batch.INSERT, F.batch.GET, F.batch.GET, F.batch.REMOVE][i % 4]
        k = pool[rng.integers(0, len(pool), 400)]
        v = rng.integers(0, 256, (400, 8), dtype=np.uint8) if kind == F.batch.INSERT else None
        queue.append((0, kind, k, v))
    g_res, g_out = run_batch(tables, queue, False)
    o_res, o_out = oracle_replay(tables, queue)
    assert g_res == o_res
    for i, (ti, kind, k, v) in enumerate(queue):
        if kind == F.batch.GET:
            assert np.array_equal(g_out[i][1].astype(bool), o_out[i][1])
            assert np.array_equal(g_out[i][0], o_out[i][0])
    gf, gk, gv = g.snapshot()
    of_, ok, ov = o.snapshot()
    assert np.array_equal(gf, of_) and np.array_equal(gk, ok) and np.array_equal(gv, ov)


def test_batch_ops_larger_than_any_earlier_call():
    """Fresh tables whose queued ops are far larger than any call they have
    seen: the per-table scratch grows to the largest op before any wave's
    descriptors are written (the small op queued first must not keep a stale
    scratch address)."""
    import flash_map as F

    rng = np.random.default_rng(9)
    tables, queue = [], []
    for ks, vs in [(8, 8), (32, 128)]:
        cap = 1 << 17
        g = gpu_map(cap, ks, vs)
        o = OracleAdapter(cap, ks, vs)
        tables.append({"g": g, "o": o, "ks": ks, "vs": vs, "known": []})
    for ti, t in enumerate(tables):
        for n in (100, 60_000, 3_000):
            queue.append((ti, F.batch.INSERT, _keys(rng, n, t["ks"]), _keys(rng, n, t["vs"])))
        queue.append((ti, F.batch.REMOVE, queue[-2][2][: 20_000], None))
        queue.append((ti, F.batch.GET, queue[-3][2], None))
    g_res, g_out = run_batch(tables, queue, False)
    o_res, o_out = oracle_replay(tables, queue)
    assert g_res == o_res
    for i, (ti, kind, k, v) in enumerate(queue):
        if kind == F.batch.GET:
            assert np.array_equal(g_out[i][1].astype(bool), o_out[i][1])
            assert np.array_equal(g_out[i][0], o_out[i][0])
    for t in tables:
        gf, gk, gv = t["g"].snapshot()
        of_, ok, ov = t["o"].snapshot()
        assert np.array_equal(gf, of_) and np.array_equal(gk, ok) and np.array_equal(gv, ov)


def test_batch_run_time_record_sizes():
    """Record sizes without a compiled specialisation (12-byte keys, 20-byte
    values) run the grouped kernels' generic path; results still equal the
    queue-order replay."""
    import flash_map as F

    rng = np.random.default_rng(12)
    tables = []
    for cap in (1 << 12, 1 << 13):
        tables.append({"g": gpu_map(cap, 12, 20), "o": OracleAdapter(cap, 12, 20), "ks": 12, "vs": 20, "known": []})
    queue = []
    for i in range(24):
        ti = i % 2
        t = tables[ti]
        kind = [F.batch.INSERT, F.batch.GET, F.batch.REMOVE, F.batch.INSERT][i % 4]
        n = int(rng.integers(50, 900))
        if kind == F.batch.INSERT:
            k = _keys(rng, n, 12)
            t["known"].append(k)
            queue.append((ti, kind, k, _keys(rng, n, 20)))
        else:
            pool = np.concatenate(t["known"]) if t["known"] else _keys(rng, 8, 12)
            queue.append((ti, kind, pool[rng.integers(0, len(pool), n)], None))
    for graph in (False,):
        g_res, g_out = run_batch(tables, queue, graph)
        o_res, o_out = oracle_replay(tables, queue)
        assert g_res == o_res
        for i, (ti, kind, k, v) in enumerate(queue):
            if kind == F.batch.GET:
                assert np.array_equal(g_out[i][1].astype(bool), o_out[i][1])
                assert np.array_equal(g_out[i][0], o_out[i][0])
    for t in tables:
        gf, gk, gv = t["g"].snapshot()
        of_, ok, ov = t["o"].snapshot()
        assert np.array_equal(gf, of_) and np.array_equal(gk, ok) and np.array_equal(gv, ov)


@pytest.mark.parametrize("graph", [False, True])
def test_batch_sixteen_tables_up_to_2_20_slots(graph):
    """16 tables of 2^12..2^20 slots, 150 ops of up to 50,000 keys: the
    persistent queue kernel (every shape here is a compile-time one) against
    the oracle replaying the queue in order."""
    import flash_map as F

    tables, queue = make_queue(21, ntables=16, nops=150, cap_bits=(12, 20), sizes=(16, 50_000))
    g_res, g_out = run_batch(tables, queue, graph)
    o_res, o_out = oracle_replay(tables, queue)
    for i, ((ti, kind, k, v), gr, orr) in enumerate(zip(queue, g_res, o_res)):
        assert gr == orr, f"op {i} kind {kind} n {len(k)}: gpu {gr} oracle {orr}"
        if kind == F.batch.GET and len(k):
            ov, of = g_out[i]
            ev, ef = o_out[i]
            assert np.array_equal(of.astype(bool), ef) and np.array_equal(ov, ev), f"op {i}"
    for t in tables:
        assert t["g"].len() == t["o"].len()
        for x, y in zip(t["g"].snapshot(), t["o"].snapshot()):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("graph", [False, True])
def test_batch_near_full_inserts_between_queue_launches(graph):
    """Inserts that take their tables to load 0.97 and beyond run on the
    component path between persistent launches; gets and removes on the same
    and other tables before and after them keep queue order."""
    import flash_map as F

    rng = np.random.default_rng(33)
    tables = []
    for i, (ks, vs) in enumerate([(8, 8), (32, 128), (8, 8)]):
        cap = 1 << 13
        g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
        k, v = _keys(rng, int(cap * 0.85), ks), _keys(rng, int(cap * 0.85), vs)
        assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
        tables.append({"g": g, "o": o, "ks": ks, "vs": vs, "known": [k]})
    queue = []
    for rep in range(3):
        for ti, t in enumerate(tables):
            cap = t["g"].capacity()
            n = int(cap * (0.05 if rep < 2 else 0.2))  # the last round is oversized for some
            k, v = _keys(rng, n, t["ks"]), _keys(rng, n, t["vs"])
            queue.append((ti, F.batch.INSERT, k, v))
            t["known"].append(k)
            known = np.concatenate(t["known"])
            queue.append((ti, F.batch.GET, known[rng.integers(0, len(known), 3000)], None))
            queue.append((ti, F.batch.REMOVE, known[rng.integers(0, len(known), 300)], None))
    g_res, g_out = run_batch(tables, queue, graph)
    o_res, o_out = oracle_replay(tables, queue)
    for i, ((ti, kind, k, v), gr, orr) in enumerate(zip(queue, g_res, o_res)):
        assert gr == orr, f"op {i} kind {kind} n {len(k)}: gpu {gr} oracle {orr}"
        if kind == F.batch.GET:
            ov, of = g_out[i]
            ev, ef = o_out[i]
            assert np.array_equal(of.astype(bool), ef) and np.array_equal(ov, ev), f"op {i}"
    for t in tables:
        assert t["g"].len() == t["o"].len()
        for x, y in zip(t["g"].snapshot(), t["o"].snapshot()):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("graph", [False, True])
def test_batch_large_and_high_load_inserts(graph):
    """The insert routes of the queue, each between gets and removes on the
    same table: an insert of 2^18 keys and inserts that take a table to load
    0.9 and 0.96 run between persistent launches on the direct passes (the
    components they leave on the component path); an insert of 24,000 keys
    that ends below 0.9 from 0.5 stays in the queue, where components too
    large for a warp go to the op's last unit."""
    import flash_map as F

    rng = np.random.default_rng(41)
    specs = [((8, 8), 1 << 20, 0.5, [1 << 18]),         # large: external direct
             ((32, 128), 1 << 16, 0.5, [24_000]),         # in queue, ends at 0.87
             ((8, 8), 1 << 16, 0.6, [int((1 << 16) * 0.3), int((1 << 16) * 0.06)])]  # to 0.9, then 0.96
    tables, queue = [], []
    for (ks, vs), cap, load0, sizes in specs:
        g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
        k, v = _keys(rng, int(cap * load0), ks), _keys(rng, int(cap * load0), vs)
        assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
        tables.append({"g": g, "o": o, "ks": ks, "vs": vs, "known": [k]})
    for ti, ((ks, vs), cap, load0, sizes) in enumerate(specs):
        t = tables[ti]
        for n in sizes:
            known = np.concatenate(t["known"])
            queue.append((ti, F.batch.GET, known[rng.integers(0, len(known), 5000)], None))
            k, v = _keys(rng, n, ks), _keys(rng, n, vs)
            k[: n // 20] = known[rng.integers(0, len(known), n // 20)]  # updates
            queue.append((ti, F.batch.INSERT, k, v))
            t["known"].append(k)
            known = np.concatenate(t["known"])
            queue.append((ti, F.batch.GET, known[rng.integers(0, len(known), 5000)], None))
            queue.append((ti, F.batch.REMOVE, known[rng.integers(0, len(known), 2000)], None))
    g_res, g_out = run_batch(tables, queue, graph)
    o_res, o_out = oracle_replay(tables, queue)
    for i, ((ti, kind, k, v), gr, orr) in enumerate(zip(queue, g_res, o_res)):
        assert gr == orr, f"op {i} kind {kind} n {len(k)}: gpu {gr} oracle {orr}"
        if kind == F.batch.GET:
            ov, of = g_out[i]
            ev, ef = o_out[i]
            assert np.array_equal(of.astype(bool), ef) and np.array_equal(ov, ev), f"op {i}"
    for t in tables:
        assert t["g"].len() == t["o"].len()
        for x, y in zip(t["g"].snapshot(), t["o"].snapshot()):
            assert np.array_equal(x, y)


def _clustered(cap, n, first_home, span, ks, salt=0):
    """n distinct keys whose identity-hash homes lie in [first_home,
    first_home + span): one run of n entries, one insert component."""
    homes = first_home + (np.arange(n, dtype=np.uint64) % np.uint64(span))
    x = (np.arange(n, dtype=np.uint64) + np.uint64(1 + salt)) * np.uint64(cap) + homes
    out = np.zeros((n, ks), np.uint8)
    out[:, :8] = x.view(np.uint8).reshape(n, 8)
    return out


@pytest.mark.parametrize("graph", [False, True])
def test_batch_queue_fallbacks(graph):
    """The queue's slow paths against the oracle: an insert whose component
    (10,000 ops homed in 100 slots) is too large for the block pass and runs
    on the op's end unit; a remove of 3,000 keys of that cluster (one group
    between EMPTY slots, too large for a warp) and removes on a table with no
    EMPTY slot at all, both on the end unit's ordered 32-op chunks; gets after
    each."""
    import flash_map as F

    rng = np.random.default_rng(43)
    tables = []
    ca, cb = 1 << 14, 1 << 12
    ga, oa = gpu_map(ca, 8, 8), OracleAdapter(ca, 8, 8)
    k0 = _keys(rng, ca // 4, 8)
    assert ga.bulk_insert(k0, k0) == oa.bulk_insert(k0, k0)
    tables.append({"g": ga, "o": oa, "ks": 8, "vs": 8, "known": [k0]})
    gb, ob = gpu_map(cb, 32, 128), OracleAdapter(cb, 32, 128)
    kb, vb = _keys(rng, cb, 32), _keys(rng, cb, 128)
    assert gb.bulk_insert(kb, vb) == ob.bulk_insert(kb, vb) == cb  # full: no EMPTY slot
    rm0 = kb[rng.choice(cb, 100, replace=False)]
    assert gb.bulk_remove(rm0) == ob.bulk_remove(rm0) == 100  # tombstones, still no EMPTY slot
    tables.append({"g": gb, "o": ob, "ks": 32, "vs": 128, "known": [kb]})
    kc = _clustered(ca, 10_000, 1000, 100, 8)
    kc = kc[rng.permutation(len(kc))]
    vc = _keys(rng, len(kc), 8)
    queue = [(0, F.batch.INSERT, kc, vc),
             (0, F.batch.GET, np.concatenate([kc[:3000], k0[:1000]]), None),
             (0, F.batch.REMOVE, kc[rng.choice(len(kc), 3000, replace=False)], None),
             (0, F.batch.GET, kc, None),
             (1, F.batch.REMOVE, np.concatenate([kb[rng.choice(cb, 700, replace=False)], _keys(rng, 300, 32)]), None),
             (1, F.batch.GET, kb, None)]
    g_res, g_out = run_batch(tables, queue, graph)
    o_res, o_out = oracle_replay(tables, queue)
    for i, ((ti, kind, k, v), gr, orr) in enumerate(zip(queue, g_res, o_res)):
        assert gr == orr, f"op {i} kind {kind} n {len(k)}: gpu {gr} oracle {orr}"
        if kind == F.batch.GET:
            ov, of = g_out[i]
            ev, ef = o_out[i]
            assert np.array_equal(of.astype(bool), ef) and np.array_equal(ov, ev), f"op {i}"
    for t in tables:
        assert t["g"].len() == t["o"].len()
        for x, y in zip(t["g"].snapshot(), t["o"].snapshot()):
            assert np.array_equal(x, y)
