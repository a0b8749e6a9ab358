"""AsyncFlashMap (the counterpart of src/async_map.rs:32-147) and the plain
per-request server built on it.

The reference wraps the map in an RwLock and runs each bulk call on
spawn_blocking: gets share the read lock, insert / remove / clear take the
write lock (async_map.rs:48-93).  Checked here: the lock lets readers overlap
and keeps writers alone (CPU); gets issued together between writes all see
the state after the last write, equal to the oracle (GPU); and the plain
server's per-request results equal the arrival-order replay (GPU)."""
import threading

import numpy as np
import pytest

from fm_testutil import OracleAdapter, gpu_map


def test_rwlock_readers_overlap_and_writers_are_alone():
    from flash_map.async_map import _RwLock

    lock = _RwLock()
    both_in = threading.Barrier(2, timeout=5)  # two readers must be inside at once
    log = []

    def reader(i):
        lock.acquire_read()
        try:
            both_in.wait()
            log.append(("r", i))
        finally:
            lock.release_read()

    ts = [threading.Thread(target=reader, args=(i,)) for i in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(10)
    assert sorted(log) == [("r", 0), ("r", 1)]

    # a writer waits for the reader inside, and a reader arriving meanwhile
    # waits for the writer (writer preference)
    inside = threading.Event()
    release = threading.Event()
    order = []

    def long_reader():
        lock.acquire_read()
        inside.set()
        release.wait(5)
        order.append("reader1 out")
        lock.release_read()

    def writer():
        lock.acquire_write()
        order.append("writer")
        lock.release_write()

    def late_reader():
        lock.acquire_read()
        order.append("reader2")
        lock.release_read()

    t1 = threading.Thread(target=long_reader)
    t1.start()
    inside.wait(5)
    t2 = threading.Thread(target=writer)
    t2.start()
    while not lock._waiting_writers:
        pass
    t3 = threading.Thread(target=late_reader)
    t3.start()
    release.set()
    for t in (t1, t2, t3):
        t.join(10)
    assert order == ["reader1 out", "writer", "reader2"]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
def test_async_map_concurrent_gets_between_ordered_writes(shape):
    import asyncio

    import flash_map as F

    ks, vs = shape
    cap = 1 << 16
    rng = np.random.default_rng(11)
    g = gpu_map(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    am = F.AsyncFlashMap(g)

    async def run():
        present = []
        for phase in range(4):
            k = rng.integers(0, 256, (5000, ks), dtype=np.uint8)
            v = rng.integers(0, 256, (5000, vs), dtype=np.uint8)
            assert await am.bulk_insert(k, v) == o.bulk_insert(k, v)
            present.append(k)
            pool = np.concatenate(present)
            qs = [np.concatenate([pool[rng.integers(0, len(pool), 3000)],
                                  rng.integers(0, 256, (1000, ks), dtype=np.uint8)]) for _ in range(8)]
            res = await asyncio.gather(*(am.bulk_get(q) for q in qs))  # share the read lock
            for q, (gv, gf) in zip(qs, res):
                ov, of = o.bulk_get(q)
                assert np.array_equal(gf, of) and np.array_equal(gv, ov)
            rm = pool[rng.integers(0, len(pool), 2000)]
            assert await am.bulk_remove(rm) == o.bulk_remove(rm)
            assert am.len() == o.len()
        await am.clear()
        assert am.is_empty()

    asyncio.run(run())


@pytest.mark.gpu
@pytest.mark.parametrize("realtime", [True, False])
def test_async_plain_server_equals_arrival_order_replay(realtime):
    import flash_map as F
    import oracle as O
    from flash_map.serve import AsyncPlainServer
    from test_serve import make_requests

    ks, vs = 32, 128
    cap = 1 << 18
    rng = np.random.default_rng(12)
    g = gpu_map(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    pk = rng.integers(0, 256, (int(cap * 0.45), ks), dtype=np.uint8)
    pv = rng.integers(0, 256, (len(pk), vs), dtype=np.uint8)
    assert g.bulk_insert(pk, pv) == o.bulk_insert(pk, pv)
    reqs = make_requests(12, ks, vs, pk, n_req=200)
    AsyncPlainServer(g).serve(reqs, realtime=realtime)
    for i, r in enumerate(reqs):
        assert r.done >= r.arrival or not realtime
        if r.kind == F.batch.GET:
            ev, ef = o.bulk_get(r.keys)
            assert np.array_equal(r.out_found.astype(bool), ef), f"request {i}"
            assert np.array_equal(r.out_values, ev), f"request {i}"
        elif r.kind == F.batch.INSERT:
            try:
                exp = (o.bulk_insert(r.keys, r.values), 0)
            except O.TableFull:
                exp = (0, 5)
            assert (r.result, r.status) == exp, f"request {i}"
        else:
            assert (r.result, r.status) == (o.bulk_remove(r.keys), 0), f"request {i}"
    assert g.len() == o.len()
    for x, y in zip(g.snapshot(), o.snapshot()):
        assert np.array_equal(x, y)
