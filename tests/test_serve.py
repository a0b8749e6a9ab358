"""Served form: requests arriving as a Poisson stream are served with
continuous batching; each request's result in the mix must equal its result
alone, i.e. the sequential oracle replaying the requests one at a time in
arrival order (get values and found masks, insert/remove counts, TableFull),
and the final table must match the oracle's slot for slot."""
import numpy as np
import pytest

from fm_testutil import OracleAdapter, gpu_map

pytestmark = pytest.mark.gpu


def make_requests(seed, ks, vs, present, n_req=240, rate=20000.0, sizes=(16, 20000)):
    import flash_map as F
    from flash_map.serve import Request

    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n_req))
    reqs = []
    known = [present]
    for i in range(n_req):
        kind = int(rng.choice([F.batch.INSERT, F.batch.GET, F.batch.REMOVE], p=[0.3, 0.6, 0.1]))
        n = int(np.exp(rng.uniform(np.log(sizes[0]), np.log(sizes[1]))))
        if kind == F.batch.INSERT:
            k = rng.integers(0, 256, (n, ks), dtype=np.uint8)
            v = rng.integers(0, 256, (n, vs), dtype=np.uint8)
            known.append(k)
        else:
            pool = np.concatenate(known)
            npres = int(n * 0.8)
            r = np.minimum((rng.random(npres) ** 10 * len(pool)).astype(np.int64), len(pool) - 1)  # skewed
            k = np.concatenate([pool[r], rng.integers(0, 256, (n - npres, ks), dtype=np.uint8)])
            k = k[rng.permutation(n)]
            v = None
        reqs.append(Request(kind, k, v, arrival=float(t[i])))
    return reqs


@pytest.mark.parametrize("piece", [None, 1000])
@pytest.mark.parametrize("shape", [(32, 128), (8, 8)])
def test_served_results_equal_arrival_order_replay(shape, piece, monkeypatch):
    """piece=1000: requests go through the server in pieces of 1000 keys
    (multi-piece gets, removes and inserts, the whole-request TableFull
    precheck of a pieced insert)."""
    import flash_map as F
    import flash_map.serve as S
    from flash_map.serve import FlashMapServer

    if piece:
        monkeypatch.setattr(S, "PIECE", piece)

    ks, vs = shape
    cap = 1 << 18
    rng = np.random.default_rng(6)
    g = gpu_map(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    pk = rng.integers(0, 256, (int(cap * 0.45), ks), dtype=np.uint8)
    pv = rng.integers(0, 256, (len(pk), vs), dtype=np.uint8)
    assert g.bulk_insert(pk, pv) == o.bulk_insert(pk, pv)
    reqs = make_requests(6, ks, vs, pk)
    srv = FlashMapServer(g, budget=64 << 20)
    srv.warmup()  # must leave the served table as it is
    srv.serve(reqs, realtime=True)
    assert srv.batches < len(reqs)  # requests were coalesced into batches
    for i, r in enumerate(reqs):
        assert r.done >= r.arrival
        if r.kind == F.batch.GET:
            ev, ef = o.bulk_get(r.keys)
            assert np.array_equal(r.out_found.astype(bool), ef), f"request {i}"
            assert np.array_equal(r.out_values, ev), f"request {i}"
        elif r.kind == F.batch.INSERT:
            import oracle as O

            try:
                exp = (o.bulk_insert(r.keys, r.values), 0)
            except O.TableFull:
                exp = (0, 5)
            assert (r.result, r.status) == exp, f"request {i}"
        else:
            assert (r.result, r.status) == (o.bulk_remove(r.keys), 0), f"request {i}"
    assert g.len() == o.len()
    gf, gk, gv = g.snapshot()
    of_, ok, ov = o.snapshot()
    assert np.array_equal(gf, of_) and np.array_equal(gk, ok) and np.array_equal(gv, ov)


def test_served_budget_smaller_than_a_request():
    """A request larger than the whole staging budget is still served (alone),
    and the results still equal the arrival-order replay."""
    import flash_map as F
    from flash_map.serve import FlashMapServer

    cap = 1 << 16
    rng = np.random.default_rng(8)
    g = gpu_map(cap, 8, 8)
    o = OracleAdapter(cap, 8, 8)
    reqs = make_requests(8, 8, 8, rng.integers(0, 256, (64, 8), dtype=np.uint8), n_req=40, sizes=(16, 4000))
    srv = FlashMapServer(g, budget=4096)
    srv.serve(reqs, realtime=False)
    for r in reqs:
        if r.kind == F.batch.GET:
            ev, ef = o.bulk_get(r.keys)
            assert np.array_equal(r.out_found.astype(bool), ef) and np.array_equal(r.out_values, ev)
        elif r.kind == F.batch.INSERT:
            assert r.result == o.bulk_insert(r.keys, r.values)
        else:
            assert r.result == o.bulk_remove(r.keys)
