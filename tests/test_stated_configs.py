"""The account-shape and skewed duplicate-heavy workloads at their stated
sizes, on the GPU through the C ABI against the sequential CPU oracle.

  * account shape: FlashMap<[u8;32],[u8;128]>, with_capacity(10,000,000)
    (2^24 slots), 8,000,000 distinct pairs inserted as 80 bulk_insert calls
    of 100,000, one bulk_get of 8,000,000 keys (half present, half fresh
    random keys, shuffled), one bulk_remove of a random 10% of the present
    keys (800,000), then every key again;
  * skewed: FlashMap<u64,u64>, with_capacity(100,000,000) (2^27 slots),
    filled to 0.9 of the capacity with 4,000,000-key batches of which 20% are
    repeats of keys earlier in the same batch carrying new values (the later
    position wins), then 10 bulk_get batches of 5,000,000 (90% Zipf(1.1)
    over the present keys, 10% absent) with a 1,000,000-key bulk_remove after
    every other one.

Each call's returned count, len, every get result (found mask and value
bytes) and the whole table after the inserts and at the end (metadata word
of every slot, key and value bytes of every occupied slot) must equal the
oracle's: integer data, compared bit for bit.  Keys and values are seeded
uniform random bytes (numpy), of the configurations' shapes and sizes.
Each test holds about 3-4 GB on the device and 6-8 GB of host memory."""
import numpy as np
import pytest

from fm_testutil import OracleAdapter, gpu_map

pytestmark = pytest.mark.gpu


def _same_layout(g, o):
    gf, gk, gv = g.snapshot()
    of, ok, ov = o.snapshot()
    assert np.array_equal(gf, of), f"flags differ at {np.nonzero(gf != of)[0][:10]}"
    del gf, of
    assert np.array_equal(gk, ok), "keys differ"
    del gk, ok
    assert np.array_equal(gv, ov), "values differ"


def _same_gets(g, o, q):
    gv, gfnd = g.bulk_get(q)
    ov, ofnd = o.bulk_get(q)
    assert np.array_equal(gfnd, ofnd), f"found differs at {np.nonzero(gfnd != ofnd)[0][:10]}"
    assert np.array_equal(gv, ov), "values differ"
    return int(gfnd.sum())


def test_account_shape_stated_size():
    cap_req, n, call = 10_000_000, 8_000_000, 100_000
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    vals = rng.integers(0, 256, (n, 128), dtype=np.uint8)
    g = gpu_map(cap_req, 32, 128)
    o = OracleAdapter(cap_req, 32, 128)
    assert g.capacity() == o.capacity() == 1 << 24
    for b in range(0, n, call):
        assert g.bulk_insert(keys[b:b + call], vals[b:b + call]) == o.bulk_insert(keys[b:b + call],
                                                                                 vals[b:b + call])
    assert g.len() == o.len() == n  # distinct keys (collisions of 32 random bytes are negligible)
    _same_layout(g, o)
    q = np.concatenate([keys[rng.choice(n, n // 2, replace=False)],
                        rng.integers(0, 256, (n - n // 2, 32), dtype=np.uint8)])
    q = q[rng.permutation(n)]
    assert _same_gets(g, o, q) == n // 2
    del q
    rm = keys[rng.choice(n, n // 10, replace=False)]
    assert g.bulk_remove(rm) == o.bulk_remove(rm) == n // 10
    assert g.len() == o.len() == n - n // 10
    _same_gets(g, o, keys)
    _same_layout(g, o)


def test_skewed_duplicate_heavy_stated_size():
    cap_req, batch = 100_000_000, 4_000_000
    rng = np.random.default_rng(4)
    g = gpu_map(cap_req, 8, 8)
    o = OracleAdapter(cap_req, 8, 8)
    cap = g.capacity()
    assert cap == o.capacity() == 1 << 27
    target = int(cap * 0.9)
    present = []
    while o.len() < target:
        b = min(batch, int((target - o.len()) / 0.8) + 1)
        nfresh = b - b // 5
        fresh = rng.integers(0, 1 << 64, nfresh, dtype=np.uint64)  # 2-bit packed 32-mers: uniform 64 bits
        fresh = fresh[: max(1, min(nfresh, target - o.len()))]
        rep = fresh[rng.integers(0, len(fresh), b // 5)]
        keys = np.concatenate([fresh, rep])
        keys = keys[rng.permutation(len(keys))]
        vals = rng.integers(0, 1 << 64, len(keys), dtype=np.uint64)
        assert g.bulk_insert(keys, vals) == o.bulk_insert(keys, vals)
        assert g.len() == o.len()
        present.append(fresh)
    assert o.len() == target
    _same_layout(g, o)
    present = np.concatenate(present)
    for r in range(10):
        nz = 4_500_000
        z = np.minimum(rng.zipf(1.1, nz) - 1, len(present) - 1)
        q = np.concatenate([present[z], rng.integers(0, 1 << 64, 5_000_000 - nz, dtype=np.uint64)])
        q = q[rng.permutation(len(q))]
        _same_gets(g, o, q)
        if r % 2 == 1:
            rm = present[rng.integers(0, len(present), 1_000_000)]
            assert g.bulk_remove(rm) == o.bulk_remove(rm)
            assert g.len() == o.len()
    _same_layout(g, o)
