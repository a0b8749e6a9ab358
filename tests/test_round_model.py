"""CPU check of the round scheduling of the insert/remove kernels: the ops a
round selects are applied in random orders and must reproduce the oracle's
sequential layout exactly (tests/round_model.py mirrors the kernel rules)."""
import numpy as np
import pytest

import oracle as O
from round_model import ModelTable


def _compare(m, o):
    mf, mk, mv = m.snapshot()
    of, ok, ov = o.snapshot()
    assert np.array_equal(mf, of)
    assert np.array_equal(mk, ok)
    assert np.array_equal(mv, ov)


@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("cap", [16, 64, 256])
def test_round_scheduling_matches_sequential(seed, cap):
    rng = np.random.default_rng(seed * 1000 + cap)
    ks, vs = 8, 4
    mode = seed % 2
    m = ModelTable(cap, ks, vs, mode)
    o = O.OracleMap(cap, ks, vs, mode)
    # narrow key space -> long clusters, duplicates and collisions
    pool = [bytes(rng.integers(0, 256, 1, dtype=np.uint8)) + bytes([int(rng.integers(0, 3))]) + bytes(6)
            for _ in range(cap * 2)]
    live = []
    for r in range(14):
        if r % 3 == 2 and live:
            n = int(rng.integers(1, max(2, cap // 4)))
            keys = [live[int(i)] for i in rng.integers(0, len(live), n)]
            a = m.bulk_remove(keys, rng)
            b = o.bulk_remove(np.frombuffer(b"".join(keys), np.uint8).reshape(n, ks))
            assert a == b
        else:
            n = int(rng.integers(1, max(2, cap // 3)))
            if len(o) + n > cap:
                continue
            keys = [pool[int(i)] for i in rng.integers(0, len(pool), n)]
            vals = [bytes(rng.integers(0, 256, vs, dtype=np.uint8)) for _ in range(n)]
            a = m.bulk_insert(keys, vals, rng)
            b = o.bulk_insert(np.frombuffer(b"".join(keys), np.uint8).reshape(n, ks),
                              np.frombuffer(b"".join(vals), np.uint8).reshape(n, vs))
            assert a == b
            live.extend(keys)
        assert m.len == len(o)
        _compare(m, o)


def test_round_scheduling_full_table_serial():
    """No free slot anywhere: one op per round (the serial fallback)."""
    rng = np.random.default_rng(3)
    cap = 16
    m = ModelTable(cap, 8, 8)
    o = O.OracleMap(cap, 8, 8)
    keys = [int(i * 16).to_bytes(8, "little") for i in range(14)]
    m.bulk_insert(keys, keys, rng)
    o.bulk_insert(np.frombuffer(b"".join(keys), np.uint8).reshape(14, 8),
                  np.frombuffer(b"".join(keys), np.uint8).reshape(14, 8))
    extra = [int(i).to_bytes(8, "little") for i in range(100, 108)]
    m.len = 0  # bypass the precheck like the uncounted insert
    m.bulk_insert(extra, extra, rng)
    with pytest.raises(O.ProbeLimit):
        o.bulk_insert_uncounted(np.frombuffer(b"".join(extra), np.uint8).reshape(8, 8),
                                np.frombuffer(b"".join(extra), np.uint8).reshape(8, 8))
    _compare(m, o)
