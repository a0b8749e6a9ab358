"""Shared helpers for the parity tests: a uniform map interface over the
oracle (CPU checker) and the B200 backend, seeded workload generators, and
replay of the golden fixtures."""
from __future__ import annotations

import json
import os

import numpy as np

import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


class OracleAdapter:
    """OracleMap with the FlashMap method names."""

    def __init__(self, capacity, key_size, value_size, hash_mode=0):
        self.m = O.OracleMap(capacity, key_size, value_size, hash_mode)
        self.key_size, self.value_size = key_size, value_size

    def bulk_insert(self, k, v):
        return self.m.bulk_insert(k, v)

    def bulk_get(self, k):
        return self.m.bulk_get(k)

    def bulk_remove(self, k):
        return self.m.bulk_remove(k)

    def bulk_insert_uncounted(self, k, v):
        return self.m.bulk_insert_uncounted(k, v)

    def recount(self):
        return self.m.recount()

    def clear(self):
        self.m.clear()

    def len(self):
        return len(self.m)

    def is_empty(self):
        return len(self.m) == 0

    def capacity(self):
        return self.m.capacity

    def load_factor(self):
        return len(self.m) / self.m.capacity

    def snapshot(self):
        return self.m.snapshot()


def gpu_map(capacity, key_size, value_size, hash_mode=0):
    import flash_map as F

    return F.FlashMap(capacity, key_size, value_size, F.HashStrategy(hash_mode))


def make_map(kind, capacity, key_size, value_size, hash_mode=0):
    if kind == "oracle":
        return OracleAdapter(capacity, key_size, value_size, hash_mode)
    return gpu_map(capacity, key_size, value_size, hash_mode)


def table_full_types():
    import flash_map as F

    return (O.TableFull, F.TableFull)


def le(i, size=8):
    """u64::to_le_bytes as a (n, size) uint8 array (zero-padded past 8 bytes)."""
    a = np.asarray(i, dtype=np.uint64).reshape(-1)
    b = a.view(np.uint8).reshape(len(a), 8)
    if size == 8:
        return np.ascontiguousarray(b)
    out = np.zeros((len(a), size), np.uint8)
    out[:, : min(size, 8)] = b[:, : min(size, 8)]
    return out


def load_json(name):
    with open(os.path.join(GOLDEN, name)) as fh:
        return json.load(fh)


def hx(s, cols):
    a = np.frombuffer(bytes.fromhex(s), np.uint8)
    return a.reshape(-1, cols) if cols else a.reshape(len(a), 0)


def replay_layout_case(case, m):
    """Replay a golden layout case on map `m`; returns the final snapshot."""
    ks, vs = case["key_size"], case["value_size"]
    for st in case["steps"]:
        keys = hx(st["keys"], ks)
        if st["op"] == "insert":
            c = m.bulk_insert(keys, hx(st["values"], vs))
        else:
            c = m.bulk_remove(keys)
        assert c == st["count"], (st["op"], c, st["count"])
    assert m.len() == case["len"]
    return m.snapshot()


def expected_layout(case):
    cap, ks, vs = case["capacity"], case["key_size"], case["value_size"]
    f = np.frombuffer(bytes.fromhex(case["flags"]), np.uint32)
    k = hx(case["keys"], ks)
    v = hx(case["values"], vs)
    assert len(f) == cap
    return f, k, v


# ---------------------------------------------------------------------------
# Seeded generators
# ---------------------------------------------------------------------------
def splitmix64(seed, n):
    """splitmix64 stream (Steele, Lea, Flood 2014), n outputs from `seed`."""
    x = np.uint64(seed)
    out = np.empty(n, np.uint64)
    g = np.uint64(0x9E3779B97F4A7C15)
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = x + g * idx
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        out[:] = z ^ (z >> np.uint64(31))
    return out


def mix64(x):
    with np.errstate(over="ignore"):
        z = np.asarray(x, np.uint64) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def churn_workload(rng, cap, ks, vs, rounds, narrow=True):
    """A sequence of (op, keys, values) with heavy collisions, in-batch
    duplicates and remove->insert churn (the layout-sensitive regime)."""
    ops = []
    live = []
    pool = rng.integers(0, 256, (max(cap, 64), ks), dtype=np.uint8)
    if narrow and ks >= 2:
        pool[:, 1:min(ks, 8)] = 0
        pool[:, 1] = rng.integers(0, 3, len(pool))
    occupied = 0
    for r in range(rounds):
        n = int(rng.integers(1, max(2, cap // 5)))
        if r % 3 == 2 and live:
            idx = rng.integers(0, len(live), n)
            keys = np.array([live[i] for i in idx], np.uint8).reshape(n, ks)
            ops.append(("remove", keys, None))
            continue
        keys = pool[rng.integers(0, len(pool), n)]
        vals = rng.integers(0, 256, (n, vs), dtype=np.uint8)
        if occupied + n > cap:
            break
        occupied += n
        ops.append(("insert", keys, vals))
        live.extend(list(keys))
    return ops
