"""Error paths under host-side failure injection (fm_inject_fault).

The reference maps CUDA failures onto FlashMapError::GpuAlloc, Transfer and
KernelLaunch (src/error.rs:5-27; raised from src/gpu.rs:45-105, 111-191,
193-273).  A real failure cannot be provoked here without faulting a GPU, so
the library fails on the host instead: the armed site returns the error its
CUDA call would have returned and the call is not made.  Each test checks the
reported error type, that the table stays consistent (len against a recount,
layout against the oracle), and that the next call works."""
import numpy as np
import pytest

from fm_testutil import OracleAdapter

pytestmark = pytest.mark.gpu


def _load_oracle(o, g):
    """The oracle with the GPU table's state (after a failure the GPU holds
    some prefix of the failed call that the oracle cannot know)."""
    f, k, v = g.snapshot()
    o.m.flags()[:] = f
    o.m.keys()[:] = k
    o.m.values()[:] = v
    o.m.set_len(g.recount())


def _same(g, o):
    assert g.len() == o.len()
    for x, y in zip(g.snapshot(), o.snapshot()):
        assert np.array_equal(x, y)


@pytest.fixture(autouse=True)
def _disarm():
    from flash_map import _native

    yield
    _native.inject_fault(_native.FAULT_NONE)


def test_alloc_failure_at_create_and_first_insert():
    import flash_map as F
    from flash_map import _native

    _native.inject_fault(_native.FAULT_ALLOC, 2)  # the third table array
    with pytest.raises(F.GpuAlloc):
        F.FlashMap(1 << 12, 8, 8)
    g = F.FlashMap(1 << 12, 8, 8)
    o = OracleAdapter(1 << 12, 8, 8)
    rng = np.random.default_rng(1)
    k = rng.integers(0, 256, (3000, 8), dtype=np.uint8)
    _native.inject_fault(_native.FAULT_ALLOC, 0)  # the staging or scratch allocation of the first insert
    with pytest.raises(F.GpuAlloc):
        g.bulk_insert(k, k)
    assert g.len() == 0 and g.recount() == 0
    assert g.bulk_insert(k, k) == o.bulk_insert(k, k)
    _same(g, o)


def test_transfer_failure_in_a_pieced_insert_keeps_completed_pieces():
    import flash_map as F
    from flash_map import _native

    cap, n, piece = 1 << 18, 150_000, 1 << 16  # three host pieces
    rng = np.random.default_rng(2)
    k = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    v = rng.integers(0, 256, (n, 128), dtype=np.uint8)
    g = F.FlashMap(cap, 32, 128)
    o = OracleAdapter(cap, 32, 128)
    # uploads: piece 0 keys (pass 0), values (1), piece 1 keys (2), values (3),
    # piece 2 keys (4): piece 1 has not run when piece 2's upload fails
    _native.inject_fault(_native.FAULT_TRANSFER, 4)
    with pytest.raises(F.Transfer):
        g.bulk_insert(k, v)
    o.bulk_insert(k[:piece], v[:piece])
    assert g.len() == g.recount() == o.len()
    _same(g, o)
    assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
    _same(g, o)


def test_transfer_failure_in_get_leaves_table_unchanged():
    import flash_map as F
    from flash_map import _native

    rng = np.random.default_rng(3)
    k = rng.integers(0, 256, (20_000, 8), dtype=np.uint8)
    g = F.FlashMap(1 << 16, 8, 8)
    g.bulk_insert(k, k)
    before = g.snapshot()
    _native.inject_fault(_native.FAULT_TRANSFER, 1)
    with pytest.raises(F.Transfer):
        g.bulk_get(k)
    for x, y in zip(before, g.snapshot()):
        assert np.array_equal(x, y)
    vals, found = g.bulk_get(k)
    assert found.all() and np.array_equal(vals, k)


def _clustered(cap, n, first_home, span, ks):
    """n keys whose identity-hash homes lie in [first_home, first_home + span):
    a run of n entries, so stored distances reach about n."""
    homes = first_home + (np.arange(n, dtype=np.uint64) % np.uint64(span))
    x = (np.arange(n, dtype=np.uint64) + np.uint64(1)) * np.uint64(cap) + homes
    out = np.zeros((n, ks), np.uint8)
    out[:, :8] = x.view(np.uint8).reshape(n, 8)
    return out


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
def test_failed_remove_with_chunk_summaries_then_remove(shape):
    """A remove on a full table (no EMPTY slot, so every op goes to the
    rounds) whose largest stored distance is far above 256 (so the call builds
    per-chunk summaries and marks) fails after its first pass of rounds; the
    next removes on the table must still make progress and match the oracle
    from the state the failure left."""
    import flash_map as F
    from flash_map import _native

    ks, vs = shape
    cap = 1 << 13
    rng = np.random.default_rng(4 + ks)
    k = np.concatenate([_clustered(cap, 1500, 300, 40, ks),
                        rng.integers(0, 256, (cap - 1500, ks), dtype=np.uint8)])
    v = rng.integers(0, 256, (len(k), vs), dtype=np.uint8)
    g = F.FlashMap(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    assert g.bulk_insert(k, v) == o.bulk_insert(k, v) == cap
    flags = g.snapshot()[0]
    assert (flags >> 4).max() >= 256 and not ((flags & 0xF) == 0).any()
    rm = k[rng.choice(len(k), 4000, replace=False)]
    # no EMPTY slot: the direct remove leaves every op to the rounds; the
    # fault fires at the readback after the first pass of those rounds (the
    # direct remove's readback is the pass before it)
    _native.inject_fault(_native.FAULT_ROUND, 1)
    with pytest.raises(F.KernelLaunch):
        g.bulk_remove(rm)
    _load_oracle(o, g)
    assert g.len() == o.len()
    rm2 = np.concatenate([rm, k[rng.choice(len(k), 2000, replace=False)]])
    assert g.bulk_remove(rm2) == o.bulk_remove(rm2)
    _same(g, o)
    more = rng.integers(0, 256, (1000, ks), dtype=np.uint8)
    mv = rng.integers(0, 256, (1000, vs), dtype=np.uint8)
    assert g.bulk_insert(more, mv) == o.bulk_insert(more, mv)
    assert g.bulk_remove(more[::2]) == o.bulk_remove(more[::2])
    _same(g, o)


def test_unknown_fault_site_is_rejected():
    import flash_map as F
    from flash_map import _native

    with pytest.raises(F.KernelLaunch):
        _native.inject_fault(99)
