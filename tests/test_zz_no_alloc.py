"""fm_bulk_insert_device_noalloc: the insert for processes that must not
allocate device memory once they run -- device memory reserved up front under
a fixed budget, or held by a caching allocator such as PyTorch's, where a
cudaMalloc at insert time could fail and a cudaFree would synchronize the
device.  It keeps its per-call scratch in a fixed array inside the library.

Called here through the C ABI from an ordinary host thread and checked
against fm_bulk_insert_device on the same inputs, call after call (counts,
len, every get result and the whole table layout must be identical: integer
data, so the tolerance is zero), against the sequential CPU oracle, and for
unchanged free device memory around calls after the first.  This file is
collected last so that a run stopping at the first failure has already run
every other test."""
import ctypes as C

import numpy as np
import pytest

from fm_testutil import OracleAdapter

pytestmark = pytest.mark.gpu


def _noalloc_insert(m, d_keys, d_vals, n, stream):
    from flash_map import _native
    from flash_map.errors import raise_for_status

    out = C.c_uint64(0)
    rc = _native.load_library().fm_bulk_insert_device_noalloc(m._h, d_keys.data_ptr(), d_vals.data_ptr(), n,
                                                                C.byref(out), stream.cuda_stream)
    raise_for_status(rc, _native.last_error(), m.len(), m.capacity())
    return out.value


def _same_tables(a, b):
    assert a.len() == b.len()
    for x, y in zip(a.snapshot(), b.snapshot()):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("shape", [(32, 128), (8, 8)])
def test_noalloc_insert_matches_allocating_insert(shape):
    import torch

    import flash_map as F

    ks, vs = shape
    cap = 1 << 17  # the precheck counts every op of a call (len + n <= capacity)
    rng = np.random.default_rng(ks + vs)
    a = F.FlashMap(cap, ks, vs)  # allocating path
    b = F.FlashMap(cap, ks, vs)  # allocation-free path
    o = OracleAdapter(cap, ks, vs)
    s = torch.cuda.current_stream()
    n1, n2 = 40000, 30000
    k1 = rng.integers(0, 256, (n1, ks), dtype=np.uint8)
    v1 = rng.integers(0, 256, (n1, vs), dtype=np.uint8)
    k1[-500:] = k1[:500]  # in-batch duplicates: later position wins
    # second call: updates of first-call keys, new keys, and duplicates
    k2 = np.concatenate([k1[rng.choice(n1, n2 // 2, replace=False)],
                         rng.integers(0, 256, (n2 - n2 // 2, ks), dtype=np.uint8)])
    k2 = k2[rng.permutation(n2)]
    v2 = rng.integers(0, 256, (n2, vs), dtype=np.uint8)
    for kk, vv in ((k1, v1), (k2, v2)):
        dk = torch.from_numpy(kk).cuda()
        dv = torch.from_numpy(vv).cuda()
        ca = a.bulk_insert_device(dk, dv, len(kk), s)
        cb = _noalloc_insert(b, dk, dv, len(kk), s)
        torch.cuda.synchronize()
        assert ca == cb == o.bulk_insert(kk, vv)
        _same_tables(a, b)
        _same_tables(b, o)
    q = np.concatenate([k1, k2, rng.integers(0, 256, (5000, ks), dtype=np.uint8)])
    va, fa = a.bulk_get(q)
    vb, fb = b.bulk_get(q)
    assert np.array_equal(fa, fb) and np.array_equal(va, vb)


@pytest.mark.parametrize("shape", [(32, 128), (8, 8)])
def test_noalloc_insert_after_removes_near_full(shape):
    """Removes first (tombstones to reuse, a raised largest stored distance
    travelling into and out of the library's array), then inserts that take
    the table past load 0.95, where rounds stall and the remaining ops run one
    at a time; then a remove after them.  Free device memory is the same
    before and after every call but the first."""
    import torch

    import flash_map as F

    ks, vs = shape
    cap = 1 << 15
    rng = np.random.default_rng(7 + ks)
    a = F.FlashMap(cap, ks, vs)
    b = F.FlashMap(cap, ks, vs)
    o = OracleAdapter(cap, ks, vs)
    s = torch.cuda.current_stream()
    k0 = rng.integers(0, 256, (int(cap * 0.8), ks), dtype=np.uint8)
    v0 = rng.integers(0, 256, (len(k0), vs), dtype=np.uint8)
    dk, dv = torch.from_numpy(k0).cuda(), torch.from_numpy(v0).cuda()
    assert a.bulk_insert_device(dk, dv, len(k0), s) == _noalloc_insert(b, dk, dv, len(k0), s) == \
        o.bulk_insert(k0, v0)
    rm = k0[rng.choice(len(k0), len(k0) // 4, replace=False)]
    assert a.bulk_remove(rm) == b.bulk_remove(rm) == o.bulk_remove(rm)
    _same_tables(a, b)
    room = cap - b.len()
    sizes = [room // 2, room // 2 - 64, 60]  # loads about 0.8, 0.996, 0.998
    for n in sizes:
        kk = rng.integers(0, 256, (n, ks), dtype=np.uint8)
        vv = rng.integers(0, 256, (n, vs), dtype=np.uint8)
        dk, dv = torch.from_numpy(kk).cuda(), torch.from_numpy(vv).cuda()
        ca = a.bulk_insert_device(dk, dv, n, s)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        cb = _noalloc_insert(b, dk, dv, n, s)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0  # nothing allocated or freed
        assert ca == cb == o.bulk_insert(kk, vv)
        _same_tables(a, b)
        _same_tables(b, o)
    assert b.load_factor() > 0.95
    rm2 = np.concatenate([k0[: len(k0) // 2], kk])
    assert a.bulk_remove(rm2) == b.bulk_remove(rm2) == o.bulk_remove(rm2)
    _same_tables(a, b)
    _same_tables(b, o)


def test_noalloc_rejects_batches_above_the_limit():
    import torch

    import flash_map as F
    from flash_map import _native

    limit = 65536  # FM_NOALLOC_MAX_OPS in include/flashmap_b200.h
    m = F.FlashMap(1 << 18, 8, 8)
    keys = torch.zeros((limit + 1, 8), dtype=torch.uint8, device="cuda")
    with pytest.raises(F.KernelLaunch, match="FM_NOALLOC_MAX_OPS"):
        _noalloc_insert(m, keys, keys, limit + 1, torch.cuda.current_stream())
    assert m.len() == 0
    assert "FM_NOALLOC_MAX_OPS" in _native.last_error()
