"""fm_bulk_insert_device_noalloc: the insert for callers that cannot allocate
GPU memory when they insert (host callbacks, where cudaMalloc is illegal;
pre-reserved memory budgets).  It keeps its scratch in a fixed array inside
the library instead of allocating.  Called here through the C ABI and checked
against fm_bulk_insert_device on the same inputs, two calls in a row: counts,
len, every get result and the whole table layout must be identical (integer
data, so the tolerance is zero).  This file is collected last so that a run
stopping at the first failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_insert(m, d_keys, d_vals, n, stream):
    from flash_map import _native
    from flash_map.errors import raise_for_status

    out = C.c_uint64(0)
    rc = _native.load_library().fm_bulk_insert_device_noalloc(m._h, d_keys.data_ptr(), d_vals.data_ptr(), n,
                                                                C.byref(out), stream.cuda_stream)
    raise_for_status(rc, _native.last_error(), m.len(), m.capacity())
    return out.value


@pytest.mark.parametrize("shape", [(32, 128), (8, 8)])
def test_noalloc_insert_matches_allocating_insert(shape):
    import torch

    import flash_map as F

    ks, vs = shape
    cap = 1 << 17  # the precheck counts every op of a call (len + n <= capacity)
    rng = np.random.default_rng(ks + vs)
    a = F.FlashMap(cap, ks, vs)  # allocating path
    b = F.FlashMap(cap, ks, vs)  # allocation-free path
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
        assert ca == cb
        assert a.len() == b.len()
        for x, y in zip(a.snapshot(), b.snapshot()):
            assert np.array_equal(x, y)
    q = np.concatenate([k1, k2, rng.integers(0, 256, (5000, ks), dtype=np.uint8)])
    va, fa = a.bulk_get(q)
    vb, fb = b.bulk_get(q)
    assert np.array_equal(fa, fb) and np.array_equal(va, vb)


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
