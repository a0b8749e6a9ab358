"""The reference's integration tests (tests/correctness.rs:1-392), run against
both the CPU oracle and the B200 backend (through the C ABI).  The test names
and assertions follow the reference file line by line."""
import numpy as np
import pytest

from fm_testutil import le, make_map, table_full_types

BACKENDS = ["oracle", pytest.param("gpu", marks=pytest.mark.gpu)]


@pytest.fixture(params=BACKENDS)
def kind(request):
    return request.param


def test_insert_and_get(kind):  # correctness.rs:4-22
    m = make_map(kind, 1024, 8, 8)
    i = np.arange(100, dtype=np.uint64)
    assert m.bulk_insert(le(i), le(i * 100)) == 100
    assert m.len() == 100
    vals, found = m.bulk_get(le(i))
    assert found.all()
    assert np.array_equal(vals, le(i * 100))


def test_get_missing_keys(kind):  # correctness.rs:25-39
    m = make_map(kind, 1024, 8, 8)
    i = np.arange(10, dtype=np.uint64)
    m.bulk_insert(le(i), le(i))
    _, found = m.bulk_get(le(np.arange(100, 110, dtype=np.uint64)))
    assert not found.any()


def test_update_existing_keys(kind):  # correctness.rs:42-65
    m = make_map(kind, 1024, 8, 8)
    i = np.arange(10, dtype=np.uint64)
    assert m.bulk_insert(le(i), le(i)) == 10
    assert m.bulk_insert(le(i), le(i + 1000)) == 0
    assert m.len() == 10
    vals, found = m.bulk_get(le(i))
    assert found.all() and np.array_equal(vals, le(i + 1000))


def test_remove_keys(kind):  # correctness.rs:68-95
    m = make_map(kind, 1024, 8, 8)
    i = np.arange(100, dtype=np.uint64)
    m.bulk_insert(le(i), le(i))
    assert m.len() == 100
    rk = le(np.arange(50, dtype=np.uint64))
    assert m.bulk_remove(rk) == 50
    assert m.len() == 50
    _, found = m.bulk_get(rk)
    assert not found.any()
    _, found = m.bulk_get(le(np.arange(50, 100, dtype=np.uint64)))
    assert found.all()


def test_insert_after_remove_reuses_tombstones(kind):  # correctness.rs:98-124
    m = make_map(kind, 64, 8, 8)
    i = np.arange(10, dtype=np.uint64)
    m.bulk_insert(le(i), le(i))
    m.bulk_remove(le(i))
    assert m.len() == 0
    j = np.arange(100, 110, dtype=np.uint64)
    assert m.bulk_insert(le(j), le(j * 2)) == 10
    vals, found = m.bulk_get(le(j))
    assert found.all() and np.array_equal(vals, le(j * 2))


def test_clear_resets_map(kind):  # correctness.rs:127-145
    m = make_map(kind, 1024, 8, 8)
    i = np.arange(100, dtype=np.uint64)
    m.bulk_insert(le(i), le(i))
    assert m.len() == 100
    m.clear()
    assert m.len() == 0 and m.is_empty()
    _, found = m.bulk_get(le(i))
    assert not found.any()


def test_murmur3_hash_strategy(kind):  # correctness.rs:148-164
    m = make_map(kind, 1024, 8, 8, hash_mode=1)
    i = np.arange(100, dtype=np.uint64)
    m.bulk_insert(le(i), le(i * 7))
    vals, found = m.bulk_get(le(i))
    assert found.all() and np.array_equal(vals, le(i * 7))


def test_large_keys_and_values(kind):  # correctness.rs:167-191
    m = make_map(kind, 4096, 32, 64)
    i = np.arange(500, dtype=np.uint64)
    keys, vals = le(i, 32), le(i * 42, 64)
    m.bulk_insert(keys, vals)
    assert m.len() == 500
    got, found = m.bulk_get(keys)
    assert found.all() and np.array_equal(got, vals)


def test_load_factor_and_capacity(kind):  # correctness.rs:194-199
    m = make_map(kind, 1024, 8, 8)
    assert m.load_factor() == 0.0
    assert m.capacity() >= 1024
    assert m.capacity() & (m.capacity() - 1) == 0


def test_empty_operations_are_no_ops(kind):  # correctness.rs:202-211
    m = make_map(kind, 64, 8, 8)
    empty = np.zeros((0, 8), np.uint8)
    assert m.bulk_insert(empty, empty) == 0
    vals, found = m.bulk_get(empty)
    assert len(found) == 0
    assert m.bulk_remove(empty) == 0


def test_table_full_error(kind):  # correctness.rs:214-227
    m = make_map(kind, 16, 8, 8)
    i = np.arange(16, dtype=np.uint64)
    m.bulk_insert(le(i), le(i))
    with pytest.raises(table_full_types()) as ei:
        m.bulk_insert(le([99]), le([99]))
    assert ei.value.occupied == 16 and ei.value.capacity == 16
    assert m.len() == 16  # the precheck runs before any mutation


def test_debug_formatting():  # correctness.rs:230-236 (GPU backend's repr)
    pytest.importorskip("torch")
    import torch

    if not torch.cuda.is_available():
        pytest.skip("needs a GPU")
    m = make_map("gpu", 256, 8, 8)
    s = repr(m)
    assert "FlashMap" in s and "len" in s and "capacity" in s


def test_u64_key_value_types(kind):  # correctness.rs:239-250
    m = make_map(kind, 1024, 8, 8)
    i = np.arange(50, dtype=np.uint64)
    m.bulk_insert(i, i * i)
    vals, found = m.bulk_get(i)
    assert found.all() and np.array_equal(vals.view(np.uint64).ravel(), i * i)


@pytest.mark.parametrize("load_pct", [80, 90, 95])
def test_robin_hood_high_load_correctness(kind, load_pct):  # correctness.rs:257-285
    cap = 1024
    n = cap * load_pct // 100
    m = make_map(kind, cap, 8, 8)
    i = np.arange(n, dtype=np.uint64)
    assert m.bulk_insert(le(i), le(i * 7)) == n
    assert m.len() == n
    vals, found = m.bulk_get(le(i))
    assert found.all() and np.array_equal(vals, le(i * 7))


def test_robin_hood_miss_exits_early(kind):  # correctness.rs:288-309
    cap = 1024
    n = cap * 90 // 100
    m = make_map(kind, cap, 8, 8)
    i = np.arange(n, dtype=np.uint64)
    m.bulk_insert(le(i), le(i))
    _, found = m.bulk_get(le(np.arange(10_000, 10_500, dtype=np.uint64)))
    assert not found.any()


def test_robin_hood_insert_remove_reinsert(kind):  # correctness.rs:312-362
    cap = 512
    n = cap * 80 // 100
    m = make_map(kind, cap, 8, 8)
    i = np.arange(n, dtype=np.uint64)
    m.bulk_insert(le(i), le(i))
    assert m.bulk_remove(le(np.arange(n // 2, dtype=np.uint64))) == n // 2
    j = np.arange(10_000, 10_000 + n // 2, dtype=np.uint64)
    assert m.bulk_insert(le(j), le(j * 3)) == n // 2
    surv = np.arange(n // 2, n, dtype=np.uint64)
    vals, found = m.bulk_get(le(surv))
    assert found.all() and np.array_equal(vals, le(surv))
    vals, found = m.bulk_get(le(j))
    assert found.all() and np.array_equal(vals, le(j * 3))


def test_robin_hood_update_at_high_load(kind):  # correctness.rs:365-392
    cap = 1024
    n = cap * 45 // 100
    m = make_map(kind, cap, 8, 8)
    i = np.arange(n, dtype=np.uint64)
    m.bulk_insert(le(i), le(i))
    assert m.bulk_insert(le(i), le(i + 999)) == 0
    assert m.len() == n
    vals, found = m.bulk_get(le(i))
    assert found.all() and np.array_equal(vals, le(i + 999))
