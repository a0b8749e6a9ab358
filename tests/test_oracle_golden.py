"""The oracle against the golden fixtures (made by the reference's own
src/kernels.cu, see tests/golden/make_golden.py) and the reference's own unit
tests for the hashes (src/hash.rs:88-118)."""
import numpy as np
import pytest

import oracle as O
from fm_testutil import OracleAdapter, expected_layout, load_json, replay_layout_case


def test_identity_hash_known_answers():
    # src/hash.rs:92-104
    assert O.hash_key(bytes([1, 2, 3, 4, 5, 6, 7, 8, 99, 99]), 0) == int.from_bytes(bytes([1, 2, 3, 4, 5, 6, 7, 8]), "little")
    assert O.hash_key(bytes([0xAB, 0xCD]), 0) == 0xCDAB


def test_murmur3_reference_unit_tests():
    # src/hash.rs:107-117: different keys differ, deterministic
    assert O.hash_key(bytes([1, 2, 3, 4]), 1) != O.hash_key(bytes([5, 6, 7, 8]), 1)
    assert O.hash_key(bytes([10] * 32), 1) == O.hash_key(bytes([10] * 32), 1)


def test_hash_golden_vectors():
    vecs = load_json("hashes.json")
    assert len(vecs) > 200
    for v in vecs:
        k = bytes.fromhex(v["key"])
        assert O.hash_key(k, 0) == v["identity"], v
        assert O.hash_key(k, 1) == v["murmur3"], v


@pytest.mark.parametrize("case_id", range(7))
def test_layout_golden(case_id):
    case = load_json("layouts.json")[case_id]
    m = OracleAdapter(case["capacity"], case["key_size"], case["value_size"], case["hash_mode"])
    f, k, v = replay_layout_case(case, m)
    ef, ek, ev = expected_layout(case)
    assert np.array_equal(f, ef)
    assert np.array_equal(k, ek)
    assert np.array_equal(v, ev)


def test_capacity_rules():
    # gpu.rs:50-54 (0 -> ZeroCapacity; next_power_of_two) vs rayon_cpu.rs:64 (max 16)
    with pytest.raises(ValueError):
        O.capacity_for(0, 0)
    assert O.capacity_for(1, 0) == 1
    assert O.capacity_for(10_000_000, 0) == 1 << 24
    assert O.capacity_for(100_000_000, 0) == 1 << 27
    assert O.capacity_for(1, 1) == 16
    assert O.capacity_for(0, 1) == 16
