"""Every lookup kernel configuration the autotuner can choose (lanes per
query 1 / 4 / 8 / 16 / 32; with one lane, 1, 2 or 4 queries per thread probed
in lockstep), forced through the tuning cache that fm_autotune reads, must
give the sequential oracle's results bit for bit: found mask and value bytes,
hits and misses, on tables with tombstones."""
import numpy as np
import pytest

from fm_testutil import OracleAdapter, gpu_map

pytestmark = pytest.mark.gpu

CONFIGS = [(1, 64, 1), (1, 32, 2), (1, 16, 4), (4, 32, 1), (8, 16, 1), (16, 8, 1), (32, 8, 1)]
SHAPES = {(8, 8): 0, (32, 128): 1, (32, 64): 2, (32, 32): 3, (8, 32): 4}


def _force(tmp_path, lanes, bps, qpt):
    from flash_map import _native

    path = tmp_path / f"tune_{lanes}_{bps}_{qpt}.txt"
    with open(path, "w") as f:
        for sh in SHAPES.values():
            for b in range(3):  # load buckets
                f.write(f"{sh} {b} {lanes} {bps} {qpt}\n")
    _native.autotune(0, str(path))


@pytest.mark.parametrize("shape", [(8, 8), (32, 128)])
def test_every_lookup_configuration_matches_the_oracle(shape, tmp_path):
    ks, vs = shape
    cap = 1 << 16
    rng = np.random.default_rng(60 + ks)
    g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
    k = rng.integers(0, 256, (int(cap * 0.8), ks), dtype=np.uint8)
    v = rng.integers(0, 256, (len(k), vs), dtype=np.uint8)
    assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
    rm = k[rng.choice(len(k), len(k) // 10, replace=False)]
    assert g.bulk_remove(rm) == o.bulk_remove(rm)
    q = np.concatenate([k[rng.integers(0, len(k), 30_001)], rng.integers(0, 256, (20_003, ks), dtype=np.uint8)])
    ev, ef = o.bulk_get(q)
    try:
        for lanes, bps, qpt in CONFIGS:
            _force(tmp_path, lanes, bps, qpt)
            gv, gf = g.bulk_get(q)
            assert np.array_equal(gf, ef), (lanes, bps, qpt)
            assert np.array_equal(gv, ev), (lanes, bps, qpt)
    finally:
        _force(tmp_path, 1, 64, 1)  # the untuned default for the tests after this one


def test_autotune_writes_lookup_and_insert_choices(tmp_path):
    """fm_autotune times the lookup configurations and the insert warp pass's
    tile width per record shape and load bucket and writes both to its cache;
    inserts and lookups under the tuned choices still match the oracle."""
    from flash_map import _native

    path = tmp_path / "tune.txt"
    _native.autotune(0, str(path))  # no cache yet: measures and writes it
    lines = path.read_text().split("\n")
    gets = [x for x in lines if x and not x.startswith("ins")]
    ins = [x.split() for x in lines if x.startswith("ins")]
    assert len(gets) == 5 * 3 and len(ins) == 5 * 3
    assert all(int(x[3]) in (8, 16, 32) for x in ins)
    _native.autotune(0, str(path))  # read back from the cache
    rng = np.random.default_rng(71)
    for ks, vs in ((8, 8), (32, 128)):
        cap = 1 << 15
        g, o = gpu_map(cap, ks, vs), OracleAdapter(cap, ks, vs)
        for frac in (0.5, 0.3, 0.1):
            k = rng.integers(0, 256, (int(cap * frac), ks), dtype=np.uint8)
            v = rng.integers(0, 256, (len(k), vs), dtype=np.uint8)
            assert g.bulk_insert(k, v) == o.bulk_insert(k, v)
        for x, y in zip(g.snapshot(), o.snapshot()):
            assert np.array_equal(x, y)
