"""Generate the golden fixtures in this directory from the reference's own code.

Runs the reference's src/kernels.cu compiled as host C++ (oracle/_ref,
built by `make -C oracle ref` from the sources under the reference tree):
  * hashes.json  -- fm_identity_hash / fm_murmur3_hash outputs for seeded
                    keys of every length 0..64 (kernels.cu:42-88, which equal
                    src/hash.rs:32-77 line for line);
  * layouts.json -- final table layouts after seeded insert sequences run by
                    flashmap_bulk_insert (kernels.cu:224-313), one simulated
                    thread at a time in index order, over tables whose
                    tombstones were placed by removes (the remove rule of
                    src/rayon_cpu.rs:276-323), including in-batch duplicate
                    keys and tombstone reuse.

Only runs where the reference tree exists; the fixtures are committed.
Usage: python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402


def hashes():
    rng = np.random.default_rng(20261203)
    out = []
    R = O.ref_host()
    for ksz in range(0, 65):
        for rep in range(4):
            k = rng.integers(0, 256, max(ksz, 1), dtype=np.uint8)[:ksz]
            if rep == 1:
                k = np.zeros(ksz, np.uint8)
            buf = np.ascontiguousarray(k) if ksz else np.zeros(1, np.uint8)
            out.append({
                "key": bytes(k).hex(),
                "identity": int(R.ref_identity_hash(buf.ctypes.data, ksz)),
                "murmur3": int(R.ref_murmur3_hash(buf.ctypes.data, ksz)),
            })
    # the reference's own unit-test inputs (src/hash.rs:92-117)
    for k in ([1, 2, 3, 4, 5, 6, 7, 8, 99, 99], [0xAB, 0xCD], [1, 2, 3, 4], [5, 6, 7, 8], [10] * 32):
        buf = np.array(k, np.uint8)
        out.append({"key": bytes(buf).hex(),
                    "identity": int(R.ref_identity_hash(buf.ctypes.data, len(k))),
                    "murmur3": int(R.ref_murmur3_hash(buf.ctypes.data, len(k)))})
    return out


def layouts():
    cases = []
    rng = np.random.default_rng(7)
    specs = [(64, 8, 8, 0), (256, 8, 8, 0), (256, 8, 8, 1), (128, 32, 64, 0), (64, 5, 3, 1), (32, 12, 20, 0),
             (16, 8, 8, 0)]
    for cap, ks, vs, mode in specs:
        rt = O.RefHostTable(cap, ks, vs, mode)
        om = O.OracleMap(cap, ks, vs, mode)
        steps = []
        live = []
        for rnd in range(12):
            n = int(rng.integers(1, max(2, cap // 6)))
            keys = rng.integers(0, 256, (n, ks), dtype=np.uint8)
            keys[:, 1:min(ks, 8)] = 0  # few distinct homes: long clusters
            if live and n > 3:
                keys[: n // 3] = np.array(live)[rng.integers(0, len(live), n // 3)]
            if n > 4:
                keys[-1] = keys[0]  # in-batch duplicate, later position wins
            vals = rng.integers(0, 256, (n, vs), dtype=np.uint8)
            if len(om) + n > cap:
                break
            c_ref = rt.bulk_insert(keys, vals)
            c_or = om.bulk_insert(keys, vals)
            assert c_ref == c_or
            steps.append({"op": "insert", "keys": keys.tobytes().hex(), "values": vals.tobytes().hex(),
                          "count": int(c_ref)})
            live = list({bytes(k): k for k in list(live) + list(keys)}.values())
            if rnd % 2 == 1 and live:
                rm = np.array(live)[rng.integers(0, len(live), max(1, len(live) // 4))]
                r = om.bulk_remove(rm)
                steps.append({"op": "remove", "keys": rm.tobytes().hex(), "count": int(r)})
                rt.load(om.flags().copy(), om.keys().copy(), om.values().copy())
        f, k, v = rt.snapshot()
        cases.append({"capacity": cap, "key_size": ks, "value_size": vs, "hash_mode": mode, "steps": steps,
                      "flags": f.tobytes().hex(), "keys": k.tobytes().hex(), "values": v.tobytes().hex(),
                      "len": int(len(om))})
    return cases


if __name__ == "__main__":
    O.build()
    with open(os.path.join(HERE, "hashes.json"), "w") as fh:
        json.dump(hashes(), fh, indent=0)
    with open(os.path.join(HERE, "layouts.json"), "w") as fh:
        json.dump(layouts(), fh, indent=0)
    print("wrote hashes.json, layouts.json")
