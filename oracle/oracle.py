"""ctypes front end for the CPU oracle (``libfm_oracle.so``) and for the
reference's own ``src/kernels.cu`` compiled as host code (``_ref/libref_host.so``).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import this module; the product package
(``flash_map``) never does.

The oracle restates bajpainaman/flash-map 0.5.0's ``src/rayon_cpu.rs`` with
every bulk call applied one operation at a time in index order (the
single-threaded semantics), ``src/hash.rs`` for the hashes, the load-factor
precheck of ``src/gpu.rs:198-206`` and the capacity rule of
``src/gpu.rs:50-54``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfm_oracle.so")
REF_HOST_PATH = os.path.join(HERE, "_ref", "libref_host.so")
# The reference source tree (bajpainaman/flash-map 0.5.0), needed only to
# build the checker under _ref/; FLASHMAP_REFERENCE_TREE names it.
REF_TREE = os.environ.get("FLASHMAP_REFERENCE_TREE", "")

EMPTY, OCCUPIED, TOMBSTONE, INSERTING = 0, 1, 2, 3
ERR_TABLE_FULL = 5
ERR_ZERO_CAPACITY = 6
ERR_PROBE_LIMIT = 9


class _Traffic(C.Structure):
    _fields_ = [
        ("ops", C.c_uint64),
        ("table_sectors_read", C.c_uint64),
        ("table_sectors_written", C.c_uint64),
        ("stream_bytes_in", C.c_uint64),
        ("stream_bytes_out", C.c_uint64),
    ]


def build(quiet: bool = True) -> None:
    """Compile the oracle (and, when the reference tree exists, the reference
    checker).  Only the checker is built here; nothing is run."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True, stdout=out)
    if REF_TREE and os.path.isdir(os.path.join(REF_TREE, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_TREE}"], check=True, stdout=out)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        u8p = C.POINTER(C.c_uint8)
        vp = C.c_void_p
        L.fmo_create.restype = vp
        L.fmo_create.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        L.fmo_destroy.argtypes = [vp]
        L.fmo_capacity_for.argtypes = [C.c_uint64, C.c_int, C.POINTER(C.c_uint64)]
        L.fmo_hash.restype = C.c_uint64
        L.fmo_hash.argtypes = [vp, C.c_uint32, C.c_uint32]
        L.fmo_bulk_insert.argtypes = [vp, vp, vp, C.c_uint64, C.POINTER(C.c_uint64)]
        L.fmo_bulk_insert_uncounted.restype = C.c_int
        L.fmo_bulk_insert_uncounted.argtypes = [vp, vp, vp, C.c_uint64]
        L.fmo_bulk_get.argtypes = [vp, vp, C.c_uint64, vp, vp]
        L.fmo_bulk_remove.restype = C.c_uint64
        L.fmo_bulk_remove.argtypes = [vp, vp, C.c_uint64]
        L.fmo_clear.argtypes = [vp]
        L.fmo_recount.restype = C.c_uint64
        L.fmo_recount.argtypes = [vp]
        L.fmo_len.restype = C.c_uint64
        L.fmo_len.argtypes = [vp]
        L.fmo_capacity.restype = C.c_uint64
        L.fmo_capacity.argtypes = [vp]
        for name in ("fmo_flags", "fmo_keys", "fmo_values"):
            getattr(L, name).restype = vp
            getattr(L, name).argtypes = [vp]
        L.fmo_set_len.argtypes = [vp, C.c_uint64]
        L.fmo_traffic_enable.argtypes = [vp, C.c_int]
        L.fmo_traffic_get.argtypes = [vp, C.c_int, C.POINTER(_Traffic)]
        L.fmo_traffic_reset.argtypes = [vp]
        L.fmo_mt_bulk_insert.argtypes = [vp, vp, vp, C.c_uint64, C.POINTER(C.c_uint64), C.c_int]
        L.fmo_mt_bulk_get.argtypes = [vp, vp, C.c_uint64, vp, vp, C.c_int]
        L.fmo_mt_bulk_remove.restype = C.c_uint64
        L.fmo_mt_bulk_remove.argtypes = [vp, vp, C.c_uint64, C.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def as_key_bytes(keys, key_size: int) -> np.ndarray:
    """Keys as a C-contiguous (n, key_size) uint8 array."""
    a = np.asarray(keys)
    if a.dtype == np.uint8 and a.ndim == 2:
        assert a.shape[1] == key_size
        return np.ascontiguousarray(a)
    a = np.ascontiguousarray(a)
    b = a.view(np.uint8).reshape(len(a), -1)
    assert b.shape[1] == key_size, (b.shape, key_size)
    return b


def capacity_for(requested: int, rule: int = 0) -> int:
    out = C.c_uint64(0)
    rc = lib().fmo_capacity_for(requested, rule, C.byref(out))
    if rc == ERR_ZERO_CAPACITY:
        raise ValueError("capacity must be positive")
    return out.value


def hash_key(key: bytes, mode: int) -> int:
    buf = np.frombuffer(bytes(key), dtype=np.uint8).copy() if len(key) else np.zeros(1, np.uint8)
    return lib().fmo_hash(_ptr(buf), len(key), mode)


class TableFull(Exception):
    def __init__(self, occupied: int, capacity: int):
        self.occupied = occupied
        self.capacity = capacity
        self.load_factor = occupied / capacity * 100.0
        super().__init__(f"table full: {occupied} occupied of {capacity} capacity")


class ProbeLimit(Exception):
    """An insert walk passed 2*capacity+2 slots on a table with no free slot
    (the reference's loop would not terminate).  Every op of the call ran."""


class OracleMap:
    """Sequential FlashMap restatement over SoA host arrays."""

    def __init__(self, capacity: int, key_size: int, value_size: int, hash_mode: int = 0,
                 capacity_rule: int = 0):
        self.capacity = capacity_for(capacity, capacity_rule)
        self.key_size = key_size
        self.value_size = value_size
        self.hash_mode = hash_mode
        self._t = lib().fmo_create(self.capacity, key_size, value_size, hash_mode)
        if not self._t:
            raise MemoryError("oracle table allocation failed")

    def __del__(self):
        t = getattr(self, "_t", None)
        if t:
            lib().fmo_destroy(t)
            self._t = None

    # -- bulk ops -----------------------------------------------------------
    def bulk_insert(self, keys, values) -> int:
        k = as_key_bytes(keys, self.key_size)
        v = as_key_bytes(values, self.value_size) if self.value_size else np.zeros((len(k), 0), np.uint8)
        assert len(k) == len(v)
        out = C.c_uint64(0)
        rc = lib().fmo_bulk_insert(self._t, _ptr(k), _ptr(v), len(k), C.byref(out))
        if rc == ERR_TABLE_FULL:
            raise TableFull(len(self), self.capacity)
        if rc == ERR_PROBE_LIMIT:
            raise ProbeLimit()
        return out.value

    def bulk_insert_uncounted(self, keys, values) -> None:
        k = as_key_bytes(keys, self.key_size)
        v = as_key_bytes(values, self.value_size)
        rc = lib().fmo_bulk_insert_uncounted(self._t, _ptr(k), _ptr(v), len(k))
        if rc == ERR_PROBE_LIMIT:
            raise ProbeLimit()

    def bulk_get(self, keys):
        k = as_key_bytes(keys, self.key_size)
        n = len(k)
        vals = np.zeros((n, self.value_size), np.uint8)
        found = np.zeros(n, np.uint8)
        if n:
            lib().fmo_bulk_get(self._t, _ptr(k), n, _ptr(vals), _ptr(found))
        return vals, found.astype(bool)

    def bulk_remove(self, keys) -> int:
        k = as_key_bytes(keys, self.key_size)
        return lib().fmo_bulk_remove(self._t, _ptr(k), len(k)) if len(k) else 0

    def clear(self) -> None:
        lib().fmo_clear(self._t)

    def recount(self) -> int:
        return lib().fmo_recount(self._t)

    def __len__(self) -> int:
        return lib().fmo_len(self._t)

    def set_len(self, n: int) -> None:
        lib().fmo_set_len(self._t, n)

    # -- multithreaded CAS restatement (timing baseline only) ---------------
    def mt_bulk_insert(self, keys, values, threads: int) -> int:
        k = as_key_bytes(keys, self.key_size)
        v = as_key_bytes(values, self.value_size)
        out = C.c_uint64(0)
        rc = lib().fmo_mt_bulk_insert(self._t, _ptr(k), _ptr(v), len(k), C.byref(out), threads)
        if rc == ERR_TABLE_FULL:
            raise TableFull(len(self), self.capacity)
        return out.value

    def mt_bulk_get(self, keys, threads: int):
        k = as_key_bytes(keys, self.key_size)
        vals = np.zeros((len(k), self.value_size), np.uint8)
        found = np.zeros(len(k), np.uint8)
        lib().fmo_mt_bulk_get(self._t, _ptr(k), len(k), _ptr(vals), _ptr(found), threads)
        return vals, found.astype(bool)

    def mt_bulk_remove(self, keys, threads: int) -> int:
        k = as_key_bytes(keys, self.key_size)
        return lib().fmo_mt_bulk_remove(self._t, _ptr(k), len(k), threads)

    # -- raw state ----------------------------------------------------------
    def flags(self) -> np.ndarray:
        p = lib().fmo_flags(self._t)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint32)), (self.capacity,))

    def keys(self) -> np.ndarray:
        p = lib().fmo_keys(self._t)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)),
                                     (self.capacity, max(self.key_size, 1)))[:, : self.key_size]

    def values(self) -> np.ndarray:
        p = lib().fmo_values(self._t)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)),
                                     (self.capacity, max(self.value_size, 1)))[:, : self.value_size]

    def snapshot(self):
        """Copies of (flags, keys, values) for OCCUPIED slots only: the
        observable layout (free slots keep stale bytes in the reference)."""
        f = self.flags().copy()
        occ = (f & 0xF) == OCCUPIED
        k = self.keys().copy()
        v = self.values().copy()
        k[~occ] = 0
        v[~occ] = 0
        return f, k, v

    # -- traffic accounting -------------------------------------------------
    def traffic(self, on: bool = True) -> None:
        lib().fmo_traffic_enable(self._t, 1 if on else 0)

    def traffic_reset(self) -> None:
        lib().fmo_traffic_reset(self._t)

    def traffic_get(self, kind: str) -> dict:
        kinds = {"get": 0, "insert": 1, "remove": 2}
        t = _Traffic()
        lib().fmo_traffic_get(self._t, kinds[kind], C.byref(t))
        return {f: getattr(t, f) for f, _ in _Traffic._fields_}


# ---------------------------------------------------------------------------
# The reference's own kernels.cu, compiled for the host (checker only).
# ---------------------------------------------------------------------------
_ref = None


def ref_host_available() -> bool:
    return os.path.exists(REF_HOST_PATH) or bool(REF_TREE and os.path.isdir(os.path.join(REF_TREE, "src")))


def ref_host():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_HOST_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_TREE}"], check=True)
        L = C.CDLL(REF_HOST_PATH)
        vp = C.c_void_p
        L.ref_identity_hash.restype = C.c_uint64
        L.ref_identity_hash.argtypes = [vp, C.c_uint]
        L.ref_murmur3_hash.restype = C.c_uint64
        L.ref_murmur3_hash.argtypes = [vp, C.c_uint]
        L.ref_seq_bulk_insert.restype = C.c_uint
        L.ref_seq_bulk_insert.argtypes = [vp, vp, vp, vp, vp, C.c_ulonglong, C.c_uint, C.c_uint,
                                          C.c_uint, C.c_uint]
        L.ref_clear.argtypes = [vp, C.c_ulonglong]
        L.ref_count.restype = C.c_uint
        L.ref_count.argtypes = [vp, C.c_ulonglong]
        _ref = L
    return _ref


class RefHostTable:
    """SoA arrays driven by the reference's own insert kernel, run one thread
    at a time (checker for the oracle's insert layout)."""

    def __init__(self, capacity: int, key_size: int, value_size: int, hash_mode: int = 0):
        assert capacity & (capacity - 1) == 0
        self.capacity, self.key_size, self.value_size, self.hash_mode = capacity, key_size, value_size, hash_mode
        self.flags = np.zeros(capacity, np.uint32)
        self.keys = np.zeros((capacity, key_size), np.uint8)
        self.values = np.zeros((capacity, value_size), np.uint8)

    def load(self, flags, keys, values):
        self.flags[:] = flags
        self.keys[:] = keys
        self.values[:] = values

    def bulk_insert(self, keys, values) -> int:
        k = as_key_bytes(keys, self.key_size)
        v = as_key_bytes(values, self.value_size)
        return ref_host().ref_seq_bulk_insert(_ptr(self.keys), _ptr(self.flags), _ptr(self.values),
                                              _ptr(k), _ptr(v), self.capacity - 1, self.key_size,
                                              self.value_size, len(k), self.hash_mode)

    def snapshot(self):
        f = self.flags.copy()
        occ = (f & 0xF) == OCCUPIED
        k = self.keys.copy()
        v = self.values.copy()
        k[~occ] = 0
        v[~occ] = 0
        return f, k, v
