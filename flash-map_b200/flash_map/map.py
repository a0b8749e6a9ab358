"""``FlashMap`` / ``FlashMapBuilder`` / ``HashStrategy`` over the B200 backend.

Host-side mirror of the reference's public API for the GPU path
(bajpainaman/flash-map 0.5.0, src/lib.rs:94-450 and src/gpu.rs:32-712):
the same constructors, bulk operations, errors and device-resident calls,
with Rust's ``FlashMap<K, V>`` generics expressed as fixed key/value byte
sizes.  Keys and values are numpy arrays: either ``(n, size)`` ``uint8`` or a
1-D array whose dtype item size equals the record size (``np.uint64`` for
``u64``).  Every call goes through ``libflashmap_b200.so``; there is no CPU
path in this package.
"""
from __future__ import annotations

import ctypes as C
import enum
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _native
from .errors import GpuRequired, NoBackend, raise_for_status

ArrayLike = Union[np.ndarray, Sequence]


class HashStrategy(enum.IntEnum):
    """``HashStrategy`` (src/hash.rs:2-27); the value is ``to_mode()``."""

    Identity = 0
    Murmur3 = 1

    def to_mode(self) -> int:
        return int(self)


def _size_of(t) -> int:
    """Record size in bytes from an int, a numpy dtype/scalar type or a
    ``("u8", n)`` style byte-array spec."""
    if isinstance(t, int):
        return t
    if isinstance(t, tuple) and len(t) == 2:
        return int(t[1])
    return np.dtype(t).itemsize


def as_records(a: ArrayLike, size: int, what: str) -> np.ndarray:
    """C-contiguous ``(n, size)`` uint8 view/copy of an array of records."""
    arr = np.asarray(a)
    if arr.dtype == np.uint8 and arr.ndim == 2:
        if arr.shape[1] != size:
            raise ValueError(f"{what}: expected records of {size} bytes, got {arr.shape[1]}")
        return np.ascontiguousarray(arr)
    if arr.ndim == 0:
        arr = arr.reshape(1)
    arr = np.ascontiguousarray(arr)
    if arr.dtype.itemsize * (arr.size // max(len(arr), 1)) != size and len(arr):
        raise ValueError(f"{what}: dtype {arr.dtype} does not match {size}-byte records")
    return arr.view(np.uint8).reshape(len(arr), size)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _dev_ptr(x, nbytes: Optional[int] = None, what: str = "buffer") -> int:
    """Raw device pointer from a torch tensor / object with data_ptr() / int.
    With nbytes, a tensor (anything with numel() and element_size()) must
    hold at least that many bytes: the kernels read and write count records
    from the pointer and cannot see the buffer's end (a raw pointer is the
    caller's to size)."""
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if nbytes is not None and hasattr(x, "numel") and hasattr(x, "element_size"):
            have = int(x.numel()) * int(x.element_size())
            if have < nbytes:
                raise ValueError(f"{what}: {have} bytes, the call needs {nbytes}")
        return int(x.data_ptr())
    raise TypeError("device buffer must be a raw pointer or expose data_ptr()")


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    raise TypeError("stream must be a raw cudaStream_t or a torch.cuda.Stream")


class FlashMap:
    """GPU-native hash map with bulk-only operations (src/lib.rs:84-351)."""

    def __init__(self, capacity: int, key_size: int, value_size: int,
                 hash_strategy: HashStrategy = HashStrategy.Identity, device_id: int = 0):
        L = _native.load_library()
        h = C.c_void_p()
        rc = L.fm_create(capacity, key_size, value_size, int(hash_strategy), device_id, C.byref(h))
        raise_for_status(rc, _native.last_error())
        self._h = h
        self._L = L
        self.key_size = key_size
        self.value_size = value_size
        self.hash_strategy = HashStrategy(hash_strategy)

    # -- construction (lib.rs:105-117) ---------------------------------------
    @classmethod
    def with_capacity(cls, capacity: int, key=np.uint64, value=np.uint64) -> "FlashMap":
        return FlashMapBuilder(capacity).build(key, value)

    @staticmethod
    def builder(capacity: int) -> "FlashMapBuilder":
        return FlashMapBuilder(capacity)

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.fm_destroy(h)
            self._h = C.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        raise_for_status(rc, _native.last_error(), self.len(), self.capacity())

    # -- host-facing bulk API (lib.rs:123-162, gpu.rs:111-332) ---------------
    def bulk_get(self, keys: ArrayLike, out_values: Optional[np.ndarray] = None,
                 out_found: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
        """Look up keys.  Returns ``(values, found)``: ``values`` is
        ``(n, value_size)`` uint8 with zeros for misses, ``found`` a bool mask
        (the ``Vec<Option<V>>`` of the reference, split).  Preallocated
        C-contiguous host buffers (``(n, value_size)`` and ``(n,)`` uint8, for
        example pinned memory) may be passed to avoid per-call allocation; the
        found mask is then returned as those uint8 bytes."""
        k = as_records(keys, self.key_size, "keys")
        n = len(k)
        given = out_found is not None
        vals = np.zeros((n, self.value_size), np.uint8) if out_values is None else out_values
        found = np.zeros(n, np.uint8) if out_found is None else out_found
        if vals.shape != (n, self.value_size) or vals.dtype != np.uint8 or not vals.flags.c_contiguous:
            raise ValueError("out_values must be a C-contiguous (n, value_size) uint8 array")
        if found.shape != (n,) or found.dtype != np.uint8:
            raise ValueError("out_found must be an (n,) uint8 array")
        if n:
            self._check(self._L.fm_bulk_get(self._h, _ptr(k), n, _ptr(vals), _ptr(found)))
        return vals, (found if given else found.astype(bool))

    def bulk_get_options(self, keys: ArrayLike) -> List[Optional[bytes]]:
        """``bulk_get`` as a list of ``Optional[bytes]`` (``Vec<Option<V>>``)."""
        vals, found = self.bulk_get(keys)
        return [bytes(vals[i]) if found[i] else None for i in range(len(found))]

    def bulk_insert(self, keys: ArrayLike, values: ArrayLike) -> int:
        """Insert pairs (keys[i], values[i]); returns the number of new keys.
        Duplicate keys inside one batch resolve to the later position."""
        k = as_records(keys, self.key_size, "keys")
        v = as_records(values, self.value_size, "values") if self.value_size else np.zeros((len(k), 0), np.uint8)
        if len(k) != len(v):
            raise ValueError("keys and values differ in length")
        out = C.c_uint64(0)
        if len(k):
            self._check(self._L.fm_bulk_insert(self._h, _ptr(k), _ptr(v), len(k), C.byref(out)))
        return out.value

    def bulk_insert_pairs(self, pairs: Sequence[Tuple[bytes, bytes]]) -> int:
        """``bulk_insert(&[(K, V)])`` with the pairs split into SoA (gpu.rs:212-217)."""
        ks = np.frombuffer(b"".join(p[0] for p in pairs), np.uint8).reshape(len(pairs), self.key_size)
        vs = np.frombuffer(b"".join(p[1] for p in pairs), np.uint8).reshape(len(pairs), self.value_size)
        return self.bulk_insert(ks, vs)

    def bulk_remove(self, keys: ArrayLike) -> int:
        k = as_records(keys, self.key_size, "keys")
        out = C.c_uint64(0)
        if len(k):
            self._check(self._L.fm_bulk_remove(self._h, _ptr(k), len(k), C.byref(out)))
        return out.value

    def len(self) -> int:
        return self._L.fm_len(self._h)

    def __len__(self) -> int:
        return self.len()

    def is_empty(self) -> bool:
        return self.len() == 0

    def capacity(self) -> int:
        return self._L.fm_capacity(self._h)

    def load_factor(self) -> float:
        return self._L.fm_load_factor(self._h)

    def clear(self) -> None:
        self._check(self._L.fm_clear(self._h))

    # -- device-resident API (lib.rs:213-350, gpu.rs:376-712) ---------------
    def device(self) -> int:
        return self._L.fm_device(self._h)

    def bulk_get_device(self, d_keys, count: int, d_out_values, d_out_found, stream=None) -> None:
        """Lookup with keys and outputs in caller-owned device memory.
        Misses write zeros.  Stream-ordered on ``stream``; does not sync."""
        ks, vs = self.key_size, self.value_size
        self._check(self._L.fm_bulk_get_device(self._h, _dev_ptr(d_keys, count * ks, "keys"), count,
                                               _dev_ptr(d_out_values, count * vs, "out_values"),
                                               _dev_ptr(d_out_found, count, "out_found"), _stream_ptr(stream)))

    def bulk_get_values_device(self, d_keys, count: int, d_out_values, stream=None) -> None:
        self._check(self._L.fm_bulk_get_values_device(self._h, _dev_ptr(d_keys, count * self.key_size, "keys"), count,
                                                      _dev_ptr(d_out_values, count * self.value_size, "out_values"),
                                                      _stream_ptr(stream)))

    def bulk_insert_device(self, d_keys, d_values, count: int, stream=None) -> int:
        out = C.c_uint64(0)
        self._check(self._L.fm_bulk_insert_device(self._h, _dev_ptr(d_keys, count * self.key_size, "keys"),
                                                  _dev_ptr(d_values, count * self.value_size, "values"), count,
                                                  C.byref(out), _stream_ptr(stream)))
        return out.value

    def bulk_insert_device_uncounted(self, d_keys, d_values, count: int, stream=None) -> None:
        self._check(self._L.fm_bulk_insert_device_uncounted(self._h, _dev_ptr(d_keys, count * self.key_size, "keys"),
                                                            _dev_ptr(d_values, count * self.value_size, "values"),
                                                            count, _stream_ptr(stream)))

    def bulk_remove_device(self, d_keys, count: int, stream=None) -> int:
        out = C.c_uint64(0)
        self._check(self._L.fm_bulk_remove_device(self._h, _dev_ptr(d_keys, count * self.key_size, "keys"), count,
                                                  C.byref(out), _stream_ptr(stream)))
        return out.value

    def recount(self) -> int:
        out = C.c_uint64(0)
        self._check(self._L.fm_recount(self._h, C.byref(out)))
        return out.value

    def copy_from(self, other: "FlashMap", stream=None) -> None:
        """Device-side copy of `other` (same capacity and record sizes) into
        this table: slots, len and probe facts (fm_copy)."""
        self._check(self._L.fm_copy(self._h, other._h, _stream_ptr(stream)))

    # -- per-kernel device timing (instrumentation) -------------------------
    def kernel_timing(self, on: bool = True, reset: bool = False) -> None:
        """Record CUDA events around this table's kernel launches while on."""
        if reset:
            self._check(self._L.fm_kernel_times_reset(self._h))
        self._check(self._L.fm_kernel_timing(self._h, 1 if on else 0))

    def kernel_times(self) -> dict:
        """{kernel class: (total device ms, launches)} since the last reset;
        waits for the recorded launches."""
        n = 13
        ms = (C.c_double * n)()
        cnt = (C.c_uint64 * n)()
        self._check(self._L.fm_kernel_times(self._h, ms, cnt, n))
        out = {}
        for i in range(n):
            name = self._L.fm_kernel_class_name(i)
            if name and cnt[i]:
                out[name.decode()] = (ms[i], int(cnt[i]))
        return out

    # -- raw table access (layout checks) -----------------------------------
    def snapshot(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(flags, keys, values) of the whole table, free slots' key/value
        bytes zeroed (they are not observable through the API)."""
        cap = self.capacity()
        f = np.zeros(cap, np.uint32)
        k = np.zeros((cap, self.key_size), np.uint8)
        v = np.zeros((cap, self.value_size), np.uint8)
        self._check(self._L.fm_snapshot(self._h, _ptr(f), _ptr(k), _ptr(v)))
        occ = (f & 0xF) == 1
        k[~occ] = 0
        v[~occ] = 0
        return f, k, v

    def load(self, flags: np.ndarray, keys: np.ndarray, values: np.ndarray, length: int) -> None:
        f = np.ascontiguousarray(flags, dtype=np.uint32)
        k = np.ascontiguousarray(keys, dtype=np.uint8)
        v = np.ascontiguousarray(values, dtype=np.uint8)
        self._check(self._L.fm_load(self._h, _ptr(f), _ptr(k), _ptr(v), length))

    def __repr__(self) -> str:  # lib.rs:353-370
        return (f"FlashMap {{ backend: \"GPU\", len: {self.len()}, capacity: {self.capacity()}, "
                f"load_factor: \"{self.load_factor() * 100.0:.1f}%\" }}")


class FlashMapBuilder:
    """``FlashMapBuilder`` (src/lib.rs:376-449) for the GPU backend."""

    def __init__(self, capacity: int):
        self._capacity = capacity
        self._hash = HashStrategy.Identity
        self._device = 0
        self._force_cpu = False

    def hash_strategy(self, strategy: HashStrategy) -> "FlashMapBuilder":
        self._hash = HashStrategy(strategy)
        return self

    def device_id(self, device: int) -> "FlashMapBuilder":
        self._device = device
        return self

    def force_cpu(self) -> "FlashMapBuilder":
        self._force_cpu = True
        return self

    def build(self, key=np.uint64, value=np.uint64) -> FlashMap:
        if self._force_cpu:
            # The CPU backend is the reference crate's own Rayon code; this
            # package is only the GPU backend and never substitutes a CPU path.
            raise NoBackend("force_cpu: this package provides only the GPU backend")
        return FlashMap(self._capacity, _size_of(key), _size_of(value), self._hash, self._device)


__all__ = ["FlashMap", "FlashMapBuilder", "HashStrategy", "GpuRequired", "as_records"]
