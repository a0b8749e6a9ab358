"""Batched form: many bulk operations over many tables in one submission.

A :class:`FlashMapBatch` holds a queue of device-resident bulk operations
(``get`` / ``insert`` / ``remove`` on :class:`~flash_map.FlashMap` tables of one
GPU).  Running it gives the result of calling ``bulk_get_device`` /
``bulk_insert_device`` / ``bulk_remove_device`` one by one in queue order --
including each insert's ``TableFull`` precheck against the table's count at
that point -- but the library runs every op as device-driven kernels on
stream lanes (a table's writes in order, its lookups between them at the same
time, different tables at once), with no host round trip between ops
(``FLASHMAP_BATCH_MODE=queue``: one persistent kernel per record shape
instead; batches with run-time record sizes: waves of grouped kernels).
:meth:`FlashMapBatch.capture` records the whole submission into a CUDA graph
that later :meth:`run` calls replay.  No op may read or write a buffer that
another op of the batch writes.

No counterpart in the reference (bajpainaman/flash-map 0.5.0); it is the
batching form built around the same bulk semantics (src/lib.rs:123-162).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any, List, Optional, Sequence, Tuple

from . import _native
from .errors import raise_for_status
from .map import FlashMap, _dev_ptr, _stream_ptr

GET, INSERT, REMOVE = 0, 1, 2


@dataclass
class BatchOp:
    """One queued op.  Buffers are device tensors (or raw device pointers):
    ``keys`` n x K bytes; ``values`` n x V bytes for inserts; ``out_values`` /
    ``out_found`` (n x V, n bytes) for gets, either may be None."""
    kind: int
    table: FlashMap
    n: int
    keys: Any
    values: Any = None
    out_values: Any = None
    out_found: Any = None


class FlashMapBatch:
    def __init__(self, ops: Sequence[BatchOp]):
        if not ops:
            raise ValueError("empty batch")
        self._L = _native.load_library()
        self._ops = list(ops)  # keeps the buffers alive
        arr = (_native.FmOp * len(ops))()
        for i, o in enumerate(ops):
            a = arr[i]
            a.table = o.table._h.value
            a.kind = int(o.kind)
            a.n = int(o.n)
            n, ks, vs = int(o.n), o.table.key_size, o.table.value_size
            a.d_keys = _dev_ptr(o.keys, n * ks, f"op {i} keys") if o.keys is not None else None
            a.d_values = _dev_ptr(o.values, n * vs, f"op {i} values") if o.values is not None else None
            a.d_out_values = _dev_ptr(o.out_values, n * vs, f"op {i} out_values") if o.out_values is not None else None
            a.d_out_found = _dev_ptr(o.out_found, n, f"op {i} out_found") if o.out_found is not None else None
        self._arr = arr
        h = C.c_void_p()
        rc = self._L.fm_batch_create(arr, len(ops), C.byref(h))
        if rc:
            raise_for_status(rc, _native.last_error(), 0, 0)
        self._h = h

    @property
    def waves(self) -> int:
        return int(self._L.fm_batch_waves(self._h))

    def capture(self, stream) -> None:
        """Record the submission into a CUDA graph on `stream` (not the legacy
        default stream); later run() calls replay it."""
        rc = self._L.fm_batch_capture(self._h, _stream_ptr(stream))
        if rc:
            raise_for_status(rc, _native.last_error(), 0, 0)

    def run(self, stream=None) -> None:
        """Enqueue the submission on `stream` (graph replay once captured)."""
        rc = self._L.fm_batch_run(self._h, _stream_ptr(stream))
        if rc:
            raise_for_status(rc, _native.last_error(), 0, 0)

    def wait(self) -> List[Tuple[int, int]]:
        """Wait for the run; returns per op (result, status): result = new keys
        (insert) / removed keys (remove); status 0 or the op's error code
        (5 TableFull, 9 probe limit, ...)."""
        rc = self._L.fm_batch_wait(self._h, self._arr)
        if rc:
            raise_for_status(rc, _native.last_error(), 0, 0)
        return [(int(a.result), int(a.status)) for a in self._arr]

    PHASE_KINDS = ("get", "begin", "ins_find", "ins_flow", "ins_exec", "ins_warp", "rem_find", "rem_exec", "end",
                   "ins_big")

    def profile(self, on: bool = True) -> None:
        """Record per-phase device times of the persistent launches (queue
        mode only; set before capture)."""
        rc = self._L.fm_batch_profile(self._h, 1 if on else 0)
        if rc:
            raise_for_status(rc, _native.last_error(), 0, 0)

    def phase_times(self) -> List[dict]:
        """Per phase of the last run (after wait): step, kind, op, units and
        device times in ns (start of the first unit, end of the last, summed
        dependency waits, summed unit run times)."""
        cap = 1 << 16
        rows = (C.c_uint64 * (8 * cap))()
        n = C.c_uint32(0)
        rc = self._L.fm_batch_phase_times(self._h, rows, cap, C.byref(n))
        if rc:
            raise_for_status(rc, _native.last_error(), 0, 0)
        out = []
        for r in range(n.value):
            w = rows[8 * r: 8 * r + 8]
            out.append({"step": int(w[0]), "kind": self.PHASE_KINDS[int(w[1])], "op": int(w[2]),
                        "units": int(w[3]), "t0": int(w[4]), "t1": int(w[5]), "wait": int(w[6]),
                        "busy": int(w[7])})
        return out

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.fm_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass
