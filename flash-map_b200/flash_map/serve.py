"""Served form: continuous batching of bulk requests on a device-resident table.

Requests (get / insert / remove of a key set, each with an arrival time)
reach a :class:`FlashMapServer` in arrival order.  Two threads run them:

* the stager admits arrived requests, oldest first, while their device
  staging (keys, values, outputs) fits the memory budget, uploads their
  inputs on its own copy stream and hands them on;
* the executor takes every admitted request that is ready, runs them as one
  :class:`~flash_map.FlashMapBatch` on the compute stream (arrival-order
  sequential semantics: each request's result is the one it would get alone
  at its turn) or, when only one is ready, as the plain device-pointer call,
  downloads the get results, stamps completion times and releases the
  budget.

So requests that arrive while a batch is on the GPU are admitted as memory
frees up, their uploads overlap the running batch, and they join the next
batch.  :class:`PlainServer` is the per-request baseline: one host-API bulk
call per request in arrival order (the reference's ``AsyncFlashMap`` serves
each request with one bulk call under a lock, src/async_map.rs:48-93).

No counterpart in the reference (bajpainaman/flash-map 0.5.0).
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .batch import GET, INSERT, REMOVE, BatchOp, FlashMapBatch
from .errors import FM_ERR_PROBE_LIMIT, FM_ERR_TABLE_FULL, TableFull
from .map import FlashMap


@dataclass
class Request:
    """One client request.  keys: (n, K) uint8 host array (pinned memory
    gives overlapped uploads); values: (n, V) for inserts.  After service:
    result (new / removed key count), status (0 or an FM error code), and
    for gets out_values (n, V) / out_found (n,) host arrays."""
    kind: int
    keys: np.ndarray
    values: Optional[np.ndarray] = None
    arrival: float = 0.0
    result: int = 0
    status: int = 0
    out_values: Optional[np.ndarray] = None
    out_found: Optional[np.ndarray] = None
    done: float = -1.0
    _dev: list = field(default_factory=list, repr=False)

    @property
    def n(self) -> int:
        return len(self.keys)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def staging_bytes(r: Request, key_size: int, value_size: int) -> int:
    n = r.n
    if r.kind == INSERT:
        return n * (key_size + value_size)
    if r.kind == GET:
        return n * (key_size + value_size + 1)
    return n * key_size


class FlashMapServer:
    """Continuous batching over one FlashMap.  `budget` bounds the device
    bytes staged for admitted, unfinished requests; a request larger than the
    whole budget is served alone once everything before it has finished."""

    def __init__(self, table: FlashMap, budget: int = 20 << 30, out_pool=None):
        import torch

        self.t = table
        self.budget = budget
        self.torch = torch
        self.dev = torch.device("cuda", table.device())
        self.copy_stream = torch.cuda.Stream(self.dev)
        self.stream = torch.cuda.Stream(self.dev)
        self.out_pool = out_pool  # optional callable(n, V) -> (pinned vals, pinned found) for get results
        self.batches = 0
        self.batch_sizes: List[int] = []

    def serve(self, requests: List[Request], realtime: bool = True) -> float:
        """Serves `requests` (sorted by arrival; arrival times in seconds from
        the start).  realtime: a request is admitted no earlier than its
        arrival.  Returns the wall time from the start to the last completion."""
        torch = self.torch
        K, V = self.t.key_size, self.t.value_size
        ready = collections.deque()
        cv = threading.Condition()
        state = {"used": 0, "admitted": 0, "error": None}
        t0 = time.perf_counter()

        def stager():
            try:
                for r in requests:
                    if realtime:
                        wait = r.arrival - (time.perf_counter() - t0)
                        if wait > 0:
                            time.sleep(wait)
                    need = staging_bytes(r, K, V)
                    with cv:
                        while state["used"] > 0 and state["used"] + need > self.budget:
                            cv.wait()
                        state["used"] += need
                    with torch.cuda.stream(self.copy_stream):
                        dk = torch.from_numpy(np.ascontiguousarray(r.keys)).to(self.dev, non_blocking=True)
                        dv = (torch.from_numpy(np.ascontiguousarray(r.values)).to(self.dev, non_blocking=True)
                              if r.kind == INSERT else None)
                        ov = torch.empty((r.n, V), dtype=torch.uint8, device=self.dev) if r.kind == GET else None
                        of = torch.empty((r.n,), dtype=torch.uint8, device=self.dev) if r.kind == GET else None
                        ev = torch.cuda.Event()
                        ev.record(self.copy_stream)
                    r._dev = [dk, dv, ov, of, ev, need]
                    with cv:
                        ready.append(r)
                        state["admitted"] += 1
                        cv.notify_all()
            except Exception as e:  # pragma: no cover - surfaced by serve()
                with cv:
                    state["error"] = e
                    cv.notify_all()

        th = threading.Thread(target=stager, daemon=True)
        th.start()
        served = 0
        end = t0
        while served < len(requests):
            with cv:
                while not ready and state["error"] is None:
                    cv.wait()
                if state["error"] is not None:
                    raise state["error"]
                group = list(ready)
                ready.clear()
            for r in group:
                self.stream.wait_event(r._dev[4])
            if len(group) == 1:
                # a lone request: the plain device call, without batch set-up
                res = [self._run_one(group[0])]
            else:
                ops = [BatchOp(r.kind, self.t, r.n, r._dev[0], r._dev[1], r._dev[2], r._dev[3]) for r in group]
                b = FlashMapBatch(ops)
                b.run(self.stream)
                res = b.wait()
                b.close()
            # results home: get outputs downloaded on the compute stream
            outs = []
            with torch.cuda.stream(self.stream):
                for r in group:
                    if r.kind == GET:
                        if self.out_pool is not None:
                            hv, hf = self.out_pool(r.n, V)
                        else:
                            hv = torch.empty((r.n, V), dtype=torch.uint8).pin_memory()
                            hf = torch.empty((r.n,), dtype=torch.uint8).pin_memory()
                        hv.copy_(r._dev[2], non_blocking=True)
                        hf.copy_(r._dev[3], non_blocking=True)
                        outs.append((r, hv, hf))
            self.stream.synchronize()
            now = time.perf_counter() - t0
            freed = 0
            for r, (cnt, st) in zip(group, res):
                r.result, r.status, r.done = cnt, st, now
                freed += r._dev[5]
                r._dev = []
            for r, hv, hf in outs:
                r.out_values, r.out_found = hv.numpy(), hf.numpy()
            with cv:
                state["used"] -= freed
                cv.notify_all()
            served += len(group)
            self.batches += 1
            self.batch_sizes.append(len(group))
            end = time.perf_counter()
        th.join()
        return end - t0


    def _run_one(self, r: Request):
        """A lone request: the device-pointer call on the compute stream, with
        TableFull and the probe limit reported as the op's status, as a batch
        reports them; any other failure raises."""
        import ctypes as C

        from .map import _dev_ptr

        dk, dv, ov, of = r._dev[:4]
        L, h, s = self.t._L, self.t._h, self.stream.cuda_stream
        out = C.c_uint64(0)
        if r.kind == GET:
            rc = L.fm_bulk_get_device(h, _dev_ptr(dk), r.n, _dev_ptr(ov), _dev_ptr(of), s)
        elif r.kind == INSERT:
            rc = L.fm_bulk_insert_device(h, _dev_ptr(dk), _dev_ptr(dv), r.n, C.byref(out), s)
        else:
            rc = L.fm_bulk_remove_device(h, _dev_ptr(dk), r.n, C.byref(out), s)
        if rc in (FM_ERR_TABLE_FULL, FM_ERR_PROBE_LIMIT):
            return 0, rc
        self.t._check(rc)
        return int(out.value), 0


class PlainServer:
    """Baseline: each request is one host-API bulk call (inputs uploaded and
    results downloaded by the call), served one at a time in arrival order."""

    def __init__(self, table: FlashMap, out_pool=None):
        self.t = table
        self.out_pool = out_pool  # optional callable(n, V) -> (host vals, host found) buffers for get results

    def serve(self, requests: List[Request], realtime: bool = True) -> float:
        t0 = time.perf_counter()
        for r in requests:
            if realtime:
                wait = r.arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
            if r.kind == GET:
                if self.out_pool is not None:
                    hv, hf = self.out_pool(r.n, self.t.value_size)
                    hv, hf = np.asarray(hv), np.asarray(hf)
                    self.t.bulk_get(r.keys, out_values=hv, out_found=hf)
                    r.out_values, r.out_found = hv, hf
                else:
                    r.out_values, f = self.t.bulk_get(r.keys)
                    r.out_found = f.astype(np.uint8)
            elif r.kind == INSERT:
                try:
                    r.result = self.t.bulk_insert(r.keys, r.values)
                except TableFull:
                    r.result, r.status = 0, 5
            else:
                r.result = self.t.bulk_remove(r.keys)
            r.done = time.perf_counter() - t0
        return time.perf_counter() - t0


def latency_summary(requests: List[Request]) -> dict:
    lat = np.array([r.latency for r in requests]) * 1e3
    return {"p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
            "p999_ms": round(float(np.percentile(lat, 99.9)), 3), "max_ms": round(float(lat.max()), 3)}
