"""Served form: continuous batching of bulk requests on a device-resident table.

Requests (get / insert / remove of a key set, each with an arrival time)
reach a :class:`FlashMapServer` in arrival order.  Three threads serve them:

* the stager admits arrived requests, oldest first, while their device
  staging (keys, values, outputs) fits the memory budget and uploads their
  inputs on its own copy stream, in pieces of at most ``PIECE`` keys, so a
  large request starts on the GPU after its first piece instead of its
  whole upload;
* the executor takes every staged piece that is ready and runs them as one
  :class:`~flash_map.FlashMapBatch` on the compute stream (arrival-order
  sequential semantics: each request's result is the one it would get alone
  at its turn) or, when only one is ready, as the plain device-pointer call;
  get results go down on a download stream behind the group's compute, while
  the executor moves on to the next group.  An insert in several pieces
  keeps the TableFull precheck of the whole request: its first piece starts
  a group, where the host compares the table's exact count plus the whole
  request with the capacity (a rejected request's pieces do not run; the
  later pieces of an accepted one always fit);
* the completer waits for each group's downloads, stamps completion times
  (a request is done with its last piece) and releases the budget.

So requests that arrive while a group is on the GPU are staged meanwhile,
their uploads and the previous group's downloads overlap the running group,
and they join the next group.  :class:`PlainServer` is the per-request
baseline: one host-API bulk call per request in arrival order (the
reference's ``AsyncFlashMap`` serves each request with one bulk call under a
lock, src/async_map.rs:48-93).

No counterpart in the reference (bajpainaman/flash-map 0.5.0).
"""
from __future__ import annotations

import collections
import queue
import threading
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .batch import GET, INSERT, REMOVE, BatchOp, FlashMapBatch
from .errors import FM_ERR_PROBE_LIMIT, FM_ERR_TABLE_FULL, TableFull
from .map import FlashMap

PIECE = 1 << 18  # keys per staged piece of a request


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
    _left: int = field(default=0, repr=False)

    @property
    def n(self) -> int:
        return len(self.keys)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def staging_bytes(r: Request, key_size: int, value_size: int, n: Optional[int] = None) -> int:
    n = r.n if n is None else n
    if r.kind == INSERT:
        return n * (key_size + value_size)
    if r.kind == GET:
        return n * (key_size + value_size + 1)
    return n * key_size


class _Piece:
    """Keys [off, off + n) of a request, staged on the device."""
    __slots__ = ("req", "off", "n", "dk", "dv", "ov", "of", "ev", "need", "in_ring")

    def __init__(self, req, off, n, need):
        self.req, self.off, self.n, self.need = req, off, n, need
        self.dk = self.dv = self.ov = self.of = self.ev = None
        self.in_ring = False


def _al(nbytes: int) -> int:
    return (nbytes + 255) & ~255


class _Ring:
    """First-in first-out space in one device buffer.  Pieces are released
    in the order they were staged (groups complete in order), so the free
    space is the ring between the newest and the oldest live piece."""

    def __init__(self, buf):
        self.buf = buf
        self.size = buf.numel()
        self.live = collections.deque()  # offsets, oldest first
        self.head = 0

    def take(self, need: int) -> Optional[int]:
        if not self.live:
            off = 0
        else:
            tail = self.live[0]
            if self.head > tail:  # live [tail, head): free at the end, then before tail
                if self.head + need <= self.size:
                    off = self.head
                elif need <= tail:
                    off = 0
                else:
                    return None
            elif self.head + need <= tail:  # wrapped: free [head, tail)
                off = self.head
            else:
                return None
        self.live.append(off)
        self.head = off + need
        return off

    def give(self) -> None:
        self.live.popleft()
        if not self.live:
            self.head = 0


# Device memory the server leaves free beside its staging buffer (kernel
# scratch, the framework's other buffers): a tenth of what is free, at most
# 2 GiB.
HEADROOM_MAX = 2 << 30


class FlashMapServer:
    """Continuous batching over one FlashMap.  Requests are admitted against
    device memory: the staging buffer the server owns is the budget, or the
    free HBM (cudaMemGetInfo) less a headroom when less is free, and at most
    `ring_bytes` when given.  The device bytes staged for admitted, unfinished
    pieces are carved from it; a piece larger than it is served alone once
    everything before it has finished."""

    def __init__(self, table: FlashMap, budget: int = 20 << 30, out_pool=None, ring_bytes: Optional[int] = None):
        import torch

        self.t = table
        self.budget = budget
        self.torch = torch
        self.dev = torch.device("cuda", table.device())
        self.copy_stream = torch.cuda.Stream(self.dev)
        free = torch.cuda.mem_get_info(self.dev)[0]
        room = max(256, free - min(HEADROOM_MAX, free // 10))
        self.staging_bytes = min(budget, room, ring_bytes if ring_bytes is not None else budget)
        # pieces are carved from staging space the server owns, so staging
        # never waits on the framework's allocator
        with torch.cuda.stream(self.copy_stream):
            self._ring = _Ring(torch.empty(max(256, self.staging_bytes) & ~255, dtype=torch.uint8,
                                           device=self.dev))
        self.stream = torch.cuda.Stream(self.dev)
        self.down_stream = torch.cuda.Stream(self.dev)
        self.out_pool = out_pool  # optional callable(n, V) -> (pinned vals, pinned found) for get results
        self.batches = 0
        self.batch_sizes: List[int] = []

    def warmup(self) -> None:
        """Runs each kind of op, alone and as a batch, on a small scratch
        table of the same record sizes, so that first-use costs (kernel
        loading, the batch buffers) fall outside served requests.  The served
        table is not touched."""
        torch = self.torch
        K, V = self.t.key_size, self.t.value_size
        scratch = FlashMap(1 << 12, K, V, device_id=self.t.device())
        try:
            g = torch.Generator(device=self.dev)
            g.manual_seed(0)
            k = torch.randint(0, 256, (512, K), dtype=torch.uint8, device=self.dev, generator=g)
            v = torch.randint(0, 256, (512, V), dtype=torch.uint8, device=self.dev, generator=g)
            ov = torch.empty((512, V), dtype=torch.uint8, device=self.dev)
            of = torch.empty((512,), dtype=torch.uint8, device=self.dev)
            scratch.bulk_insert_device(k, v, 256, self.stream)
            scratch.bulk_get_device(k, 512, ov, of, self.stream)
            scratch.bulk_remove_device(k, 64, self.stream)
            ops = [BatchOp(INSERT, scratch, 256, k[256:], v[256:]), BatchOp(GET, scratch, 512, k, None, ov, of),
                   BatchOp(REMOVE, scratch, 64, k[64:])]
            b = FlashMapBatch(ops)
            b.run(self.stream)
            b.wait()
            b.close()
            self.stream.synchronize()
        finally:
            scratch.close()

    def serve(self, requests: List[Request], realtime: bool = True) -> float:
        """Serves `requests` (sorted by arrival; arrival times in seconds from
        the start).  realtime: a request is admitted no earlier than its
        arrival.  Returns the wall time from the start to the last completion."""
        torch = self.torch
        K, V = self.t.key_size, self.t.value_size
        ready = collections.deque()
        cv = threading.Condition()
        state = {"used": 0, "error": None, "end": 0.0}
        done_q: "queue.Queue" = queue.Queue()
        ring = self._ring
        t0 = time.perf_counter()

        def stager():
            try:
                for r in requests:
                    if realtime:
                        wait = r.arrival - (time.perf_counter() - t0)
                        if wait > 0:
                            time.sleep(wait)
                    offs = list(range(0, r.n, PIECE)) if r.n else [0]
                    r._left = len(offs)
                    if r.kind == GET:
                        if self.out_pool is not None:
                            hv, hf = self.out_pool(r.n, V)
                        else:
                            hv = torch.empty((r.n, V), dtype=torch.uint8).pin_memory()
                            hf = torch.empty((r.n,), dtype=torch.uint8).pin_memory()
                        r._host = (hv, hf)
                    for off in offs:
                        n = min(PIECE, r.n - off)
                        pc = _Piece(r, off, n, staging_bytes(r, K, V, n))
                        parts = [n * K] + ([n * V] if r.kind == INSERT else []) + (
                            [n * V, n] if r.kind == GET else [])
                        rneed = sum(_al(x) for x in parts)
                        at = None
                        with cv:
                            if rneed <= ring.size:
                                # (after a piece staged alone, nothing until it is done)
                                while state["used"] > 0 or (at := ring.take(rneed)) is None:
                                    cv.wait()
                                pc.in_ring = True
                            else:  # alone: once everything staged before it is done
                                while ring.live or state["used"] > 0:
                                    cv.wait()
                                state["used"] += pc.need
                        with torch.cuda.stream(self.copy_stream):
                            if at is not None:
                                views = []
                                for x in parts:
                                    views.append(ring.buf[at:at + x])
                                    at += _al(x)
                            else:
                                views = [torch.empty(x, dtype=torch.uint8, device=self.dev) for x in parts]
                            pc.dk = views[0].view(n, K)
                            pc.dk.copy_(torch.from_numpy(np.ascontiguousarray(r.keys[off:off + n])), non_blocking=True)
                            if r.kind == INSERT:
                                pc.dv = views[1].view(n, V)
                                pc.dv.copy_(torch.from_numpy(np.ascontiguousarray(r.values[off:off + n])),
                                            non_blocking=True)
                            if r.kind == GET:
                                pc.ov, pc.of = views[1].view(n, V), views[2]
                            pc.ev = torch.cuda.Event()
                            pc.ev.record(self.copy_stream)
                        with cv:
                            ready.append(pc)
                            cv.notify_all()
            except Exception as e:  # pragma: no cover - surfaced by serve()
                with cv:
                    state["error"] = e
                    cv.notify_all()

        def completer():
            try:
                while True:
                    item = done_q.get()
                    if item is None:
                        return
                    ev, group, res = item
                    if ev is not None:
                        ev.synchronize()
                    now = time.perf_counter() - t0
                    freed = 0
                    given = 0
                    for pc, (cnt, st) in zip(group, res):
                        r = pc.req
                        r.result += cnt
                        if st and not r.status:
                            r.status = st
                        r._left -= 1
                        if r._left == 0:
                            if r.kind == GET:
                                hv, hf = r._host
                                r.out_values, r.out_found = np.asarray(hv), np.asarray(hf)
                                del r._host
                            r.done = now
                            state["end"] = max(state["end"], now)
                        if pc.in_ring:
                            given += 1
                        else:
                            freed += pc.need
                        pc.dk = pc.dv = pc.ov = pc.of = pc.ev = None
                    with cv:
                        for _ in range(given):
                            ring.give()
                        state["used"] -= freed
                        cv.notify_all()
            except Exception as e:  # pragma: no cover - surfaced by serve()
                with cv:
                    state["error"] = e
                    cv.notify_all()

        th = threading.Thread(target=stager, daemon=True)
        tc = threading.Thread(target=completer, daemon=True)
        th.start()
        tc.start()
        total = sum(len(range(0, r.n, PIECE)) if r.n else 1 for r in requests)
        ran = 0
        cap = self.t.capacity()
        try:
            while ran < total:
                with cv:
                    while not ready and state["error"] is None:
                        cv.wait()
                    if state["error"] is not None:
                        raise state["error"]
                    group = list(ready)
                    ready.clear()
                    # the first piece of a multi-piece insert starts a group
                    for idx in range(1, len(group)):
                        if group[idx].off == 0 and group[idx].req.kind == INSERT and group[idx].req.n > PIECE:
                            ready.extendleft(reversed(group[idx:]))
                            del group[idx:]
                            break
                head = group[0]
                if head.off == 0 and head.req.kind == INSERT and head.req.n > PIECE:
                    # every earlier group has finished: len is exact here
                    head.req._reject = self.t.len() + head.req.n > cap
                skip = [pc for pc in group if getattr(pc.req, "_reject", False)]
                if skip:
                    done_q.put((None, skip, [(0, FM_ERR_TABLE_FULL)] * len(skip)))
                    ran += len(skip)
                    group = [pc for pc in group if not getattr(pc.req, "_reject", False)]
                    if not group:
                        continue
                for pc in group:
                    self.stream.wait_event(pc.ev)
                if len(group) == 1:
                    # a lone piece: the plain device call, without batch set-up
                    res = [self._run_one(group[0])]
                else:
                    ops = [BatchOp(pc.req.kind, self.t, pc.n, pc.dk, pc.dv, pc.ov, pc.of) for pc in group]
                    b = FlashMapBatch(ops)
                    b.run(self.stream)
                    res = b.wait()
                    b.close()
                # get results go down behind the group, on their own stream
                ev = None
                gets = [pc for pc in group if pc.req.kind == GET]
                if gets:
                    done_compute = torch.cuda.Event()
                    done_compute.record(self.stream)
                    self.down_stream.wait_event(done_compute)
                    with torch.cuda.stream(self.down_stream):
                        for pc in gets:
                            hv, hf = pc.req._host
                            hv[pc.off:pc.off + pc.n].copy_(pc.ov, non_blocking=True)
                            hf[pc.off:pc.off + pc.n].copy_(pc.of, non_blocking=True)
                    ev = torch.cuda.Event()
                    ev.record(self.down_stream)
                done_q.put((ev, group, res))
                ran += len(group)
                self.batches += 1
                self.batch_sizes.append(len(group))
        finally:
            done_q.put(None)
            tc.join()
        th.join()
        if state["error"] is not None:
            raise state["error"]
        return state["end"]

    def _run_one(self, pc: _Piece):
        """A lone piece: the device-pointer call on the compute stream, with
        TableFull and the probe limit reported as the op's status, as a batch
        reports them; any other failure raises."""
        import ctypes as C

        from .map import _dev_ptr

        L, h, s = self.t._L, self.t._h, self.stream.cuda_stream
        out = C.c_uint64(0)
        kind = pc.req.kind
        if kind == GET:
            rc = L.fm_bulk_get_device(h, _dev_ptr(pc.dk), pc.n, _dev_ptr(pc.ov), _dev_ptr(pc.of), s)
        elif kind == INSERT:
            rc = L.fm_bulk_insert_device(h, _dev_ptr(pc.dk), _dev_ptr(pc.dv), pc.n, C.byref(out), s)
        else:
            rc = L.fm_bulk_remove_device(h, _dev_ptr(pc.dk), pc.n, C.byref(out), s)
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


class AsyncPlainServer:
    """Per-request plain calls through :class:`~flash_map.AsyncFlashMap`, as
    the reference's async wrapper serves them (src/async_map.rs:48-93): each
    request is one host-API bulk call run off the event loop under the
    wrapper's reader/writer lock, issued when it arrives, so gets overlap one
    another while inserts and removes run alone.  Every request also waits
    for the earlier requests it conflicts with -- a write for all of them, a
    get for the earlier writes -- so each result is its arrival-order result,
    the same as :class:`FlashMapServer` gives."""

    def __init__(self, table: FlashMap, out_pool=None, workers: int = 8):
        self.t = table
        self.out_pool = out_pool  # optional callable(n, V) -> (host vals, host found) buffers for get results
        self.workers = workers

    def serve(self, requests: List[Request], realtime: bool = True) -> float:
        import asyncio
        from concurrent.futures import ThreadPoolExecutor

        from .async_map import AsyncFlashMap

        am = AsyncFlashMap(self.t)
        V = self.t.value_size

        async def one(r: Request, deps, t0):
            if deps:
                await asyncio.gather(*deps)
            if r.kind == GET:
                if self.out_pool is not None:
                    hv, hf = self.out_pool(r.n, V)
                    hv, hf = np.asarray(hv), np.asarray(hf)
                    await am._run(False, lambda: self.t.bulk_get(r.keys, out_values=hv, out_found=hf))
                    r.out_values, r.out_found = hv, hf
                else:
                    vals, found = await am.bulk_get(r.keys)
                    r.out_values, r.out_found = vals, found.astype(np.uint8)
            elif r.kind == INSERT:
                try:
                    r.result = await am.bulk_insert(r.keys, r.values)
                except TableFull:
                    r.result, r.status = 0, FM_ERR_TABLE_FULL
            else:
                r.result = await am.bulk_remove(r.keys)
            r.done = time.perf_counter() - t0

        async def main():
            loop = asyncio.get_running_loop()
            loop.set_default_executor(ThreadPoolExecutor(max_workers=self.workers))
            t0 = time.perf_counter()
            last_write = None
            reads = []
            tasks = []
            for r in requests:
                if realtime:
                    wait = r.arrival - (time.perf_counter() - t0)
                    if wait > 0:
                        await asyncio.sleep(wait)
                if r.kind == GET:
                    deps = [last_write] if last_write is not None else []
                    task = asyncio.ensure_future(one(r, deps, t0))
                    reads.append(task)
                else:
                    deps = ([last_write] if last_write is not None else []) + reads
                    task = asyncio.ensure_future(one(r, deps, t0))
                    last_write, reads = task, []
                tasks.append(task)
            await asyncio.gather(*tasks)
            return time.perf_counter() - t0

        return asyncio.run(main())


def latency_summary(requests: List[Request]) -> dict:
    lat = np.array([r.latency for r in requests]) * 1e3
    return {"p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
            "p999_ms": round(float(np.percentile(lat, 99.9)), 3), "max_ms": round(float(lat.max()), 3)}
