"""``AsyncFlashMap``: asyncio counterpart of src/async_map.rs:32-147.

The reference wraps the map in ``Arc<RwLock<FlashMap>>`` and runs every bulk
call on ``spawn_blocking``: gets take the read lock (so they may overlap),
insert/remove/clear take the write lock.  Here the blocking calls run on the
event loop's default executor under the same reader/writer discipline.
"""
from __future__ import annotations

import asyncio
import threading

from .errors import AsyncJoin
from .map import FlashMap


class _RwLock:
    """Writer-preferring reader/writer lock for threads."""

    def __init__(self):
        self._cv = threading.Condition()
        self._readers = 0
        self._writer = False
        self._waiting_writers = 0

    def acquire_read(self):
        with self._cv:
            while self._writer or self._waiting_writers:
                self._cv.wait()
            self._readers += 1

    def release_read(self):
        with self._cv:
            self._readers -= 1
            if self._readers == 0:
                self._cv.notify_all()

    def acquire_write(self):
        with self._cv:
            self._waiting_writers += 1
            while self._writer or self._readers:
                self._cv.wait()
            self._waiting_writers -= 1
            self._writer = True

    def release_write(self):
        with self._cv:
            self._writer = False
            self._cv.notify_all()


class AsyncFlashMap:
    def __init__(self, inner: FlashMap):
        self._inner = inner
        self._lock = _RwLock()

    async def _run(self, write: bool, fn, *args):
        def job():
            (self._lock.acquire_write if write else self._lock.acquire_read)()
            try:
                return fn(*args)
            finally:
                (self._lock.release_write if write else self._lock.release_read)()

        try:
            return await asyncio.get_running_loop().run_in_executor(None, job)
        except asyncio.CancelledError as e:  # mirrors JoinError -> AsyncJoin
            raise AsyncJoin(str(e)) from e

    async def bulk_get(self, keys):
        return await self._run(False, self._inner.bulk_get, keys)

    async def bulk_insert(self, keys, values) -> int:
        return await self._run(True, self._inner.bulk_insert, keys, values)

    async def bulk_remove(self, keys) -> int:
        return await self._run(True, self._inner.bulk_remove, keys)

    async def clear(self) -> None:
        return await self._run(True, self._inner.clear)

    def len(self) -> int:
        return self._inner.len()

    def is_empty(self) -> bool:
        return self._inner.len() == 0

    def capacity(self) -> int:
        return self._inner.capacity()

    def load_factor(self) -> float:
        return self._inner.load_factor()
