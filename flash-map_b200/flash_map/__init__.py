"""FlashMap B200 backend: host-side API over ``libflashmap_b200.so``.

Mirrors the public surface of bajpainaman/flash-map 0.5.0 (src/lib.rs,
src/async_map.rs, src/error.rs, src/hash.rs) for the GPU path.
"""
from .async_map import AsyncFlashMap
from .batch import BatchOp, FlashMapBatch
from .errors import (AsyncJoin, CudaInit, FlashMapError, GpuAlloc, GpuRequired, KernelLaunch, LockPoisoned,
                     NoBackend, TableFull, Transfer, ZeroCapacity)
from .map import FlashMap, FlashMapBuilder, HashStrategy, as_records
from ._native import EXPORTS, LIB_PATH, load_library

__all__ = [
    "FlashMap", "FlashMapBuilder", "HashStrategy", "AsyncFlashMap", "FlashMapError", "CudaInit", "GpuAlloc",
    "KernelLaunch", "Transfer", "TableFull", "ZeroCapacity", "NoBackend", "GpuRequired", "LockPoisoned",
    "AsyncJoin", "as_records", "EXPORTS", "LIB_PATH", "load_library", "BatchOp", "FlashMapBatch",
]
