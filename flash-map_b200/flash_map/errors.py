"""Error types of the FlashMap B200 backend.

Mirrors ``FlashMapError`` of bajpainaman/flash-map 0.5.0 (src/error.rs:3-40):
one exception class per variant, with the same fields and messages.  C status
codes from ``libflashmap_b200.so`` map onto them in ``raise_for_status``.
"""
from __future__ import annotations


class FlashMapError(Exception):
    """Base class (the ``FlashMapError`` enum)."""


class CudaInit(FlashMapError):
    def __init__(self, msg: str):
        super().__init__(f"CUDA initialization failed: {msg}")


class GpuAlloc(FlashMapError):
    def __init__(self, msg: str):
        super().__init__(f"GPU memory allocation failed: {msg}")


class KernelLaunch(FlashMapError):
    def __init__(self, msg: str):
        super().__init__(f"kernel launch failed: {msg}")


class Transfer(FlashMapError):
    def __init__(self, msg: str):
        super().__init__(f"host-device transfer failed: {msg}")


class TableFull(FlashMapError):
    def __init__(self, occupied: int, capacity: int):
        self.occupied = occupied
        self.capacity = capacity
        self.load_factor = occupied / capacity * 100.0
        super().__init__(
            f"table full: {occupied} occupied of {capacity} capacity "
            f"(load factor {self.load_factor:.1f}%)"
        )


class ZeroCapacity(FlashMapError):
    def __init__(self):
        super().__init__("capacity must be positive")


class NoBackend(FlashMapError):
    def __init__(self, msg: str = "no backend available: enable 'cuda' or 'rayon' feature"):
        super().__init__(msg)


class GpuRequired(FlashMapError):
    def __init__(self):
        super().__init__("device-resident API requires GPU backend (currently using Rayon)")


class LockPoisoned(FlashMapError):
    def __init__(self):
        super().__init__("internal lock poisoned")


class AsyncJoin(FlashMapError):
    def __init__(self, msg: str):
        super().__init__(f"async task join failed: {msg}")


# C status codes (include/flashmap_b200.h)
FM_OK = 0
FM_ERR_CUDA_INIT = 1
FM_ERR_GPU_ALLOC = 2
FM_ERR_KERNEL_LAUNCH = 3
FM_ERR_TRANSFER = 4
FM_ERR_TABLE_FULL = 5
FM_ERR_ZERO_CAPACITY = 6
FM_ERR_INVALID_ARG = 7
FM_ERR_DEVICE_TIMEOUT = 8
FM_ERR_PROBE_LIMIT = 9


def raise_for_status(rc: int, msg: str, occupied: int = 0, capacity: int = 1) -> None:
    if rc == FM_OK:
        return
    if rc == FM_ERR_CUDA_INIT:
        raise CudaInit(msg)
    if rc == FM_ERR_GPU_ALLOC:
        raise GpuAlloc(msg)
    if rc == FM_ERR_TRANSFER:
        raise Transfer(msg)
    if rc == FM_ERR_TABLE_FULL:
        raise TableFull(occupied, capacity)
    if rc == FM_ERR_ZERO_CAPACITY:
        raise ZeroCapacity()
    # INVALID_ARG, DEVICE_TIMEOUT, PROBE_LIMIT and KERNEL_LAUNCH all surface as
    # KernelLaunch with the library's message.
    raise KernelLaunch(msg or f"status {rc}")
