"""ctypes binding of ``libflashmap_b200.so`` (the C ABI in include/flashmap_b200.h).

The shared library is built in-tree (``make -C flash-map_b200``).  There is no
fallback: if the library is missing or cannot be loaded, every entry point
raises ``CudaInit``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from .errors import CudaInit

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# The in-tree build; FLASHMAP_B200_LIB names another build of the same ABI.
LIB_PATH = os.environ.get("FLASHMAP_B200_LIB") or os.path.join(PKG_DIR, "libflashmap_b200.so")

# Every exported symbol of include/flashmap_b200.h.
EXPORTS = (
    "fm_create", "fm_destroy", "fm_bulk_get", "fm_bulk_insert", "fm_bulk_remove", "fm_len",
    "fm_capacity", "fm_load_factor", "fm_clear", "fm_device", "fm_bulk_get_device",
    "fm_bulk_get_values_device", "fm_bulk_insert_device", "fm_bulk_insert_device_uncounted",
    "fm_bulk_remove_device", "fm_recount", "fm_last_error", "fm_launch_count", "fm_snapshot", "fm_load",
    "fm_bulk_insert_device_noalloc", "fm_kernel_timing", "fm_kernel_times", "fm_kernel_times_reset",
    "fm_kernel_class_name", "fm_batch_create", "fm_batch_capture", "fm_batch_run", "fm_batch_wait",
    "fm_batch_waves", "fm_batch_destroy", "fm_autotune", "fm_tuned_get_config", "fm_copy",
    "fm_inject_fault", "fm_batch_profile", "fm_batch_phase_times",
)


class FmOp(C.Structure):
    """struct fm_op of include/flashmap_b200.h."""
    _fields_ = [
        ("table", C.c_void_p),
        ("kind", C.c_uint32),
        ("n", C.c_uint64),
        ("d_keys", C.c_void_p),
        ("d_values", C.c_void_p),
        ("d_out_values", C.c_void_p),
        ("d_out_found", C.c_void_p),
        ("result", C.c_uint64),
        ("status", C.c_int),
    ]

_lock = threading.Lock()
_lib = None


def _declare(L) -> None:
    vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int
    u64p = C.POINTER(C.c_uint64)
    L.fm_create.restype = i32
    L.fm_create.argtypes = [u64, u32, u32, u32, i32, C.POINTER(vp)]
    L.fm_destroy.restype = None
    L.fm_destroy.argtypes = [vp]
    L.fm_bulk_get.restype = i32
    L.fm_bulk_get.argtypes = [vp, vp, u64, vp, vp]
    L.fm_bulk_insert.restype = i32
    L.fm_bulk_insert.argtypes = [vp, vp, vp, u64, u64p]
    L.fm_bulk_remove.restype = i32
    L.fm_bulk_remove.argtypes = [vp, vp, u64, u64p]
    L.fm_len.restype = u64
    L.fm_len.argtypes = [vp]
    L.fm_capacity.restype = u64
    L.fm_capacity.argtypes = [vp]
    L.fm_load_factor.restype = C.c_double
    L.fm_load_factor.argtypes = [vp]
    L.fm_clear.restype = i32
    L.fm_clear.argtypes = [vp]
    L.fm_device.restype = i32
    L.fm_device.argtypes = [vp]
    L.fm_bulk_get_device.restype = i32
    L.fm_bulk_get_device.argtypes = [vp, vp, u64, vp, vp, vp]
    L.fm_bulk_get_values_device.restype = i32
    L.fm_bulk_get_values_device.argtypes = [vp, vp, u64, vp, vp]
    L.fm_bulk_insert_device.restype = i32
    L.fm_bulk_insert_device.argtypes = [vp, vp, vp, u64, u64p, vp]
    L.fm_bulk_insert_device_uncounted.restype = i32
    L.fm_bulk_insert_device_uncounted.argtypes = [vp, vp, vp, u64, vp]
    L.fm_bulk_remove_device.restype = i32
    L.fm_bulk_remove_device.argtypes = [vp, vp, u64, u64p, vp]
    L.fm_bulk_insert_device_noalloc.restype = i32
    L.fm_bulk_insert_device_noalloc.argtypes = [vp, vp, vp, u64, u64p, vp]
    L.fm_recount.restype = i32
    L.fm_recount.argtypes = [vp, u64p]
    L.fm_launch_count.restype = u64
    L.fm_launch_count.argtypes = []
    L.fm_last_error.restype = C.c_char_p
    L.fm_last_error.argtypes = []
    L.fm_snapshot.restype = i32
    L.fm_snapshot.argtypes = [vp, vp, vp, vp]
    L.fm_load.restype = i32
    L.fm_load.argtypes = [vp, vp, vp, vp, u64]
    L.fm_kernel_timing.restype = i32
    L.fm_kernel_timing.argtypes = [vp, i32]
    L.fm_kernel_times.restype = i32
    L.fm_kernel_times.argtypes = [vp, C.POINTER(C.c_double), u64p, u32]
    L.fm_kernel_times_reset.restype = i32
    L.fm_kernel_times_reset.argtypes = [vp]
    L.fm_kernel_class_name.restype = C.c_char_p
    L.fm_kernel_class_name.argtypes = [u32]
    L.fm_batch_create.restype = i32
    L.fm_batch_create.argtypes = [C.POINTER(FmOp), u32, C.POINTER(vp)]
    L.fm_batch_capture.restype = i32
    L.fm_batch_capture.argtypes = [vp, vp]
    L.fm_batch_run.restype = i32
    L.fm_batch_run.argtypes = [vp, vp]
    L.fm_batch_wait.restype = i32
    L.fm_batch_wait.argtypes = [vp, C.POINTER(FmOp)]
    L.fm_batch_waves.restype = u32
    L.fm_batch_waves.argtypes = [vp]
    L.fm_batch_destroy.restype = None
    L.fm_batch_destroy.argtypes = [vp]
    L.fm_batch_profile.restype = i32
    L.fm_batch_profile.argtypes = [vp, i32]
    L.fm_batch_phase_times.restype = i32
    L.fm_batch_phase_times.argtypes = [vp, C.POINTER(C.c_uint64), u32, C.POINTER(u32)]
    L.fm_copy.restype = i32
    L.fm_copy.argtypes = [vp, vp, vp]
    L.fm_autotune.restype = i32
    L.fm_autotune.argtypes = [i32, C.c_char_p]
    L.fm_tuned_get_config.restype = i32
    L.fm_tuned_get_config.argtypes = [u32, u32, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.fm_inject_fault.restype = i32
    L.fm_inject_fault.argtypes = [u32, u32]


def load_library(path: str = LIB_PATH):
    """Load the shared library (once).  Raises CudaInit when it is absent."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(path):
                raise CudaInit(f"native library not built: {path} (run `make -C flash-map_b200`)")
            try:
                L = C.CDLL(path)
            except OSError as e:  # pragma: no cover - depends on the host
                raise CudaInit(f"cannot load {path}: {e}") from e
            _declare(L)
            _lib = L
        return _lib


def launch_count() -> int:
    """Kernels launched by the library in this process (instrumentation)."""
    return load_library().fm_launch_count()


def autotune(device: int = 0, cache_path: str = None) -> None:
    """Time the lookup kernel configurations on `device` and use the fastest
    per record shape and load (fm_autotune)."""
    from .errors import raise_for_status

    rc = load_library().fm_autotune(device, cache_path.encode() if cache_path else None)
    raise_for_status(rc, last_error())


def tuned_get_config(key_size: int, value_size: int, load: float):
    """(lanes per query, blocks per SM) the lookups of such a table use."""
    lanes, bps = C.c_int(0), C.c_int(0)
    load_library().fm_tuned_get_config(key_size, value_size, load, C.byref(lanes), C.byref(bps))
    return lanes.value, bps.value


FAULT_NONE, FAULT_ALLOC, FAULT_TRANSFER, FAULT_ROUND = 0, 1, 2, 3


def inject_fault(site: int, after: int = 0) -> None:
    """Arm one host-side failure (fm_inject_fault): the after-th next pass
    through `site` fails as if its CUDA call had failed.  Tests only."""
    from .errors import raise_for_status

    raise_for_status(load_library().fm_inject_fault(site, after), last_error())


def last_error() -> str:
    msg = load_library().fm_last_error()
    return msg.decode() if msg else ""
