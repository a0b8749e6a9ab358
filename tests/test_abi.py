"""The C ABI library loads and exports every symbol include/flashmap_b200.h
declares; the host packages map status codes onto the reference's error
variants (src/error.rs).  No compute call needs a GPU here."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "flashmap_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|uint32_t|uint64_t|double|const char\*)\s+(fm_\w+)\s*\(", src, re.M)))


def test_header_declares_the_gpu_rs_surface():
    syms = declared_symbols()
    for s in ("fm_create", "fm_destroy", "fm_bulk_get", "fm_bulk_insert", "fm_bulk_remove", "fm_len",
              "fm_capacity", "fm_load_factor", "fm_clear", "fm_device", "fm_bulk_get_device",
              "fm_bulk_get_values_device", "fm_bulk_insert_device", "fm_bulk_insert_device_uncounted",
              "fm_recount", "fm_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    import flash_map

    lib = ctypes.CDLL(flash_map.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) == set(flash_map.EXPORTS)


def test_status_codes_map_to_reference_errors():
    from flash_map import errors as E

    cases = {1: E.CudaInit, 2: E.GpuAlloc, 3: E.KernelLaunch, 4: E.Transfer, 6: E.ZeroCapacity, 7: E.KernelLaunch,
             8: E.KernelLaunch, 9: E.KernelLaunch}
    for rc, cls in cases.items():
        with pytest.raises(cls):
            E.raise_for_status(rc, "x")
    with pytest.raises(E.TableFull) as ei:
        E.raise_for_status(5, "", occupied=16, capacity=16)
    assert ei.value.occupied == 16 and ei.value.load_factor == 100.0
    assert str(ei.value) == "table full: 16 occupied of 16 capacity (load factor 100.0%)"
    E.raise_for_status(0, "")


def test_no_gpu_fails_loudly():
    """Without a usable GPU the product path raises; it never falls back."""
    import flash_map as F

    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(F.CudaInit):
        F.FlashMap.with_capacity(1024)


def test_builder_force_cpu_is_refused():
    import flash_map as F

    with pytest.raises(F.NoBackend):
        F.FlashMap.builder(64).force_cpu().build()


def test_zero_capacity_before_device_use():
    import flash_map as F

    with pytest.raises(F.ZeroCapacity):
        F.FlashMap(0, 8, 8)


def test_device_buffers_smaller_than_the_call_are_refused():
    """The kernels read and write count records from each device pointer and
    cannot see a buffer's end: a tensor that holds fewer bytes than the call
    needs is refused on the host, before any launch."""
    import torch

    from flash_map.map import _dev_ptr

    t = torch.zeros((50, 32), dtype=torch.uint8)
    assert _dev_ptr(t, 50 * 32, "keys") == t.data_ptr()
    with pytest.raises(ValueError, match="keys: 1600 bytes, the call needs 3200"):
        _dev_ptr(t, 100 * 32, "keys")
    w = torch.zeros(100, dtype=torch.int64)  # sized in bytes, not elements
    assert _dev_ptr(w, 800, "values") == w.data_ptr()
    assert _dev_ptr(12345, 1 << 40) == 12345  # a raw pointer is the caller's to size
