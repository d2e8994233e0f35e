"""Conservation sums through the entry point that allocates nothing.

flb_reduce_conservation_noalloc serves callers that must not have this library
call cudaMalloc: programs whose GPU memory comes only from their own caching
pool (allocating outside it breaks their accounting and can stall their
streams), or loops that may not wait on an allocation.  They pass their own
device arrays; the reduction keeps its scratch in a fixed array inside the
library.  These tests call it through the C ABI and compare it with the
allocating flb_reduce_conservation on the same lattice, on consecutive calls
(every call reuses the scratch the previous call left behind).  This file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

import freelb_b200 as F
from freelb_b200 import _capi as C

pytestmark = pytest.mark.gpu

STORAGE = {"fp32": C.STORAGE_FP32, "fp16s": C.STORAGE_FP16S, "fp64": C.STORAGE_FP64,
           "fp32s": C.STORAGE_FP32S}


def noalloc_sums(lat, key):
    """Call the no-allocation reduction on the lattice's own device arrays."""
    lib = C.load()
    pops, flags = ctypes.c_void_p(), ctypes.c_void_p()
    C.call("flb_device_pointers", lat._h, ctypes.byref(pops), ctypes.byref(flags), None, None)
    layout = lat.layout()
    out = (ctypes.c_double * 4)()
    rc = lib.flb_reduce_conservation_noalloc(pops, flags, ctypes.byref(layout),
                                             STORAGE[lat.storage], 1.0, key, out, None)
    assert rc == 0, lib.flb_last_error().decode()
    return np.array(out[:])


def assert_same_sums(got, want):
    # same FP64 sums, different summation order
    scale = max(1.0, float(np.max(np.abs(want))))
    assert np.all(np.abs(got - want) <= 1e-12 * scale), (got, want)


@pytest.mark.parametrize("storage", ["fp32", "fp16s", "fp64", "fp32s"])
def test_noalloc_matches_allocating_reduction_on_consecutive_calls(gpu_ok, storage):
    lat = F.cavity(40, tau=0.55, ulid=0.1, storage=storage)
    lat.step(25)
    for key in (2, 0xFF):
        first = noalloc_sums(lat, key)
        assert_same_sums(first, lat.conservation(key))
        second = noalloc_sums(lat, key)       # same state: identical result
        assert np.array_equal(first, second)
    lat.step(7)                                # new state, scratch still holds the old sums
    assert_same_sums(noalloc_sums(lat, 2), lat.conservation(2))


def test_noalloc_smaller_lattice_after_larger(gpu_ok):
    """A small lattice after a large one reads only the scratch slots it wrote."""
    big = F.cavity(96, storage="fp32")
    big.step(3)
    assert_same_sums(noalloc_sums(big, 0xFF), big.conservation(0xFF))
    small = F.cavity(12, storage="fp32")
    small.step(5)
    assert_same_sums(noalloc_sums(small, 2), small.conservation(2))
    assert_same_sums(noalloc_sums(small, 2), small.conservation(2))


def test_noalloc_rejects_layouts_beyond_its_scratch(gpu_ok):
    """Lattices above 268,435,456 padded cells are refused before any GPU work."""
    lat = F.cavity(8, storage="fp32")
    lib = C.load()
    pops, flags = ctypes.c_void_p(), ctypes.c_void_p()
    C.call("flb_device_pointers", lat._h, ctypes.byref(pops), ctypes.byref(flags), None, None)
    L = C.Layout()
    L.nx, L.ny, L.nz = 1024, 1024, 300
    L.pitch_x = 1024
    L.plane = 1024 * 1024
    L.dir_stride = L.plane * 300
    L.elem_bytes = 4
    out = (ctypes.c_double * 4)()
    rc = lib.flb_reduce_conservation_noalloc(pops, flags, ctypes.byref(L), C.STORAGE_FP32, 1.0,
                                             2, out, None)
    assert rc == -1    # FLB_ERR_INVALID
    assert "268435456" in lib.flb_last_error().decode()


def test_noalloc_rejects_host_memory(gpu_ok):
    """Arrays that are not device memory of the current device are refused
    before any GPU work (the scratch and the kernels are the current device's)."""
    lat = F.cavity(8, storage="fp32")
    lib = C.load()
    host = np.zeros(19 * lat.layout().dir_stride, dtype=np.float32)
    flags = ctypes.c_void_p()
    C.call("flb_device_pointers", lat._h, None, ctypes.byref(flags), None, None)
    out = (ctypes.c_double * 4)()
    rc = lib.flb_reduce_conservation_noalloc(ctypes.c_void_p(host.ctypes.data), flags,
                                             ctypes.byref(lat.layout()), C.STORAGE_FP32, 1.0,
                                             2, out, None)
    assert rc == -1    # FLB_ERR_INVALID
    assert "device memory" in lib.flb_last_error().decode()
