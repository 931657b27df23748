"""gtsc_delta_decode_noalloc: the delta decode for callers that cannot allocate device memory (a
host framework owning every allocation through its own pool).  It must give exactly what the
allocating gtsc_decode(GTSC_DELTA) gives, on consecutive calls that share its static scratch, up to
its stated limit of 2^24 values, and it must leave the device's memory as it found it.

This file is collected last on purpose: a run that stops at the first failure has run every other
test before it."""
import ctypes
import gc

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_VALUES = 1 << 24
CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT = 5   # cuda.h, CUmemPool_attribute
CU_MEMPOOL_ATTR_USED_MEM_CURRENT = 7


def _column(rng, npt, n):
    if np.issubdtype(npt, np.floating):
        return rng.normal(0, 100, n).astype(npt)
    return rng.integers(np.iinfo(npt).min // 2, np.iinfo(npt).max // 2, n).astype(npt)


def _noalloc(G, dtype, meta, deltas, n_deltas, out):
    return G.lib().gtsc_delta_decode_noalloc(dtype, meta.ptr, deltas.ptr if n_deltas else None, n_deltas,
                                             out.ptr, None)


def _check_against_allocating_decode(G, dtype, x):
    meta, deltas = G.encode(G.DELTA, dtype, G.to_device(x))
    expected = G.to_host(G.decode(G.DELTA, dtype, [meta, deltas]))
    out = G.alloc(max(x.nbytes, 16))
    G.check(_noalloc(G, dtype, meta, deltas, x.size - 1, out), "delta_decode_noalloc")
    got = G.to_host(out)[:x.nbytes]
    assert got.tobytes() == expected.tobytes() == x.tobytes()


@pytest.mark.parametrize("dtype,npt", [(2, np.int32), (3, np.int64), (4, np.float32), (1, np.int16)])
def test_noalloc_delta_decode_matches_allocating_decode(G, rng, dtype, npt):
    for n in (1 << 20, 70001):  # two calls in a row, the second one smaller than the first
        _check_against_allocating_decode(G, dtype, _column(rng, npt, n))


def test_noalloc_capacity_boundary_and_single_value(G, rng):
    """Exactly 2^24 values (n_deltas = 2^24 - 1, every one of the 8192 scratch tiles in use), then a
    column of one value (no deltas at all), then the full size again."""
    _check_against_allocating_decode(G, 2, _column(rng, np.int32, MAX_VALUES))
    _check_against_allocating_decode(G, 2, np.array([123456789], np.int32))
    _check_against_allocating_decode(G, 3, _column(rng, np.int64, MAX_VALUES))


def _device_memory_state():
    """(default pool bytes in use, default pool bytes reserved, free device bytes) of the current
    device, from the driver API."""
    cu = ctypes.CDLL("libcuda.so.1")
    dev = ctypes.c_int(0)
    assert cu.cuCtxGetDevice(ctypes.byref(dev)) == 0
    pool = ctypes.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(ctypes.byref(pool), dev) == 0
    used, reserved = ctypes.c_uint64(0), ctypes.c_uint64(0)
    assert cu.cuMemPoolGetAttribute(pool, CU_MEMPOOL_ATTR_USED_MEM_CURRENT, ctypes.byref(used)) == 0
    assert cu.cuMemPoolGetAttribute(pool, CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT, ctypes.byref(reserved)) == 0
    free, total = ctypes.c_size_t(0), ctypes.c_size_t(0)
    assert cu.cuMemGetInfo_v2(ctypes.byref(free), ctypes.byref(total)) == 0
    return used.value, reserved.value, free.value


def test_noalloc_allocates_no_device_memory(G, rng):
    """Around two calls (after a first one that may load the library's module on the device), the
    default memory pool's used and reserved bytes and the device's free memory do not move."""
    x = _column(rng, np.int32, 3 << 20)
    meta, deltas = G.encode(G.DELTA, 2, G.to_device(x))
    outs = [G.alloc(x.nbytes) for _ in range(2)]
    G.check(_noalloc(G, 2, meta, deltas, x.size - 1, outs[0]), "delta_decode_noalloc")
    G.lib().gtsc_stream_synchronize(None)
    gc.collect()
    gc.disable()  # no buffer of an earlier test is released inside the window
    try:
        before = _device_memory_state()
        for o in outs:
            G.check(_noalloc(G, 2, meta, deltas, x.size - 1, o), "delta_decode_noalloc")
        after = _device_memory_state()
    finally:
        gc.enable()
    assert after == before, (before, after)
    for o in outs:
        assert G.to_host(o).tobytes() == x.tobytes()


def test_noalloc_rejects_sizes_beyond_its_scratch(G):
    L = G.lib()
    first, deltas, out = G.alloc(16), G.alloc(64), G.alloc(64)
    big = MAX_VALUES  # n_deltas + 1 > 2^24: refused before any device work
    st = L.gtsc_delta_decode_noalloc(2, first.ptr, deltas.ptr, big, out.ptr, None)
    assert st == -3
    assert b"2^24" in L.gtsc_last_error()
