"""gtsc_delta_decode_noalloc: the delta decode for callers that cannot allocate device memory (a
host framework owning every allocation through its own pool).  It must give exactly what the
allocating gtsc_decode(GTSC_DELTA) gives, on consecutive calls that share its static scratch.

This file is collected last on purpose: a run that stops at the first failure has run every other
test before it."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,npt", [(2, np.int32), (3, np.int64), (4, np.float32), (1, np.int16)])
def test_noalloc_delta_decode_matches_allocating_decode(G, rng, dtype, npt):
    L = G.lib()
    for n in (1 << 20, 70001):  # two calls in a row, the second one smaller than the first
        if np.issubdtype(npt, np.floating):
            x = rng.normal(0, 100, n).astype(npt)
        else:
            x = rng.integers(np.iinfo(npt).min // 2, np.iinfo(npt).max // 2, n).astype(npt)
        meta, deltas = G.encode(G.DELTA, dtype, G.to_device(x))
        expected = G.to_host(G.decode(G.DELTA, dtype, [meta, deltas]))
        out = G.alloc(x.nbytes)
        es = x.itemsize
        G.check(L.gtsc_delta_decode_noalloc(dtype, meta.ptr, deltas.ptr, deltas.nbytes // es, out.ptr, None),
                "delta_decode_noalloc")
        got = G.to_host(out)
        assert got.tobytes() == expected.tobytes() == x.tobytes()


def test_noalloc_rejects_sizes_beyond_its_scratch(G):
    L = G.lib()
    first, deltas, out = G.alloc(16), G.alloc(64), G.alloc(64)
    big = 1 << 24  # n_deltas + 1 > 2^24: refused before any device work
    st = L.gtsc_delta_decode_noalloc(2, first.ptr, deltas.ptr, big, out.ptr, None)
    assert st == -3
    assert b"2^24" in L.gtsc_last_error()
