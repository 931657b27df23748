"""The column-chunk pipeline (ParallelTSCompressor::Compress's chunk loop on the batched engine):
chunks from host memory come back as per-group framed buffers whose blobs are the per-column
trees' blobs, successive chunks reuse the engines, and the device decode restores every column."""
import ctypes

import numpy as np
import pytest

import oracle as OR
from test_tree_gpu import PATHS, ts_like, pattern_b

pytestmark = pytest.mark.gpu


def test_pipeline_chunks(G, O, rng):
    trees, sizes, dts = [], [], []
    n_cols = 13
    for i in range(n_cols):
        n = [1, 100, 5000, 70001, 3000][i % 5]
        trees.append(G.tree_from_path(PATHS[i % len(PATHS)], OR.INT))
        sizes.append(4 * n)
        dts.append(OR.INT)
    P = G.Pipeline(sizes, dts, trees, groups=4)
    assert P.groups == 4
    cap = 8 * sum(sizes) + 4096 * n_cols
    framed = np.zeros(cap, np.uint8)
    for chunk in range(3):
        cols = [(ts_like(rng, s // 4) if chunk % 2 == 0 else pattern_b(rng, s // 4)) for s in sizes]
        if chunk == 2:
            gb = P.roundtrip_host([c.ctypes.data for c in cols], framed.ctypes.data, cap)
        else:
            gb = P.compress_host([c.ctypes.data for c in cols], framed.ctypes.data, cap)
        pos = 0
        seen = set()
        for g in range(P.groups):
            part = framed[pos:pos + int(gb[g])]
            pos += int(gb[g])
            members = P.group_columns(g)
            blobs = G.split_framed(part)
            assert len(blobs) == len(members)
            for c, b in zip(members, blobs):
                assert np.array_equal(b, O.tree_compress(trees[c], cols[c])), (chunk, c)
                seen.add(c)
        assert seen == set(range(n_cols))
        if chunk != 2:
            P.decompress()
        for c, x in enumerate(cols):
            _, d_out = P.column(c)
            out = np.zeros(x.nbytes, np.uint8)
            if x.nbytes:
                G.check(G.lib().gtsc_memcpy(out.ctypes.data, d_out, x.nbytes, 2, None), "d2h")
            assert out.tobytes() == x.tobytes(), (chunk, c)
