"""Compression trees and planners on the GPU against the oracle (tree/compression_tree_unittest.cpp and
optimizer/optimizer_unittest.cpp are the reference's tests of these): byte-identical blobs, bit-exact
round trips, predicted size == actual, and the same tree chosen by both planners."""
import numpy as np
import pytest

import oracle as OR

pytestmark = pytest.mark.gpu

FIRST = [[], [OR.FLOAT2INT], [OR.DELTA], [OR.SCALE], [OR.DELTA, OR.FLOAT2INT], [OR.SCALE, OR.FLOAT2INT]]
SECOND = [[OR.DICT, OR.AFL, OR.NONE, OR.AFL, OR.NONE], [OR.CONST, OR.AFL, OR.NONE],
          [OR.RLE, OR.AFL, OR.NONE, OR.AFL, OR.NONE], [OR.AFL, OR.NONE],
          [OR.PATCH, OR.AFL, OR.NONE, OR.AFL, OR.NONE]]
PATHS = [a + b for a in FIRST for b in SECOND]


def ts_like(rng, n):
    """timestamps-like int column (stands in for the reference's missing info.log test file)"""
    return (np.cumsum(rng.exponential(30, n)).astype(np.int64) % (1 << 30)).astype(np.int32)


def pattern_a(rng, n, npt):
    """runs of a few values with rare outliers (stands in for GetFakeDataWithPatternA)"""
    x = np.repeat(rng.integers(0, 8, n // 16 + 1) * 1.5, 16)[:n]
    idx = rng.choice(n, max(n // 200, 1), replace=False)
    x[idx] = 1e6
    return x.astype(npt)


def pattern_b(rng, n):
    """piecewise random walks with jumps (stands in for GetFakeDataWithPatternB)"""
    x = np.cumsum(rng.integers(-3, 4, n))
    x[n // 2:] += 10000
    return np.clip(x, -10000, 20000).astype(np.int32)


def roundtrip(G, O, nodes, x):
    nodes = np.asarray(nodes, np.int16)
    dev = G.to_device(x)
    blob = G.tree_compress(nodes, dev)
    hb = G.to_host(blob)
    ob = O.tree_compress(nodes, x)
    assert hb.size == ob.size and np.array_equal(hb, ob), (G.tree_names(nodes), hb.size, ob.size)
    out, dt = G.tree_decompress(blob)
    assert dt == nodes[1]
    assert G.to_host(out).tobytes() == x.tobytes(), G.tree_names(nodes)
    return hb.size


@pytest.mark.parametrize("path", PATHS, ids=["-".join(OR.ENC_NAMES[e] for e in p) for p in PATHS])
def test_generated_paths_roundtrip_and_predicted_size(G, O, rng, path):
    """optimizer_unittest.cpp:64-81, compression_tree_unittest.cpp:238-258"""
    x = ts_like(rng, 20000)
    nodes = G.tree_from_path(path, OR.INT)
    assert np.array_equal(nodes, O.tree_from_path(path, OR.INT))
    size = roundtrip(G, O, nodes, x)
    assert G.tree_predict_size(nodes, G.to_device(x)) == size == O.tree_predict_size(nodes, x)


TREES = [
    ([OR.DELTA, OR.NONE], OR.INT, "int"),
    ([OR.DELTA, OR.SCALE, OR.NONE], OR.INT, "int"),
    ([OR.DICT, OR.SCALE, OR.DELTA, OR.NONE, OR.DELTA, OR.NONE], OR.INT, "int"),
    ([OR.PATCH, OR.DICT, OR.DELTA, OR.NONE, OR.SCALE, OR.NONE, OR.DELTA, OR.NONE], OR.INT, "int"),
    ([OR.SCALE, OR.DELTA, OR.PATCH, OR.AFL, OR.NONE, OR.NONE], OR.INT, "ts"),
    ([OR.PATCH, OR.CONST, OR.NONE, OR.FLOAT2INT, OR.RLE, OR.CONST, OR.NONE, OR.SCALE, OR.AFL, OR.NONE],
     OR.FLOAT, "a"),
    ([OR.DELTA, OR.FLOAT2INT, OR.AFL, OR.NONE], OR.FLOAT, "prec3"),
    ([OR.SCALE, OR.DELTA, OR.GFC, OR.NONE, OR.NONE], OR.FLOAT, "prec3"),
    ([OR.GFC, OR.NONE, OR.NONE], OR.FLOAT, "a"),
    ([OR.DICT, OR.NONE, OR.NONE], OR.FLOAT, "a"),
    ([OR.DICT, OR.SCALE, OR.DELTA, OR.GFC, OR.NONE, OR.NONE, OR.DELTA, OR.FLOAT2INT, OR.AFL, OR.NONE],
     OR.FLOAT, "a"),
    ([OR.DELTA, OR.PATCH, OR.DELTA, OR.AFL, OR.NONE, OR.DELTA, OR.AFL, OR.NONE], OR.TIME, "ts"),
    ([OR.DELTA, OR.RLE, OR.AFL, OR.NONE, OR.AFL, OR.NONE], OR.INT, "b"),
    ([OR.PATCH, OR.DELTA, OR.SCALE, OR.AFL, OR.NONE, OR.DELTA, OR.SCALE, OR.AFL, OR.NONE], OR.INT, "b"),
    ([OR.GFC, OR.NONE, OR.NONE], OR.DOUBLE, "prec3"),
    ([OR.DELTA, OR.GFC, OR.NONE, OR.NONE], OR.DOUBLE, "prec3"),
    # ComplexTree_Patch (compression_tree_unittest.cpp:124-150): an outside patch root
    ([OR.PATCH_OUTSIDE, OR.DICT, OR.DELTA, OR.NONE, OR.SCALE, OR.NONE, OR.DELTA, OR.NONE], OR.INT, "int"),
    ([OR.PATCH_OUTSIDE, OR.AFL, OR.NONE, OR.AFL, OR.NONE], OR.INT, "ts"),
    ([OR.SCALE, OR.PATCH_OUTSIDE, OR.GFC, OR.NONE, OR.NONE, OR.NONE], OR.DOUBLE, "prec3"),
]


@pytest.mark.parametrize("path,dt,kind", TREES)
@pytest.mark.parametrize("n", [10, 1000, 10000])
def test_reference_tree_shapes(G, O, rng, path, dt, kind, n):
    """tree shapes of compression_tree_unittest.cpp:70-536"""
    npt = OR.NP_TYPES[dt]
    if kind == "int":
        x = rng.integers(-1000, 1000, n).astype(npt)
    elif kind == "ts":
        x = ts_like(rng, n).astype(npt)
    elif kind == "a":
        x = pattern_a(rng, n, npt)
    elif kind == "b":
        x = pattern_b(rng, n).astype(npt)
    else:
        x = np.round(rng.normal(0, 100, n), 3).astype(npt)
    nodes = G.tree_from_path(path, dt)
    roundtrip(G, O, nodes, x)


def planner_columns(rng):
    n = 3000
    yield OR.INT, (np.cumsum(rng.integers(-8, 9, n)) + 10 ** 6).astype(np.int32)
    yield OR.INT, np.repeat(rng.integers(0, 16, n // 32 + 1), 32)[:n].astype(np.int32)
    yield OR.INT, (np.minimum(rng.zipf(1.1, n), 5000) - 1).astype(np.int32)
    yield OR.INT, np.full(n, 12345, np.int32)
    x = rng.integers(0, 256, n).astype(np.int32)
    x[rng.choice(n, 30, replace=False)] = rng.integers(0, 2 ** 31 - 1, 30)
    yield OR.INT, x
    yield OR.TIME, np.cumsum(rng.exponential(1000, n)).astype(np.int64)
    yield OR.DOUBLE, np.round(100 * np.sin(np.arange(n) / 50) + rng.normal(0, 0.01, n), 2)
    yield OR.FLOAT, np.round(rng.normal(50, 10, n), 2).astype(np.float32)
    yield OR.SHORT, rng.integers(0, 100, n).astype(np.int16)


def test_exhaustive_planner_matches_oracle(G, O, rng):
    for dt, x in planner_columns(rng):
        nodes, size = G.plan_exhaustive(dt, G.to_device(x))
        onodes, osize = O.plan_exhaustive(dt, x)
        assert np.array_equal(nodes, onodes), (dt, G.tree_names(nodes), G.tree_names(onodes))
        assert size == osize
        roundtrip(G, O, nodes, x)


def test_optimize_tree_matches_oracle(G, O, rng):
    for dt, x in planner_columns(rng):
        if dt not in (OR.INT,):
            continue  # the reference's AFL size predictor only exists for int (afl_encoding.cu:281-293)
        nodes, size = G.optimize_tree(dt, G.to_device(x))
        onodes, osize = O.optimize_tree(dt, x)
        assert np.array_equal(nodes, onodes) and size == osize


def test_corrupt_blob_fails_cleanly(G, O, rng):
    x = ts_like(rng, 5000)
    nodes = G.tree_from_path([OR.DELTA, OR.PATCH, OR.AFL, OR.NONE, OR.AFL, OR.NONE], OR.INT)
    blob = O.tree_compress(nodes, x)
    for cut in [3, 9, 20, blob.size // 2, blob.size - 1]:
        with pytest.raises(G.GtscError):
            G.tree_decompress(G.to_device(blob[:cut]))
    bad = blob.copy()
    bad[0] = 99  # unknown encoding type
    with pytest.raises(G.GtscError):
        G.tree_decompress(G.to_device(bad))
    with pytest.raises(G.GtscError):
        G.tree_compress(np.array([OR.DELTA, OR.INT], np.int16), G.to_device(x))  # leaf is not none
