"""The library against the reference's own encoders and compression tree, run on the same GPU.

oracle/_ref/libref_enc.so is the reference's compression/, util/ and tree/ sources compiled as
they are (oracle/Makefile, target refenc; oracle/ref_enc_shim.cu).  Here the library's streams
and blobs are byte-compared with what the reference itself returns for the same columns, at sizes
up to 2^22 values: every encoding the reference implements for each type
(Encoding::Encode through the factory's Get(data), as tree/compression_node.cpp:103-110 calls
it) and the benchmark configurations' trees (CompressionTree::Compress).  The reference's
decoders are not run; the library decodes the reference's own blobs instead.

The reference's launch policy (core/execution_policy.hpp:24-33) covers at most 65535 * 1024
elements per kernel (its kernels index with blockIdx.x only), so its outputs are only complete
below 2^26 values; the sizes here stay below that.  Code slots that the reference fills from values
read past the end of its input (unique_encoding.cu:56-61) are cleared on both sides before the
comparison (tests/golden/refcases.py).
"""
import os
import sys

import numpy as np
import pytest

import oracle as OR
from gputimeseriescompressionoptimizer_b200 import workloads as W

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import refcases as RC  # noqa: E402

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not os.path.exists(OR.REF_ENC_PATH),
                       reason="oracle/_ref/libref_enc.so not built (make -C oracle refenc where the reference is)"),
]

SEED = 0xFEED
ENC_SIZES = [4097, 1 << 18]
TREE_SIZES = [1 << 16, 1 << 22]
CONFIG_TREES = [
    ("walk", OR.INT, [OR.DELTA, OR.AFL, OR.NONE]),
    ("walk", OR.INT, [OR.DELTA, OR.SCALE, OR.AFL, OR.NONE]),
    ("runs", OR.INT, [OR.RLE, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("zipf", OR.INT, [OR.DICT, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("const", OR.INT, [OR.CONST, OR.AFL, OR.NONE]),
    ("outliers", OR.INT, [OR.PATCH, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("outliers", OR.INT, [OR.PATCH_OUTSIDE, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("price", OR.FLOAT, [OR.FLOAT2INT, OR.DELTA, OR.AFL, OR.NONE]),
    ("walk", OR.TIME, [OR.DELTA, OR.RLE, OR.AFL, OR.NONE, OR.DELTA, OR.AFL, OR.NONE]),
]


def _ref_encode_or_skip(enc, dt, x):
    try:
        res = OR.ref_encode(enc, dt, x)
    except OR.OracleError as e:
        pytest.skip(f"the reference refuses {OR.ENC_NAMES[enc]} on type {dt}: {e}")
    if not res:
        # e.g. AflEncoding::EncodeDouble returns no buffers (compression/afl/afl_encoding.hpp)
        pytest.skip(f"the reference returns no streams for {OR.ENC_NAMES[enc]} on type {dt}")
    return res


@pytest.mark.parametrize("n", ENC_SIZES)
@pytest.mark.parametrize("dt", RC.DTYPES)
@pytest.mark.parametrize("enc", RC.ENCODINGS, ids=[OR.ENC_NAMES[e] for e in RC.ENCODINGS])
def test_encoding_matches_reference(G, enc, dt, n):
    for j, kind in enumerate(RC.kinds_of(dt)):
        x = W.column(kind, dt, n, SEED + 31 * j + enc)
        if RC.lossy_in_reference(enc, dt, x):
            continue
        ref = RC.canonical(enc, dt, _ref_encode_or_skip(enc, dt, x))
        parts = G.encode(enc, dt, G.to_device(x))
        ours = RC.canonical(enc, dt, [G.to_host(p) for p in parts])
        assert len(ours) == len(ref), (OR.ENC_NAMES[enc], kind)
        for k, (a, b) in enumerate(zip(ours, ref)):
            assert a.size == b.size and np.array_equal(a, b), \
                f"{OR.ENC_NAMES[enc]} dt={dt} {kind} n={n} stream {k}: sizes {a.size} vs {b.size}"
        # the library decodes the reference's streams back to the column
        back = G.to_host(G.decode(enc, dt, [G.to_device(r) for r in ref]))
        assert back.tobytes() == x.tobytes(), f"{OR.ENC_NAMES[enc]} dt={dt} {kind} n={n} decode"


@pytest.mark.parametrize("n", TREE_SIZES)
@pytest.mark.parametrize("case", range(len(CONFIG_TREES)))
def test_tree_matches_reference(G, case, n):
    kind, dt, path = CONFIG_TREES[case]
    x = W.column(kind, dt, n, SEED + 1000 + case)
    nodes = OR.tree_from_path(path, dt)
    ref = OR.ref_tree_compress(nodes, x)
    blob = G.tree_compress(nodes, G.to_device(x))
    ours = G.to_host(blob)
    assert ours.size == ref.size and np.array_equal(ours, ref), (G.tree_names(nodes), ours.size, ref.size)
    out, odt = G.tree_decompress(G.to_device(ref))
    assert odt == dt and G.to_host(out).tobytes() == x.tobytes()


@pytest.mark.parametrize("case", range(len(CONFIG_TREES)))
def test_batch_matches_reference(G, case):
    """The batched engine's blob of a configuration column equals the reference tree's blob."""
    kind, dt, path = CONFIG_TREES[case]
    n = 1 << 20
    x = W.column(kind, dt, n, SEED + 2000 + case)
    nodes = OR.tree_from_path(path, dt)
    ref = OR.ref_tree_compress(nodes, x)
    st = G.Stream()
    dev = G.to_device(x)
    b = G.Batch([dev], [dt], [nodes], st)
    b.compress()
    b.status()
    p, nb = b.output()
    blobs = G.split_framed(G.to_host(G.DeviceBuffer(p, nb, owned=False)))
    assert len(blobs) == 1
    assert blobs[0].size == ref.size and np.array_equal(blobs[0], ref)
