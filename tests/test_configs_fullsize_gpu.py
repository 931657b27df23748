"""The benchmark configurations at their stated sizes against the oracle.

Each configuration's column is generated with its seeded generator at full size and compressed
three ways -- the single encoding (config 1) or the configuration's compression tree through
gtsc_tree_compress, and all columns together through the batched engine -- and every stream is
byte-compared with the oracle's CompressionTree::Compress (tree/compression_tree.cpp:98-155) of the
same column.  Every decode (of our blob and of the oracle's blob) must give back the input bit for
bit, NaN payloads, +-inf and -0.0 included (GFC: gfc_encoding_impl_double.cu:31-90,
gfc_encoding_impl_float.cu).

Sizes: config 1 is 2^20 int32 values at bit width 11; configs 2a-2e are 2^26 int32 values each;
config 3 is 2^26 float64 values plus the same series as float32.  The oracle runs in host threads
(its C calls release the GIL), so the whole module takes a minute or two on a many-core host.
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

import oracle as OR
from gputimeseriescompressionoptimizer_b200 import workloads as W

pytestmark = pytest.mark.gpu

N_CHAIN = 1 << 26
SEED = 0xB200

# (config, generator, data type, compression tree as a pre-order encoding list)
CONFIGS = [
    ("2a delta-afl", "walk", OR.INT, [OR.DELTA, OR.AFL, OR.NONE]),
    ("2a delta-scale-afl", "walk", OR.INT, [OR.DELTA, OR.SCALE, OR.AFL, OR.NONE]),
    ("2b rle-afl-afl", "runs", OR.INT, [OR.RLE, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("2c dict-afl-afl", "zipf", OR.INT, [OR.DICT, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("2d const-afl", "const", OR.INT, [OR.CONST, OR.AFL, OR.NONE]),
    ("2e patch-afl-afl", "outliers", OR.INT, [OR.PATCH, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("3 gfc double", "price", OR.DOUBLE, [OR.GFC, OR.NONE, OR.NONE]),
    ("3 gfc float", "price", OR.FLOAT, [OR.GFC, OR.NONE, OR.NONE]),
]
IDS = [c[0].replace(" ", "_") for c in CONFIGS]


def _threads():
    return max(1, min(len(CONFIGS), os.cpu_count() or 1))


@pytest.fixture(scope="module")
def columns(G):
    """Every configuration's column, its tree and the oracle's blob of it."""
    def one(k):
        name, kind, dt, path = CONFIGS[k]
        x = W.column(kind, dt, N_CHAIN, SEED + 2 + (k if kind != "price" else 8))
        nodes = OR.tree_from_path(path, dt)
        return x, nodes, OR.tree_compress(nodes, x)

    with cf.ThreadPoolExecutor(_threads()) as ex:
        return list(ex.map(one, range(len(CONFIGS))))


def test_config1_afl_single_encoding(G, O):
    """2^20 int32 uniform in [0, 2^11): AFL alone at bit width 11, byte-compared with the oracle
    (afl_encoding.cu:15-56) and decoded bit-exact."""
    rng = np.random.default_rng(SEED + 1)
    x = rng.integers(0, 1 << 11, 1 << 20).astype(np.int32)
    parts = G.encode(G.AFL, G.INT, G.to_device(x))
    host = [G.to_host(p) for p in parts]
    expect = O.encode(O.AFL, O.INT, x)
    assert host[0][0] == 11 and host[1].size == 1441792
    assert len(host) == len(expect)
    for h, e in zip(host, expect):
        assert np.array_equal(h, e)
    assert G.to_host(G.decode(G.AFL, G.INT, parts)).tobytes() == x.tobytes()


def test_config1_afl_matches_reference_host_code(G, O):
    """The same stream against the reference's own run_afl_compress_cpu<int,1> (afl_gpu.cu), when
    it was built into oracle/_ref."""
    if not O.build_ref():
        pytest.skip("the reference's AFL host path was not built")
    rng = np.random.default_rng(SEED + 1)
    x = rng.integers(0, 1 << 11, 1 << 20).astype(np.int32)
    parts = G.encode(G.AFL, G.INT, G.to_device(x))
    assert np.array_equal(G.to_host(parts[1]), O.ref_afl_compress(O.INT, x, 11))


@pytest.mark.parametrize("k", range(len(CONFIGS)), ids=IDS)
def test_tree_full_size(G, O, columns, k):
    """gtsc_tree_compress of the configuration's tree at 2^26 values: blob byte-identical to the
    oracle's, our decode and the decode of the oracle's blob bit-exact."""
    x, nodes, ob = columns[k]
    dev = G.to_device(x)
    blob = G.tree_compress(nodes, dev)
    hb = G.to_host(blob)
    assert hb.size == ob.size, (CONFIGS[k][0], hb.size, ob.size)
    assert np.array_equal(hb, ob), CONFIGS[k][0]
    out, dt = G.tree_decompress(blob)
    assert dt == CONFIGS[k][2]
    assert G.to_host(out).tobytes() == x.tobytes(), CONFIGS[k][0]
    del out
    out2, _ = G.tree_decompress(G.to_device(ob))
    assert G.to_host(out2).tobytes() == x.tobytes(), CONFIGS[k][0] + " (oracle's blob)"


def test_batch_full_size(G, O, columns):
    """All configurations' columns in one batch: each framed blob byte-identical to the oracle's,
    and the batched decompress bit-exact, over two replayed steps."""
    st = G.Stream()
    devs = [G.to_device(x) for x, _, _ in columns]
    b = G.Batch(devs, [c[2] for c in CONFIGS], [n for _, n, _ in columns], st)
    for step in range(2):
        b.compress()
        b.status()
        p, nb = b.output()
        blobs = G.split_framed(G.to_host(G.DeviceBuffer(p, nb, owned=False)))
        assert len(blobs) == len(columns)
        for k, (x, _, ob) in enumerate(columns):
            assert blobs[k].size == ob.size and np.array_equal(blobs[k], ob), (step, CONFIGS[k][0])
        outs = [G.alloc(x.nbytes) for x, _, _ in columns]
        b.decompress(p, nb, outs)
        b.status()
        for k, (x, _, _) in enumerate(columns):
            assert G.to_host(outs[k]).tobytes() == x.tobytes(), (step, CONFIGS[k][0])
        del outs


def test_config_streams_have_expected_shape(columns):
    """Sanity of the generators against the configurations' stated properties (from the oracle's
    blobs): delta->AFL of the walk needs 32 bits (negative deltas, no zigzag), RLE of runs with mean
    length 32 gives about 2^21 runs, the const column compresses to its stencil, GFC is lossless."""
    walk_blob = columns[0][2]
    # header(8) + delta meta(4) | header(8) + AFL meta: byte 0 is the bit width
    assert walk_blob[8 + 4 + 8] == 32
    runs_x = columns[2][0]
    n_runs = int(np.count_nonzero(runs_x[1:] != runs_x[:-1])) + 1
    assert 1.8e6 < n_runs < 2.4e6
    assert columns[4][2].size < (N_CHAIN // 8) + 4096
