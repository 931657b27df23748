"""Every encoding on the GPU against the oracle: byte-identical streams, bit-exact decode (NaN
payloads, +-0, +-inf included), and decode of the oracle's stream.  Mirrors the reference's
per-encoding round-trip tests (compression/*/`*_unittest.cpp`) with byte-level checks added."""
import numpy as np
import pytest

import oracle as OR

pytestmark = pytest.mark.gpu

INT_TYPES = [(OR.CHAR, np.int8), (OR.SHORT, np.int16), (OR.INT, np.int32), (OR.TIME, np.int64)]
FP_TYPES = [(OR.FLOAT, np.float32), (OR.DOUBLE, np.float64)]
ALL_TYPES = INT_TYPES + FP_TYPES
SIZES = [0, 1, 2, 7, 33, 1000, 2049, 65537]


def gen(kind, npt, n, rng):
    """Seeded column generators covering the encodings' interesting cases."""
    fp = np.issubdtype(npt, np.floating)
    if kind == "uniform":
        x = rng.normal(0, 1000, n) if fp else rng.integers(-100, 100, n)
    elif kind == "walk":
        x = np.cumsum(rng.integers(-8, 9, n)) + 1000
        x = x / 100.0 if fp else x
    elif kind == "runs":
        x = np.repeat(rng.integers(0, 16, n + 1), rng.integers(1, 16, n + 1))[:n]
        x = x / 4.0 if fp else x
    elif kind == "const":
        x = np.full(n, 7)
    elif kind == "zipf":
        x = np.minimum(rng.zipf(1.3, n), 5000) - 1
    elif kind == "outliers":
        x = rng.integers(0, 256, n)
        k = max(n // 100, 0)
        if k:
            idx = rng.choice(n, k, replace=False)
            x[idx] = rng.integers(0, 2 ** 14, k)
    else:
        raise ValueError(kind)
    x = np.asarray(x)
    if not fp:
        info = np.iinfo(npt)
        x = np.clip(x, info.min, info.max)
    x = x.astype(npt)
    if fp and n > 20:
        # special values: NaN with payloads and both signs, infinities, signed zeros
        bits = x.view(np.uint32 if npt == np.float32 else np.uint64)
        if npt == np.float32:
            bits[3], bits[9] = 0x7fc00001, 0xffa00005
        else:
            bits[3], bits[9] = 0x7ff8000000000123, 0xfff4000000000007
        x[4], x[5], x[6], x[7] = np.inf, -np.inf, -0.0, 0.0
    return x


KINDS = ["uniform", "walk", "runs", "const", "zipf", "outliers"]


def check_encoding(G, O, enc, dt, x):
    dev = G.to_device(x)
    parts = G.encode(enc, dt, dev)
    host = [G.to_host(p) for p in parts]
    expect = O.encode(enc, dt, x)
    assert len(host) == len(expect), (OR.ENC_NAMES[enc], len(host), len(expect))
    for k, (h, e) in enumerate(zip(host, expect)):
        assert h.size == e.size and np.array_equal(h, e), \
            f"{OR.ENC_NAMES[enc]} dt={dt} n={x.size} part {k}: sizes {h.size} vs {e.size}"
    back = G.to_host(G.decode(enc, dt, parts))
    assert back.tobytes() == x.tobytes(), f"{OR.ENC_NAMES[enc]} dt={dt} n={x.size} round trip"
    # the GPU decodes the oracle's stream too
    back2 = G.to_host(G.decode(enc, dt, [G.to_device(e) for e in expect]))
    assert back2.tobytes() == x.tobytes()


@pytest.mark.parametrize("dt,npt", ALL_TYPES)
@pytest.mark.parametrize("enc", [OR.DELTA, OR.SCALE, OR.NONE])
@pytest.mark.parametrize("n", SIZES)
def test_elementwise_encodings(G, O, rng, enc, dt, npt, n):
    for kind in ["uniform", "walk"]:
        check_encoding(G, O, enc, dt, gen(kind, npt, n, rng))


@pytest.mark.parametrize("dt,npt", ALL_TYPES)
@pytest.mark.parametrize("enc", [OR.RLE, OR.DICT, OR.CONST, OR.PATCH, OR.PATCH_OUTSIDE])
@pytest.mark.parametrize("n", SIZES)
def test_split_and_run_encodings(G, O, rng, enc, dt, npt, n):
    for kind in KINDS:
        check_encoding(G, O, enc, dt, gen(kind, npt, n, rng))


@pytest.mark.parametrize("dt,npt", ALL_TYPES)
@pytest.mark.parametrize("n", SIZES + [32768, 32769, 100000])
def test_gfc(G, O, rng, dt, npt, n):
    for kind in ["uniform", "walk", "runs"]:
        check_encoding(G, O, OR.GFC, dt, gen(kind, npt, n, rng))


@pytest.mark.parametrize("dt,npt", ALL_TYPES)
@pytest.mark.parametrize("n", SIZES)
def test_float_to_int(G, O, rng, dt, npt, n):
    for kind in ["uniform", "walk", "const"]:
        x = gen(kind, npt, n, rng)
        if np.issubdtype(npt, np.floating) and kind == "walk":
            x = np.round(x.astype(np.float64), 2).astype(npt)
        check_encoding(G, O, OR.FLOAT2INT, dt, x)


def test_gfc_price_series(G, O, rng):
    """GFC on the price-like series of the GFC workload (scaled down), float64 and float32."""
    t = np.arange(1 << 18)
    x = np.round(100 * np.sin(2 * np.pi * t / 1000) + rng.normal(0, 0.01, t.size), 2)
    bits = x.view(np.uint64)
    idx = rng.choice(x.size, x.size // 1000, replace=False)
    bits[idx] = 0x7ff0000000000000 | rng.integers(1, 1 << 52, idx.size, dtype=np.uint64) | \
        (rng.integers(0, 2, idx.size, dtype=np.uint64) << 63)
    x[5], x[6], x[7] = np.inf, -np.inf, -0.0
    check_encoding(G, O, OR.GFC, OR.DOUBLE, x)
    check_encoding(G, O, OR.GFC, OR.FLOAT, x.astype(np.float32))


@pytest.mark.parametrize("dt,npt", ALL_TYPES)
@pytest.mark.parametrize("n", [1, 2, 3, 100, 10000, 70001])
def test_statistics(G, O, rng, dt, npt, n):
    for kind in KINDS:
        x = gen(kind, npt, n, rng)
        if np.issubdtype(npt, np.floating) and kind in ("walk", "uniform"):
            x = np.round(x.astype(np.float64), 3).astype(npt)
        got = G.stats(dt, G.to_device(x))
        exp = O.stats(dt, x)
        for f in ("min_bit_cnt", "precision", "sorted", "size"):
            assert getattr(got, f) == getattr(exp, f), (f, kind, getattr(got, f), getattr(exp, f))
        for f in ("min", "max"):
            a, b = getattr(got, f), getattr(exp, f)
            assert (np.isnan(a) and np.isnan(b)) or a == b, (f, kind, a, b)
        assert got.rl_metric == exp.rl_metric, (kind, got.rl_metric, exp.rl_metric)
        if np.issubdtype(npt, np.floating):
            # floating sums are order dependent in the reference (thrust::reduce): the two
            # summation orders may differ by the rounding bound 2*n*eps*mean(|x|)
            if np.isfinite(exp.mean):
                eps = np.finfo(npt).eps
                tol = 2 * n * eps * float(np.mean(np.abs(x.astype(np.float64)))) + 1e-12
                assert abs(got.mean - exp.mean) <= tol, (got.mean, exp.mean, tol)
        else:
            assert got.mean == exp.mean


def test_precision_table_matches_glibc(G, O):
    """The device logf table used for _getFloatPrecision equals the host KAT values."""
    for k, v in enumerate([1.0, 0.1, 0.01, 0.001, 1e-4, 1e-5, 1e-6, 1e-7]):
        x = np.full(64, 3 + v, np.float32)
        assert G.stats(OR.FLOAT, G.to_device(x)).precision == O.stats(OR.FLOAT, x).precision


def test_corrupt_streams_fail_cleanly(G, O, rng):
    x = rng.integers(0, 100, 5000).astype(np.int32)
    for enc in (OR.RLE, OR.DICT, OR.PATCH, OR.CONST, OR.GFC):
        for dt, src in ((OR.INT, x), (OR.DOUBLE, x.astype(np.float64))):
            parts = [G.to_host(p) for p in G.encode(enc, dt, G.to_device(src))]
            for k in range(1, len(parts)):
                if parts[k].size < 8:
                    continue
                cut = [G.to_device(p if j != k else p[: p.size // 2]) for j, p in enumerate(parts)]
                try:
                    G.decode(enc, dt, cut)
                except G.GtscError as e:
                    assert e.status in (-4, -3)


@pytest.mark.parametrize("dt,npt,bits,expected", [
    (OR.DOUBLE, np.float64, 0x7ff8000000000123, -2 ** 31), (OR.DOUBLE, np.float64, 0xfff4000000000007, -2 ** 31),
    (OR.FLOAT, np.float32, 0x7fc00001, 0), (OR.FLOAT, np.float32, 0xffa00005, 0)])
def test_device_nan_to_int_conversion(G, O, dt, npt, bits, expected):
    """RlMetric converts `int value = data[idx]` on the device (cuda_array_statistics.cu:103): the
    B200's conversion of NaN (INT_MIN for double, 0 for float) is what the oracle restates."""
    x = np.array([0, expected, expected], npt)
    x.view(np.uint64 if npt == np.float64 else np.uint32)[0] = bits
    assert G.stats(dt, G.to_device(x)).rl_metric == 2.0 == O.stats(dt, x).rl_metric


def float_cases(rng):
    for n in [0, 1, 7, 8, 9, 1000, 100001]:
        x = np.round(rng.normal(0, 100, n), 2).astype(np.float32)
        yield "mixed", x
        yield "positive", np.abs(x)
        yield "negative", -np.abs(x) - np.float32(1)
        if n >= 16:
            y = x.copy()
            y[3] = np.float32(-0.0)
            y[5] = np.float32(np.inf)
            y[6] = -np.float32(np.inf)
            bits = y.view(np.uint32)
            bits[7] = np.uint32(0xffc00123)  # a negative NaN with a payload
            yield "specials", y
            z = np.abs(x)
            z[2] = np.float32(-0.0)  # all positive but one -0.0: the sign must survive
            yield "minus_zero", z


def test_afl_float_split(G, O, rng):
    """AflEncoding's float path (afl_encoding.cu:116-254): mantissa / exponent AFL streams and the
    sign byte or stencil, byte-identical to the oracle, bit-exact round trip"""
    for name, x in float_cases(rng):
        ref = O.encode(OR.AFL, OR.FLOAT, x)
        parts = G.encode(G.AFL, G.FLOAT, G.to_device(x))
        assert len(parts) == len(ref) == 2
        for a, b in zip(parts, ref):
            assert np.array_equal(G.to_host(a), b), (name, x.size)
        out = G.decode(G.AFL, G.FLOAT, parts)
        assert G.to_host(out).tobytes() == x.tobytes(), (name, x.size)
        if x.size:  # sign byte: 1 all sign bits clear, 2 all set, 0 a stencil follows
            neg = int(np.signbit(x).sum())
            expect = 1 if neg == 0 else 2 if neg == x.size else 0
            assert int(G.to_host(parts[0])[8]) == expect, name
            if name == "minus_zero":
                assert expect == 0


def test_afl_float_in_trees(G, O, rng):
    x = np.round(rng.normal(0, 10, 20000), 1).astype(np.float32)
    for path in ([OR.AFL, OR.NONE], [OR.DELTA, OR.AFL, OR.NONE], [OR.PATCH, OR.AFL, OR.NONE, OR.AFL, OR.NONE]):
        nodes = G.tree_from_path(path, OR.FLOAT)
        blob = G.tree_compress(nodes, G.to_device(x))
        assert np.array_equal(G.to_host(blob), O.tree_compress(nodes, x))
        out, _ = G.tree_decompress(blob)
        assert G.to_host(out).tobytes() == x.tobytes()
        assert G.tree_predict_size(nodes, G.to_device(x)) == O.tree_predict_size(nodes, x)
    with pytest.raises(G.GtscError):  # double: EncodeDouble returns no buffers in the reference
        G.encode(G.AFL, G.DOUBLE, G.to_device(x.astype(np.float64)))


@pytest.mark.parametrize("dt,npt", ALL_TYPES)
@pytest.mark.parametrize("n", SIZES + [4095, 4096, 4097, 300001])
def test_unique(G, O, rng, dt, npt, n):
    """The standalone UniqueEncoding (unique_encoding.cu:133-181, 261-304): sorted table of the
    distinct bit patterns and packed codes, byte-identical to the oracle."""
    for kind in KINDS:
        check_encoding(G, O, OR.UNIQUE, dt, gen(kind, npt, n, rng))


@pytest.mark.parametrize("dt,npt", ALL_TYPES)
def test_unique_table_sizes(G, O, rng, dt, npt):
    """1 distinct value (1-bit codes), 2^k and 2^k + 1 distinct values around the code widths, and
    every value distinct (a table too large for shared memory, one code per word)."""
    info = np.iinfo(npt) if not np.issubdtype(npt, np.floating) else None
    for m in [1, 2, 3, 4, 5, 16, 17, 255, 256, 257, 40000]:
        if info is not None and m > info.max - info.min + 1:
            continue
        vals = rng.permutation(np.arange(m)) - m // 2
        vals = vals.astype(npt) if info is None else np.clip(vals, info.min, info.max).astype(npt)
        x = vals[rng.integers(0, m, 50000)]
        x[:m] = vals
        check_encoding(G, O, OR.UNIQUE, dt, x)
        meta = G.to_host(G.encode(OR.UNIQUE, dt, G.to_device(x))[0])
        assert int(meta[:8].view(np.uint64)[0]) == np.unique(x.view(f"u{x.itemsize}")).size


def test_unique_large(G, rng):
    """2^24 int32 with ~10^6 distinct values: round trip and table size (size-independent checks)."""
    n = 1 << 24
    x = rng.integers(-(1 << 30), 1 << 30, 1 << 20).astype(np.int32)[rng.integers(0, 1 << 20, n)]
    parts = G.encode(OR.UNIQUE, OR.INT, G.to_device(x))
    meta = G.to_host(parts[0])
    table = meta[16:].view(np.int32)
    assert np.array_equal(table, np.unique(x))
    assert G.to_host(G.decode(OR.UNIQUE, OR.INT, parts), np.int32).tobytes() == x.tobytes()


def test_unique_in_trees_and_corrupt_codes(G, O, rng):
    x = rng.integers(0, 50, 20000).astype(np.int32)
    for path in ([OR.UNIQUE, OR.NONE], [OR.UNIQUE, OR.AFL, OR.NONE], [OR.DELTA, OR.UNIQUE, OR.AFL, OR.NONE]):
        nodes = G.tree_from_path(path, OR.INT)
        blob = G.tree_compress(nodes, G.to_device(x))
        assert np.array_equal(G.to_host(blob), O.tree_compress(nodes, x))
        out, _ = G.tree_decompress(blob)
        assert G.to_host(out).tobytes() == x.tobytes()
    # 3 distinct values -> 2-bit codes; code 3 points past the table
    y = np.array([5, 6, 7, 5], np.int32)
    meta, data = O.encode(OR.UNIQUE, OR.INT, y)
    bad = data.copy()
    bad[0] |= 0b11
    with pytest.raises(G.GtscError) as e:
        G.decode(OR.UNIQUE, OR.INT, [G.to_device(meta), G.to_device(bad)])
    assert e.value.status == -4


EXACT_PREDICTORS = [OR.NONE, OR.DELTA, OR.SCALE, OR.RLE, OR.DICT, OR.CONST, OR.UNIQUE]


@pytest.mark.parametrize("dt,npt", ALL_TYPES)
@pytest.mark.parametrize("n", [0, 1, 33, 4097, 65537])
def test_size_predictors(G, O, rng, dt, npt, n):
    """GetMetadataSize / GetCompressedSize == the emitted sizes (the reference's TestGetMetadataSize /
    TestGetCompressedSize, test/compression_unittest_base.hpp:32-54) for the exact predictors; the
    reference's fixed formulas for the others."""
    es = np.dtype(npt).itemsize
    for kind in KINDS:
        x = gen(kind, npt, n, rng)
        dev = G.to_device(x)
        for enc in EXACT_PREDICTORS + ([OR.AFL] if dt != OR.DOUBLE else []):
            parts = O.encode(enc, dt, x)
            meta, data = G.predict_sizes(enc, dt, dev)
            if n == 0:  # the reference's formulas: only none and dict have no empty guard
                assert (meta, data) == ({OR.NONE: 8, OR.DICT: 1}.get(enc, 0), 0)
                continue
            if enc == OR.AFL and dt == OR.FLOAT:
                assert meta == (9 if n else 0)
            else:
                assert meta == parts[0].size, (OR.ENC_NAMES[enc], kind)
            assert data == sum(p.size for p in parts[1:]), (OR.ENC_NAMES[enc], kind)
        stencil = (n + 7) // 8 + 1 if n else 0
        assert G.predict_sizes(OR.PATCH, dt, dev) == (stencil, n * es)
        assert G.predict_sizes(OR.FLOAT2INT, dt, dev) == ((4 if n else 0), n * es)
        assert G.predict_sizes(OR.GFC, dt, dev) == (12, 0)
