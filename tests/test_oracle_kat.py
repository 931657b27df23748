"""Pins the CPU oracle against the reference's own known-answer tests (restated) and against the
reference's AFL host implementation compiled from its sources (oracle/_ref).  CPU only."""
import numpy as np
import pytest

import oracle as OR


# ---- BITLEN / ALT_BITLEN (src/test/macros_unittest.cu:5-139) --------------------------------
@pytest.mark.parametrize("dt,mn,mx,expected", [
    (OR.INT, 0, 0, 1), (OR.INT, 0, 1, 1), (OR.INT, 0, 12345, 14), (OR.INT, 0, 2147268225, 31),
    (OR.INT, -12345, -12345, 32), (OR.INT, -2147268227, 147268227, 32), (OR.SHORT, 0, 12345, 14),
    (OR.CHAR, 0, 45, 6), (OR.TIME, 0, 22147268225, 35)])
def test_bitlen_kat(O, dt, mn, mx, expected):
    assert O.lib().or_bitlen(dt, mn, mx) == expected


@pytest.mark.parametrize("v,expected", [(12345, 14), (2147268225, 31), (-12345, 32),
                                        (-2147268227, 32), (0, 1), (1, 1)])
def test_alt_bitlen_kat(O, v, expected):
    assert O.lib().or_alt_bitlen(v) == expected


# ---- _getFloatPrecision (util/statistics/cuda_array_statistics_unittest.cpp:21-83) ----------
@pytest.mark.parametrize("x,expected", [(123.0, 0), (123123123123.0, 0), (-123123123.0, 0), (123.1, 1),
                                        (123.34, 2), (13.3412312, 6), (1231201.2312, 1),
                                        (12312311.33412312, 0)])
def test_float_precision_kat(O, x, expected):
    assert O.lib().or_float_precision(np.float32(x)) == expected


# ---- Sorted / RlMetric / Mean (cuda_array_statistics_unittest.cpp:103-187), size 10000 -------
N = 10000


def test_sorted_kat(O):
    h = np.array([i // 100 if i % 50 == 0 else N for i in range(N)], np.int32)
    assert O.stats(OR.INT, h).sorted == 0
    h = np.array([i // 100 + 39 for i in range(N)], np.int32)
    assert O.stats(OR.INT, h).sorted == 1


def test_rlmetric_kat(O):
    const = np.full(N, 100, np.int32)
    assert O.lib().or_rl_metric(OR.INT, const.ctypes.data, const.nbytes, 4) == 4.0
    consec = np.arange(N, dtype=np.int32)
    assert O.lib().or_rl_metric(OR.INT, consec.ctypes.data, consec.nbytes, 4) == 1.0
    pairs = (np.arange(N) // 2).astype(np.int32)
    assert O.stats(OR.INT, pairs).rl_metric == 1.5


def test_mean_kat(O):
    assert O.stats(OR.INT, np.arange(N, dtype=np.int32)).mean == float((N - 1) // 2)


# ---- stencil pack / unpack (util/stencil/stencil_unittest.cpp:10-34) -------------------------
@pytest.mark.parametrize("n", [1, 7, 8, 9, 1000, 1001])
def test_stencil_pack_unpack(O, rng, n):
    st = rng.integers(0, 2, n).astype(np.int32)
    packed = np.zeros(n // 8 + 2, np.uint8)
    nb = O.lib().or_stencil_pack(st.ctypes.data, n, packed.ctypes.data)
    assert nb == (n + 7) // 8 + 1 and nb < 4 * n
    assert packed[0] == n % 8
    # tail bits repeat the last element (stencil.cu:27)
    if n % 8:
        tail = (packed[nb - 1] >> (n % 8)) & 1
        assert tail == st[-1]
    out = np.zeros(n + 8, np.int32)
    m = O.lib().or_stencil_unpack(packed.ctypes.data, nb, out.ctypes.data, n + 8)
    assert m == n and np.array_equal(out[:n], st)


# ---- split / merge ordering (util/splitter/splitter_unittest.cpp:63-170) ----------------------
def test_split_manual_complex(O, rng):
    # a patch split is Splitter::Split on the stencil x < threshold: check stable ordering
    n = 1000
    x = rng.integers(0, 100, n).astype(np.int32)
    x[: n // 4] = 95
    x[n // 2: 3 * n // 4] = 99
    x[0] = 0
    parts = O.encode(OR.PATCH, OR.INT, x)
    st = np.unpackbits(parts[0][1:], bitorder="little")[:n].astype(bool)
    t = int(99 - 0.1 * 99)
    assert np.array_equal(st, x < t)
    assert np.array_equal(parts[1].view(np.int32), x[st])
    assert np.array_equal(parts[2].view(np.int32), x[~st])


# ---- AFL against the reference's own host implementation (afl_gpu.cu:6-65) ------------------
@pytest.mark.parametrize("dt,npt", [(OR.CHAR, np.int8), (OR.SHORT, np.int16), (OR.INT, np.int32),
                                    (OR.TIME, np.int64)])
def test_afl_oracle_matches_reference(O, rng, dt, npt):
    if not OR.build_ref():
        pytest.skip("reference AFL sources not available")
    W = 8 * np.dtype(npt).itemsize
    for n in [1, 31, 32, 33, 1000, 4097]:
        for b in sorted({1, 3, 5, 7, 11, W - 1}):
            if b >= W:
                continue
            x = rng.integers(0, 2 ** b, n).astype(npt)
            x[0] = 2 ** b - 1
            meta, data = O.encode(OR.AFL, dt, x)
            assert meta[0] == b and meta[2] == 0 and meta[3] == 0
            assert np.array_equal(O.ref_afl_compress(dt, x, b), data)
            assert np.array_equal(O.ref_afl_decompress(dt, data, b, n), x)


@pytest.mark.parametrize("dt,npt", [(OR.SHORT, np.int16), (OR.INT, np.int32), (OR.TIME, np.int64)])
def test_afl_layouts_match_reference(O, rng, dt, npt):
    """The oracle's bit-position restatement of both packed layouts against the reference's own
    run_afl_compress_cpu / run_afl_decompress_cpu <T,1|32> and afl_decompress_base_value_gpu
    (afl_gpu.cu:5-65, 197-222).  The reference's host bit extraction is defined for b < W only."""
    if not OR.build_ref():
        pytest.skip("reference AFL sources not available")
    W = 8 * np.dtype(npt).itemsize
    for n in [1, 31, 32, 33, 32 * W - 1, 32 * W, 32 * W + 1, 3 * 32 * W + 77, 20000]:
        for b in sorted({1, 3, 7, W // 2 + 1, W - 1}):
            x = rng.integers(0, 2 ** b, n).astype(npt)
            x[-1] = 2 ** b - 1
            p1 = OR.afl_layout_pack(1, dt, x, b)
            p32 = OR.afl_layout_pack(32, dt, x, b)
            assert p32.size == OR.afl_layout_words(32, dt, b, n) * x.itemsize
            assert np.array_equal(O.ref_afl_compress(dt, x, b), p1)
            assert np.array_equal(O.ref_afl32_compress(dt, x, b), p32)
            assert np.array_equal(O.ref_afl32_decompress(dt, p32, b, n), x)
            assert np.array_equal(OR.afl_layout_values(1, dt, p1, b, n), x)
            assert np.array_equal(OR.afl_layout_values(32, dt, p32, b, n), x)
            if dt != OR.SHORT:
                for i in sorted({0, n // 3, n - 1}):
                    assert O.ref_afl_value(dt, 1, p1, b, i) == x[i]
                    assert O.ref_afl_value(dt, 32, p32, b, i) == x[i]


def test_afl_config1_sizes(O, rng):
    """2^20 int32 uniform in [0, 2^11): b = 11, 1 441 792 data bytes + 4 metadata bytes."""
    x = rng.integers(0, 2 ** 11, 1 << 20).astype(np.int32)
    x[0] = 2 ** 11 - 1
    meta, data = O.encode(OR.AFL, OR.INT, x)
    assert meta.size == 4 and meta[0] == 11 and meta[1] == 0
    assert data.size == 1441792
    if OR.build_ref():
        assert np.array_equal(O.ref_afl_compress(OR.INT, x, 11), data)


# ---- outside patch (outside_patch_encoding.cu:22-60, stencil_operators.hpp:14-25) -----------
def _stencil_bits(st):
    """Stencil::pack layout: rest byte, then LSB-first bits, the tail repeating the last element."""
    n = st.size
    pad = (-n) % 8
    full = np.concatenate([st, np.full(pad, st[-1])]).astype(np.uint8)
    return np.concatenate([[n % 8], np.packbits(full, bitorder="little")]).astype(np.uint8)


def test_outside_patch_kat(O, rng):
    """low = (int)(min + 0.1 * dist), high = (int)(max - 0.1 * dist); elements in [low, high] go to
    out1, the others (both tails) to out2, in order."""
    x = rng.integers(-1000, 1000, 5000).astype(np.int32)
    x[7], x[9] = -1000, 999
    mn, mx = int(x.min()), int(x.max())
    dist = mx - mn
    lo, hi = int(mn + 0.1 * dist), int(mx - 0.1 * dist)   # truncation toward zero, as static_cast<int>
    inside = (x >= lo) & (x <= hi)
    meta, o1, o2 = O.encode(OR.PATCH_OUTSIDE, OR.INT, x)
    assert np.array_equal(o1.view(np.int32), x[inside])
    assert np.array_equal(o2.view(np.int32), x[~inside])
    assert np.array_equal(meta, _stencil_bits(inside))
    assert np.array_equal(O.decode(OR.PATCH_OUTSIDE, OR.INT, [meta, o1, o2]).view(np.int32), x)
    assert np.array_equal(O.decode(OR.PATCH, OR.INT, [meta, o1, o2]).view(np.int32), x)


def test_outside_patch_nan_is_inside(O):
    """OutsideOperator returns true unless x > high or x < low: NaN compares false both ways."""
    x = np.array([0.0, 100.0, 50.0, np.nan, 5.0, 95.0], np.float64)
    meta, o1, o2 = O.encode(OR.PATCH_OUTSIDE, OR.DOUBLE, x)
    # min/max skip NaN: 0 and 100, bounds 10 and 90
    got = o1.view(np.float64)
    assert got.size == 2 and got[0] == 50.0 and np.isnan(got[1])
    assert np.array_equal(o2.view(np.float64), [0.0, 100.0, 5.0, 95.0])


def test_outside_patch_tree_serialises_as_patch(O, rng):
    """A tree with an outside patch node records EncodingType::patch (6) in its header and decodes."""
    x = rng.integers(0, 1 << 12, 3000).astype(np.int32)
    nodes = O.tree_from_path([OR.PATCH_OUTSIDE, OR.AFL, OR.NONE, OR.AFL, OR.NONE], OR.INT)
    blob = O.tree_compress(nodes, x)
    assert blob[:2].view(np.int16)[0] == OR.PATCH
    out, dt = O.tree_decompress(blob, x.nbytes)
    assert dt == OR.INT and np.array_equal(out.view(np.int32), x)
