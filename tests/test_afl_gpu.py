"""AFL on the GPU against the oracle: byte-identical stream, bit-exact decode
(compression/afl/afl_encoding_unittest.cpp is the reference's test of this encoding)."""
import numpy as np
import pytest

import oracle as OR

pytestmark = pytest.mark.gpu

TYPES = [(OR.CHAR, np.int8), (OR.SHORT, np.int16), (OR.INT, np.int32), (OR.TIME, np.int64)]


def gpu_encode(G, enc, dt, x):
    parts = G.encode(enc, dt, G.to_device(x))
    return parts, [G.to_host(p) for p in parts]


@pytest.mark.parametrize("dt,npt", TYPES)
@pytest.mark.parametrize("n", [0, 1, 31, 32, 33, 1000, 2047, 2048, 2049, 100003])
def test_afl_matches_oracle(G, O, rng, dt, npt, n):
    W = 8 * np.dtype(npt).itemsize
    for b in sorted({1, 5, 11, W - 1, W}):
        if b > W:
            continue
        if b == W:
            x = rng.integers(np.iinfo(npt).min, np.iinfo(npt).max, n, dtype=npt, endpoint=True)
        else:
            x = rng.integers(0, 2 ** b, n).astype(npt)
        parts, host = gpu_encode(G, OR.AFL, dt, x)
        expect = O.encode(OR.AFL, dt, x)
        assert len(host) == len(expect) == 2
        for h, e in zip(host, expect):
            assert np.array_equal(h, e), (dt, n, b)
        back = G.to_host(G.decode(OR.AFL, dt, parts), npt)
        assert back.tobytes() == x.tobytes()


def test_afl_config1(G, O, rng):
    """2^20 int32 uniform in [0, 2^11), b = 11: stream byte-identical to the oracle."""
    x = rng.integers(0, 2 ** 11, 1 << 20).astype(np.int32)
    parts, host = gpu_encode(G, OR.AFL, OR.INT, x)
    meta, data = O.encode(OR.AFL, OR.INT, x)
    assert host[0].tobytes() == meta.tobytes() and host[1].tobytes() == data.tobytes()
    assert host[1].size == 1441792
    assert np.array_equal(G.to_host(G.decode(OR.AFL, OR.INT, parts), np.int32), x)


def test_afl_decode_unaligned_stream(G, O, rng):
    """Decoding straight out of a serialized blob: the stream may start at any byte."""
    x = rng.integers(0, 2 ** 13, 5000).astype(np.int32)
    meta, data = O.encode(OR.AFL, OR.INT, x)
    for off in range(1, 8):
        blob = np.concatenate([np.zeros(off, np.uint8), data])
        dev = G.to_device(blob)
        view = G.DeviceBuffer(dev.ptr + off, data.size, owned=False)
        out = G.decode(OR.AFL, OR.INT, [G.to_device(meta), view])
        assert np.array_equal(G.to_host(out, np.int32), x)


@pytest.mark.parametrize("dt,npt", TYPES)
def test_afl_aligned_layout(G, O, rng, dt, npt):
    """The aligned layout (run_afl_compress_gpu<T,32>, afl_gpu.cu:67-81) byte-identical to the
    oracle's restatement, which is pinned to the reference's run_afl_compress_cpu<T,32>."""
    W = 8 * np.dtype(npt).itemsize
    for n in [0, 1, 31, 32, 33, 32 * W - 1, 32 * W, 32 * W + 1, 5 * 32 * W + 77, 100003]:
        for b in sorted({1, 5, W // 2 + 1, W - 1, W}):
            if b == W:
                x = rng.integers(np.iinfo(npt).min, np.iinfo(npt).max, n, dtype=npt, endpoint=True)
            else:
                x = rng.integers(0, 2 ** b, n).astype(npt)
            packed = G.afl_pack(dt, b, G.to_device(x), n, omega=32)
            expect = OR.afl_layout_pack(32, dt, x, b)
            assert G.to_host(packed).tobytes() == expect.tobytes(), (dt, n, b)
            back = G.to_host(G.afl_unpack(dt, b, packed, n, omega=32), npt)
            assert back.tobytes() == x.tobytes(), (dt, n, b)


@pytest.mark.parametrize("dt,npt", TYPES)
@pytest.mark.parametrize("omega", [1, 32])
def test_afl_random_access(G, O, rng, dt, npt, omega):
    """run_afl_decompress_value_gpu<T,omega> (afl_gpu.cu:83-121, 197-222): every element, and a
    gather of random positions, decoded on its own from either layout."""
    W = 8 * np.dtype(npt).itemsize
    for n in [1, 33, 32 * W + 5, 70001]:
        for b in sorted({1, 7, W - 3, W}):
            if b == W:
                x = rng.integers(np.iinfo(npt).min, np.iinfo(npt).max, n, dtype=npt, endpoint=True)
            else:
                x = rng.integers(0, 2 ** b, n).astype(npt)
            packed = G.afl_pack(dt, b, G.to_device(x), n, omega=omega)
            host = G.to_host(packed)
            assert host.tobytes() == OR.afl_layout_pack(omega, dt, x, b).tobytes(), (dt, n, b, omega)
            every = G.to_host(G.afl_values(dt, b, packed, omega, n=n), npt)
            assert every.tobytes() == x.tobytes(), (dt, n, b, omega)
            idx = rng.integers(0, n, 4097).astype(np.uint64)
            got = G.to_host(G.afl_values(dt, b, packed, omega, index=G.to_device(idx)), npt)
            assert got.tobytes() == x[idx.astype(np.int64)].tobytes()
            assert got.tobytes() == OR.afl_layout_values(omega, dt, host, b, n, idx).tobytes()


def test_afl_layouts_large(G, rng):
    """2^26 int32 at b = 17 in the aligned layout: round trip and a random gather (size-independent
    properties at full size)."""
    n = 1 << 26
    x = rng.integers(0, 2 ** 17, n, dtype=np.int32)
    packed = G.afl_pack(OR.INT, 17, G.to_device(x), n, omega=32)
    assert packed.nbytes == n * 17 // 8
    back = G.to_host(G.afl_unpack(OR.INT, 17, packed, n, omega=32), np.int32)
    assert np.array_equal(back, x)
    idx = rng.integers(0, n, 1 << 16).astype(np.uint64)
    got = G.to_host(G.afl_values(OR.INT, 17, packed, 32, index=G.to_device(idx)), np.int32)
    assert np.array_equal(got, x[idx.astype(np.int64)])


def test_afl_layout_arguments(G):
    buf = G.to_device(np.zeros(64, np.int32))
    with pytest.raises(G.GtscError) as e:
        G.afl_pack(OR.FLOAT, 5, buf, 64, omega=32)
    assert e.value.status == -2
    with pytest.raises(G.GtscError):
        G.afl_pack(OR.INT, 33, buf, 64, omega=32)
    with pytest.raises(G.GtscError):
        G.afl_values(OR.INT, 5, buf, 7, n=4)


def test_afl_float_rejected(G):
    with pytest.raises(G.GtscError) as e:
        G.encode(OR.AFL, OR.DOUBLE, G.to_device(np.zeros(4, np.float64)))
    assert e.value.status == -2
