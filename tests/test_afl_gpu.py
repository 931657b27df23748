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


def test_afl_float_rejected(G):
    with pytest.raises(G.GtscError) as e:
        G.encode(OR.AFL, OR.DOUBLE, G.to_device(np.zeros(4, np.float64)))
    assert e.value.status == -2
