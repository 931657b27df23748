"""CompressionOptimizer::CompressData on the GPU against the oracle restatement: over a stream of
parts, the same blob for every part (byte-identical), the same full-update / correction decisions,
the same optimal tree and the same edge statistics (exact doubles); every blob decodes to its part
(the reference's CompressDecompressNPartsData, optimizer/optimizer_unittest.cpp:233-280)."""
import numpy as np
import pytest

import oracle as OR
from oracle import maintenance as M

pytestmark = pytest.mark.gpu


def plateaus(part, size, period, step, lo, hi, dtype):
    """a staircase of plateaus that moves by `step` every `period` elements and bounces between lo
    and hi, with a spike to hi at every step (the shape of the reference's pattern A)"""
    i = np.arange(part * size, (part + 1) * size)
    k = i // period
    span = max(int((hi - lo) / step), 1)
    pos = k % (2 * span)
    level = lo + step * np.where(pos < span, pos, 2 * span - pos)
    out = np.where(i % period == 0, hi, level)
    return out.astype(dtype)


def extremes_and_ramps(part, size, period, lo, hi, dtype, rng):
    """blocks of `period` elements alternating between noisy extremes and a V-shaped ramp (the shape of
    the reference's pattern B)"""
    i = np.arange(part * size, (part + 1) * size)
    x = i % period
    step = (hi - lo) / (period // 2)
    ramp = np.where(x < period // 2, hi - x * step, hi - (period - x) * step)
    noise = rng.integers(0, 6, size)
    ext = np.where(i % 2 == 0, hi - noise, lo + noise)
    out = np.where((i // period) % 2 == 0, ext, ramp)
    return out.astype(dtype)


def run_parts(G, parts, dt):
    gopt, oopt = G.Optimizer(dt), M.Optimizer(dt)
    for k, x in enumerate(parts):
        blob, full, corr = gopt.compress(G.to_device(x))
        oblob, ofull, ocorr = oopt.compress(x)
        assert (full, corr) == (ofull, ocorr), k
        hb = G.to_host(blob)
        assert hb.tobytes() == oblob.tobytes(), k
        out, odt = G.tree_decompress(blob)
        assert odt == dt and G.to_host(out).tobytes() == x.tobytes(), k
        gn, gr = gopt.tree()
        on, orr = M.nodes_of(oopt.opt.root)
        assert np.array_equal(gn, on) and np.array_equal(gr, orr), k
    st = gopt.statistics()
    for no in range(62):
        assert st.entries(no) == oopt.stats.e[no], no
    return gopt


def test_optimizer_pattern_a_int_25_parts(G, rng):
    parts = [plateaus(p, 20000, 10, 1, -100, 10 ** 6, np.int32) for p in range(25)]
    run_parts(G, parts, OR.INT)


def test_optimizer_patterns_ab_int(G, rng):
    parts = []
    for p in range(12):
        parts.append(plateaus(p, 20000, 100, 1, -100, 10 ** 6, np.int32))
        parts.append(extremes_and_ramps(p, 20000, 60000, -10 ** 4, 10 ** 4, np.int32, rng))
    run_parts(G, parts, OR.INT)


def test_optimizer_float_parts(G, rng):
    parts = [plateaus(p, 20000, 100, 1.5, -10.0, 1e6, np.float32) for p in range(5)]
    parts += [extremes_and_ramps(p, 20000, 60000, -1e4, 1e4, np.float32, rng) for p in range(6)]
    run_parts(G, parts, OR.FLOAT)


def test_optimizer_random_and_time_parts(G, rng):
    run_parts(G, [rng.integers(10, 10000, 30000).astype(np.int32) for _ in range(3)], OR.INT)
    ts = [np.cumsum(rng.exponential(1000, 15000)).astype(np.int64) + 10 ** 12 for _ in range(11)]
    run_parts(G, ts, OR.TIME)
    dbl = [np.round(np.cumsum(rng.normal(0, 1, 15000)), 2) for _ in range(4)]
    run_parts(G, dbl, OR.DOUBLE)
