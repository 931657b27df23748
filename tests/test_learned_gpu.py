"""The learned planner on the GPU: its feature kernel and its FP32 forward / backward kernels
against the CPU oracle (oracle/learned.py), training, save / load, the exhaustive fallback, and the
ablation of the trained network (what it gains over the methods without it)."""
import os

import numpy as np
import pytest

import oracle as OR
from oracle import learned as OL
from gputimeseriescompressionoptimizer_b200 import workloads as W

pytestmark = pytest.mark.gpu


class _View:
    def __init__(self, ptr, nbytes):
        self.ptr, self.nbytes = ptr, nbytes


def feature_columns(rng):
    cols = []
    for dt in range(6):
        npt = OR.NP_TYPES[dt]
        for n in [0, 1, 2, 3, 100, 10000, 25000]:
            if dt >= 4:
                x = np.round(rng.normal(0, 50, n), 2).astype(npt)
                if n > 10:
                    x[3] = np.nan
                    x[5] = -0.0
            else:
                x = rng.integers(-60, 60, n).astype(npt)
            cols.append((dt, x))
    for i in range(40):
        kind, dt, n_total, x = W.training_column(1000 + i)
        cols.append((dt, x))
    for kind, dt, x in W.tick_chunk(n_cols=10, rows=20000):
        cols.append((dt, x))
    return cols


def test_features_match_oracle(G, rng):
    cols = feature_columns(rng)
    devs = [G.to_device(x) for _, x in cols]
    f = G.to_host(G.planner_features(devs, [dt for dt, _ in cols]), np.float32).reshape(len(cols), -1)
    for i, (dt, x) in enumerate(cols):
        ref = OL.features(x, dt)
        assert np.allclose(f[i], ref, rtol=1e-5, atol=2e-6), (i, dt, x.size, np.flatnonzero(~np.isclose(f[i], ref)))


def make_classes():
    return [[OR.AFL, OR.NONE], [OR.DELTA, OR.AFL, OR.NONE], [OR.GFC, OR.NONE, OR.NONE],
            [OR.DICT, OR.NONE, OR.AFL, OR.NONE], [OR.FLOAT2INT, OR.AFL, OR.NONE], [OR.NONE],
            [OR.RLE, OR.AFL, OR.NONE, OR.NONE], [OR.DELTA, OR.GFC, OR.NONE, OR.NONE]]


def test_gradient_matches_oracle(G, rng):
    cls = make_classes()
    P = G.Planner(cls, seed=3)
    valid = P.valid()
    n = 300
    x = rng.normal(0, 1, (n, 32)).astype(np.float32)
    dts = rng.integers(0, 6, n)
    x[:, :6] = 0
    x[np.arange(n), dts] = 1
    lab = np.array([rng.choice(np.flatnonzero(valid[:, d])) for d in dts], np.int32)
    lab[::17] = -1
    mu = rng.normal(0, 0.1, 32).astype(np.float32)
    sd = rng.uniform(0.5, 2, 32).astype(np.float32)
    params, _, _ = P.get_params()
    params = (params + rng.normal(0, 0.05, params.size)).astype(np.float32)
    P.set_params(params, mu, sd)
    loss, g = P.gradient(G.to_device(x), lab)
    mask = valid[:, dts].T.astype(bool)
    ref_loss, ref_g = OL.loss_and_grad(params, len(cls), x, mu.astype(np.float64), sd.astype(np.float64), lab, mask)
    assert abs(loss - ref_loss) < 1e-5 * max(1, abs(ref_loss))
    assert np.allclose(g, ref_g, rtol=1e-3, atol=2e-6), np.max(np.abs(g - ref_g))
    # the gradient is reproducible bit for bit (fixed summation order)
    loss2, g2 = P.gradient(G.to_device(x), lab)
    assert loss2 == loss and np.array_equal(g, g2)


def test_forward_matches_oracle_and_save_load(G, rng):
    cls = make_classes()
    P = G.Planner(cls, seed=5)
    valid = P.valid()
    n = 200
    x = rng.normal(0, 1, (n, 32)).astype(np.float32)
    dts = rng.integers(0, 6, n).astype(np.int32)
    x[:, :6] = 0
    x[np.arange(n), dts] = 1
    d = G.to_device(x)
    c1, p1 = P.predict(d, dts)
    params, mu, sd = P.get_params()
    z = OL.logits(params, len(cls), x, mu.astype(np.float64), sd.astype(np.float64))
    for r in range(n):
        zz = np.where(valid[:, dts[r]], z[r], -np.inf)
        assert c1[r] == int(np.argmax(zz))
        pr = np.exp(zz - zz.max())
        assert abs(p1[r] - pr.max() / pr.sum()) < 1e-4
    Q = G.Planner(model=P.save())
    c2, p2 = Q.predict(d, dts)
    assert np.array_equal(c1, c2) and np.array_equal(p1, p2)


def test_training_learns_a_separable_rule(G, rng):
    """labels that depend on two features: the trained network reproduces them"""
    cls = make_classes()[:4]
    P = G.Planner(cls, seed=11)
    n = 2000
    x = rng.normal(0, 1, (n, 32)).astype(np.float32)
    x[:, :6] = 0
    x[:, OR.INT] = 1
    lab = ((x[:, 10] > 0).astype(np.int32) * 2 + (x[:, 20] > 0.5)).astype(np.int32)
    valid = P.valid()
    lab = np.where(valid[lab, OR.INT], lab, 0).astype(np.int32)
    d = G.to_device(x)
    before, _ = P.gradient(d, lab)
    after = P.train(d, lab, epochs=60, batch=128, lr=3e-3)
    pred, conf = P.predict(d, np.full(n, OR.INT, np.int32))
    assert after < 0.5 * before
    assert np.mean(pred == lab) > 0.95


def test_plan_learned_fallback(G, rng):
    cls = make_classes()
    P = G.Planner(cls, seed=2)
    cols = [W.training_column(2000 + i) for i in range(12)]
    devs = [G.to_device(x) for _, _, _, x in cols]
    dts = [dt for _, dt, _, _ in cols]
    every = P.plan(devs, dts, min_confidence=1.01)  # nothing is that confident: all exhaustive
    for (nodes, fb), d, dt in zip(every, devs, dts):
        assert fb
        sb = G.sample_bytes(dt, d.nbytes)
        ex, _ = G.plan_exhaustive(dt, G.DeviceBuffer(d.ptr, sb, owned=False))
        assert np.array_equal(nodes, ex)
    none = P.plan(devs, dts, min_confidence=0.0)
    for (nodes, fb), d, dt, (_, _, _, x) in zip(none, devs, dts, cols):
        assert not fb
        blob = G.tree_compress(nodes, d)  # any chosen tree is lossless
        out, _ = G.tree_decompress(blob)
        assert G.to_host(out).tobytes() == x.tobytes()


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)),
                                                    "gputimeseriescompressionoptimizer_b200", "planner_model.bin")),
                    reason="trained model not present")
def test_trained_planner_ablation(G, rng):
    """Held-out columns (seeds the training never saw): the trained network with its fallback stays
    within 3% of the exhaustive planner's mean compression ratio, and does better than the same
    network untrained and than always proposing the most common tree."""
    P = G.Planner.load()
    cols = [W.training_column(500000 + i) for i in range(300)]
    devs = [G.to_device(x) for _, _, _, x in cols]
    dts = [dt for _, dt, _, _ in cols]

    def mean_ratio(trees):
        r = []
        for (nodes, _), d, (_, _, _, x) in zip(trees, devs, cols):
            r.append(x.nbytes / G.tree_compress(nodes, d).nbytes)
        return float(np.mean(r))

    exhaustive = []
    for d, dt in zip(devs, dts):
        nodes, _ = G.plan_exhaustive(dt, d)
        exhaustive.append((nodes, True))
    learned = P.plan(devs, dts, min_confidence=0.5)
    network_only = P.plan(devs, dts, min_confidence=0.0)
    _, mu, sd = P.get_params()
    untrained = G.Planner(_classes(P), seed=99)
    untrained.set_params(None, mu, sd)
    naive = untrained.plan(devs, dts, min_confidence=0.0)
    top = _classes(P)
    valid = P.valid()
    const = []
    for dt in dts:
        k = int(np.flatnonzero(valid[:, dt])[0])  # the most common class valid for the type
        const.append((G.tree_from_path(top[k], dt), False))
    r_ex, r_ln, r_net = mean_ratio(exhaustive), mean_ratio(learned), mean_ratio(network_only)
    r_un, r_const = mean_ratio(naive), mean_ratio(const)
    assert r_ln >= 0.97 * r_ex, (r_ln, r_ex)
    assert r_net > r_un and r_net > r_const, (r_net, r_un, r_const)


def _classes(P):
    """the class table of a planner, read back from its model file"""
    b = P.save()
    K = int(np.frombuffer(b[8:12], np.int32)[0])
    pos = 8 + 12 + 4 * 64 + 4 * int(P.n_params)
    out = []
    for _ in range(K):
        ln = int(np.frombuffer(b[pos:pos + 4], np.int32)[0])
        out.append(np.frombuffer(b[pos + 4:pos + 4 + 2 * ln], np.int16).tolist())
        pos += 4 + 2 * ln
    return out
