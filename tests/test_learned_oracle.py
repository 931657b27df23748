"""The CPU oracle of the learned planner checked on its own (no GPU): the MLP gradient against
central finite differences, and the feature definitions on hand-made columns."""
import numpy as np

import oracle as OR
from oracle import learned as OL


def test_mlp_gradient_matches_finite_differences(rng):
    K = 7
    n = OL.N_FEATURES * OL.HIDDEN + OL.HIDDEN + OL.HIDDEN * OL.HIDDEN + OL.HIDDEN + OL.HIDDEN * K + K
    p = rng.normal(0, 0.2, n)
    x = rng.normal(0, 1, (24, OL.N_FEATURES))
    lab = rng.integers(0, K, 24)
    lab[3] = -1
    mask = rng.random((24, K)) < 0.8
    mask[np.arange(24), np.maximum(lab, 0)] = True
    mu, sd = rng.normal(0, 0.1, OL.N_FEATURES), rng.uniform(0.5, 2, OL.N_FEATURES)
    _, g = OL.loss_and_grad(p, K, x, mu, sd, lab, mask)
    eps = 1e-6
    for i in rng.choice(n, 40, replace=False):
        q = p.copy()
        q[i] += eps
        a, _ = OL.loss_and_grad(q, K, x, mu, sd, lab, mask)
        q[i] -= 2 * eps
        b, _ = OL.loss_and_grad(q, K, x, mu, sd, lab, mask)
        assert abs((a - b) / (2 * eps) - g[i]) < 1e-6 + 1e-4 * abs(g[i])


def test_features_on_known_columns():
    f = OL.features(np.full(100, 7, np.int32), OR.INT)
    assert f[OR.INT] == 1 and f[10] == 1 and f[11] == 1 and f[13] == np.float32(0.01) and f[15] == 1
    assert f[18] == 0 and f[21] == np.float32(1 / 32) and f[30] == 1
    f = OL.features(np.arange(1000, dtype=np.int64), OR.TIME)
    assert f[10] == 1 and f[11] == 0 and f[13] == 1 and f[30] == 1 and f[23] == 0
    assert f[21] == np.float32(1 / 64)  # deltas all 1: BITLEN(1, 1) = 1 bit
    f = OL.features(np.array([1.5, 2.25, np.nan, -0.0], np.float32), OR.FLOAT)
    assert f[8] == np.float32(0.25) and f[26] == 1  # a NaN keeps multiplying: precision 10
    f = OL.features(np.zeros(0, np.int16), OR.SHORT)
    assert f[OR.SHORT] == 1 and not f[6:].any()
