"""Seeded synthetic workloads with the shapes, sizes and value distributions of the benchmark
configurations (no public dataset is involved; these generators stand in for real columns).

Generators (one per column kind):
  walk      random walk, steps uniform in [-8, 8], starting at 10^6
  runs      runs of geometric length (mean 32) drawn from 16 distinct values in [0, 2^20)
  zipf      Zipf(s=1.1) symbols over 5000 ids
  const     a constant column
  outliers  99% uniform in [0, 2^8), 1% uniform in [0, 2^31)
  price     round(100*sin(2*pi*t/1000) + N(0, 0.01), 2) with 0.1% NaN (random payloads, both
            signs), some +-inf and -0.0

Integer generators give float columns their values converted to the float type; the price
generator gives integer columns round(100 * price) (its NaN/inf positions become 0).
"""
import numpy as np

from . import CHAR, SHORT, INT, TIME, FLOAT, DOUBLE, NP_TYPES

KINDS = ["walk", "runs", "zipf", "const", "outliers", "price"]


def _zipf_ids(rng, n, s=1.1, ids=5000):
    p = 1.0 / np.arange(1, ids + 1) ** s
    p /= p.sum()
    return rng.choice(ids, n, p=p)


def gen_values(kind, n, rng):
    """float64 (price) or int64 values of a generator."""
    if kind == "walk":
        return 10 ** 6 + np.cumsum(rng.integers(-8, 9, n))
    if kind == "runs":
        vals = rng.choice(1 << 20, 16, replace=False)
        nruns = max(8, int(n / 32 * 1.5) + 8)
        lens = rng.geometric(1 / 32, nruns)
        while lens.sum() < n:
            lens = np.concatenate([lens, rng.geometric(1 / 32, nruns)])
        idx = rng.integers(0, 16, lens.size)
        # next run value differs from the previous one
        for i in range(1, idx.size):
            if idx[i] == idx[i - 1]:
                idx[i] = (idx[i] + 1) % 16
        return np.repeat(vals[idx], lens)[:n]
    if kind == "zipf":
        return _zipf_ids(rng, n)
    if kind == "const":
        return np.full(n, int(rng.integers(0, 1 << 20)))
    if kind == "outliers":
        x = rng.integers(0, 1 << 8, n)
        k = n // 100
        if k:
            pos = rng.choice(n, k, replace=False)
            x[pos] = rng.integers(0, 1 << 31, k)
        return x
    if kind == "price":
        t = np.arange(n)
        return np.round(100 * np.sin(2 * np.pi * t / 1000) + rng.normal(0, 0.01, n), 2)
    raise ValueError(kind)


def inject_specials(x, rng):
    """0.1% NaN with random payloads and both signs, a few +-inf and -0.0 (in place)."""
    n = x.size
    if n < 16:
        return x
    k = max(n // 1000, 1)
    pos = rng.choice(n, k + 6, replace=False)
    if x.dtype == np.float64:
        bits = x.view(np.uint64)
        pay = rng.integers(1, 1 << 52, k, dtype=np.uint64)
        sign = rng.integers(0, 2, k, dtype=np.uint64) << np.uint64(63)
        bits[pos[:k]] = np.uint64(0x7ff0000000000000) | pay | sign
    else:
        bits = x.view(np.uint32)
        pay = rng.integers(1, 1 << 23, k, dtype=np.uint32)
        sign = rng.integers(0, 2, k, dtype=np.uint32) << np.uint32(31)
        bits[pos[:k]] = np.uint32(0x7f800000) | pay | sign
    x[pos[k]], x[pos[k + 1]] = np.inf, -np.inf
    x[pos[k + 2]] = -0.0
    return x


def column(kind, dtype, n, seed):
    """One synthetic column as a numpy array of the data type's numpy dtype."""
    rng = np.random.default_rng(seed)
    v = gen_values(kind, n, rng)
    npt = NP_TYPES[dtype]
    if np.issubdtype(npt, np.floating):
        x = np.asarray(v, np.float64).astype(npt)
        if kind == "price":
            inject_specials(x, rng)
        return x
    if kind == "price":
        v = np.round(np.nan_to_num(v) * 100)
    info = np.iinfo(npt)
    return np.clip(np.asarray(v, np.int64), info.min, info.max).astype(npt)


def mixed_columns(ncols=512, seed=0xB204, min_len=4096, max_len=1 << 24):
    """The batched mixed workload: lengths log-uniform in [4096, 16M], types int32:float32:float64
    = 2:1:1, each column's generator chosen uniformly.  Returns [(kind, dtype, n, seed)]."""
    rng = np.random.default_rng(seed)
    types = [INT, INT, FLOAT, DOUBLE]
    out = []
    for c in range(ncols):
        n = int(np.floor(np.exp(rng.uniform(np.log(min_len), np.log(max_len)))))
        out.append((KINDS[rng.integers(0, len(KINDS))], types[rng.integers(0, 4)], n, seed * 1000 + c))
    return out
