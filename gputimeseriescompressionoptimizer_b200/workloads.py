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


# ------------------------------------------------------------------------------ tick table
TICK_COLUMNS = ["ts", "price", "volume", "symbol", "flags"]


def tick_chunk(n_cols=40, rows=1 << 20, chunk=0, seed=0x71C4):
    """One chunk of the streaming tick table: n_cols columns of `rows` rows, chunk index `chunk`
    (chunks of the same column continue one another).  Column c has kind TICK_COLUMNS[c % 5]:
      ts      int64 microseconds, monotone, exponential gaps with mean 1 ms
      price   float64 random walk in 0.01 ticks, rounded to 2 decimals
      volume  int32 Zipf(1.5) lot sizes x 100
      symbol  int32 Zipf(1.1) ids over 5000
      flags   int32, every 4th flags column constant, the others over 4 values
    Returns [(kind, dtype, array)]."""
    out = []
    for c in range(n_cols):
        kind = TICK_COLUMNS[c % len(TICK_COLUMNS)]
        rng = np.random.default_rng([seed, c, chunk])
        base = np.random.default_rng([seed, c]).integers(0, 1 << 20)
        if kind == "ts":
            start = 1_700_000_000_000_000 + chunk * rows * 1000
            x = (start + np.cumsum(rng.exponential(1000.0, rows))).astype(np.int64)
            out.append((kind, TIME, x))
        elif kind == "price":
            ticks = rng.integers(-1, 2, rows).cumsum() + (base % 100000) + 1000 + chunk * 7
            out.append((kind, DOUBLE, np.round(ticks * 0.01, 2)))
        elif kind == "volume":
            out.append((kind, INT, (np.minimum(rng.zipf(1.5, rows), 10000) * 100).astype(np.int32)))
        elif kind == "symbol":
            out.append((kind, INT, _zipf_ids(rng, rows).astype(np.int32)))
        else:
            if (c // len(TICK_COLUMNS)) % 4 == 0:
                out.append((kind, INT, np.full(rows, int(base % 16), np.int32)))
            else:
                out.append((kind, INT, rng.integers(0, 4, rows).astype(np.int32)))
    return out


# ------------------------------------------------------------------------------ planner training
TRAIN_KINDS = KINDS + ["ts", "tick_price", "volume", "flags", "uniform", "sawtooth"]


def training_column(seed, m=10000):
    """One seeded training column for the learned planner: (kind, dtype, nominal length, the first
    min(m, length) values).  Four in ten come from the benchmark generators (column(), fresh seeds),
    fifteen in a hundred from the tick-table generators, the rest from the family below whose
    parameters are drawn per column."""
    rng = np.random.default_rng([0x7EA1, seed])
    n_total = int(np.floor(np.exp(rng.uniform(np.log(1024), np.log(1 << 24)))))
    n = min(m, n_total)
    u = rng.random()
    if u < 0.40:
        kind = KINDS[rng.integers(0, len(KINDS))]
        dtype = [INT, INT, FLOAT, DOUBLE, TIME, SHORT][rng.integers(0, 6)]
        return kind, dtype, n_total, column(kind, dtype, n, (0x7EA1 << 20) + seed)
    if u < 0.55:
        chunk = tick_chunk(n_cols=5, rows=n, chunk=int(rng.integers(0, 1000)), seed=int(rng.integers(1 << 30)))
        kind, dtype, x = chunk[rng.integers(0, 5)]
        return "tick_" + kind, dtype, n_total, x
    kind = TRAIN_KINDS[rng.integers(0, len(TRAIN_KINDS))]
    dtype = [INT, INT, FLOAT, DOUBLE, TIME, SHORT, CHAR][rng.integers(0, 7)]
    v = None
    if kind == "walk":
        step = int(rng.integers(1, 65))
        v = int(rng.integers(-10 ** 6, 10 ** 7)) + np.cumsum(rng.integers(-step, step + 1, n))
    elif kind == "runs":
        k = int(rng.integers(2, 65))
        mean = float(np.exp(rng.uniform(np.log(2), np.log(256))))
        vals = rng.integers(0, 1 << int(rng.integers(4, 30)), k)
        lens = rng.geometric(1 / mean, n)
        v = np.repeat(vals[rng.integers(0, k, n)], lens)[:n]
    elif kind == "zipf":
        a = float(rng.uniform(1.01, 2.0))
        ids = int(np.exp(rng.uniform(np.log(10), np.log(100000))))
        v = np.minimum(rng.zipf(a, n), ids) - 1 + int(rng.integers(0, 1000))
    elif kind == "const":
        v = np.full(n, int(rng.integers(-1000, 1 << 20)))
    elif kind == "outliers":
        bits = int(rng.integers(2, 17))
        v = rng.integers(0, 1 << bits, n)
        k = int(n * rng.uniform(0.0005, 0.05))
        if k:
            v[rng.choice(n, k, replace=False)] = rng.integers(0, 1 << 31, k)
    elif kind in ("price", "tick_price"):
        dec = int(rng.integers(1, 5))
        if kind == "price":
            t = np.arange(n)
            x = np.round(float(rng.uniform(1, 1000)) * np.sin(2 * np.pi * t / float(rng.uniform(100, 5000)))
                         + rng.normal(0, float(rng.uniform(0.001, 1)), n), dec)
        else:
            x = np.round((rng.integers(-1, 2, n).cumsum() + int(rng.integers(100, 100000))) * 10.0 ** -dec, dec)
        v = x
    elif kind == "ts":
        gap = float(np.exp(rng.uniform(0, np.log(10 ** 6))))
        v = (int(rng.integers(0, 1 << 40)) + np.cumsum(rng.exponential(gap, n))).astype(np.int64)
    elif kind == "volume":
        v = (np.minimum(rng.zipf(float(rng.uniform(1.2, 3)), n), 10000) * int(rng.choice([1, 10, 100]))).astype(np.int64)
    elif kind == "flags":
        v = rng.integers(0, int(rng.integers(1, 5)), n)
    elif kind == "uniform":
        v = rng.integers(0, 1 << int(rng.integers(1, 40)), n)
    else:  # sawtooth
        period = int(rng.integers(2, 1000))
        v = (np.arange(n) % period) * int(rng.integers(1, 100))
    npt = NP_TYPES[dtype]
    if np.issubdtype(npt, np.floating):
        x = np.asarray(v, np.float64).astype(npt)
        if rng.random() < 0.15:
            inject_specials(x, rng)
        return kind, dtype, n_total, x
    if np.asarray(v).dtype.kind == "f":
        v = np.round(np.nan_to_num(np.asarray(v)) * 10 ** 2)
    info = np.iinfo(npt)
    return kind, dtype, n_total, np.clip(np.asarray(v, np.int64), info.min, info.max).astype(npt)
