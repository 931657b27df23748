"""CPU restatement of the learned tree planner's numerics: the 32 column features and the MLP's
forward pass, loss and gradients (numpy, float64).

TEST INFRASTRUCTURE ONLY.  The reference has no learned planner (its planners are
CompressionOptimizer::FullStatisticsUpdate / OptimizeTree, optimizer/compression_optimizer.cpp);
this file restates the library's own definitions so that its feature kernel and its FP32 forward /
backward kernels can be checked.  Float precision steps use the oracle's restatement of
_getFloatPrecision (util/statistics/cuda_array_statistics.cu:37-44).
"""
import ctypes

import numpy as np

from . import lib, NP_TYPES, FLOAT, DOUBLE

N_FEATURES = 32
HIDDEN = 64
SAMPLE = 10000


# ------------------------------------------------------------------------------ features
def _key(bits, es, fp):
    """order key (uint64) of raw bits, as the library's order_key"""
    b = bits.astype(np.uint64)
    if fp and es == 4:
        neg = (b & np.uint64(0x80000000)) != 0
        return np.where(neg, (~b) & np.uint64(0xffffffff), b | np.uint64(0x80000000))
    if fp and es == 8:
        neg = (b & np.uint64(1 << 63)) != 0
        return np.where(neg, ~b, b | np.uint64(1 << 63))
    s = _sext(b, es)
    return s.astype(np.uint64) ^ np.uint64(1 << 63)


def _sext(b, es):
    sh = np.uint64(64 - 8 * es)
    return ((b.astype(np.uint64) << sh).view(np.int64) >> sh.astype(np.int64))


def _bits_of(v):
    v = np.asarray(v, np.uint64)
    out = np.zeros(v.shape, np.int64)
    x = v.copy()
    while np.any(x):
        nz = x != 0
        out[nz] += 1
        x = x >> np.uint64(1)
    return out


def _bitlen_signed(mn, mx, es):
    if mn < 0:
        return 8 * es
    return 1 if mx == 0 else int(mx).bit_length()


def _unkey(k, es, fp):
    k = np.uint64(k)
    if fp and es == 4:
        v = int(k) & 0xffffffff
        return (v & 0x7fffffff) if v & 0x80000000 else (~v) & 0xffffffff
    if fp and es == 8:
        v = int(k)
        return (v & ((1 << 63) - 1)) if v & (1 << 63) else (~v) & ((1 << 64) - 1)
    s = int(k) ^ (1 << 63)
    return s if es == 8 else s & ((1 << (8 * es)) - 1)


def _as_double(bits_int, es, fp):
    if fp and es == 4:
        return float(np.array([bits_int], np.uint32).view(np.float32)[0])
    if fp and es == 8:
        return float(np.array([bits_int], np.uint64).view(np.float64)[0])
    return float(int(_sext(np.array([bits_int], np.uint64), es)[0]))


def features(x, dtype, n_total=None):
    """The 32 planner features of column x (numpy array of the data type's numpy dtype)."""
    es = np.dtype(NP_TYPES[dtype]).itemsize
    fp = dtype in (FLOAT, DOUBLE)
    W = 8 * es
    n_total = x.size if n_total is None else n_total
    m = min(n_total, SAMPLE)
    s = np.ascontiguousarray(x[:m])
    ubits = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[es]
    b = s.view(ubits).astype(np.uint64)
    f = np.zeros(N_FEATURES, np.float64)
    f[dtype] = 1
    f[6] = np.log2(n_total + 1.0) / 32
    f[7] = m / SAMPLE
    if m == 0:
        return f.astype(np.float32)
    if fp:
        nan = np.isnan(s)
        inf = np.isinf(s)
    else:
        nan = np.zeros(m, bool)
        inf = np.zeros(m, bool)
    keys = _key(b, es, fp)
    f[8] = nan.sum() / m
    f[9] = inf.sum() / m
    if m > 1:
        if fp:
            with np.errstate(invalid="ignore"):
                uns = np.sum(s[1:] < s[:-1])
        else:
            uns = np.sum(s[1:].astype(np.int64) < s[:-1].astype(np.int64))
    else:
        uns = 0
    f[10] = 1.0 if uns == 0 else 0.0
    same = int(np.sum(b[1:] == b[:-1])) if m > 1 else 0
    f[11] = same / (m - 1) if m > 1 else 0
    runs = m - same
    f[12] = np.log2(m / runs) / 14
    sk = np.sort(keys)
    bound = np.ones(m, bool)
    bound[1:] = sk[1:] != sk[:-1]
    distinct = int(bound.sum())
    f[13] = distinct / m
    f[14] = np.log2(distinct) / 14
    starts = np.flatnonzero(bound)
    mult = np.diff(np.append(starts, m))
    top = np.sort(mult)[::-1]
    f[15] = top[0] / m
    f[16] = top[:4].sum() / m
    nk = keys[~nan]
    any_ = nk.size > 0
    kmin = int(nk.min()) if any_ else 0
    kmax = int(nk.max()) if any_ else 0
    krange = kmax - kmin
    if not fp:
        mn = int(_sext(np.array([_unkey(kmin, es, fp)], np.uint64), es)[0]) if any_ else 0
        mx = int(_sext(np.array([_unkey(kmax, es, fp)], np.uint64), es)[0]) if any_ else 0
        f[17] = _bitlen_signed(mn, mx, es) / W
    else:
        f[17] = int(krange).bit_length() / W
    f[18] = int(krange).bit_length() / W
    kp90 = int(sk[((m - 1) * 9) // 10])
    f[19] = (kp90 - kmin).bit_length() / W if any_ and kp90 > kmin else 0
    if any_:
        tk = kmin + int(float(krange) * 0.9)
        lo = int(np.searchsorted(sk, np.uint64(tk), side="left"))
        hi = int(np.searchsorted(sk, np.uint64(kmax), side="right"))
        f[20] = (hi - lo) / m
    if m > 1:
        d = _sext((b[1:] - b[:-1]) & np.uint64((1 << W) - 1 if W < 64 else (1 << 64) - 1), es)
        dmin, dmax = int(d.min()), int(d.max())
        f[21] = _bitlen_signed(dmin, dmax, es) / W
        f[22] = ((dmax - dmin) & ((1 << 64) - 1)).bit_length() / W
        f[23] = np.sum(d < 0) / (m - 1)
        ad = np.abs(d.astype(object)).astype(np.uint64) if es == 8 else np.abs(d).astype(np.uint64)
        f[24] = _bits_of(ad).sum() / (m - 1) / W
        xo = (b[1:] ^ b[:-1])
        f[25] = ((_bits_of(xo) + 7) // 8).sum() / (m - 1) / es
    if fp:
        L = lib()
        L.or_float_precision.restype = ctypes.c_int
        steps = max(L.or_float_precision(ctypes.c_float(float(v))) for v in s.astype(np.float32))
        f[26] = steps / 10
        mnv = _as_double(_unkey(kmin, es, fp), es, fp) if any_ else 0.0
        mxv = _as_double(_unkey(kmax, es, fp), es, fp) if any_ else 0.0
        sc = 10.0 ** min(steps, 10) if steps < 10 else 0
        ok = steps < 10 and any_ and inf.sum() == 0 and mnv * sc > -2147483648.0 and mxv * sc < 2147483647.0
        f[27] = 1.0 if ok else 0.0
        f[28] = np.log2(1.0 + (mxv - mnv) * sc) / 32 if ok else 1.0
        with np.errstate(invalid="ignore"):
            dv = s.astype(np.float64)
            f[29] = np.sum((~nan) & (~inf) & (dv == np.rint(dv))) / m
    else:
        f[28] = int(krange).bit_length() / 32
        f[29] = 1.0
    if m > 2:
        d = _sext((b[1:] - b[:-1]) & np.uint64((1 << W) - 1 if W < 64 else (1 << 64) - 1), es)
        du = d.astype(np.uint64)
        d2 = _sext((du[1:] - du[:-1]) & np.uint64((1 << W) - 1 if W < 64 else (1 << 64) - 1), es)
        f[30] = np.sum(d2 == 0) / (m - 2)
        a2 = np.abs(d2.astype(object)).astype(np.uint64) if es == 8 else np.abs(d2).astype(np.uint64)
        f[31] = _bits_of(a2).sum() / (m - 2) / W
    return f.astype(np.float32)


# ------------------------------------------------------------------------------ MLP
def unpack(params, K):
    p = np.asarray(params, np.float64)
    o = 0
    shapes = [(N_FEATURES, HIDDEN), (HIDDEN,), (HIDDEN, HIDDEN), (HIDDEN,), (HIDDEN, K), (K,)]
    out = []
    for sh in shapes:
        n = int(np.prod(sh))
        out.append(p[o:o + n].reshape(sh))
        o += n
    return out


def loss_and_grad(params, K, x, mu, sd, labels, mask):
    """Mean softmax cross-entropy over the rows with label >= 0 (softmax over mask[row]) and its
    gradient, flattened in the library's parameter order."""
    W1, b1, W2, b2, W3, b3 = unpack(params, K)
    xn = (np.asarray(x, np.float64) - mu) / sd
    z1 = xn @ W1 + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0)
    z = h2 @ W3 + b3
    lab = np.asarray(labels)
    rows = lab >= 0
    nv = rows.sum()
    zm = np.where(mask, z, -np.inf)
    mx = zm.max(axis=1, keepdims=True)
    e = np.where(mask, np.exp(z - mx), 0.0)
    p = e / e.sum(axis=1, keepdims=True)
    loss = 0.0
    dz = p.copy()
    for r in range(z.shape[0]):
        if rows[r]:
            loss += -np.log(p[r, lab[r]])
            dz[r, lab[r]] -= 1
        else:
            dz[r] = 0
    dz /= nv
    gW3 = h2.T @ dz
    gb3 = dz.sum(0)
    dh2 = (dz @ W3.T) * (h2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (h1 > 0)
    gW1 = xn.T @ dh1
    gb1 = dh1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss / nv, g


def logits(params, K, x, mu, sd):
    W1, b1, W2, b2, W3, b3 = unpack(params, K)
    xn = (np.asarray(x, np.float64) - mu) / sd
    h1 = np.maximum(xn @ W1 + b1, 0)
    h2 = np.maximum(h1 @ W2 + b2, 0)
    return h2 @ W3 + b3
