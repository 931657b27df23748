"""The cases of the reference-encoder fixtures, shared by their generator and their tests.

The fixtures hold what the reference's own encoders and compression tree (compiled from its
sources, oracle/ref_enc_shim.cu) produce on the GPU for seeded synthetic columns:
make_reference_fixtures.py runs them on a machine with a GPU and writes reference_encoders.npz;
tests/test_oracle_reference_fixtures.py checks the CPU oracle against that file without a GPU.

Inputs are stored in the file (the generators are not relied on to give the same values under
another numpy).  Streams of at most FULL_LIMIT input values are stored whole; larger ones as their
SHA-256 and size.
"""
import hashlib

import numpy as np

import oracle as OR
from gputimeseriescompressionoptimizer_b200 import workloads as W

SEED = 0x5EED
FULL_LIMIT = 1000
SIZES = [1, 2, 33, 1000, 4099]
INT_KINDS = ["walk", "runs", "zipf", "const", "outliers", "price"]
FLOAT_KINDS = ["price", "walk", "const", "runs"]
DTYPES = [OR.CHAR, OR.SHORT, OR.INT, OR.TIME, OR.FLOAT, OR.DOUBLE]
ENCODINGS = [OR.DELTA, OR.AFL, OR.SCALE, OR.RLE, OR.DICT, OR.UNIQUE, OR.PATCH, OR.NONE, OR.FLOAT2INT,
             OR.CONST, OR.PATCH_OUTSIDE]
TREE_SIZE = 5000
# compression trees as pre-order encoding lists, with the generator and type they run on
TREES = [
    ("walk", OR.INT, [OR.DELTA, OR.AFL, OR.NONE]),
    ("walk", OR.INT, [OR.DELTA, OR.SCALE, OR.AFL, OR.NONE]),
    ("runs", OR.INT, [OR.RLE, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("zipf", OR.INT, [OR.DICT, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("const", OR.INT, [OR.CONST, OR.AFL, OR.NONE]),
    ("outliers", OR.INT, [OR.PATCH, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("outliers", OR.INT, [OR.PATCH_OUTSIDE, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("walk", OR.TIME, [OR.DELTA, OR.RLE, OR.AFL, OR.NONE, OR.DELTA, OR.AFL, OR.NONE]),
    ("runs", OR.SHORT, [OR.RLE, OR.DELTA, OR.AFL, OR.NONE, OR.SCALE, OR.AFL, OR.NONE]),
    ("zipf", OR.INT, [OR.DICT, OR.NONE, OR.PATCH, OR.SCALE, OR.AFL, OR.NONE, OR.NONE]),
    ("price", OR.FLOAT, [OR.FLOAT2INT, OR.DELTA, OR.AFL, OR.NONE]),
    ("price", OR.FLOAT, [OR.FLOAT2INT, OR.SCALE, OR.AFL, OR.NONE]),
    ("walk", OR.DOUBLE, [OR.SCALE, OR.NONE]),
    ("runs", OR.FLOAT, [OR.RLE, OR.AFL, OR.NONE, OR.NONE]),
    ("zipf", OR.TIME, [OR.UNIQUE, OR.AFL, OR.NONE]),
]


def kinds_of(dt):
    return FLOAT_KINDS if dt in (OR.FLOAT, OR.DOUBLE) else INT_KINDS


def column(kind, dt, n, k):
    """The input of case k (its own seed)."""
    return W.column(kind, dt, n, SEED + 7919 * k)


def digest(b):
    return hashlib.sha256(np.ascontiguousarray(b).tobytes()).hexdigest()


def unique_tail_mask(stream, header_bytes, m, table_count):
    """A copy of a unique-coded stream with the code slots past its m values cleared.

    UniqueEncoding::CompressUnique (compression/unique/unique_encoding.cu:48-76) fills the last
    output word from values read past the end of its input; the oracle writes zero codes there.
    The stream is [header_bytes][uint32 words], 32 / bits codes per word."""
    s = np.array(stream, np.uint8, copy=True)
    if m == 0 or s.size <= header_bytes:
        return s
    bits = int(OR.lib().or_alt_bitlen(int(table_count) - 1))
    per = 32 // bits
    used = m % per
    if used == 0:
        return s
    off = header_bytes + 4 * ((m - 1) // per)
    if off + 4 > s.size:
        return s
    w = int(s[off:off + 4].view(np.uint32)[0])
    w &= (1 << (bits * used)) - 1
    s[off:off + 4] = np.frombuffer(np.uint32(w).tobytes(), np.uint8)
    return s


def lossy_in_reference(enc, dt, x):
    """Cases where the reference's own stream loses data and the library keeps every bit on
    purpose: the standalone unique coder's table merges -0.0 into +0.0 and cannot find NaNs
    (thrust::unique and == in compression/unique/unique_encoding.cu:35-46), while the library keeps
    distinct bit patterns."""
    if enc != OR.UNIQUE or dt not in (OR.FLOAT, OR.DOUBLE):
        return False
    x = np.asarray(x)
    return bool(np.isnan(x).any() or (np.signbit(x) & (x == 0)).any())


def canonical(enc, dt, streams):
    """The encoder's streams with the code slots past the last value cleared, which the reference
    fills from values read past the end of its input (unique_encoding.cu:56-61)."""
    out = [np.asarray(s, np.uint8) for s in streams]
    es = np.dtype(OR.NP_TYPES[dt]).itemsize
    if enc == OR.DICT and len(out) >= 2 and out[1].size >= 16:
        cnt, m = (int(v) for v in out[1][:16].view(np.uint64))
        out[1] = unique_tail_mask(out[1], 16 + cnt * es, m, cnt)
    if enc == OR.UNIQUE and len(out) >= 2 and out[0].size >= 16:
        cnt, m = (int(v) for v in out[0][:16].view(np.uint64))
        out[1] = unique_tail_mask(out[1], 0, m, cnt)
    return out
