"""ctypes bindings of the CPU oracle (oracle/liboracle.so) and of the reference's own AFL host path
(oracle/_ref/libref_afl.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline
legs, never by the product package.  Builds itself with `make` on first use when the shared object
is missing.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_afl.so")

# data types and encodings (compression/encoding_type.hpp:17-30)
CHAR, SHORT, INT, TIME, FLOAT, DOUBLE = range(6)
DELTA, AFL, SCALE, RLE, DICT, UNIQUE, PATCH, NONE, FLOAT2INT, CONST, GFC = range(11)
PATCH_OUTSIDE = 11  # PatchType::outside (patch_encoding_factory.hpp:47-55), serialised as PATCH
NP_TYPES = {CHAR: np.int8, SHORT: np.int16, INT: np.int32, TIME: np.int64,
            FLOAT: np.float32, DOUBLE: np.float64}
DTYPE_OF = {np.dtype(v): k for k, v in NP_TYPES.items()}
ENC_NAMES = ["delta", "afl", "scale", "rle", "dict", "unique", "patch", "none", "floatToInt",
             "constData", "gfc", "patch(outside)"]


class OracleError(RuntimeError):
    pass


class Stats(ctypes.Structure):
    _fields_ = [("min", ctypes.c_double), ("max", ctypes.c_double),
                ("min_bit_cnt", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("sorted", ctypes.c_int32), ("rl_metric", ctypes.c_float),
                ("mean", ctypes.c_double), ("size", ctypes.c_uint64)]


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


# the reference's source tree (read only when building oracle/_ref; absent on machines that only
# run the prebuilt files)
REF_SRC = os.environ.get("GTSC_REFERENCE_SRC", "/root/reference/src")


def build_ref():
    """Compile the reference AFL host path; returns False when the reference tree is absent."""
    if not os.path.isdir(REF_SRC):
        return os.path.exists(REF_PATH)
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True)
    return True


# the reference's own encoders and compression tree, built from its sources (oracle/Makefile,
# target refenc; oracle/ref_enc_shim.cu); they run on the GPU
REF_ENC_PATH = os.path.join(HERE, "_ref", "libref_enc.so")


def build_ref_enc():
    """Compile the reference encoders; returns whether the library exists afterwards."""
    if os.path.isdir(REF_SRC):
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "refenc", f"REF={REF_SRC}"], check=True)
    return os.path.exists(REF_ENC_PATH)


_lib = None
_ref = None


NATIVE_PATH = os.path.join(HERE, "_native", "liboracle.so")


def select_native():
    """Build the oracle -O3 -march=native for this host (oracle/_native, never shipped elsewhere)
    and route every later call through it.  Used only by the timed CPU legs of bench.py; parity
    checks run on the default build.  Returns a description of the build."""
    global _lib
    subprocess.run(["make", "-s", "-C", HERE, "native"], check=True)
    _lib = _bind(ctypes.CDLL(NATIVE_PATH))
    return "C oracle, gcc -O3 -march=native -ffp-contract=off"


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = _bind(ctypes.CDLL(LIB_PATH))
    return _lib


def _bind(L):
    """Declare the argument and result types of the oracle's C functions on a loaded library."""
    u8p = ctypes.POINTER(ctypes.c_uint8)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    L.or_encode.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                            u64p, ctypes.POINTER(ctypes.c_int)]
    L.or_decode.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                            ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                            ctypes.c_void_p, ctypes.c_uint64, u64p]
    L.or_bitlen.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int64]
    L.or_alt_bitlen.argtypes = [ctypes.c_int]
    L.or_stats.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Stats)]
    L.or_rl_metric.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int]
    L.or_rl_metric.restype = ctypes.c_float
    L.or_float_precision.argtypes = [ctypes.c_float]
    L.or_stencil_pack.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    L.or_stencil_pack.restype = ctypes.c_uint64
    L.or_stencil_unpack.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64]
    L.or_stencil_unpack.restype = ctypes.c_int64
    L.or_tree_from_path.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    L.or_tree_compress.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                   ctypes.c_void_p, ctypes.c_uint64, u64p]
    L.or_tree_decompress.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                                     u64p, ctypes.POINTER(ctypes.c_int)]
    L.or_tree_predict_size.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, u64p]
    for f in (L.or_plan_exhaustive, L.or_optimize_tree):
        f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int,
                      ctypes.POINTER(ctypes.c_int), u64p]
    L.or_sample_bytes.argtypes = [ctypes.c_int, ctypes.c_uint64]
    L.or_sample_bytes.restype = ctypes.c_uint64
    del u8p
    return L


def ref():
    """The reference's own AFL host implementation, or None when it was not built."""
    global _ref
    if _ref is None and os.path.exists(REF_PATH):
        _ref = ctypes.CDLL(REF_PATH)
    return _ref


_ref_enc = None


def ref_enc():
    """The reference's encoders and tree (a CUDA library), or None when it was not built."""
    global _ref_enc
    if _ref_enc is None and os.path.exists(REF_ENC_PATH):
        L = ctypes.CDLL(REF_ENC_PATH)
        vp, u64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)
        L.ref_enc_error.restype = ctypes.c_char_p
        L.ref_enc_free.argtypes = [vp]
        L.ref_enc_encode.argtypes = [ctypes.c_int, ctypes.c_int, vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(vp), u64p]
        L.ref_enc_decode.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp), u64p,
                                     ctypes.POINTER(vp), u64p]
        L.ref_tree_compress.argtypes = [vp, ctypes.c_int, vp, ctypes.c_uint64, ctypes.POINTER(vp), u64p]
        L.ref_tree_decompress.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(vp), u64p]
        _ref_enc = L
    return _ref_enc


def _ref_take(L, p, n):
    """Copy a host buffer the reference shim allocated into numpy and free it."""
    out = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint8)), (max(n, 1),))[:n].copy() \
        if n else np.zeros(0, np.uint8)
    L.ref_enc_free(p)
    return out


def _ref_check(L, rc, what):
    if rc != 0:
        raise OracleError(f"reference {what}: {L.ref_enc_error().decode()}")


def ref_encode(enc, dtype, data):
    """The reference's Encoding::Encode (through its factory's Get(data)) -> [metadata, out1, ...]."""
    L = ref_enc()
    src = as_bytes(data)
    nres = ctypes.c_int(0)
    outs = (ctypes.c_void_p * 4)()
    sizes = (ctypes.c_uint64 * 4)()
    rc = L.ref_enc_encode(enc, dtype, _ptr(src), src.size, ctypes.byref(nres), outs, sizes)
    res = [_ref_take(L, outs[i], sizes[i]) for i in range(nres.value)]
    _ref_check(L, rc, f"encode {ENC_NAMES[enc]}")
    return res


def ref_decode(enc, dtype, parts):
    """The reference's Encoding::Decode (through its factory's Get()) -> byte array."""
    L = ref_enc()
    parts = [as_bytes(p) for p in parts]
    ptrs = (ctypes.c_void_p * len(parts))(*[_ptr(p) for p in parts])
    sizes = (ctypes.c_uint64 * len(parts))(*[p.size for p in parts])
    out = ctypes.c_void_p()
    ob = ctypes.c_uint64(0)
    rc = L.ref_enc_decode(enc, dtype, len(parts), ptrs, sizes, ctypes.byref(out), ctypes.byref(ob))
    res = _ref_take(L, out, ob.value) if out.value else np.zeros(0, np.uint8)
    _ref_check(L, rc, f"decode {ENC_NAMES[enc]}")
    return res


def ref_tree_compress(nodes, data):
    """The reference's CompressionTree::Compress of a pre-order (encoding, type) node list."""
    L = ref_enc()
    nodes = np.asarray(nodes, np.int16)
    src = as_bytes(data)
    out = ctypes.c_void_p()
    ob = ctypes.c_uint64(0)
    rc = L.ref_tree_compress(_ptr(nodes), nodes.size // 2, _ptr(src), src.size, ctypes.byref(out), ctypes.byref(ob))
    res = _ref_take(L, out, ob.value) if out.value else np.zeros(0, np.uint8)
    _ref_check(L, rc, "tree compress")
    return res


def ref_tree_decompress(blob):
    """The reference's CompressionTree::Decompress."""
    L = ref_enc()
    blob = as_bytes(blob)
    out = ctypes.c_void_p()
    ob = ctypes.c_uint64(0)
    rc = L.ref_tree_decompress(_ptr(blob), blob.size, ctypes.byref(out), ctypes.byref(ob))
    res = _ref_take(L, out, ob.value) if out.value else np.zeros(0, np.uint8)
    _ref_check(L, rc, "tree decompress")
    return res


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None and a.size else None


def as_bytes(a):
    return np.ascontiguousarray(a).view(np.uint8).reshape(-1)


def _check(rc, what):
    if rc != 0:
        raise OracleError(f"{what} failed with status {rc}")


def encode(enc, dtype, data):
    """Encoding::Encode -> list of byte arrays [metadata, out1, (out2)]."""
    src = as_bytes(data)
    n = src.size
    cap = 5 * n + 65536  # RLE of 1-byte values: 4 bytes of run length per value
    outs = [np.zeros(cap, np.uint8) for _ in range(3)]
    ob = (ctypes.c_uint64 * 3)()
    n_out = ctypes.c_int(0)
    _check(lib().or_encode(enc, dtype, _ptr(src), n, _ptr(outs[0]), _ptr(outs[1]), _ptr(outs[2]),
                           cap, ob, ctypes.byref(n_out)), f"encode {ENC_NAMES[enc]}")
    return [outs[i][:ob[i]].copy() for i in range(n_out.value)]


def decode(enc, dtype, parts, cap=None):
    """Encoding::Decode -> byte array."""
    parts = [as_bytes(p) for p in parts] + [np.zeros(0, np.uint8)] * (3 - len(parts))
    if cap is None:
        cap = 64 * sum(p.size for p in parts) + 4096
    out = np.zeros(cap, np.uint8)
    ob = ctypes.c_uint64(0)
    _check(lib().or_decode(enc, dtype, _ptr(parts[0]), parts[0].size, _ptr(parts[1]), parts[1].size,
                           _ptr(parts[2]), parts[2].size, _ptr(out), cap, ctypes.byref(ob)),
           f"decode {ENC_NAMES[enc]}")
    return out[:ob.value].copy()


def stats(dtype, data):
    s = Stats()
    src = as_bytes(data)
    _check(lib().or_stats(dtype, _ptr(src), src.size, ctypes.byref(s)), "stats")
    return s


def tree_from_path(encs, dtype):
    p = np.asarray(encs, np.int16)
    nodes = np.zeros(256, np.int16)
    r = lib().or_tree_from_path(_ptr(p), p.size, dtype, _ptr(nodes), 128)
    if r < 0:
        raise OracleError(f"tree_from_path failed {r}")
    return nodes[:2 * r].copy()


def tree_compress(nodes, data):
    nodes = np.asarray(nodes, np.int16)
    src = as_bytes(data)
    cap = 8 * src.size + 65536
    out = np.zeros(cap, np.uint8)
    ob = ctypes.c_uint64(0)
    _check(lib().or_tree_compress(_ptr(nodes), nodes.size // 2, _ptr(src), src.size, _ptr(out), cap,
                                  ctypes.byref(ob)), "tree_compress")
    return out[:ob.value].copy()


def tree_decompress(blob, cap):
    blob = as_bytes(blob)
    out = np.zeros(max(cap, 1), np.uint8)
    ob = ctypes.c_uint64(0)
    dt = ctypes.c_int(0)
    _check(lib().or_tree_decompress(_ptr(blob), blob.size, _ptr(out), cap, ctypes.byref(ob),
                                    ctypes.byref(dt)), "tree_decompress")
    return out[:ob.value].copy(), dt.value


def tree_predict_size(nodes, data):
    nodes = np.asarray(nodes, np.int16)
    src = as_bytes(data)
    sz = ctypes.c_uint64(0)
    _check(lib().or_tree_predict_size(_ptr(nodes), nodes.size // 2, _ptr(src), src.size,
                                      ctypes.byref(sz)), "tree_predict_size")
    return sz.value


def _plan(fn, dtype, data):
    src = as_bytes(data)
    nodes = np.zeros(1024, np.int16)
    nn = ctypes.c_int(0)
    sz = ctypes.c_uint64(0)
    _check(fn(dtype, _ptr(src), src.size, _ptr(nodes), 512, ctypes.byref(nn), ctypes.byref(sz)), "plan")
    return nodes[:2 * nn.value].copy(), sz.value


def plan_exhaustive(dtype, data):
    """FullStatisticsUpdate + max-ratio pick on `data` (already the sample)."""
    return _plan(lib().or_plan_exhaustive, dtype, data)


def optimize_tree(dtype, data):
    return _plan(lib().or_optimize_tree, dtype, data)


def sample_bytes(dtype, nbytes):
    return lib().or_sample_bytes(dtype, nbytes)


# ------------------------------------------------------------------ reference AFL host path
_REF_T = {CHAR: ("char", np.int8), SHORT: ("short", np.int16), INT: ("int", np.int32),
          TIME: ("long", np.int64)}


def ref_afl_compress(dtype, data, bit_length):
    """run_afl_compress_cpu<T,1> of the reference (afl_gpu.cu:6-30) -> packed words as bytes."""
    R = ref()
    name, npt = _REF_T[dtype]
    x = np.ascontiguousarray(data, npt)
    W = 8 * x.itemsize
    words = (bit_length * x.size + W - 1) // W
    out = np.zeros(max(words, 1), npt)
    fn = getattr(R, f"ref_afl_compress_{name}")
    fn.argtypes = [ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulong, ctypes.c_ulong]
    fn(bit_length, _ptr(x), _ptr(out), x.size, words)
    return out[:words].view(np.uint8).copy()


def afl_layout_words(omega, dtype, b, n):
    L = lib()
    L.or_afl_words.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint64]
    L.or_afl_words.restype = ctypes.c_uint64
    return L.or_afl_words(omega, dtype, b, n)


def afl_layout_pack(omega, dtype, data, b):
    """The packed stream of `data` in the FL (omega 1) or aligned (omega 32) layout, as bytes."""
    L = lib()
    x = np.ascontiguousarray(data)
    words = afl_layout_words(omega, dtype, b, x.size)
    out = np.zeros(max(words * x.itemsize, 1), np.uint8)
    L.or_afl_pack.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                              ctypes.c_void_p, ctypes.c_uint64]
    r = L.or_afl_pack(omega, dtype, b, _ptr(x), x.size, _ptr(out), words)
    if r:
        raise OracleError(r)
    return out[:words * x.itemsize].copy()


def afl_layout_values(omega, dtype, packed, b, n, idx=None):
    """Elements idx (or 0..n-1) of a packed stream, in the dtype's integer type."""
    L = lib()
    npt = _REF_T[dtype][1]
    es = np.dtype(npt).itemsize
    comp = np.ascontiguousarray(packed, np.uint8)
    ix = None if idx is None else np.ascontiguousarray(idx, np.uint64)
    m = n if ix is None else ix.size
    out = np.zeros(max(m, 1), npt)
    L.or_afl_values.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    r = L.or_afl_values(omega, dtype, b, _ptr(comp), comp.size // es, None if ix is None else _ptr(ix), m,
                        _ptr(out))
    if r:
        raise OracleError(r)
    return out[:m].copy()


def ref_afl32_compress(dtype, data, bit_length):
    """run_afl_compress_cpu<T,32> of the reference (afl_gpu.cu:5-30) -> packed words as bytes."""
    R = ref()
    name, npt = _REF_T[dtype]
    x = np.ascontiguousarray(data, npt)
    words = afl_layout_words(32, dtype, bit_length, x.size)
    out = np.zeros(max(words, 1) + 64, npt)
    fn = getattr(R, f"ref_afl32_compress_{name}")
    fn.argtypes = [ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulong, ctypes.c_ulong]
    fn(bit_length, _ptr(x), _ptr(out), x.size, words)
    assert not out[words:].any()
    return out[:words].view(np.uint8).copy()


def ref_afl32_decompress(dtype, packed, bit_length, n):
    """run_afl_decompress_cpu<T,32> of the reference (afl_gpu.cu:43-65)."""
    R = ref()
    name, npt = _REF_T[dtype]
    W = np.dtype(npt).itemsize
    comp = np.zeros((packed.size + W - 1) // W + 64, npt)
    comp.view(np.uint8)[:packed.size] = packed
    out = np.zeros(max(n, 1), npt)
    fn = getattr(R, f"ref_afl32_decompress_{name}")
    fn.argtypes = [ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulong]
    fn(bit_length, _ptr(comp), _ptr(out), n)
    return out[:n].copy()


def ref_afl_value(dtype, omega, packed, bit_length, i):
    """afl_decompress_base_value_gpu<T,omega> of the reference (afl_gpu.cu:197-222), int or long."""
    R = ref()
    name, npt = _REF_T[dtype]
    W = np.dtype(npt).itemsize
    comp = np.zeros((packed.size + W - 1) // W + 64, npt)
    comp.view(np.uint8)[:packed.size] = packed
    fn = getattr(R, f"ref_afl_value_{name}")
    fn.argtypes = [ctypes.c_uint, ctypes.c_int, ctypes.c_void_p, ctypes.c_ulong]
    fn.restype = ctypes.c_long if name == "long" else ctypes.c_int
    return fn(bit_length, omega, _ptr(comp), i)


def ref_afl_decompress(dtype, packed, bit_length, n):
    R = ref()
    name, npt = _REF_T[dtype]
    W = np.dtype(npt).itemsize
    comp = np.zeros((packed.size + W - 1) // W + 2, npt)
    comp.view(np.uint8)[:packed.size] = packed
    out = np.zeros(max(n, 1), npt)
    fn = getattr(R, f"ref_afl_decompress_{name}")
    fn.argtypes = [ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulong]
    fn(bit_length, _ptr(comp), _ptr(out), n)
    return out[:n].copy()
