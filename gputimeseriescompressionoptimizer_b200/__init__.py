"""gputimeseriescompressionoptimizer_b200 -- B200-native lightweight column compression.

Python host side over the C ABI of libgtsc.so (declared in include/gtsc.h).  The CUDA library is
the only implementation: importing this package loads it, and every call fails loudly when it is
missing or when no GPU is present -- there is no CPU fallback.

Low-level API (device buffers in, device buffers out)::

    import gputimeseriescompressionoptimizer_b200 as g
    col = g.to_device(np.arange(1000, dtype=np.int32))
    parts = g.encode(g.AFL, g.INT, col)          # [metadata, data] on the GPU
    back = g.decode(g.AFL, g.INT, parts)
    assert (g.to_host(back, np.int32) == np.arange(1000)).all()

The reference-shaped classes (EncodingType, DataType, Encoding factories, CompressionTree,
CompressionOptimizer, ...) live in `gputimeseriescompressionoptimizer_b200.api`.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgtsc.so")

# DataType codes (this library's; the reference's live in an unavailable submodule)
CHAR, SHORT, INT, TIME, FLOAT, DOUBLE = range(6)
# EncodingType codes (compression/encoding_type.hpp:17-30)
DELTA, AFL, SCALE, RLE, DICT, UNIQUE, PATCH, NONE, FLOAT_TO_INT, CONST, GFC = range(11)
# the outside variant of the patch encoding (PatchType::outside); serialised as PATCH
PATCH_OUTSIDE = 11
ENCODING_NAMES = ["delta", "afl", "scale", "rle", "dict", "unique", "patch", "none", "floatToInt",
                  "constData", "gfc", "patch(outside)"]
NP_TYPES = {CHAR: np.int8, SHORT: np.int16, INT: np.int32, TIME: np.int64, FLOAT: np.float32,
            DOUBLE: np.float64}

STATUS_NAMES = {0: "OK", -1: "ERR_ARG", -2: "ERR_TYPE", -3: "ERR_CAPACITY", -4: "ERR_FORMAT",
                -5: "ERR_UNSUPPORTED", -6: "ERR_CUDA", -7: "ERR_TIMEOUT", -8: "ERR_NO_DEVICE"}


class GtscError(RuntimeError):
    """A libgtsc call returned a non-zero status."""

    def __init__(self, status, what, message):
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Buffer(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p), ("bytes", ctypes.c_uint64)]


class Column(ctypes.Structure):
    _fields_ = [("d_data", ctypes.c_void_p), ("bytes", ctypes.c_uint64), ("dtype", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class DataStatistics(ctypes.Structure):
    """DataStatistics (util/statistics/cuda_array_statistics.hpp:24-34)."""
    _fields_ = [("min", ctypes.c_double), ("max", ctypes.c_double),
                ("min_bit_cnt", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("sorted", ctypes.c_int32), ("rl_metric", ctypes.c_float),
                ("mean", ctypes.c_double), ("size", ctypes.c_uint64)]


_lib = None


def lib():
    """The loaded libgtsc.so.  Raises when the extension was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libgtsc.so not built ({LIB_PATH}); run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        vp, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32
        L.gtsc_last_error.restype = ctypes.c_char_p
        L.gtsc_version.restype = ctypes.c_char_p
        L.gtsc_dtype_size.argtypes = [i32]
        L.gtsc_malloc.argtypes = [ctypes.POINTER(vp), u64, vp]
        L.gtsc_free.argtypes = [vp, vp]
        L.gtsc_memcpy.argtypes = [vp, vp, u64, i32, vp]
        L.gtsc_memcpy_async.argtypes = [vp, vp, u64, i32, vp]
        L.gtsc_stream_synchronize.argtypes = [vp]
        L.gtsc_encode.argtypes = [i32, i32, vp, u64, ctypes.POINTER(Buffer), ctypes.POINTER(ctypes.c_uint32), vp]
        L.gtsc_decode.argtypes = [i32, i32, ctypes.POINTER(Buffer), ctypes.c_uint32, ctypes.POINTER(Buffer), vp]
        u32 = ctypes.c_uint32
        L.gtsc_stats.argtypes = [i32, vp, u64, ctypes.POINTER(DataStatistics), vp]
        L.gtsc_afl_compress_gpu.argtypes = [i32, u32, vp, u64, vp, u64, vp]
        L.gtsc_afl_decompress_gpu.argtypes = [i32, u32, vp, u64, vp, u64, vp]
        i16p, i32p, u64p = ctypes.POINTER(ctypes.c_int16), ctypes.POINTER(i32), ctypes.POINTER(u64)
        L.gtsc_tree_from_path.argtypes = [i16p, i32, i32, i16p, i32, i32p]
        L.gtsc_tree_compress.argtypes = [i16p, i32, vp, u64, ctypes.POINTER(Buffer), vp]
        L.gtsc_tree_decompress.argtypes = [vp, u64, ctypes.POINTER(Buffer), i32p, vp]
        L.gtsc_tree_predict_size.argtypes = [i16p, i32, vp, u64, u64p, vp]
        L.gtsc_plan_exhaustive.argtypes = [i32, vp, u64, i16p, i32, i32p, u64p, vp]
        L.gtsc_optimize_tree.argtypes = [i32, vp, u64, i16p, i32, i32p, u64p, vp]
        L.gtsc_sample_bytes.argtypes = [i32, u64]
        L.gtsc_sample_bytes.restype = u64
        L.gtsc_delta_decode_noalloc.argtypes = [i32, vp, vp, u64, vp, vp]
        L.gtsc_selftest_lookback_timeout.argtypes = [ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double), vp]
        i16, f64 = ctypes.c_int16, ctypes.c_double
        L.gtsc_optimizer_create.argtypes = [i32, ctypes.POINTER(vp)]
        L.gtsc_optimizer_compress.argtypes = [vp, vp, u64, vp, vp, vp, vp]
        L.gtsc_optimizer_tree.argtypes = [vp, vp, vp, i32, vp]
        L.gtsc_optimizer_statistics.argtypes = [vp, ctypes.POINTER(vp)]
        L.gtsc_optimizer_destroy.argtypes = [vp]
        L.gtsc_edge_stats_create.argtypes = [i32, ctypes.POINTER(vp)]
        L.gtsc_edge_stats_destroy.argtypes = [vp]
        L.gtsc_edge_stats_set.argtypes = [vp, i32, i16, i16, f64]
        L.gtsc_edge_stats_update.argtypes = [vp, i32, i16, i16, f64]
        L.gtsc_edge_stats_get.argtypes = [vp, i32, i16, i16, vp]
        L.gtsc_edge_stats_best.argtypes = [vp, i32, i16, i16, i32, vp, vp, vp]
        L.gtsc_edge_stats_entries.argtypes = [vp, i32, vp, vp, i32, vp]
        L.gtsc_tree_edges.argtypes = [vp, i32, vp, vp, vp, i32, vp]
        L.gtsc_tree_update_statistics.argtypes = [vp, vp, i32, vp]
        L.gtsc_optimal_tree_create.argtypes = [vp, vp, i32, vp, ctypes.POINTER(vp)]
        L.gtsc_optimal_tree_set_ratio.argtypes = [vp, i32, f64]
        L.gtsc_optimal_tree_try_correct.argtypes = [vp, vp]
        L.gtsc_optimal_tree_get.argtypes = [vp, vp, vp, i32, vp]
        L.gtsc_optimal_tree_destroy.argtypes = [vp]
        L.gtsc_predict_sizes.argtypes = [i32, i32, vp, u64, ctypes.POINTER(u64), ctypes.POINTER(u64), vp]
        L.gtsc_afl32_bytes.argtypes = [i32, u32, u64]
        L.gtsc_afl32_bytes.restype = u64
        L.gtsc_afl32_compress_gpu.argtypes = [i32, u32, vp, u64, vp, u64, vp]
        L.gtsc_afl32_decompress_gpu.argtypes = [i32, u32, vp, u64, vp, u64, vp]
        L.gtsc_afl_values_gpu.argtypes = [i32, u32, i32, vp, u64, vp, u64, vp, vp]
        L.gtsc_stream_create.argtypes = [ctypes.POINTER(vp)]
        L.gtsc_stream_destroy.argtypes = [vp]
        L.gtsc_batch_create.argtypes = [ctypes.POINTER(Column), ctypes.c_uint32, i16p, i32p,
                                        ctypes.POINTER(vp), vp]
        L.gtsc_batch_set_inputs.argtypes = [vp, ctypes.POINTER(vp), vp]
        L.gtsc_batch_compress.argtypes = [vp, vp]
        L.gtsc_batch_output.argtypes = [vp, ctypes.POINTER(vp), u64p, vp]
        L.gtsc_batch_blob_sizes.argtypes = [vp, u64p, vp]
        L.gtsc_batch_decompress.argtypes = [vp, vp, u64, ctypes.POINTER(vp), vp]
        L.gtsc_batch_status.argtypes = [vp, vp]
        L.gtsc_batch_launches.argtypes = [vp, i32]
        L.gtsc_batch_set_schedule.argtypes = [vp, i32]
        L.gtsc_batch_create_tuned.argtypes = [ctypes.POINTER(Column), ctypes.c_uint32, i16p, i32p,
                                              ctypes.POINTER(Tuning), ctypes.POINTER(vp), vp]
        L.gtsc_batch_get_tuning.argtypes = [vp, ctypes.POINTER(Tuning)]
        L.gtsc_batch_autotune.argtypes = [vp, ctypes.POINTER(Tuning), vp]
        L.gtsc_batch_schedule.argtypes = [vp]
        L.gtsc_batch_destroy.argtypes = [vp]
        L.gtsc_batch_profile.argtypes = [vp, i32, i32p, ctypes.POINTER(ctypes.c_float), u64p, u64p, i32, i32p, vp]
        L.gtsc_pipeline_create.argtypes = [ctypes.POINTER(Column), u32, i16p, i32p, i32, ctypes.POINTER(vp)]
        L.gtsc_pipeline_groups.argtypes = [vp]
        L.gtsc_pipeline_group_columns.argtypes = [vp, i32, i32p, i32, i32p]
        L.gtsc_pipeline_compress_host.argtypes = [vp, ctypes.POINTER(vp), vp, u64, u64p]
        L.gtsc_pipeline_decompress.argtypes = [vp]
        L.gtsc_pipeline_roundtrip_host.argtypes = [vp, ctypes.POINTER(vp), vp, u64, u64p]
        L.gtsc_pipeline_column.argtypes = [vp, i32, ctypes.POINTER(vp), ctypes.POINTER(vp)]
        L.gtsc_pipeline_destroy.argtypes = [vp]
        f32p = ctypes.POINTER(ctypes.c_float)
        L.gtsc_planner_features.argtypes = [ctypes.POINTER(Column), u32, vp, vp]
        L.gtsc_planner_create.argtypes = [i16p, i32p, i32, u64, ctypes.POINTER(vp)]
        L.gtsc_planner_load.argtypes = [vp, u64, ctypes.POINTER(vp)]
        L.gtsc_planner_save.argtypes = [vp, vp, u64, u64p]
        L.gtsc_planner_destroy.argtypes = [vp]
        L.gtsc_planner_classes.argtypes = [vp]
        L.gtsc_planner_param_count.argtypes = [vp]
        L.gtsc_planner_param_count.restype = u64
        L.gtsc_planner_get_params.argtypes = [vp, f32p, f32p, f32p]
        L.gtsc_planner_set_params.argtypes = [vp, f32p, f32p, f32p]
        L.gtsc_planner_valid.argtypes = [vp, ctypes.POINTER(ctypes.c_uint8)]
        L.gtsc_planner_gradient.argtypes = [vp, vp, i32p, u32, f32p, f32p, vp]
        L.gtsc_planner_train.argtypes = [vp, vp, i32p, u32, i32, i32, ctypes.c_float, u64, f32p, vp]
        L.gtsc_planner_predict.argtypes = [vp, vp, i32p, u32, i32p, f32p, vp]
        L.gtsc_plan_learned.argtypes = [vp, ctypes.POINTER(Column), u32, ctypes.c_float, i16p, i32, i32p, i32p, vp]
        _lib = L
    return _lib


def check(status, what):
    if status != 0:
        msg = lib().gtsc_last_error().decode(errors="replace")
        raise GtscError(status, what, msg)


class DeviceBuffer:
    """Owned device allocation (freed with gtsc_free when collected)."""

    __slots__ = ("ptr", "nbytes", "_owned")

    def __init__(self, ptr, nbytes, owned=True):
        self.ptr = ptr or None
        self.nbytes = int(nbytes)
        self._owned = owned and bool(ptr)

    def __del__(self):
        if getattr(self, "_owned", False) and _lib is not None:
            _lib.gtsc_free(self.ptr, None)
            self._owned = False

    def __len__(self):
        return self.nbytes

    def __repr__(self):
        return f"DeviceBuffer(0x{self.ptr or 0:x}, {self.nbytes} B)"


def alloc(nbytes, stream=None):
    p = ctypes.c_void_p()
    check(lib().gtsc_malloc(ctypes.byref(p), nbytes, stream), "gtsc_malloc")
    return DeviceBuffer(p.value, nbytes)


def to_device(array, stream=None):
    a = np.ascontiguousarray(array)
    buf = alloc(a.nbytes, stream)
    if a.nbytes:
        check(lib().gtsc_memcpy(buf.ptr, a.ctypes.data, a.nbytes, 1, stream), "gtsc_memcpy h2d")
        check(lib().gtsc_stream_synchronize(stream), "sync")
    return buf


def to_host(buf, dtype=np.uint8, stream=None):
    out = np.empty(buf.nbytes, np.uint8)
    if buf.nbytes:
        check(lib().gtsc_memcpy(out.ctypes.data, buf.ptr, buf.nbytes, 2, stream), "gtsc_memcpy d2h")
    return out.view(dtype) if np.dtype(dtype).itemsize and buf.nbytes % np.dtype(dtype).itemsize == 0 else out


def dtype_size(dtype):
    return lib().gtsc_dtype_size(dtype)


def predict_sizes(encoding, dtype, data, stream=None):
    """GetMetadataSize / GetCompressedSize of one encoding for a device column -> (meta, data) bytes."""
    m, d = ctypes.c_uint64(), ctypes.c_uint64()
    check(lib().gtsc_predict_sizes(encoding, dtype, data.ptr, data.nbytes, ctypes.byref(m), ctypes.byref(d), stream),
          "predict_sizes")
    return m.value, d.value


def afl_pack(dtype, bit_length, data, n, omega=32, stream=None):
    """Pack n integer elements into the FL (omega 1, run_afl_compress_gpu<T,1>) or aligned (omega 32,
    run_afl_compress_gpu<T,32>) layout of compression/afl/afl_gpu.cu -> DeviceBuffer."""
    L = lib()
    es = dtype_size(dtype)
    if omega == 32:
        nb = L.gtsc_afl32_bytes(dtype, bit_length, n)
        out = alloc(max(nb, es), stream)
        check(L.gtsc_afl32_compress_gpu(dtype, bit_length, data.ptr, n, out.ptr, nb, stream), "afl32 compress")
    else:
        W = 8 * es
        nb = (n * bit_length + W - 1) // W * es
        out = alloc(max(nb, es), stream)
        check(L.gtsc_afl_compress_gpu(dtype, bit_length, data.ptr, n, out.ptr, nb, stream), "afl compress")
    out.nbytes = nb
    return out


def afl_unpack(dtype, bit_length, comp, n, omega=32, stream=None):
    """All n elements of a packed stream (either layout) -> DeviceBuffer of n elements."""
    L = lib()
    out = alloc(max(n * dtype_size(dtype), 1), stream)
    out.nbytes = n * dtype_size(dtype)
    if omega == 32:
        check(L.gtsc_afl32_decompress_gpu(dtype, bit_length, comp.ptr, comp.nbytes, out.ptr, n, stream),
              "afl32 decompress")
    else:
        check(L.gtsc_afl_decompress_gpu(dtype, bit_length, comp.ptr, comp.nbytes, out.ptr, n, stream),
              "afl decompress")
    return out


def afl_values(dtype, bit_length, comp, omega, index=None, n=None, stream=None):
    """Random-access decode (run_afl_decompress_value_gpu): element index[t] (or t < n) of a packed
    stream -> DeviceBuffer.  `index` is a device buffer of uint64 positions."""
    m = index.nbytes // 8 if index is not None else int(n)
    out = alloc(max(m * dtype_size(dtype), 1), stream)
    out.nbytes = m * dtype_size(dtype)
    check(lib().gtsc_afl_values_gpu(dtype, bit_length, omega, comp.ptr, comp.nbytes,
                                    index.ptr if index is not None else None, m, out.ptr, stream),
          "afl values")
    return out


def encode(encoding, dtype, data, stream=None):
    """Encoding::Encode -> [metadata, out1, (out2)] as DeviceBuffers."""
    outs = (Buffer * 3)()
    n_out = ctypes.c_uint32(0)
    check(lib().gtsc_encode(encoding, dtype, data.ptr, data.nbytes, outs, ctypes.byref(n_out), stream),
          f"encode {ENCODING_NAMES[encoding]}")
    return [DeviceBuffer(outs[i].ptr, outs[i].bytes) for i in range(n_out.value)]


def decode(encoding, dtype, parts, stream=None):
    """Encoding::Decode of [metadata, in1, (in2)] -> DeviceBuffer."""
    ins = (Buffer * 3)()
    for i, p in enumerate(parts):
        ins[i] = Buffer(p.ptr, p.nbytes)
    out = Buffer()
    check(lib().gtsc_decode(encoding, dtype, ins, len(parts), ctypes.byref(out), stream),
          f"decode {ENCODING_NAMES[encoding]}")
    return DeviceBuffer(out.ptr, out.bytes)


def stats(dtype, data, stream=None):
    """CudaArrayStatistics::GenerateStatistics of a device column -> DataStatistics."""
    s = DataStatistics()
    check(lib().gtsc_stats(dtype, data.ptr, data.nbytes, ctypes.byref(s), stream), "stats")
    return s


# ------------------------------------------------------------------------ compression trees
def _i16(a):
    a = np.ascontiguousarray(a, np.int16)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int16))


def tree_from_path(encodings, dtype):
    """PathGenerator::GenerateTree -> node list [(enc, dtype), ...] as an int16 array of pairs."""
    p, pp = _i16(encodings)
    out = np.zeros(2 * 256, np.int16)
    n = ctypes.c_int32(0)
    check(lib().gtsc_tree_from_path(pp, p.size, dtype,
                                    out.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)), 256,
                                    ctypes.byref(n)), "tree_from_path")
    return out[:2 * n.value].copy()


def tree_compress(nodes, data, stream=None):
    """CompressionTree::Compress -> serialized blob (DeviceBuffer)."""
    nd, ndp = _i16(nodes)
    out = Buffer()
    check(lib().gtsc_tree_compress(ndp, nd.size // 2, data.ptr, data.nbytes, ctypes.byref(out), stream),
          "tree_compress")
    return DeviceBuffer(out.ptr, out.bytes)


def tree_decompress(blob, stream=None):
    """CompressionTree::Decompress -> (DeviceBuffer, root data type)."""
    out = Buffer()
    dt = ctypes.c_int32(-1)
    check(lib().gtsc_tree_decompress(blob.ptr, blob.nbytes, ctypes.byref(out), ctypes.byref(dt), stream),
          "tree_decompress")
    return DeviceBuffer(out.ptr, out.bytes), dt.value


def tree_predict_size(nodes, data, stream=None):
    nd, ndp = _i16(nodes)
    sz = ctypes.c_uint64(0)
    check(lib().gtsc_tree_predict_size(ndp, nd.size // 2, data.ptr, data.nbytes, ctypes.byref(sz), stream),
          "tree_predict_size")
    return sz.value


def _plan(fn, what, dtype, data, stream):
    out = np.zeros(2 * 1024, np.int16)
    n = ctypes.c_int32(0)
    sz = ctypes.c_uint64(0)
    check(fn(dtype, data.ptr, data.nbytes, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)), 1024,
             ctypes.byref(n), ctypes.byref(sz), stream), what)
    return out[:2 * n.value].copy(), sz.value


def plan_exhaustive(dtype, sample, stream=None):
    """FullStatisticsUpdate + max-ratio pick on a device sample -> (nodes, candidate size)."""
    return _plan(lib().gtsc_plan_exhaustive, "plan_exhaustive", dtype, sample, stream)


def optimize_tree(dtype, data, stream=None):
    """CompressionOptimizer::OptimizeTree -> (nodes, predicted size)."""
    return _plan(lib().gtsc_optimize_tree, "optimize_tree", dtype, data, stream)


def sample_bytes(dtype, nbytes):
    return lib().gtsc_sample_bytes(dtype, nbytes)


def tree_names(nodes):
    return [ENCODING_NAMES[e] for e in np.asarray(nodes)[::2]]


# ------------------------------------------------------------------------ streams and batches
def selftest_lookback_timeout(stream=None):
    """Runs one decoupled look-back whose predecessor never publishes (gtsc_selftest_lookback_timeout):
    returns (the status the waiting tile recorded, seconds the bounded wait took)."""
    err = ctypes.c_int32(0)
    sec = ctypes.c_double(0.0)
    check(lib().gtsc_selftest_lookback_timeout(ctypes.byref(err), ctypes.byref(sec), stream),
          "selftest_lookback_timeout")
    return err.value, sec.value


class Stream:
    """A non-blocking CUDA stream owned by the library (batched steps are captured on it)."""

    def __init__(self):
        p = ctypes.c_void_p()
        check(lib().gtsc_stream_create(ctypes.byref(p)), "stream_create")
        self.handle = p.value

    def synchronize(self):
        check(lib().gtsc_stream_synchronize(self.handle), "sync")

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.gtsc_stream_destroy(self.handle)
            self.handle = None


# pass kinds of the batched engine (batch.hpp BOp) and the fixed kernels of a step
PASS_NAMES = dict(enumerate(
    ["minmax", "delta_enc", "scale_sub", "afl_pack", "hist", "topk", "split", "rle_heads", "rle_lengths",
     "f2i_stats", "f2i_enc", "f2i_raw", "gfc_compress", "gfc_scan", "gfc_compact", "none_copy", "afl_unpack",
     "delta_dec", "scale_add", "merge", "rle_scan", "rle_expand", "f2i_dec", "gfc_sizes", "gfc_dec", "vmeta",
     "merge_count"]))
PASS_NAMES.update({-1: "set_streams", -2: "zero", -3: "frame_sizes", -4: "frame_layout", -5: "frame_copy",
                   -6: "parse_frames", -7: "persistent"})


class Tuning(ctypes.Structure):
    """gtsc_batch_tuning: a batch's launch parameters (and the autotuner's report)."""
    _fields_ = [("minmax_tile", ctypes.c_uint32), ("minmax_values_per_thread", ctypes.c_uint32),
                ("hist_tile", ctypes.c_uint32), ("schedule_compress", ctypes.c_int32),
                ("schedule_decompress", ctypes.c_int32), ("ms_default_compress", ctypes.c_float),
                ("ms_default_decompress", ctypes.c_float), ("ms_tuned_compress", ctypes.c_float),
                ("ms_tuned_decompress", ctypes.c_float), ("candidates", ctypes.c_int32),
                ("seconds", ctypes.c_float)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        for k in ("schedule_compress", "schedule_decompress"):
            d[k] = "persistent" if d[k] == 1 else "levels"
        for k in d:
            if isinstance(d[k], float):
                d[k] = round(d[k], 4)
        return d


def tuning(minmax_tile=8192, minmax_values_per_thread=16, hist_tile=32768, persistent_compress=False,
           persistent_decompress=False):
    t = Tuning()
    t.minmax_tile, t.minmax_values_per_thread, t.hist_tile = minmax_tile, minmax_values_per_thread, hist_tile
    t.schedule_compress = 1 if persistent_compress else 0
    t.schedule_decompress = 1 if persistent_decompress else 0
    return t


class Batch:
    """Many columns with their trees, compressed / decompressed by the batched engine.

    columns: DeviceBuffers (or objects with .ptr and .nbytes); dtypes: data type codes;
    trees: node lists (int16 pairs) per column; tuning: launch parameters (None = the defaults)."""

    def __init__(self, columns, dtypes, trees, stream, tuning=None):
        self.stream = stream
        self.n = len(columns)
        cols = (Column * self.n)()
        for i, (c, dt) in enumerate(zip(columns, dtypes)):
            cols[i] = Column(c.ptr, c.nbytes, dt, 0)
        counts = np.array([len(t) // 2 for t in trees], np.int32)
        nodes = np.ascontiguousarray(np.concatenate([np.asarray(t, np.int16) for t in trees]))
        h = ctypes.c_void_p()
        check(lib().gtsc_batch_create_tuned(cols, self.n, nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)),
                                            counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                            ctypes.byref(tuning) if tuning is not None else None, ctypes.byref(h),
                                            stream.handle), "batch_create")
        self.handle = h.value
        self.sizes = [c.nbytes for c in columns]

    def set_inputs(self, columns):
        arr = (ctypes.c_void_p * self.n)(*[c.ptr for c in columns])
        check(lib().gtsc_batch_set_inputs(self.handle, arr, self.stream.handle), "batch_set_inputs")

    def compress(self):
        check(lib().gtsc_batch_compress(self.handle, self.stream.handle), "batch_compress")

    def output(self):
        """(device pointer, bytes) of the framed output of the last compress (synchronises)."""
        p = ctypes.c_void_p()
        b = ctypes.c_uint64(0)
        check(lib().gtsc_batch_output(self.handle, ctypes.byref(p), ctypes.byref(b), self.stream.handle),
              "batch_output")
        return p.value, b.value

    def blob_sizes(self):
        out = np.zeros(self.n, np.uint64)
        check(lib().gtsc_batch_blob_sizes(self.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                          self.stream.handle), "batch_blob_sizes")
        return out

    def decompress(self, framed_ptr, framed_bytes, outputs):
        arr = (ctypes.c_void_p * self.n)(*[o.ptr for o in outputs])
        check(lib().gtsc_batch_decompress(self.handle, framed_ptr, framed_bytes, arr, self.stream.handle),
              "batch_decompress")

    def status(self):
        check(lib().gtsc_batch_status(self.handle, self.stream.handle), "batch step")

    def launches(self, compress=True):
        return lib().gtsc_batch_launches(self.handle, 1 if compress else 0)

    def set_schedule(self, persistent):
        """Replay the steps as one persistent launch per step (True) or per level (False)."""
        check(lib().gtsc_batch_set_schedule(self.handle, 1 if persistent else 0), "batch_set_schedule")

    def schedule(self):
        return "persistent" if lib().gtsc_batch_schedule(self.handle) == 1 else "levels"

    def tuning(self):
        t = Tuning()
        check(lib().gtsc_batch_get_tuning(self.handle, ctypes.byref(t)), "batch_get_tuning")
        return t

    def autotune(self):
        """Chooses the schedule, min/max tile and values per thread and histogram tile by timing them
        on this batch; returns the report (a dict).  The framed output buffer may move."""
        t = Tuning()
        check(lib().gtsc_batch_autotune(self.handle, ctypes.byref(t), self.stream.handle), "batch_autotune")
        return t.as_dict()

    def profile(self, compress=True):
        """One step launch by launch: [(pass name, ms, bytes moved at least, blocks)]."""
        cap = 4096
        ops = np.zeros(cap, np.int32)
        ms = np.zeros(cap, np.float32)
        by = np.zeros(cap, np.uint64)
        bl = np.zeros(cap, np.uint64)
        n = ctypes.c_int32(0)
        check(lib().gtsc_batch_profile(self.handle, 1 if compress else 0,
                                       ops.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                       ms.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                       by.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                       bl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), cap, ctypes.byref(n),
                                       self.stream.handle), "batch_profile")
        return [(PASS_NAMES.get(int(ops[i]), str(int(ops[i]))), float(ms[i]), int(by[i]), int(bl[i]))
                for i in range(n.value)]

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.gtsc_batch_destroy(self.handle)
            self.handle = None


# ------------------------------------------------------------------------ column-chunk pipeline
class Pipeline:
    """Column chunks from host memory (pinned for overlap) to host framed output, column groups
    pipelined over their own batch engines and streams (gtsc_pipeline_*)."""

    def __init__(self, sizes, dtypes, trees, groups=8):
        self.n = len(sizes)
        cols = (Column * self.n)()
        for i, (b, dt) in enumerate(zip(sizes, dtypes)):
            cols[i] = Column(None, int(b), dt, 0)
        counts = np.array([len(t) // 2 for t in trees], np.int32)
        nodes = np.ascontiguousarray(np.concatenate([np.asarray(t, np.int16) for t in trees]))
        h = ctypes.c_void_p()
        check(lib().gtsc_pipeline_create(cols, self.n, nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)),
                                         _i32(counts), groups, ctypes.byref(h)), "pipeline_create")
        self.handle = h.value
        self.groups = lib().gtsc_pipeline_groups(self.handle)

    def compress_host(self, host_ptrs, framed_ptr, cap):
        """host_ptrs: addresses of the host columns; framed_ptr: host buffer of cap bytes.
        Returns the bytes of every group's framed output (written back to back)."""
        arr = (ctypes.c_void_p * self.n)(*host_ptrs)
        sizes = np.zeros(self.groups, np.uint64)
        check(lib().gtsc_pipeline_compress_host(self.handle, arr, framed_ptr, cap,
                                                sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))),
              "pipeline_compress_host")
        return sizes

    def roundtrip_host(self, host_ptrs, framed_ptr, cap):
        """compress_host plus each group's device decode right after its read-back."""
        arr = (ctypes.c_void_p * self.n)(*host_ptrs)
        sizes = np.zeros(self.groups, np.uint64)
        check(lib().gtsc_pipeline_roundtrip_host(self.handle, arr, framed_ptr, cap,
                                                 sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))),
              "pipeline_roundtrip_host")
        return sizes

    def decompress(self):
        check(lib().gtsc_pipeline_decompress(self.handle), "pipeline_decompress")

    def group_columns(self, g):
        out = np.zeros(self.n, np.int32)
        k = ctypes.c_int32(0)
        check(lib().gtsc_pipeline_group_columns(self.handle, g, _i32(out), self.n, ctypes.byref(k)),
              "pipeline_group_columns")
        return out[:k.value].tolist()

    def column(self, c):
        """(device input, device output) addresses of column c."""
        a, b = ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().gtsc_pipeline_column(self.handle, c, ctypes.byref(a), ctypes.byref(b)), "pipeline_column")
        return a.value, b.value

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.gtsc_pipeline_destroy(self.handle)
            self.handle = None


# ------------------------------------------------------------------------ learned planner
N_FEATURES = 32
MODEL_PATH = os.path.join(HERE, "planner_model.bin")


def _columns(cols, dtypes):
    arr = (Column * len(cols))()
    for i, (c, dt) in enumerate(zip(cols, dtypes)):
        arr[i] = Column(c.ptr, c.nbytes, dt, 0)
    return arr


def _f32(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _i32(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def planner_features(cols, dtypes, stream=None):
    """Planner features of the columns' samples -> DeviceBuffer of len(cols) x 32 float32."""
    out = alloc(4 * N_FEATURES * max(len(cols), 1), stream)
    check(lib().gtsc_planner_features(_columns(cols, dtypes), len(cols), out.ptr, stream), "planner_features")
    return out


# --------------------------------------------------------------------- online tree maintenance
def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class EdgeStats:
    """CompressionStatistics (tree/compression_statistics.cpp): edge scores of compression trees.
    Host-only; no GPU needed."""

    def __init__(self, tree_height=5, _handle=None, _owner=None):
        self._owner = _owner
        if _handle is not None:
            self.h = _handle
            self._owned = False
        else:
            h = ctypes.c_void_p()
            check(lib().gtsc_edge_stats_create(tree_height, ctypes.byref(h)), "edge_stats_create")
            self.h, self._owned = h.value, True

    def __del__(self):
        if getattr(self, "_owned", False) and _lib is not None:
            _lib.gtsc_edge_stats_destroy(self.h)
            self._owned = False

    def set(self, edge, frm, to, value):
        check(lib().gtsc_edge_stats_set(self.h, edge, frm, to, value), "edge_stats_set")

    def update(self, edge, frm, to, ratio):
        check(lib().gtsc_edge_stats_update(self.h, edge, frm, to, ratio), "edge_stats_update")

    def get(self, edge, frm, to):
        v = ctypes.c_double()
        check(lib().gtsc_edge_stats_get(self.h, edge, frm, to, ctypes.byref(v)), "edge_stats_get")
        return v.value

    def best(self, edge, frm, to, same_beginning=False):
        """GetBest -> ((parent, child), score)"""
        a, b, v = ctypes.c_int16(), ctypes.c_int16(), ctypes.c_double()
        check(lib().gtsc_edge_stats_best(self.h, edge, frm, to, int(same_beginning), ctypes.byref(a),
                                         ctypes.byref(b), ctypes.byref(v)), "edge_stats_best")
        return (a.value, b.value), v.value

    def entries(self, edge):
        """{(parent, child): score} of one edge"""
        n = ctypes.c_int32()
        pairs = np.zeros(2 * 256, np.int16)
        vals = np.zeros(256, np.float64)
        check(lib().gtsc_edge_stats_entries(self.h, edge, _ptr(pairs), _ptr(vals), 256, ctypes.byref(n)),
              "edge_stats_entries")
        return {(int(pairs[2 * k]), int(pairs[2 * k + 1])): float(vals[k]) for k in range(n.value)}


def tree_edges(nodes):
    """CompressionTree::GetEdges -> [(edge number, parent node index, child node index)] (pre-order
    node indices)."""
    nd, _ = _i16(nodes)
    no, fr, to = (np.zeros(128, np.int32) for _ in range(3))
    n = ctypes.c_int32()
    check(lib().gtsc_tree_edges(_ptr(nd), nd.size // 2, _ptr(no), _ptr(fr), _ptr(to), 128, ctypes.byref(n)),
          "tree_edges")
    return [(int(no[k]), int(fr[k]), int(to[k])) for k in range(n.value)]


def tree_update_statistics(nodes, ratios, stats):
    nd, _ = _i16(nodes)
    r = np.ascontiguousarray(ratios, np.float64)
    check(lib().gtsc_tree_update_statistics(_ptr(nd), _ptr(r), nd.size // 2, stats.h), "tree_update_statistics")


def _read_tree(fn, h, what):
    nodes = np.zeros(2 * 1024, np.int16)
    ratios = np.zeros(1024, np.float64)
    n = ctypes.c_int32()
    check(fn(h, _ptr(nodes), _ptr(ratios), 1024, ctypes.byref(n)), what)
    return nodes[:2 * n.value].copy(), ratios[:n.value].copy()


class OptimalTree:
    """OptimalTree (optimizer/optimal_tree.cpp) over live statistics; host-only."""

    def __init__(self, nodes, ratios, stats):
        nd, _ = _i16(nodes)
        r = np.ascontiguousarray(ratios, np.float64)
        h = ctypes.c_void_p()
        check(lib().gtsc_optimal_tree_create(_ptr(nd), _ptr(r), nd.size // 2, stats.h, ctypes.byref(h)),
              "optimal_tree_create")
        self.h, self.stats = h.value, stats

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.gtsc_optimal_tree_destroy(self.h)
            self.h = None

    def set_ratio(self, node, ratio):
        check(lib().gtsc_optimal_tree_set_ratio(self.h, node, ratio), "optimal_tree_set_ratio")

    def try_correct(self):
        c = ctypes.c_int32()
        check(lib().gtsc_optimal_tree_try_correct(self.h, ctypes.byref(c)), "optimal_tree_try_correct")
        return bool(c.value)

    def tree(self):
        return _read_tree(lib().gtsc_optimal_tree_get, self.h, "optimal_tree_get")


class Optimizer:
    """CompressionOptimizer::CompressData for one column: compress() takes one part (a device
    buffer) and returns (blob DeviceBuffer, full_update, corrected)."""

    def __init__(self, dtype):
        h = ctypes.c_void_p()
        check(lib().gtsc_optimizer_create(dtype, ctypes.byref(h)), "optimizer_create")
        self.h, self.dtype = h.value, dtype

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.gtsc_optimizer_destroy(self.h)
            self.h = None

    def compress(self, data, stream=None):
        out = Buffer()
        full, corr = ctypes.c_int32(), ctypes.c_int32()
        check(lib().gtsc_optimizer_compress(self.h, data.ptr, data.nbytes, ctypes.byref(out), ctypes.byref(full),
                                            ctypes.byref(corr), stream), "optimizer_compress")
        return DeviceBuffer(out.ptr, out.bytes), bool(full.value), bool(corr.value)

    def tree(self):
        return _read_tree(lib().gtsc_optimizer_tree, self.h, "optimizer_tree")

    def statistics(self):
        h = ctypes.c_void_p()
        check(lib().gtsc_optimizer_statistics(self.h, ctypes.byref(h)), "optimizer_statistics")
        return EdgeStats(_handle=h.value, _owner=self)


class Planner:
    """The learned tree planner (an MLP over column features, exhaustive-planner fallback)."""

    def __init__(self, classes=None, seed=0, model=None):
        h = ctypes.c_void_p()
        if model is not None:
            b = np.frombuffer(bytes(model), np.uint8)
            check(lib().gtsc_planner_load(b.ctypes.data, b.size, ctypes.byref(h)), "planner_load")
        else:
            lens = np.array([len(c) for c in classes], np.int32)
            encs = np.ascontiguousarray(np.concatenate([np.asarray(c, np.int16) for c in classes]))
            check(lib().gtsc_planner_create(encs.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)), _i32(lens),
                                            len(classes), seed, ctypes.byref(h)), "planner_create")
        self.handle = h.value
        self.K = lib().gtsc_planner_classes(self.handle)

    @classmethod
    def load(cls, path=MODEL_PATH):
        with open(path, "rb") as f:
            return cls(model=f.read())

    def save(self, path=None):
        n = ctypes.c_uint64(0)
        check(lib().gtsc_planner_save(self.handle, None, 0, ctypes.byref(n)), "planner_save")
        buf = np.zeros(n.value, np.uint8)
        check(lib().gtsc_planner_save(self.handle, buf.ctypes.data, buf.size, ctypes.byref(n)), "planner_save")
        if path:
            with open(path, "wb") as f:
                f.write(buf.tobytes())
        return buf.tobytes()

    @property
    def n_params(self):
        return lib().gtsc_planner_param_count(self.handle)

    def get_params(self):
        p = np.zeros(self.n_params, np.float32)
        mu = np.zeros(N_FEATURES, np.float32)
        sd = np.zeros(N_FEATURES, np.float32)
        check(lib().gtsc_planner_get_params(self.handle, _f32(p), _f32(mu), _f32(sd)), "planner_get_params")
        return p, mu, sd

    def set_params(self, params=None, mu=None, sd=None):
        args = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (params, mu, sd)]
        check(lib().gtsc_planner_set_params(self.handle, *[None if a is None else _f32(a) for a in args]),
              "planner_set_params")

    def valid(self):
        v = np.zeros(self.K * 6, np.uint8)
        check(lib().gtsc_planner_valid(self.handle, v.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))), "valid")
        return v.reshape(self.K, 6)

    def gradient(self, d_features, labels, stream=None):
        labels = np.ascontiguousarray(labels, np.int32)
        g = np.zeros(self.n_params, np.float32)
        loss = ctypes.c_float(0)
        check(lib().gtsc_planner_gradient(self.handle, d_features.ptr, _i32(labels), labels.size, _f32(g),
                                          ctypes.byref(loss), stream), "planner_gradient")
        return loss.value, g

    def train(self, d_features, labels, epochs=100, batch=256, lr=2e-3, seed=1, stream=None):
        labels = np.ascontiguousarray(labels, np.int32)
        loss = ctypes.c_float(0)
        check(lib().gtsc_planner_train(self.handle, d_features.ptr, _i32(labels), labels.size, epochs, batch, lr,
                                       seed, ctypes.byref(loss), stream), "planner_train")
        return loss.value

    def predict(self, d_features, dtypes, stream=None):
        dtypes = np.ascontiguousarray(dtypes, np.int32)
        cls = np.zeros(dtypes.size, np.int32)
        conf = np.zeros(dtypes.size, np.float32)
        check(lib().gtsc_planner_predict(self.handle, d_features.ptr, _i32(dtypes), dtypes.size, _i32(cls),
                                         _f32(conf), stream), "planner_predict")
        return cls, conf

    def plan(self, cols, dtypes, min_confidence=0.5, stream=None):
        """Trees for the columns: [(nodes, fallback_used)]."""
        cap = 64 * max(len(cols), 1)
        nodes = np.zeros(2 * cap, np.int16)
        counts = np.zeros(len(cols), np.int32)
        fb = np.zeros(len(cols), np.int32)
        check(lib().gtsc_plan_learned(self.handle, _columns(cols, dtypes), len(cols), min_confidence,
                                      nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_int16)), cap, _i32(counts),
                                      _i32(fb), stream), "plan_learned")
        out, pos = [], 0
        for c, f in zip(counts, fb):
            out.append((nodes[2 * pos: 2 * (pos + c)].copy(), bool(f)))
            pos += c
        return out

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.gtsc_planner_destroy(self.handle)
            self.handle = None


def split_framed(framed):
    """Split a framed host buffer (uint64 column count, uint64 blob bytes per column, blobs)."""
    framed = np.ascontiguousarray(framed, np.uint8)
    nc = int(framed[:8].view(np.uint64)[0])
    lens = framed[8:8 + 8 * nc].view(np.uint64).astype(np.int64)
    pos = 8 + 8 * nc
    blobs = []
    for n in lens:
        blobs.append(framed[pos:pos + n])
        pos += n
    return blobs
