"""Times the reference's own compression tree (CompressionTree::Compress, compiled from its sources
into oracle/_ref/libref_enc.so by `make -C oracle refenc`) beside the library on the same B200.

Workloads (columns resident on the device on both sides, outputs left on the device):
  - the benchmark configurations' trees on int32 columns: 2a delta->AFL and delta->scale->AFL on the
    walk, 2b RLE->(AFL, AFL) on runs, 2c dict->(AFL, AFL) on Zipf(1.1) ids, 2d const->AFL, 2e
    patch->(AFL, AFL) on the outliers, at 67,107,840 values: the largest column the reference's
    launch policy covers (65535 blocks of 1024 threads, core/execution_policy.hpp:24-33; its kernels
    index with blockIdx.x only, so at 2^26 values it leaves the last 1024 unprocessed);
  - the mixed 512-column workload of bench.py (the learned planner's trees), every column through
    the reference's tree one after another, as its ParallelTsCompressor does per column.
Config 3 (GFC) is not timed: the reference's GFC kernels rely on implicit warp synchrony.

The library side is gtsc_tree_compress (one column per call) and the batched engine (all columns,
one CUDA graph).  Before timing, each configuration's blob is byte-compared between the two.  The
reference's API is synchronous (it allocates, copies and synchronises inside), so both sides are
timed by the host clock around whole calls, after warm-up, median of the repetitions; GB/s counts
the uncompressed input bytes.

--reference-only: the mixed workload through the reference alone (no library call), with the trees
the oracle's exhaustive planner picks -- the extra line of `bench.py --impl reference`; prints one
JSON line.

TEST INFRASTRUCTURE: a measurement script, not part of the library.  Usage:
    python oracle/time_ref_tree.py [--out FILE] [--reps 5] [--mixed-reps 1] [--reference-only]
"""
import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

import oracle as OR  # noqa: E402
import gputimeseriescompressionoptimizer_b200 as G  # noqa: E402
from gputimeseriescompressionoptimizer_b200 import workloads as W  # noqa: E402

N_REF_MAX = 65535 * 1024
CONFIGS = [
    ("2a delta-afl", "walk", [OR.DELTA, OR.AFL, OR.NONE]),
    ("2a delta-scale-afl", "walk", [OR.DELTA, OR.SCALE, OR.AFL, OR.NONE]),
    ("2b rle-afl-afl", "runs", [OR.RLE, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("2c dict-afl-afl", "zipf", [OR.DICT, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
    ("2d const-afl", "const", [OR.CONST, OR.AFL, OR.NONE]),
    ("2e patch-afl-afl", "outliers", [OR.PATCH, OR.AFL, OR.NONE, OR.AFL, OR.NONE]),
]


def _lib():
    L = OR.ref_enc()
    if L is None:
        sys.exit("oracle/_ref/libref_enc.so is missing: run make -C oracle refenc first")
    L.ref_dev_upload.restype = ctypes.c_void_p
    L.ref_dev_upload.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
    L.ref_dev_free.argtypes = [ctypes.c_void_p]
    L.ref_dev_tree_compress.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_uint64)]
    return L


def _median_time(fn, reps, warm=1):
    for _ in range(warm):
        fn()
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts))


def _ref_call(L, h, nodes):
    ob = ctypes.c_uint64(0)
    rc = L.ref_dev_tree_compress(h, nodes.ctypes.data_as(ctypes.c_void_p), nodes.size // 2, ctypes.byref(ob))
    if rc != 0:
        raise OR.OracleError(f"reference tree compress: {L.ref_enc_error().decode()}")
    return ob.value


def reference_only(L, reps):
    """The bench workload's columns through the reference's own tree compress, one after another;
    trees from the oracle's exhaustive planner; columns whose tree holds GFC left out."""
    import bench
    t0 = time.perf_counter()
    specs = bench.workload_specs()
    cols = bench.gen_columns(specs)
    trees = bench.cpu_trees(cols, specs)
    keep = [i for i, t in enumerate(trees) if OR.GFC not in [int(v) for v in np.asarray(t)[0::2]]]
    handles = [L.ref_dev_upload(OR._ptr(OR.as_bytes(cols[i])), cols[i].nbytes) for i in keep]
    if any(h is None for h in handles):
        raise OR.OracleError(f"reference upload: {L.ref_enc_error().decode()}")
    nodes = [np.asarray(trees[i], np.int16) for i in keep]
    in_bytes = sum(cols[i].nbytes for i in keep)

    def all_columns():
        for h, nd in zip(handles, nodes):
            _ref_call(L, h, nd)

    t = _median_time(all_columns, reps, warm=1)
    for h in handles:
        L.ref_dev_free(h)
    print(json.dumps({"value": round(in_bytes / 1e9 / t, 4), "unit": "GB/s", "ms": round(t * 1e3, 1),
                      "columns": len(keep), "of_columns": len(cols), "input_bytes": int(in_bytes),
                      "seconds": round(time.perf_counter() - t0, 1)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--mixed-reps", type=int, default=1)
    ap.add_argument("--reference-only", action="store_true")
    args = ap.parse_args()
    L = _lib()
    if args.reference_only:
        reference_only(L, args.mixed_reps)
        return
    st = G.Stream()
    rows = []
    for k, (name, kind, path) in enumerate(CONFIGS):
        x = W.column(kind, OR.INT, N_REF_MAX, 0xB200 + 2 + k)
        nodes = OR.tree_from_path(path, OR.INT).astype(np.int16)
        h = L.ref_dev_upload(OR._ptr(OR.as_bytes(x)), x.nbytes)
        dev = G.to_device(x)
        # parity first: the reference's blob (host copy) against the library's
        ref_blob = OR.ref_tree_compress(nodes, x)
        ours = G.to_host(G.tree_compress(nodes, dev, st.handle), stream=st.handle)
        same = bool(ours.size == ref_blob.size and np.array_equal(ours, ref_blob))
        t_ref = _median_time(lambda: _ref_call(L, h, nodes), args.reps)

        def ours_call():
            G.tree_compress(nodes, dev, st.handle)
            st.synchronize()

        t_col = _median_time(ours_call, args.reps)
        b = G.Batch([dev], [OR.INT], [nodes], st)

        def batch_call():
            b.compress()
            st.synchronize()

        t_bat = _median_time(batch_call, args.reps)
        L.ref_dev_free(h)
        del b
        gb = x.nbytes / 1e9
        rows.append({"config": name, "values": int(x.size), "input_bytes": int(x.nbytes), "identical": same,
                     "reference_ms": round(t_ref * 1e3, 3), "gtsc_tree_ms": round(t_col * 1e3, 3),
                     "gtsc_batch_ms": round(t_bat * 1e3, 3), "reference_GBps": round(gb / t_ref, 2),
                     "gtsc_tree_GBps": round(gb / t_col, 2), "gtsc_batch_GBps": round(gb / t_bat, 2),
                     "speedup_tree": round(t_ref / t_col, 2), "speedup_batch": round(t_ref / t_bat, 2)})
        print(json.dumps(rows[-1]), flush=True)
    # the mixed workload through the reference's tree, column after column
    import bench
    specs = bench.workload_specs()
    cols = bench.gen_columns(specs)
    dts = [dt for _, dt, _, _ in specs]
    devs = [G.to_device(c) for c in cols]
    trees = [t for t, _ in G.Planner.load().plan(devs, dts, bench.MIN_CONFIDENCE, st.handle)]
    # the reference cannot run GFC: those columns (and any tree holding a GFC node) are left out on
    # both sides
    keep = [i for i, t in enumerate(trees) if OR.GFC not in [int(v) for v in np.asarray(t)[0::2]]]
    handles = [L.ref_dev_upload(OR._ptr(OR.as_bytes(cols[i])), cols[i].nbytes) for i in keep]
    nodes_k = [np.asarray(trees[i], np.int16) for i in keep]
    in_bytes = sum(cols[i].nbytes for i in keep)

    def ref_all():
        for h, nd in zip(handles, nodes_k):
            _ref_call(L, h, nd)

    t_ref = _median_time(ref_all, args.mixed_reps, warm=1)
    b = G.Batch([devs[i] for i in keep], [dts[i] for i in keep], [trees[i] for i in keep], st)

    def batch_all():
        b.compress()
        st.synchronize()

    t_bat = _median_time(batch_all, max(args.reps, 3))
    for h in handles:
        L.ref_dev_free(h)
    mixed = {"config": "mixed workload without GFC columns", "columns": len(keep), "input_bytes": int(in_bytes),
             "reference_ms": round(t_ref * 1e3, 1), "gtsc_batch_ms": round(t_bat * 1e3, 3),
             "reference_GBps": round(in_bytes / 1e9 / t_ref, 2), "gtsc_batch_GBps": round(in_bytes / 1e9 / t_bat, 2),
             "speedup_batch": round(t_ref / t_bat, 1)}
    print(json.dumps(mixed), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump({"configs": rows, "mixed": mixed}, f, indent=1)


if __name__ == "__main__":
    main()
