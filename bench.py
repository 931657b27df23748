#!/usr/bin/env python
"""Benchmark of the column-compression hot path on B200: the batched mixed workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 512 synthetic columns (lengths log-uniform in [4096, 2^24], int32 : float32 : float64 =
2 : 1 : 1, generators walk / runs / zipf / const / outliers / price chosen by seed), each with the
compression tree the planner picks on its sample.  One step = compress all 512 columns into one
framed buffer and decompress it again, with the columns resident in HBM; `value` is uncompressed
GB/s.  Beside it: the plain path (one column at a time through gtsc_tree_compress /
gtsc_tree_decompress, host-synchronising as the reference's per-column calls do), the planners'
cost, the dominant kernel against the HBM roofline, an end-to-end step from pinned host memory,
the CPU oracle on the same workload, and each benchmark configuration (AFL alone, the int32
chains, GFC) measured alone.

N > 1 runs N independent replicas (one process per GPU, launched by torchrun): the columns are
independent and the path has no exchange step, so `value` is the work of all ranks over the
slowest rank's time.
"""
import argparse
import concurrent.futures as cf
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
N_COLUMNS = int(os.environ.get("GTSC_BENCH_COLUMNS", "512"))
MAX_LEN = 1 << int(os.environ.get("GTSC_BENCH_MAX_LOG2", "24"))
MIN_CONFIDENCE = 0.5         # learned planner: below this softmax probability the exhaustive search decides
TICK_CHUNKS = 4              # streaming tick table: 40 columns x 2^20 rows per chunk
E2E_GROUPS = 16              # end to end: column groups pipelined over their own streams
METRIC = "batched mixed-workload compress+decompress throughput (uncompressed GB/s)"
WORKLOAD = (f"mixed {N_COLUMNS} columns, lengths log-uniform [4096, {MAX_LEN}], int32:float32:float64 = 2:1:1, "
            "generators walk/runs/zipf/const/outliers/price, seed 0xB204")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    return p.parse_args()


def peak_hbm():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.out.close()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm = [float(r[1]) for r in rows if len(r) > 2 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 2 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip() == "Active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload_specs():
    from gputimeseriescompressionoptimizer_b200 import workloads as W
    return W.mixed_columns(N_COLUMNS, max_len=MAX_LEN)


def gen_columns(specs, max_len=None, threads=None):
    """The columns of `specs` as numpy arrays (each cut to max_len values when given)."""
    from gputimeseriescompressionoptimizer_b200 import workloads as W

    def one(s):
        kind, dt, n, seed = s
        return W.column(kind, dt, n if max_len is None else min(n, max_len), seed)

    with cf.ThreadPoolExecutor(threads or os.cpu_count() or 1) as ex:
        return list(ex.map(one, specs))


# ------------------------------------------------------------------------------- CPU legs
def cpu_model():
    """The host CPU's model name and the number of hardware threads."""
    name = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    name = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return name, os.cpu_count() or 1


def cpu_roundtrip(cols, trees, threads):
    """The oracle's CompressionTree::Compress + Decompress of every column: one task per column,
    largest columns first, `threads` host threads (ctypes releases the GIL).  A column's blob depends
    on the whole column (its min / max, histogram and run boundaries), so a column is one task.
    Returns (seconds, input bytes, blob bytes)."""
    import oracle

    order = sorted(range(len(cols)), key=lambda i: -cols[i].nbytes)

    def work(i):
        blob = oracle.tree_compress(trees[i], cols[i])
        out, _ = oracle.tree_decompress(blob, cols[i].nbytes)
        return blob.size, out.size, cols[i].nbytes

    t = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        res = list(ex.map(work, order))
    dt = time.perf_counter() - t
    assert all(o == c for _, o, c in res)
    return dt, sum(c.nbytes for c in cols), sum(b for b, _, _ in res)


DRAM_PROFILE = os.path.join(ROOT, "profiles", "batch_step_mixed512_dram.json")


def dram_traffic(prof, phase, index):
    """DRAM bytes (read + written) of launch `index` of a step phase, from the committed ncu
    capture of this workload's step (profiles/batch_step_mixed512_dram.json: per phase, the pass of
    every launch and its dram__bytes_read.sum + dram__bytes_write.sum).  Used only when the capture's
    launch sequence is the one this run profiled; otherwise (None, reason)."""
    try:
        with open(DRAM_PROFILE) as f:
            cap = json.load(f)
    except (OSError, ValueError):
        return None, "no ncu capture of this step"
    seq = [x[0] for x in prof[phase]]
    got = cap.get(phase, [])
    if [g[0] for g in got] != seq:
        return None, "the ncu capture's launch sequence differs from this build's"
    return int(got[index][1]), f"ncu dram__bytes_read.sum + dram__bytes_write.sum, {phase} launch {index} ({DRAM_PROFILE[len(ROOT) + 1:]})"


def oracle_check(cols, trees, blobs, threads=None):
    """Parity at full size: every batched blob byte-compared with the oracle's
    CompressionTree::Compress of the same column (largest columns first, all host threads).
    Returns the number of bytes checked."""
    import oracle

    order = sorted(range(len(cols)), key=lambda i: -cols[i].nbytes)

    def work(i):
        ob = oracle.tree_compress(trees[i], cols[i])
        assert ob.size == blobs[i].size and np.array_equal(ob, blobs[i]), \
            f"column {i}: batched blob differs from the oracle's"
        return cols[i].nbytes

    with cf.ThreadPoolExecutor(threads or os.cpu_count() or 1) as ex:
        return sum(ex.map(work, order))


def cpu_trees(cols, specs):
    """The oracle's exhaustive planner on each column's sample."""
    import oracle
    trees = []
    for x, (_, dt, _, _) in zip(cols, specs):
        sb = oracle.sample_bytes(dt, x.nbytes)
        nodes, _ = oracle.plan_exhaustive(dt, x.view(np.uint8)[:sb].view(x.dtype))
        trees.append(nodes)
    return trees


def reference_gpu():
    """The reference's own CompressionTree::Compress (its sources compiled for sm_100a into
    oracle/_ref/libref_enc.so) over the same workload on this GPU, compress only, the columns whose
    trees hold no GFC node (its GFC kernels rely on implicit warp synchrony), timed by
    oracle/time_ref_tree.py in a child process: the reference exits its process on a CUDA error."""
    import oracle
    if not os.path.exists(oracle.REF_ENC_PATH):
        return {"unavailable": "oracle/_ref/libref_enc.so not built (make -C oracle refenc where the reference is)"}
    script = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle", "time_ref_tree.py")
    try:
        p = subprocess.run([sys.executable, script, "--reference-only"], capture_output=True, text=True,
                           timeout=900)
    except subprocess.TimeoutExpired:
        return {"unavailable": "the reference's tree compress did not finish in 900 s"}
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    if p.returncode != 0 or not lines:
        tail = " ".join((p.stderr or "").strip().splitlines()[-2:])[-200:]
        return {"unavailable": f"the reference's run failed (status {p.returncode}): {tail}"}
    r = json.loads(lines[-1])
    r["what"] = ("the reference's own CompressionTree::Compress (compiled from its sources for sm_100a), "
                 f"compress only, {r['columns']} of {r['of_columns']} columns (those without GFC), the exhaustive "
                 "planner's trees, column after column, host clock around the synchronous calls")
    return r


def run_reference(args, world, rank):
    """A CPU implementation of the path on the same workload.  The reference has none (its
    encoders are CUDA kernels and Thrust calls), so this is the oracle restatement built -O3
    -march=native on this host, with every host thread, over the full 512-column workload per step,
    with the trees the exhaustive planner picks.  The reference's own GPU tree compress on the same
    workload is reported beside it (reference_gpu)."""
    if rank != 0:
        return
    import oracle

    build = oracle.select_native()
    model, threads = cpu_model()
    specs = workload_specs()
    cols = gen_columns(specs)
    trees = cpu_trees(cols, specs)
    for _ in range(max(args.warmup, 1)):
        cpu_roundtrip(cols, trees, threads)
    times = []
    for _ in range(args.steps):
        t, in_bytes, blob_bytes = cpu_roundtrip(cols, trees, threads)
        times.append(t)
    t = sum(times) / len(times)
    gbs = in_bytes / t / 1e9
    sample = (f"the full workload each step: all {len(cols)} columns ({in_bytes} B), trees from the exhaustive "
              f"planner on each column's sample; {build}; {threads} threads on {model}")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 4), "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32/float32/float64 (integer arithmetic on bits)",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "inputs": "host memory",
                   "step": "CompressionTree::Compress + Decompress of every column (CPU restatement)",
                   "compression_ratio": round(in_bytes / blob_bytes, 4)},
        "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": threads, "kind": "port", "sample": sample,
                         "cpu_model": model},
        "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": reference_gpu(),
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------- GPU leg
class DevView:
    """(ptr, nbytes) of a torch tensor, the shape the package's calls take."""

    def __init__(self, t):
        self.t = t
        self.ptr = t.data_ptr()
        self.nbytes = t.numel() * t.element_size()


def tick_table(g, torch, planner, st, stream, sp):
    """The streaming tick table (40 columns, 2^20-row chunks arriving one after another): per chunk
    the learned planner against the exhaustive one (time, compressed bytes, fallbacks), and the
    batched compress + decompress of the chunk with the learned trees (the engine is rebuilt only
    when a column's tree changes)."""
    from gputimeseriescompressionoptimizer_b200 import workloads as W
    batch, prev, res = None, None, []
    for ch in range(TICK_CHUNKS):
        chunk = W.tick_chunk(40, 1 << 20, ch)
        dts = [dt for _, dt, _ in chunk]
        dev = [torch.from_numpy(x.view(np.uint8)).to("cuda") for _, _, x in chunk]
        dv = [DevView(d) for d in dev]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        planned = planner.plan(dv, dts, MIN_CONFIDENCE, sp)
        torch.cuda.synchronize()
        t_ln = time.perf_counter() - t0
        t0 = time.perf_counter()
        ex = [g.plan_exhaustive(dt, g.DeviceBuffer(d.ptr, g.sample_bytes(dt, d.nbytes), owned=False), sp)[0]
              for d, dt in zip(dv, dts)]
        torch.cuda.synchronize()
        t_ex = time.perf_counter() - t0
        trees = [t for t, _ in planned]
        key = [tuple(t) for t in trees]
        if batch is None or key != prev:
            batch = g.Batch(dv, dts, trees, st)
            prev = key
        else:
            batch.set_inputs(dv)
        outs = [torch.empty_like(d) for d in dev]
        ov = [DevView(o) for o in outs]
        batch.compress()
        p, n = batch.output()
        batch.decompress(p, n, ov)
        batch.status()
        assert all(torch.equal(a, b) for a, b in zip(outs, dev)), "tick chunk round trip differs"
        sizes_ln = [b.size for b in g.split_framed(g.to_host(g.DeviceBuffer(p, n, owned=False)))]
        sizes_ex = [g.tree_compress(t, d, sp).nbytes for t, d in zip(ex, dv)]
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(3):
            batch.compress()
            batch.decompress(p, n, ov)
        ev1.record(stream)
        torch.cuda.synchronize()
        t_step = ev0.elapsed_time(ev1) / 3e3
        raw = sum(d.nbytes for d in dv)
        res.append({"chunk": ch, "plan_learned_ms": round(1e3 * t_ln, 2), "plan_exhaustive_ms": round(1e3 * t_ex, 1),
                    "fallbacks": int(sum(f for _, f in planned)),
                    "ratio_learned": round(raw / sum(sizes_ln), 4), "ratio_exhaustive": round(raw / sum(sizes_ex), 4),
                    "GBps": round(raw / t_step / 1e9, 2)})
    gaps = [1 - r["ratio_learned"] / r["ratio_exhaustive"] for r in res]
    return {"workload": "tick table: 40 columns (ts, price, volume, symbol, flags) x 2^20 rows per chunk",
            "chunks": res, "ratio_gap": round(float(np.mean(gaps)), 4),
            "fallback_rate": round(sum(r["fallbacks"] for r in res) / (40.0 * len(res)), 4),
            "planning_speedup": round(sum(r["plan_exhaustive_ms"] for r in res) /
                                      max(sum(r["plan_learned_ms"] for r in res), 1e-9), 1)}


# the benchmark configurations measured one by one beside the mixed workload: (name, generator,
# data type, values, compression tree as a pre-order encoding list)
CONFIG_COLUMNS = [
    ("1 afl", "uniform11", 2, 1 << 20, [1, 7]),
    ("2a delta-afl", "walk", 2, 1 << 26, [0, 1, 7]),
    ("2a delta-scale-afl", "walk", 2, 1 << 26, [0, 2, 1, 7]),
    ("2b rle-afl-afl", "runs", 2, 1 << 26, [3, 1, 7, 1, 7]),
    ("2c dict-afl-afl", "zipf", 2, 1 << 26, [4, 1, 7, 1, 7]),
    ("2d const-afl", "const", 2, 1 << 26, [9, 1, 7]),
    ("2e patch-afl-afl", "outliers", 2, 1 << 26, [6, 1, 7, 1, 7]),
    ("3 gfc double", "price", 5, 1 << 26, [10, 7, 7]),
    ("3 gfc float", "price", 4, 1 << 26, [10, 7, 7]),
]


def config_column(k):
    from gputimeseriescompressionoptimizer_b200 import workloads as W
    name, kind, dt, n, _ = CONFIG_COLUMNS[k]
    if kind == "uniform11":
        return np.random.default_rng(0xB201).integers(0, 1 << 11, n).astype(np.int32)
    return W.column(kind, dt, n, 0xB202 + (k if kind != "price" else 8))


def per_config(g, torch, st, stream, peak, reps, tune):
    """Each benchmark configuration alone as a one-column batch with the mixed workload's tuned
    launch parameters (its tree's compress and decompress steps, CUDA graphs, device-resident input): CUDA-event time per step (median of `reps`, the L2
    flushed before each step when the column fits in it), GB/s of uncompressed input and the
    fraction of the HBM peak on algorithmic bytes (n*s + C each way).  Config 1 also times the AFL
    pack / unpack kernels alone at its bit width 11 (run_afl_compress_gpu / run_afl_decompress_gpu)."""
    with cf.ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        cols = list(ex.map(config_column, range(len(CONFIG_COLUMNS))))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def med_time(fn, small):
        """Columns that fit in L2: each call timed alone after a 256 MB write on the same stream
        (it evicts the column from L2 and keeps the GPU busy while the host issues the call); larger
        columns: `reps` calls back to back between two events, after two warm-up calls."""
        if not small:
            for _ in range(2):
                fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / 1e3 / reps
        ts = []
        for _ in range(reps + 2):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return statistics.median(ts[2:])

    out = []
    for k, (name, kind, dt, n, path) in enumerate(CONFIG_COLUMNS):
        x = cols[k]
        dev = torch.from_numpy(x.view(np.uint8)).to("cuda")
        dv = DevView(dev)
        small = x.nbytes < (128 << 20)
        nodes = g.tree_from_path(path, dt)
        b = g.Batch([dv], [dt], [nodes], st, tuning=g.tuning(
            tune["minmax_tile"], tune["minmax_values_per_thread"], tune["hist_tile"],
            tune["schedule_compress"] == "persistent", tune["schedule_decompress"] == "persistent"))
        o = torch.empty_like(dev)
        ov = [DevView(o)]
        b.compress()
        b.status()
        p, nb = b.output()
        b.decompress(p, nb, ov)
        b.status()
        assert torch.equal(o, dev), f"config {name}: round trip differs"
        blob = int(b.blob_sizes()[0])
        tc = med_time(b.compress, small)
        td = med_time(lambda: b.decompress(p, nb, ov), small)
        b.status()
        alg = x.nbytes + blob
        row = {"config": name, "values": n, "input_bytes": x.nbytes, "blob_bytes": blob,
               "ratio": round(x.nbytes / blob, 4), "compress_ms": round(1e3 * tc, 4),
               "decompress_ms": round(1e3 * td, 4), "compress_GBps": round(x.nbytes / tc / 1e9, 1),
               "decompress_GBps": round(x.nbytes / td / 1e9, 1),
               "compress_hbm_frac": round(alg / tc / 1e9 / peak, 4),
               "decompress_hbm_frac": round(alg / td / 1e9 / peak, 4),
               "launches": [b.launches(True), b.launches(False)]}
        if k == 0:  # the AFL kernels alone at b = 11
            L = g.lib()
            words = (n * 11 + 31) // 32
            packed = torch.empty(words * 4, dtype=torch.uint8, device="cuda")
            back = torch.empty_like(dev)
            tp = med_time(lambda: g.check(L.gtsc_afl_compress_gpu(dt, 11, dv.ptr, n, packed.data_ptr(), words * 4,
                                                                   st.handle), "afl"), small)
            tu = med_time(lambda: g.check(L.gtsc_afl_decompress_gpu(dt, 11, packed.data_ptr(), words * 4,
                                                                     back.data_ptr(), n, st.handle), "afl"), small)
            assert torch.equal(back, dev)
            row["afl_kernels_b11"] = {"pack_ms": round(1e3 * tp, 4), "unpack_ms": round(1e3 * tu, 4),
                                      "pack_GBps": round((x.nbytes + words * 4) / tp / 1e9, 1),
                                      "unpack_GBps": round((x.nbytes + words * 4) / tu / 1e9, 1)}
        out.append(row)
        del b, o, ov, dev, dv
    return out


def run_ours(args, world, rank, local):
    import torch
    import gputimeseriescompressionoptimizer_b200 as g

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", device_id=torch.device("cuda", local), timeout=timedelta(seconds=600))
    L = g.lib()
    st = g.Stream()
    stream = torch.cuda.ExternalStream(st.handle)
    sp = st.handle

    specs = workload_specs()
    t0 = time.perf_counter()
    cols = gen_columns(specs)
    t_gen = time.perf_counter() - t0
    dts = [dt for _, dt, _, _ in specs]
    in_bytes = sum(c.nbytes for c in cols)
    host = [torch.from_numpy(c.view(np.uint8)).pin_memory() for c in cols]
    dev = [torch.empty(c.nbytes, dtype=torch.uint8, device="cuda") for c in cols]
    for d, h in zip(dev, host):
        d.copy_(h)
    torch.cuda.synchronize()
    dv = [DevView(d) for d in dev]

    # the learned planner (features + MLP, exhaustive fallback below min confidence) for the batch
    planner = g.Planner.load()
    planner.plan(dv[:4], dts[:4], MIN_CONFIDENCE, sp)  # warm (kernel attributes, allocations)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    planned = planner.plan(dv, dts, MIN_CONFIDENCE, sp)
    torch.cuda.synchronize()
    t_plan_learned = time.perf_counter() - t0
    trees = [t for t, _ in planned]
    fallback_rate = float(np.mean([f for _, f in planned]))

    # the plain exhaustive planner on every column's sample (the reference's CompressData full update)
    t0 = time.perf_counter()
    ex_trees = []
    for d, dt in zip(dv, dts):
        sb = g.sample_bytes(dt, d.nbytes)
        nodes, _ = g.plan_exhaustive(dt, g.DeviceBuffer(d.ptr, sb, owned=False), sp)
        ex_trees.append(nodes)
    torch.cuda.synchronize()
    t_plan_exh = time.perf_counter() - t0

    t0 = time.perf_counter()
    batch = g.Batch(dv, dts, trees, st)
    t_create = time.perf_counter() - t0
    # the autotuner: schedule, min/max tile x values per thread, histogram tile, timed on this batch
    tune = batch.autotune()
    outs = [torch.empty_like(d) for d in dev]
    ov = [DevView(o) for o in outs]

    def compress():
        batch.compress()

    framed = {}

    def decompress():
        batch.decompress(framed["p"], framed["n"], ov)

    def step():
        compress()
        decompress()

    # parity at full size: the batched blobs against the plain per-column path, and the round trip
    compress()
    batch.status()
    framed["p"], framed["n"] = batch.output()
    decompress()
    batch.status()
    framed_host = g.to_host(g.DeviceBuffer(framed["p"], framed["n"], owned=False))
    blobs = g.split_framed(framed_host)
    blob_bytes = sum(b.size for b in blobs)
    for i in range(len(cols)):
        pb = g.tree_compress(trees[i], g.DeviceBuffer(dv[i].ptr, dv[i].nbytes, owned=False), sp)
        assert np.array_equal(g.to_host(pb, stream=sp), blobs[i]), f"column {i}: batched blob differs"
        assert torch.equal(outs[i], dev[i]), f"column {i}: round trip differs"
    t0 = time.perf_counter()
    oracle_checked = oracle_check(cols, trees, blobs) if rank == 0 else 0
    t_oracle_check = time.perf_counter() - t0
    del framed_host

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def timed(fn, k):
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(k):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        t = ev0.elapsed_time(ev1) / 1e3 / k
        if dist is not None:
            tt = torch.tensor([t], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = tt.item()
        return t

    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local)
    clocks.start()
    t_step = timed(step, args.steps)
    t_comp = timed(compress, args.steps)
    t_dec = timed(decompress, args.steps)
    batch.status()

    # the plain path: one column at a time with the exhaustive planner's trees (planning timed above)
    ex_sizes = [0] * len(cols)

    def plain():
        for i in range(len(cols)):
            blob = g.tree_compress(ex_trees[i], g.DeviceBuffer(dv[i].ptr, dv[i].nbytes, owned=False), sp)
            ex_sizes[i] = blob.nbytes
            g.tree_decompress(blob, sp)

    plain()
    t_plain = timed(plain, 1)
    ex_blob_bytes = sum(ex_sizes)
    ratio_ln = [c.nbytes / b.size for c, b in zip(cols, blobs)]
    ratio_ex = [c.nbytes / e for c, e in zip(cols, ex_sizes)]

    # launch-by-launch profile (events between launches, outside the graphs), a few repeats
    prof = {}
    for name, comp in (("compress", True), ("decompress", False)):
        runs = [batch.profile(comp) for _ in range(3)]
        prof[name] = [(runs[0][j][0], min(r[j][1] for r in runs), runs[0][j][2], runs[0][j][3])
                      for j in range(len(runs[0]))]
    batch.status()
    n_launch = batch.launches(True) + batch.launches(False)
    del batch, outs, ov

    # end to end through the public API: the column-chunk pipeline (E2E_GROUPS column groups, each with its
    # batch engine and stream) from pinned host columns to pinned host framed output, each group's
    # device decode right after its read-back; the call is synchronous, timed by CUDA events
    # around it
    pipe = g.Pipeline([c.nbytes for c in cols], dts, trees, groups=E2E_GROUPS)
    cap = blob_bytes + 8 * len(cols) + 8 * E2E_GROUPS + (1 << 20)
    host_framed = torch.empty(cap, dtype=torch.uint8).pin_memory()
    host_ptrs = [h.data_ptr() for h in host]
    e2e_bytes = {}

    def e2e_step():
        sizes = pipe.roundtrip_host(host_ptrs, host_framed.data_ptr(), cap)
        e2e_bytes["d2h"] = int(sizes.sum()) + 4 * pipe.groups

    e2e_step()
    for i in range(len(cols)):  # the first end-to-end step restores every column
        _, d_out = pipe.column(i)
        chk = torch.empty_like(dev[i])
        g.check(L.gtsc_memcpy(chk.data_ptr(), d_out, dev[i].numel(), 3, sp), "d2d")
        torch.cuda.synchronize()
        assert torch.equal(chk, dev[i]), f"column {i}: end-to-end round trip differs"
        del chk
    t_e2e = timed(e2e_step, max(2, args.steps // 2))
    clk = clocks.stop()
    del pipe

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    peak, peak_kind = peak_hbm()
    allp = [(phase, *x) for phase, lst in prof.items() for x in lst]
    top = max(allp, key=lambda r: r[2])
    top_index = prof[top[0]].index(top[1:])
    traffic, traffic_src = dram_traffic(prof, top[0], top_index)
    t_prof = {k: sum(x[1] for x in v) for k, v in prof.items()}
    top_ach = top[3] / (top[2] / 1e3) / 1e9 if top[2] > 0 else 0.0
    alg_step = 2 * (in_bytes + blob_bytes + 8 + 8 * len(cols))
    value = world * in_bytes / t_step / 1e9

    # CPU baseline: the oracle (built -O3 -march=native here) on the same workload and trees, all
    # host threads, best of two after a warm-up
    import oracle
    cpu_build = oracle.select_native()
    model, threads = cpu_model()
    cpu_roundtrip(cols, trees, threads)
    ct, cin, _ = min((cpu_roundtrip(cols, trees, threads) for _ in range(2)), key=lambda r: r[0])
    cpu_gbs = cin / ct / 1e9

    tick = tick_table(g, torch, planner, st, stream, sp) if rank == 0 else None
    configs = per_config(g, torch, st, stream, peak, max(3, args.steps), tune) if rank == 0 else None
    tree_names = {}
    for t in trees:
        k = "-".join(g.tree_names(t))
        tree_names[k] = tree_names.get(k, 0) + 1
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32/float32/float64 (integer arithmetic on bits)", "data": "synthetic",
        "config": {"workload": WORKLOAD, "columns": len(cols), "input_bytes": in_bytes, "blob_bytes": blob_bytes,
                   "compression_ratio": round(in_bytes / blob_bytes, 4),
                   "inputs": f"larger than L2 ({in_bytes / 1e9:.2f} GB), no flush needed",
                   "planner": f"learned (MLP over 32 sample features, exhaustive fallback below confidence "
                              f"{MIN_CONFIDENCE})",
                   "plan_learned_ms": round(1e3 * t_plan_learned, 2), "fallback_rate": round(fallback_rate, 4),
                   "ratio_learned": round(in_bytes / blob_bytes, 4),
                   "ratio_exhaustive": round(in_bytes / ex_blob_bytes, 4),
                   "ratio_gap": round(1 - ex_blob_bytes / blob_bytes, 4),
                   "mean_column_ratio_learned": round(float(np.mean(ratio_ln)), 4),
                   "mean_column_ratio_exhaustive": round(float(np.mean(ratio_ex)), 4),
                   "blob_bytes_exhaustive": ex_blob_bytes,
                   "step": "gtsc_batch_compress + gtsc_batch_decompress (CUDA graphs), device-resident columns",
                   "compress_ms": round(1e3 * t_comp, 4), "decompress_ms": round(1e3 * t_dec, 4),
                   "hbm_frac_step": round(alg_step / t_step / 1e9 / peak, 4),
                   "algorithmic_bytes_per_step": alg_step,
                   "plain_path_ms": round(1e3 * t_plain, 2),
                   "plan_exhaustive_ms": round(1e3 * t_plan_exh, 1),
                   "speedup_vs_plain_step": round(t_plain / t_step, 2),
                   "speedup_vs_plain_with_planning": round((t_plan_exh + t_plain) / (t_plan_learned + t_step), 2),
                   "batch_create_ms": round(1e3 * t_create, 1), "generate_s": round(t_gen, 1),
                   "autotune": tune,
                   "trees": dict(sorted(tree_names.items(), key=lambda kv: -kv[1]))},
        "roofline": {"bound": "hbm", "kernel": f"{top[0]}:{top[1]}", "achieved": round(top_ach, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(top_ach / peak, 4), "peak_kind": peak_kind, "traffic": traffic,
                     "traffic_source": traffic_src,
                     "algorithmic_bytes_per_launch": top[3], "launch_ms": round(top[2], 4), "blocks": top[4],
                     "share_of_step": round(top[2] / (t_prof["compress"] + t_prof["decompress"]), 4),
                     "timing": "CUDA events around each launch of one step replayed launch by launch"},
        "launches": {k: [[x[0], round(x[1], 4), x[2], x[3]] for x in v] for k, v in prof.items()},
        "cpu_baseline": {"value": round(cpu_gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": f"the full workload: all {len(cols)} columns ({cin} B), the same trees, oracle "
                                   f"tree compress + decompress, best of 2; {cpu_build}",
                         "cpu_model": model},
        "e2e": {"value": round(world * in_bytes / t_e2e / 1e9, 3), "unit": "GB/s", "h2d_bytes_per_step": in_bytes,
                "d2h_bytes_per_step": e2e_bytes["d2h"],
                "path": f"gtsc_pipeline_roundtrip_host: {E2E_GROUPS} column groups, pinned host columns in, "
                        "framed output to pinned host memory, device decode of every group verified"},
        "gpu_launches": n_launch * args.steps,
        "parity": {"blobs_vs_oracle_bytes": oracle_checked, "oracle_check_s": round(t_oracle_check, 1),
                   "what": "every batched blob of the first step byte-compared with the oracle's "
                           "CompressionTree::Compress of its column; every column's round trip bit-exact"},
        "tick_table": tick,
        "configs": configs,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
