#!/usr/bin/env python
"""Benchmark of the column-compression hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = compress + decompress of one batch of synthetic input resident in HBM.  Prints one JSON
line (rank 0).  N > 1 runs N independent replicas (one process per GPU, launched by torchrun): the
path has no exchange step, so `value` is the work of all ranks over the slowest rank's time.
"""
import argparse
import concurrent.futures as cf
import ctypes
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

# workload: AFL fixed-width packing of one int32 column, U[0, 2^11), 11 bits per value
AFL_N = 1 << int(os.environ.get("GTSC_BENCH_AFL_LOG2N", "28"))
AFL_BITS = 11
AFL_SEED = 0xB200


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


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def gen_afl_column(n):
    rng = np.random.default_rng(AFL_SEED)
    x = rng.integers(0, 1 << AFL_BITS, n, dtype=np.int32)
    x[0] = (1 << AFL_BITS) - 1
    return x


# ------------------------------------------------------------------------------- CPU legs
def cpu_afl_reference(x, threads):
    """The reference's own AFL host path (oracle/_ref, run_afl_compress_cpu / decompress) over
    chunks of 2^16 values split across threads; returns (seconds, bytes)."""
    import oracle
    oracle.build_ref()
    R = oracle.ref()
    if R is None:
        raise RuntimeError("oracle/_ref not built")
    comp = R.ref_afl_compress_int
    comp.argtypes = [ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulong, ctypes.c_ulong]
    dec = R.ref_afl_decompress_int
    dec.argtypes = [ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulong]
    chunk = 1 << 16
    words = chunk * AFL_BITS // 32
    packed = np.zeros(x.size * AFL_BITS // 32 + 64, np.int32)
    out = np.zeros_like(x)

    def work(c):
        lo = c * chunk
        cnt = min(chunk, x.size - lo)
        w0 = lo * AFL_BITS // 32
        cw = (cnt * AFL_BITS + 31) // 32
        comp(AFL_BITS, x.ctypes.data + 4 * lo, packed.ctypes.data + 4 * w0, cnt, cw)
        dec(AFL_BITS, packed.ctypes.data + 4 * w0, out.ctypes.data + 4 * lo, cnt)

    nchunks = (x.size + chunk - 1) // chunk
    t = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(work, range(nchunks)))
    dt = time.perf_counter() - t
    assert np.array_equal(out, x), "reference AFL round trip failed"
    del words
    return dt, x.nbytes


def run_reference(args, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    n = 1 << 25
    x = gen_afl_column(n)
    for _ in range(max(args.warmup, 1)):
        cpu_afl_reference(x, threads)
    times = [cpu_afl_reference(x, threads)[0] for _ in range(args.steps)]
    t = sum(times) / len(times)
    gbs = x.nbytes / t / 1e9
    line = {
        "impl": "reference", "metric": "AFL compress+decompress throughput (uncompressed GB/s)",
        "value": round(gbs, 4), "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"afl int32 U[0,2^{AFL_BITS}) b={AFL_BITS}, CPU sample 2^25 of the 2^28-value column",
                   "inputs": "host memory"},
        "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": threads, "kind": "reference",
                         "sample": "2^25 int32 values per step"},
        "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------- GPU leg
def run_ours(args, world, rank, local):
    import torch
    import gputimeseriescompressionoptimizer_b200 as g

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    L = g.lib()

    n = AFL_N
    x = gen_afl_column(n)
    host_in = torch.from_numpy(x).pin_memory()
    host_out = torch.empty(n, dtype=torch.int32).pin_memory()
    dev_in = torch.empty(n, dtype=torch.int32, device="cuda")
    dev_in.copy_(host_in)
    torch.cuda.synchronize()
    col = g.DeviceBuffer(dev_in.data_ptr(), dev_in.numel() * 4, owned=False)

    def step():
        parts = g.encode(g.AFL, g.INT, col, sp)
        out = g.decode(g.AFL, g.INT, parts, sp)
        return parts, out

    # correctness of one step before timing
    parts, out = step()
    back = torch.empty(n, dtype=torch.int32, device="cuda")
    g.check(L.gtsc_memcpy(back.data_ptr(), out.ptr, out.nbytes, 3, sp), "copy")
    assert torch.equal(back, dev_in), "round trip failed"
    comp_bytes = sum(p.nbytes for p in parts)
    del back

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

    # dominant kernel alone: the AFL pack (2 launches of our kernels per step: minmax + pack,
    # plus the unpack)
    data_part = parts[1]
    pack = lambda: g.check(L.gtsc_afl_compress_gpu(g.INT, AFL_BITS, col.ptr, n, data_part.ptr,
                                                   data_part.nbytes, sp), "pack")
    unpack = lambda: g.check(L.gtsc_afl_decompress_gpu(g.INT, AFL_BITS, data_part.ptr, data_part.nbytes,
                                                       out.ptr, n, sp), "unpack")
    for _ in range(3):
        pack()
        unpack()
    t_pack = timed(pack, args.steps)
    t_unpack = timed(unpack, args.steps)

    # end to end through the public API: pinned host column in, decoded column back to the host
    def e2e_step():
        dev_in.copy_(host_in, non_blocking=True)
        p, o = step()
        tmp = torch.empty(0)
        g.check(L.gtsc_memcpy(host_out.data_ptr(), o.ptr, o.nbytes, 2, sp), "d2h")
        return tmp

    for _ in range(2):
        e2e_step()
    t_e2e = timed(e2e_step, max(2, args.steps // 2))
    clk = clocks.stop()

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    peak, peak_kind = peak_hbm()
    in_bytes = n * 4
    alg_pack = in_bytes + data_part.nbytes
    achieved = alg_pack / t_pack / 1e9
    value = world * in_bytes / t_step / 1e9

    # CPU baseline: the reference's AFL host path on a bounded sample, all host threads
    threads = os.cpu_count() or 1
    sample = x[: 1 << 25]
    cpu_afl_reference(sample, threads)
    ct = min(cpu_afl_reference(sample, threads)[0] for _ in range(2))
    cpu_gbs = sample.nbytes / ct / 1e9

    line = {
        "metric": "AFL compress+decompress throughput (uncompressed GB/s)",
        "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * t_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"afl: 2^28 int32 U[0,2^{AFL_BITS}) at b={AFL_BITS} (1 GiB per GPU)",
                   "inputs": "larger than L2 (1 GiB), no flush needed",
                   "step": "gtsc_encode(AFL) + gtsc_decode(AFL), device-resident input"},
        "roofline": {"bound": "hbm", "kernel": "k_afl_pack", "achieved": round(achieved, 1),
                     "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": None, "algorithmic_bytes_per_launch": alg_pack,
                     "launch_ms": round(1e3 * t_pack, 4),
                     "unpack_GBps": round((in_bytes + data_part.nbytes) / t_unpack / 1e9, 1)},
        "cpu_baseline": {"value": round(cpu_gbs, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
                         "sample": "first 2^25 values of the column, run_afl_compress_cpu + decompress"},
        "e2e": {"value": round(world * in_bytes / t_e2e / 1e9, 3), "unit": "GB/s",
                "h2d_bytes_per_step": in_bytes, "d2h_bytes_per_step": in_bytes},
        "gpu_launches": 3 * args.steps,
        "compressed_bytes": comp_bytes,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
