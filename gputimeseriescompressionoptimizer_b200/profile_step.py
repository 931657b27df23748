"""One batched compress + decompress step of the mixed workload, bracketed for a profiler.

    python -m gputimeseriescompressionoptimizer_b200.profile_step [--columns 512] [--max-log2 24]
        [--persistent] [--repeat 1] [--config NAME]

Builds the mixed workload (seeded synthetic columns, the learned planner's trees), creates the
batch, runs two untimed steps, then runs `--repeat` steps between cudaProfilerStart and
cudaProfilerStop, so that a profiler started with its capture off (ncu --profile-from-start off)
records exactly the launches of those steps.  Prints one JSON line: the step's launch sequence per
phase (pass names, as gtsc_batch_profile reports them), the step time measured with CUDA events
outside the profiled range, and the workload's size.

--config NAME replaces the mixed workload by one benchmark configuration's column and tree: 2^26
int32 values, "2a" delta->AFL on the walk, "2b" RLE->(AFL, AFL) on runs, "2c" dict->(AFL, AFL) on
Zipf(1.1) ids, "2d" const->AFL, "2e" patch->(AFL, AFL) on the outliers.
"""
import argparse
import json

import numpy as np

import gputimeseriescompressionoptimizer_b200 as E


# benchmark configurations 2a-2e: generator and tree (pre-order encodings)
CONFIGS = {
    "2a": ("walk", [E.DELTA, E.AFL, E.NONE]),
    "2b": ("runs", [E.RLE, E.AFL, E.NONE, E.AFL, E.NONE]),
    "2c": ("zipf", [E.DICT, E.AFL, E.NONE, E.AFL, E.NONE]),
    "2d": ("const", [E.CONST, E.AFL, E.NONE]),
    "2e": ("outliers", [E.PATCH, E.AFL, E.NONE, E.AFL, E.NONE]),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--columns", type=int, default=512)
    ap.add_argument("--max-log2", type=int, default=24)
    ap.add_argument("--persistent", action="store_true")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--config", default=None, choices=sorted(CONFIGS))
    args = ap.parse_args()

    import torch
    import gputimeseriescompressionoptimizer_b200 as g
    from gputimeseriescompressionoptimizer_b200 import workloads as W

    torch.cuda.set_device(0)
    st = g.Stream()
    stream = torch.cuda.ExternalStream(st.handle)
    if args.config:
        kind, path = CONFIGS[args.config]
        specs = [(kind, g.INT, 1 << 26, 0xB200)]
    else:
        specs = W.mixed_columns(args.columns, max_len=1 << args.max_log2)
    dts = [dt for _, dt, _, _ in specs]
    cols = [W.column(kind, dt, n, seed) for kind, dt, n, seed in specs]
    dev = [torch.from_numpy(c.view(np.uint8)).to("cuda") for c in cols]

    class View:
        def __init__(self, t):
            self.ptr, self.nbytes = t.data_ptr(), t.numel()

    dv = [View(d) for d in dev]
    if args.config:
        trees = [g.tree_from_path(CONFIGS[args.config][1], g.INT)]
    else:
        trees = [t for t, _ in g.Planner.load().plan(dv, dts, 0.5, st.handle)]
    b = g.Batch(dv, dts, trees, st)
    b.set_schedule(args.persistent)
    outs = [torch.empty_like(d) for d in dev]
    ov = [View(o) for o in outs]
    b.compress()
    p, n = b.output()

    def step():
        b.compress()
        b.decompress(p, n, ov)

    for _ in range(2):
        step()
    b.status()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    seq = {"compress": [x[0] for x in b.profile(True)], "decompress": [x[0] for x in b.profile(False)]}
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for _ in range(args.repeat):
        step()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    b.status()
    assert all(torch.equal(o, d) for o, d in zip(outs, dev)), "round trip differs"
    print(json.dumps({"columns": len(cols), "input_bytes": int(sum(c.nbytes for c in cols)), "blob_bytes": int(n),
                      "schedule": b.schedule(), "step_ms": round(ms, 4), "launches": seq}))


if __name__ == "__main__":
    main()
