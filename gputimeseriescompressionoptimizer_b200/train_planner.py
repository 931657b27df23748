"""Trains the learned tree planner on the GPU and writes its model file.

    python -m gputimeseriescompressionoptimizer_b200.train_planner [--columns 10000] [--out PATH]

1. Seeded training columns (workloads.training_column: the benchmark generators and the tick table
   with per-column parameters), each represented by its planner sample (first 10 000 values).
2. Labels: the tree the plain exhaustive planner (gtsc_plan_exhaustive, FullStatisticsUpdate) picks
   on that sample, as its pre-order encoding list; lists seen at least --min-count times become the
   network's classes (most frequent first, at most 64).
3. Features by the library's feature kernel; training by its FP32 forward / backward / Adam
   kernels; a held-out tenth reports accuracy, fallback rate and the compression-ratio gap of the
   chosen trees against the exhaustive planner's.
Prints one JSON line with those figures.
"""
import argparse
import collections
import concurrent.futures as cf
import json
import os
import time

import numpy as np

from . import (DeviceBuffer, Planner, Stream, alloc, check, lib, plan_exhaustive, planner_features, to_device,
               to_host, tree_compress, tree_from_path, MODEL_PATH, NP_TYPES)
from . import workloads as W


def label(cols, threads=8):
    """Exhaustive-planner trees of the columns' samples (one stream per worker thread)."""
    streams = [Stream() for _ in range(threads)]

    def work(k):
        st = streams[k % threads]
        out = []
        for i in range(k, len(cols), threads):
            _, dt, _, x = cols[i]
            dev = to_device(x, st.handle)
            nodes, _ = plan_exhaustive(dt, dev, st.handle)
            out.append((i, nodes))
        return out

    res = [None] * len(cols)
    with cf.ThreadPoolExecutor(threads) as ex:
        for lst in ex.map(work, range(threads)):
            for i, nodes in lst:
                res[i] = nodes
    return res


def device_samples(cols):
    """All samples in one device buffer (16-byte aligned slots) -> (buffer, [(ptr, nominal bytes, dtype)])."""
    offs, pos = [], 0
    for _, dt, _, x in cols:
        offs.append(pos)
        pos += (x.nbytes + 15) // 16 * 16
    host = np.zeros(max(pos, 16), np.uint8)
    for (_, _, _, x), o in zip(cols, offs):
        host[o:o + x.nbytes] = x.view(np.uint8)
    buf = to_device(host)
    views = [(buf.ptr + o, n_total * np.dtype(NP_TYPES[dt]).itemsize, dt)
             for (_, dt, n_total, _), o in zip(cols, offs)]
    return buf, views


class _View:
    def __init__(self, ptr, nbytes):
        self.ptr, self.nbytes = ptr, nbytes


def features(cols):
    buf, views = device_samples(cols)
    feats = planner_features([_View(p, b) for p, b, _ in views], [dt for _, _, dt in views])
    return buf, feats


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--columns", type=int, default=10000)
    ap.add_argument("--min-count", type=int, default=3)
    ap.add_argument("--max-classes", type=int, default=96)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--min-confidence", type=float, default=0.5)
    ap.add_argument("--out", default=MODEL_PATH)
    args = ap.parse_args()

    t0 = time.perf_counter()
    cols = [W.training_column(i) for i in range(args.columns)]
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    trees = label(cols)
    t_label = time.perf_counter() - t0
    seqs = [tuple(int(e) for e in t[::2]) for t in trees]
    counts = collections.Counter(seqs)
    classes = [s for s, c in counts.most_common(args.max_classes) if c >= args.min_count]
    index = {s: k for k, s in enumerate(classes)}
    labels = np.array([index.get(s, -1) for s in seqs], np.int32)

    buf, feats = features(cols)
    n = len(cols)
    hold = np.arange(n) % 10 == 9
    train_rows = np.flatnonzero(~hold)
    # training rows first in one feature buffer, held-out rows after
    fh = to_host(feats, np.float32).reshape(n, -1)
    order = np.concatenate([train_rows, np.flatnonzero(hold)])
    fd = to_device(np.ascontiguousarray(fh[order]))
    ftrain = DeviceBuffer(fd.ptr, 4 * fh.shape[1] * train_rows.size, owned=False)
    fhold = DeviceBuffer(fd.ptr + 4 * fh.shape[1] * train_rows.size, 4 * fh.shape[1] * int(hold.sum()), owned=False)

    P = Planner(classes, seed=7)
    t0 = time.perf_counter()
    loss = P.train(ftrain, labels[train_rows], epochs=args.epochs, batch=args.batch, lr=args.lr)
    t_train = time.perf_counter() - t0

    # held-out evaluation
    hrows = np.flatnonzero(hold)
    dts = np.array([cols[i][1] for i in hrows], np.int32)
    pred, conf = P.predict(fhold, dts)
    labelled = labels[hrows] >= 0
    acc = float(np.mean(pred[labelled] == labels[hrows][labelled])) if labelled.any() else 0.0
    fb = conf < args.min_confidence
    size_ex = size_ln = raw = 0
    for j, i in enumerate(hrows):
        _, dt, _, x = cols[i]
        dev = to_device(x)
        ex_nodes = trees[i]
        ln_nodes = ex_nodes if fb[j] else tree_from_path(list(classes[pred[j]]), dt)
        size_ex += tree_compress(ex_nodes, dev).nbytes
        size_ln += tree_compress(ln_nodes, dev).nbytes
        raw += x.nbytes
    P.save(args.out)
    print(json.dumps({
        "columns": n, "classes": len(classes), "labelled_share": round(float(np.mean(labels >= 0)), 4),
        "train_loss": round(loss, 4), "holdout_accuracy": round(acc, 4),
        "holdout_fallback_rate": round(float(fb.mean()), 4),
        "holdout_ratio_exhaustive": round(raw / size_ex, 4), "holdout_ratio_learned": round(raw / size_ln, 4),
        "holdout_ratio_gap": round(1 - (raw / size_ln) / (raw / size_ex), 4),
        "generate_s": round(t_gen, 1), "label_s": round(t_label, 1), "train_s": round(t_train, 1),
        "model": os.path.basename(args.out), "model_bytes": len(P.save()),
    }), flush=True)
    del buf


if __name__ == "__main__":
    main()
