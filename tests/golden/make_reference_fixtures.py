"""Generate reference_encoders.npz: the reference's own encoder and tree outputs on seeded columns.

    make -C oracle refenc                      # where the reference sources are (no GPU needed)
    python tests/golden/make_reference_fixtures.py [--out tests/golden/reference_encoders.npz]

Runs on a machine with a GPU: the reference's encoders are CUDA code.  oracle/_ref/libref_enc.so
is the reference's compression/, util/ and tree/ sources compiled as they are, behind the stand-in
headers of oracle/refshim/ and the entry points of oracle/ref_enc_shim.cu.  For every case of
refcases.py it stores the input column and what the reference returns: each encoding's streams
(Encoding::Encode through its factory's Get(data), as CompressionNode::Compress calls it) and each
compression tree's serialised blob (CompressionTree::Compress).  A case the reference refuses (an
exception, e.g. an encoding without an implementation for that type) is recorded with its message.

The reference exits the process on a CUDA error (CUDA_ASSERT_RETURN, core/macros.h), so the cases
run in worker processes, one per (type, generator) group; when a worker dies, its group runs again
one case per process and each case that kills its process is recorded with the reference's last
message.  The reference's decoders are not run.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import oracle as OR  # noqa: E402
import refcases as RC  # noqa: E402


def groups():
    """(group id, data type, generator) in a fixed order; inputs are numbered across groups."""
    out = []
    for dt in RC.DTYPES:
        for kind in RC.kinds_of(dt):
            out.append((len(out), dt, kind))
    return out


def run_cases(g, only, out_path):
    """Worker: the encoding cases of group g (all, or the one numbered `only`) into out_path."""
    gid, dt, kind = groups()[g]
    arrays, cases = {}, []
    j = -1
    for si, n in enumerate(RC.SIZES):
        k = gid * len(RC.SIZES) + si
        x = RC.column(kind, dt, n, k)
        key = f"in{k}"
        arrays[key] = OR.as_bytes(x).copy()
        for enc in RC.ENCODINGS:
            j += 1
            if only is not None and j != only:
                continue
            case = {"input": key, "kind": kind, "dtype": dt, "n": n, "enc": enc}
            try:
                res = OR.ref_encode(enc, dt, x)
            except OR.OracleError as e:
                case["refused"] = str(e)
                cases.append(case)
                continue
            if not res:
                case["refused"] = "no streams"
                cases.append(case)
                continue
            if RC.lossy_in_reference(enc, dt, x):
                case["lossy_in_reference"] = True
            res = RC.canonical(enc, dt, res)
            case["sizes"] = [int(r.size) for r in res]
            case["sha256"] = [RC.digest(r) for r in res]
            if n <= RC.FULL_LIMIT:
                case["streams"] = []
                for s, r in enumerate(res):
                    sk = f"g{gid}c{j}s{s}"
                    arrays[sk] = r
                    case["streams"].append(sk)
            cases.append(case)
    arrays["cases"] = np.frombuffer(json.dumps(cases).encode(), np.uint8)
    np.savez(out_path, **arrays)


def run_trees(out_path):
    """Worker: every tree of refcases.TREES."""
    arrays, cases = {}, []
    for t, (kind, dt, path) in enumerate(RC.TREES):
        x = RC.column(kind, dt, RC.TREE_SIZE, 100000 + t)
        nodes = OR.tree_from_path(path, dt)
        key = f"tin{t}"
        arrays[key] = OR.as_bytes(x).copy()
        case = {"input": key, "kind": kind, "dtype": dt, "n": RC.TREE_SIZE, "path": path,
                "nodes": [int(v) for v in nodes]}
        try:
            blob = OR.ref_tree_compress(nodes, x)
            case["size"] = int(blob.size)
            case["sha256"] = RC.digest(blob)
            arrays[f"tblob{t}"] = blob
            case["blob"] = f"tblob{t}"
        except OR.OracleError as e:
            case["refused"] = str(e)
        cases.append(case)
    arrays["cases"] = np.frombuffer(json.dumps(cases).encode(), np.uint8)
    np.savez(out_path, **arrays)


def spawn(args, tmp):
    """Runs a worker; returns (its npz or None, the tail of its error output)."""
    out = os.path.join(tmp, "w.npz")
    if os.path.exists(out):
        os.remove(out)
    p = subprocess.run([sys.executable, os.path.abspath(__file__)] + args + ["--worker-out", out],
                       capture_output=True, text=True)
    tail = " ".join((p.stderr or "").strip().splitlines()[-2:])[-300:]
    if p.returncode != 0 or not os.path.exists(out):
        return None, tail or f"exit status {p.returncode}"
    return np.load(out), tail


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "reference_encoders.npz"))
    ap.add_argument("--group", type=int, default=None)
    ap.add_argument("--case", type=int, default=None)
    ap.add_argument("--trees", action="store_true")
    ap.add_argument("--worker-out", default=None)
    args = ap.parse_args()
    if OR.ref_enc() is None:
        sys.exit("oracle/_ref/libref_enc.so is missing: run make -C oracle refenc first")
    if args.worker_out:
        if args.trees:
            run_trees(args.worker_out)
        else:
            run_cases(args.group, args.case, args.worker_out)
        return

    t0 = time.time()
    arrays, index = {}, {"encodings": [], "trees": [], "seed": RC.SEED, "full_limit": RC.FULL_LIMIT}
    per_group = len(RC.SIZES) * len(RC.ENCODINGS)

    def merge(z):
        cases = json.loads(z["cases"].tobytes().decode())
        for k in z.files:
            if k != "cases":
                arrays[k] = z[k]
        return cases

    with tempfile.TemporaryDirectory() as tmp:
        for gid, dt, kind in groups():
            z, tail = spawn(["--group", str(gid)], tmp)
            if z is not None:
                index["encodings"] += merge(z)
                continue
            print(f"group {gid} (dt={dt} {kind}) died: {tail}; running its cases one by one", flush=True)
            for j in range(per_group):
                z, tail = spawn(["--group", str(gid), "--case", str(j)], tmp)
                if z is not None:
                    index["encodings"] += merge(z)
                    continue
                si, e = divmod(j, len(RC.ENCODINGS))
                k = gid * len(RC.SIZES) + si
                arrays[f"in{k}"] = OR.as_bytes(RC.column(kind, dt, RC.SIZES[si], k)).copy()
                index["encodings"].append({"input": f"in{k}", "kind": kind, "dtype": dt, "n": RC.SIZES[si],
                                           "enc": RC.ENCODINGS[e], "refused": f"the reference exits: {tail}"})
                print(f"  case {j}: {OR.ENC_NAMES[RC.ENCODINGS[e]]} n={RC.SIZES[si]}: {tail}", flush=True)
        z, tail = spawn(["--trees"], tmp)
        if z is None:
            sys.exit(f"the tree worker died: {tail}")
        index["trees"] = merge(z)
    arrays["index"] = np.frombuffer(json.dumps(index).encode(), np.uint8)
    np.savez_compressed(args.out, **arrays)
    n_ok = sum("sizes" in c for c in index["encodings"])
    n_ref = sum("refused" in c for c in index["encodings"])
    t_ok = sum("blob" in c for c in index["trees"])
    print(json.dumps({"out": args.out, "encoding_cases": n_ok, "refused": n_ref, "trees": t_ok,
                      "bytes": os.path.getsize(args.out), "seconds": round(time.time() - t0, 1)}))


if __name__ == "__main__":
    main()
