"""Times the reference's own AFL kernels (compression/afl/afl_gpu.cu, compiled for sm_100a into
oracle/_ref/libref_afl.so by `make -C oracle ref`) beside the library's AFL kernels on the same
device, on AFL-only columns of int32 values uniform in [0, 2^b):

  compress     run_afl_compress_gpu<int, omega>        vs gtsc_afl_compress_gpu / gtsc_afl32_compress_gpu
  decompress   run_afl_decompress_gpu<int, omega>      vs gtsc_afl_decompress_gpu / gtsc_afl32_decompress_gpu
  values       run_afl_decompress_value_gpu<int, omega> vs gtsc_afl_values_gpu (every element on its own)

omega 1 is the FL layout AflEncoding uses, omega 32 the aligned layout.  Outputs are checked equal
(packed bytes against each other, unpacked values against the input) before timing.  GB/s counts the
algorithmic bytes (input read + output written) per call.  Timing: CUDA events on the legacy default
stream (where both sides launch), 3 warm-up calls, median of 20.

TEST INFRASTRUCTURE: a measurement script, not part of the library.  Usage:
    python oracle/time_ref_afl.py [--out FILE]      (needs a GPU and oracle/_ref/libref_afl.so)
"""
import argparse
import ctypes
import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import gputimeseriescompressionoptimizer_b200 as G  # noqa: E402

REF = os.path.join(HERE, "_ref", "libref_afl.so")


def timed(fn, reps=20, warm=3):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    R = ctypes.CDLL(REF)
    for f in ("ref_afl_gpu_compress_int",):
        getattr(R, f).argtypes = [ctypes.c_int, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulong,
                                  ctypes.c_ulong]
    for f in ("ref_afl_gpu_decompress_int", "ref_afl_gpu_values_int"):
        getattr(R, f).argtypes = [ctypes.c_int, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulong]
    peaks = {}
    p = os.path.join(os.path.dirname(HERE), "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            peaks = json.load(fh)
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    rows = []
    rng = np.random.default_rng(0xB200 + 1)
    for n, b in [(1 << 20, 11), (1 << 26, 11), (1 << 26, 17)]:
        x = rng.integers(0, 1 << b, n, dtype=np.int32)
        d_in = torch.from_numpy(x).cuda()
        src = G.DeviceBuffer(d_in.data_ptr(), n * 4, owned=False)
        for omega in (1, 32):
            words = G.lib().gtsc_afl32_bytes(G.INT, b, n) // 4 if omega == 32 else (n * b + 31) // 32
            pad = 64
            ref_c = torch.zeros(words + pad, dtype=torch.int32, device="cuda")
            ours_c = torch.zeros(words + pad, dtype=torch.int32, device="cuda")
            ours_buf = G.DeviceBuffer(ours_c.data_ptr(), words * 4, owned=False)
            out_r = torch.empty(n, dtype=torch.int32, device="cuda")
            out_o = torch.empty(n, dtype=torch.int32, device="cuda")
            out_o_buf = G.DeviceBuffer(out_o.data_ptr(), n * 4, owned=False)

            def ref_comp():
                assert R.ref_afl_gpu_compress_int(omega, b, d_in.data_ptr(), ref_c.data_ptr(), n, words) == 0

            def our_comp():
                if omega == 32:
                    G.check(G.lib().gtsc_afl32_compress_gpu(G.INT, b, src.ptr, n, ours_buf.ptr, words * 4, None), "c")
                else:
                    G.check(G.lib().gtsc_afl_compress_gpu(G.INT, b, src.ptr, n, ours_buf.ptr, words * 4, None), "c")

            def ref_dec():
                assert R.ref_afl_gpu_decompress_int(omega, b, ref_c.data_ptr(), out_r.data_ptr(), n) == 0

            def our_dec():
                if omega == 32:
                    G.check(G.lib().gtsc_afl32_decompress_gpu(G.INT, b, ours_buf.ptr, words * 4, out_o_buf.ptr, n,
                                                              None), "d")
                else:
                    G.check(G.lib().gtsc_afl_decompress_gpu(G.INT, b, ours_buf.ptr, words * 4, out_o_buf.ptr, n,
                                                            None), "d")

            def ref_val():
                assert R.ref_afl_gpu_values_int(omega, b, ref_c.data_ptr(), out_r.data_ptr(), n) == 0

            def our_val():
                G.check(G.lib().gtsc_afl_values_gpu(G.INT, b, omega, ours_buf.ptr, words * 4, None, n, out_o_buf.ptr,
                                                    None), "v")

            ref_comp()
            our_comp()
            torch.cuda.synchronize()
            assert torch.equal(ref_c[:words], ours_c[:words]), ("packed streams differ", n, b, omega)
            for rf, of in ((ref_dec, our_dec), (ref_val, our_val)):
                out_r.zero_()
                out_o.zero_()
                rf()
                of()
                torch.cuda.synchronize()
                assert torch.equal(out_r, d_in) and torch.equal(out_o, d_in), ("decode differs", n, b, omega)
            algo = n * 4 + words * 4
            for op, rf, of in (("compress", ref_comp, our_comp), ("decompress", ref_dec, our_dec),
                               ("values", ref_val, our_val)):
                tr, to = timed(rf), timed(of)
                rows.append({"n": n, "b": b, "omega": omega, "op": op, "ref_ms": round(tr, 4), "gtsc_ms": round(to, 4),
                             "ref_GBps": round(algo / tr / 1e6, 1), "gtsc_GBps": round(algo / to / 1e6, 1),
                             "gtsc_hbm_frac": round(algo / to / 1e6 / hbm, 3), "speedup": round(tr / to, 2)})
                print(json.dumps(rows[-1]), flush=True)
    text = "| n | b | omega | op | reference kernel ms | gtsc ms | reference GB/s | gtsc GB/s | gtsc / HBM | speed-up |\n"
    text += "|---|---|---|---|---|---|---|---|---|---|\n"
    for r in rows:
        text += (f"| 2^{int(np.log2(r['n']))} | {r['b']} | {r['omega']} | {r['op']} | {r['ref_ms']} | {r['gtsc_ms']} | "
                 f"{r['ref_GBps']} | {r['gtsc_GBps']} | {r['gtsc_hbm_frac']} | {r['speedup']}x |\n")
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(text)
    print(text)


if __name__ == "__main__":
    main()
