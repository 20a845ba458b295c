"""Time the reference kernel rebuilt for the B200 (oracle/_ref/, r2 builds)
on the benchmark workloads, with the protocol bench.py uses for the product:
the same synthetic image, a 256 MiB L2 flush before every kernel, CUDA events
around each launch.  TEST INFRASTRUCTURE ONLY (the timing bar).

    python oracle/time_ref.py [--config cfg2] [--steps 10]

Prints one JSON line per build variant; the bar is the fastest variant.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "cuda_bpc-paco_b200"))


def main():
    import torch

    import bench
    import oracle
    import ref_run

    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="cfg2")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args()
    c = bench.CONFIGS[args.config]
    img = bench.make_input(c, 1)
    passes = c["passes"]
    lut = oracle.load_luts(os.path.join(ROOT, "tests", "golden", "luts", f"{passes}_coding_pass"), passes,
                           c["levels"])
    want = ref_run.check_no_overflow(img, lut, passes)
    decodable = True
    try:
        ref_run.check_decodable(want, img.shape, lut, passes)
    except ValueError:
        decodable = False
    N = img.size
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for variant in ("r2", "r2_m32"):
        if not ref_run.available(passes, variant):
            continue
        rc = ref_run.RefCoder(c["side"], c["side"], lut, passes, variant)
        s = rc.run(0, img)
        assert np.array_equal(s, want), "reference stream differs from the oracle"
        enc_ms, dec_ms = [], []
        for k in range(args.warmup + args.steps):
            rc.a.copy_(torch.from_numpy(img.reshape(-1)))
            rc.b.fill_(-1)
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            rc.launch(0)
            e1.record()
            torch.cuda.synchronize()
            if k >= args.warmup:
                enc_ms.append(e0.elapsed_time(e1))
            if decodable:
                rc.a.copy_(torch.from_numpy(want))
                rc.b.fill_(-1)
                flush.fill_(2)
                torch.cuda.synchronize()
                e0.record()
                rc.launch(1)
                e1.record()
                torch.cuda.synchronize()
                if k >= args.warmup:
                    dec_ms.append(e0.elapsed_time(e1))
                if k == 0:
                    assert np.array_equal(rc.b.cpu().numpy().reshape(img.shape), img), "reference decode not lossless"
        te = float(np.mean(enc_ms))
        out = {"variant": variant, "config": bench.workload_name(c), "encode_ms": te,
               "encode_gcoeffs": N / te / 1e6}
        if decodable:
            td = float(np.mean(dec_ms))
            out.update({"decode_ms": td, "decode_gcoeffs": N / td / 1e6, "value": 2 * N / (te + td) / 1e6,
                        "unit": "Gcoeff/s"})
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
