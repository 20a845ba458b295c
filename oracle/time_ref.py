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

import oracle  # noqa: E402


def time_reference_kernel(c: dict, img: np.ndarray, steps: int = 10, warmup: int = 3, flush=None,
                          variants=("r2", "r2_m32")) -> dict:
    """Time the rebuilt reference kernel on `img` (configuration dict `c` of
    bench.py) with the product's protocol: an L2 flush before every launch,
    CUDA events around Kernel_launcher.  Returns the fastest variant's figures
    plus every variant's; {"unavailable": why} when it cannot run.  Guards of
    ref_run.py apply: no slot overflow, no 3-pass all-zero codeblock to decode."""
    import torch

    import ref_run
    if c.get("levels") != 5 or c.get("cb") != 64:
        return {"unavailable": "the reference is compiled for 5 DWT levels and 64x64 codeblocks"}
    passes = c["passes"]
    if not ref_run.available(passes, variants[0]):
        return {"unavailable": "oracle/_ref not built (make -C oracle ref)"}
    lut = oracle.load_luts(os.path.join(ROOT, "tests", "golden", "luts", f"{passes}_coding_pass"), passes, 5)
    try:
        want = ref_run.check_no_overflow(img, lut, passes)
    except ValueError as e:
        return {"unavailable": str(e)}
    decodable = True
    try:
        ref_run.check_decodable(want, img.shape, lut, passes)
    except ValueError:
        decodable = False
    N = img.size
    if flush is None:
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    h_img = torch.from_numpy(np.ascontiguousarray(img).reshape(-1))
    h_want = torch.from_numpy(want)
    out = {}
    for variant in variants:
        if not ref_run.available(passes, variant):
            continue
        rc = ref_run.RefCoder(img.shape[1], img.shape[0], lut, passes, variant)
        s = rc.run(0, img)
        assert np.array_equal(s, want), "reference stream differs from the oracle"
        enc_ms, dec_ms = [], []
        for k in range(warmup + steps):
            rc.a.copy_(h_img)
            rc.b.fill_(-1)
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            rc.launch(0)
            e1.record()
            torch.cuda.synchronize()
            if k >= warmup:
                enc_ms.append(e0.elapsed_time(e1))
            if decodable:
                rc.a.copy_(h_want)
                rc.b.fill_(-1)
                flush.fill_(2)
                torch.cuda.synchronize()
                e0.record()
                rc.launch(1)
                e1.record()
                torch.cuda.synchronize()
                if k >= warmup:
                    dec_ms.append(e0.elapsed_time(e1))
                if k == 0:
                    assert torch.equal(rc.b.cpu(), h_img), "reference decode not lossless"
        v = {"encode_ms": float(np.mean(enc_ms)), "encode_gcoeffs": N / float(np.mean(enc_ms)) / 1e6}
        if decodable:
            td = float(np.mean(dec_ms))
            v.update({"decode_ms": td, "decode_gcoeffs": N / td / 1e6,
                      "gcoeffs": 2 * N / (v["encode_ms"] + td) / 1e6})
        out[variant] = v
        del rc
    if not out:
        return {"unavailable": "no reference build variant found"}
    key = "gcoeffs" if decodable else "encode_gcoeffs"
    best = max(out, key=lambda k: out[k][key])
    res = dict(out[best])
    res.update({"build": best, "variants": out, "steps": steps,
                "note": "reference Kernel_launcher rebuilt for sm_100a (_sync shim), stream checked equal to the "
                        "oracle's, L2 flushed before every launch"})
    return res


def main():
    import torch  # noqa: F401

    import bench

    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="cfg2")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    args = ap.parse_args()
    c = bench.CONFIGS[args.config]
    img = bench.make_input(c, 1)
    r = time_reference_kernel(c, img, args.steps, args.warmup)
    for variant, v in r.get("variants", {}).items():
        print(json.dumps(dict(v, variant=variant, config=bench.workload_name(c))), flush=True)
    if "unavailable" in r:
        print(json.dumps(r))


if __name__ == "__main__":
    main()
