"""Benchmark of the B200 BPC-PaCo codec.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config cfg2]

One step = encode + decode of one synthetic image of the named configuration
(default cfg2: 4096x4096, 5-level CDF 5/3 DWT, 64x64 codeblocks, 3 passes).
`value` is coefficients coded per second counting both directions,
2 * X * Y / (t_encode + t_decode), with each kernel timed by CUDA events on its
launching stream and the L2 flushed (a 256 MiB write) before every kernel;
`e2e` is the same metric through the C ABI's host-buffer call (bpc_code_host:
pinned host -> device copy, kernel, device -> host copy, status read).
Under torchrun (N > 1) every rank codes its own image (weak scaling, no
collective on the data path) and the time is the max over ranks.

--impl reference times the CPU restatement of the reference coder (the
reference has no CPU implementation of its own) on all host cores, on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

# the request server runs small and large requests on separate streams and the
# host-buffer path pipelines bands on 16 streams; give each stream its own
# hardware queue (must be set before CUDA initialises)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cuda_bpc-paco_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
LUT_DIR = os.path.join(ROOT, "tests", "golden", "luts")

CONFIGS = {
    # name: side, levels, passes, cb, amp, nrect
    "cfg1": dict(side=2048, levels=5, passes=2, cb=64, amp=20.0, nrect=30),
    "cfg2": dict(side=4096, levels=5, passes=3, cb=64, amp=40.0, nrect=60),
    "cfg5": dict(side=16384, levels=5, passes=3, cb=64, amp=80.0, nrect=400, gpu_input=True),
    # cfg5's second input: i.i.d. Laplacian coefficients, every codeblock coding 16 planes
    "cfg5l": dict(side=16384, levels=5, passes=3, cb=64, laplacian=True, gpu_input=True),
    # cfg5's generator at 8192x8192 (4 warp waves, work-ordered like cfg5): the
    # case its ncu counters are captured on, under a GiB on the device
    "cfg5s": dict(side=8192, levels=5, passes=3, cb=64, amp=80.0, nrect=400, gpu_input=True),
}
METRIC = "encode/decode Gcoeff/s (bit-exact)"
# ncu counters of the coder kernels per workload, written by
# `python bench.py --ncu-import <raw csv> --workload <name>` from a capture of
# this source (see the header of the file for the capture command)
COUNTERS = os.path.join(ROOT, "profiles", "k_bpc_counters.txt")


def load_counters():
    """{(workload, direction): {calls, time_us, dram_read, dram_write, warp_inst}} per coder call"""
    out = {}
    try:
        with open(COUNTERS) as f:
            for line in f:
                t = line.split()
                if not t or t[0].startswith("#") or len(t) < 7:
                    continue
                out[(t[0], t[1])] = {"calls": int(t[2]), "time_us": float(t[3]), "dram_read": float(t[4]),
                                     "dram_write": float(t[5]), "warp_inst": float(t[6])}
    except OSError:
        pass
    return out


def ncu_import(path, workload, units_scale=1.0):
    """Lines for COUNTERS from `ncu -i <rep> --page raw --csv` output: per
    coder kernel (encoder / decoder) the mean over its captured launches."""
    import csv
    rows = list(csv.reader(open(path)))
    hdr = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    names, units = rows[hdr], rows[hdr + 1]
    col = {n: i for i, n in enumerate(names)}
    scale = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6, "GB": 1e9,
             "nsecond": 1e-3, "usecond": 1.0, "msecond": 1e3, "ns": 1e-3, "us": 1.0, "ms": 1e3,
             "inst": 1, "Kinst": 1e3, "Minst": 1e6,
             "Ginst": 1e9, "": 1}

    def val(r, m):
        i = col[m]
        return float(r[i].replace(",", "")) * scale.get(units[i], 1)

    def dram(r, which):
        """bytes read or written; from the throughput metric when the sum is absent"""
        if f"dram__bytes_{which}.sum" in col:
            return val(r, f"dram__bytes_{which}.sum")
        if which == "read" and "dram__bytes.sum.per_second" in col:  # read + write together
            i = col["dram__bytes.sum.per_second"]
            rate = {"byte/s": 1, "Kbyte/s": 1e3, "Mbyte/s": 1e6, "Gbyte/s": 1e9, "Tbyte/s": 1e12}
            per_s = float(r[i].replace(",", "")) * rate.get(units[i].replace("second", "s"), 1)
            return per_s * val(r, "gpu__time_duration.sum") * 1e-6
        return 0.0

    # per coder call: an isolated decode is a heavy launch of a few CTAs and
    # the bulk launch after it, counted together as one call
    acc = {}
    for r in rows[hdr + 2:]:
        if len(r) != len(names) or "k_bpc" not in r[col["Kernel Name"]] or "batch" in r[col["Kernel Name"]]:
            continue
        kname = r[col["Kernel Name"]]
        m = re.search(r"k_bpc<\s*\d+,\s*\d+,\s*(\w+)", kname)  # <passes, cb, encoder, ...>
        kind = "encoder" if m and m.group(1) in ("1", "true") else "decoder"
        heavy = "launch__grid_size" in col and val(r, "launch__grid_size") <= 8
        a = acc.setdefault(kind, [0, 0.0, 0.0, 0.0, 0.0])
        a[0] += 0 if heavy else 1
        a[1] += val(r, "gpu__time_duration.sum")
        a[2] += dram(r, "read")
        a[3] += dram(r, "write")
        a[4] += val(r, "smsp__inst_executed.sum")
    for kind, (n, t, rd, wr, ins) in sorted(acc.items()):
        n = max(n, 1)
        f = units_scale / n  # per call, times the workload's units over the captured case's
        print(f"{workload} {kind} {n} {t * f:.1f} {rd * f:.0f} {wr * f:.0f} {ins * f:.0f}")


def workload_name(c):
    src = ("i.i.d. Laplacian coefficients (scale 2^(level+3), 16 planes per codeblock)" if c.get("laplacian")
           else f"synthetic image, {c['levels']}-level CDF 5/3 DWT")
    return f"{c['side']}x{c['side']} {src}, {c['cb']}x{c['cb']} codeblocks, {c['passes']}-pass encode+decode"


def launches_per_call(X, Y, cb, enc, dev):
    """Kernels one work-ordered call launches: the coder, plus the cost and
    sort kernels when the image spans more than two waves of resident warps
    (4 warps x 4 encoder / 7 decoder CTAs per SM); a decode of 64x64
    codeblocks between half a wave and two waves is sorted too and isolated
    (heavy launch + bulk launch)."""
    import torch
    units = (X // cb) * (Y // cb) // (1 if cb == 64 else 2)
    resident = torch.cuda.get_device_properties(dev).multi_processor_count * 4 * (4 if enc else 7)
    if units >= 2 * resident:
        return 3
    if not enc and cb == 64 and 2 * units > resident and units > 4 * 6 * 4:
        return 4
    return 1


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def bench_config(args, c, world):
    """The workload both arms report (same keys and values)."""
    return {"workload": workload_name(c), "name": args.config, "coefficients_per_gpu": c["side"] * c["side"],
            "l2": "GPU kernels: L2 flushed (256 MiB write) before every kernel; inputs of 4 B per coefficient",
            "parallelism": f"replicas x{world}"}


def copy_floor(n_words, dev, reps=5):
    """Seconds for one encode+decode step's PCIe traffic alone: per call X*Y
    int32 host -> device and X*Y int32 device -> host from pinned memory,
    both directions at once on two streams (the host-buffer calls overlap
    them), twice (encode call + decode call).  Median of `reps`."""
    import torch
    h_in = torch.empty(n_words, dtype=torch.int32, pin_memory=True)
    h_out = torch.empty(n_words, dtype=torch.int32, pin_memory=True)
    d_a = torch.empty(n_words, dtype=torch.int32, device=dev)
    d_b = torch.empty(n_words, dtype=torch.int32, device=dev)
    s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ts = []
    for _ in range(reps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        with torch.cuda.stream(s1):
            d_a.copy_(h_in, non_blocking=True)
        with torch.cuda.stream(s2):
            h_out.copy_(d_b, non_blocking=True)
        torch.cuda.synchronize(dev)
        ts.append(time.perf_counter() - t0)
    return 2 * float(np.median(ts[1:]))


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def rank_seed(rank: int) -> int:
    """Each rank codes its own image (seed 1 + rank): images are independent,
    so the work shards by image with no exchange between ranks."""
    return 1 + rank


def max_over_ranks(x: float, device=None) -> float:
    """The slowest rank's time (the job's time); x itself when not distributed."""
    import torch
    import torch.distributed as tdist
    if not (tdist.is_available() and tdist.is_initialized()) or tdist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(img, lut_np, c, budget_s=12.0):
    """Oracle (CPU restatement) encode + decode on all host cores over a
    bounded prefix of the codeblocks."""
    import oracle
    threads = os.cpu_count() or 1
    ncb = (img.shape[0] // c["cb"]) * (img.shape[1] // c["cb"])
    # calibrate on a small prefix, then size the sample to ~budget_s
    n = min(ncb, max(threads * 4, 64))
    t0 = time.perf_counter()
    s = oracle.encode(img, lut_np, c["passes"], c["levels"], c["cb"], threads, cb_range=(0, n))
    oracle.decode(s, img.shape, lut_np, c["passes"], c["levels"], c["cb"], threads, cb_range=(0, n))
    dt = time.perf_counter() - t0
    n2 = int(min(ncb, max(n, n * budget_s / max(dt, 1e-3))))
    # the whole image may take less than the budget: code it repeatedly
    reps = 0
    t0 = time.perf_counter()
    while True:
        s = oracle.encode(img, lut_np, c["passes"], c["levels"], c["cb"], threads, cb_range=(0, n2))
        oracle.decode(s, img.shape, lut_np, c["passes"], c["levels"], c["cb"], threads, cb_range=(0, n2))
        reps += 1
        dt = time.perf_counter() - t0
        if n2 < ncb or dt >= budget_s:
            break
    coefs = reps * n2 * c["cb"] * c["cb"]
    what = f"the whole image x{reps}" if n2 == ncb else f"first {n2} of {ncb} codeblocks of the same image"
    return {"value": 2 * coefs / dt / 1e9, "unit": "Gcoeff/s", "cores": threads, "kind": "port",
            "sample": f"{what}, encode+decode, {dt:.1f} s"}


def make_input(c, seed):
    """Seeded coefficients of the configuration as a host int32 array (the
    HBM-scale configurations are generated on the GPU and copied back)."""
    import bpc_synth
    if c.get("laplacian"):
        return bpc_synth.laplacian_coefficients_gpu(c["side"], c["levels"], seed, cb=c["cb"]).cpu().numpy()
    if c.get("gpu_input"):
        return bpc_synth.synthetic_coefficients_gpu(c["side"], c["levels"], seed, amp=c["amp"],
                                                    nrect=c["nrect"]).cpu().numpy()
    return bpc_synth.synthetic_coefficients(c["side"], c["levels"], seed, amp=c["amp"], nrect=c["nrect"])


def run_reference(args, c):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    import oracle
    img = make_input(c, 1)
    lut_np = oracle.load_luts(os.path.join(LUT_DIR, f"{c['passes']}_coding_pass"), c["passes"], c["levels"])
    threads = os.cpu_count() or 1
    ncb = (img.shape[0] // c["cb"]) * (img.shape[1] // c["cb"])
    # size each step's sample so that warm-up + timed steps take ~60 s in all
    n0 = min(ncb, max(threads * 8, 128))
    t0 = time.perf_counter()
    s = oracle.encode(img, lut_np, c["passes"], c["levels"], c["cb"], threads, cb_range=(0, n0))
    oracle.decode(s, img.shape, lut_np, c["passes"], c["levels"], c["cb"], threads, cb_range=(0, n0))
    t_n0 = max(time.perf_counter() - t0, 1e-4)
    budget = 60.0 / max(1, args.warmup + args.steps)
    n = int(max(min(n0, ncb), min(ncb, n0 * budget / t_n0)))
    times = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        s = oracle.encode(img, lut_np, c["passes"], c["levels"], c["cb"], threads, cb_range=(0, n))
        oracle.decode(s, img.shape, lut_np, c["passes"], c["levels"], c["cb"], threads, cb_range=(0, n))
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    coefs = n * c["cb"] * c["cb"]
    v = 2 * coefs * len(times) / sum(times) / 1e9
    sample = f"first {n} of {ncb} codeblocks per step, encode+decode, CPU restatement"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Gcoeff/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic", "config": bench_config(args, c, world),
        "cpu_baseline": {"value": v, "unit": "Gcoeff/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "Gcoeff/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def cfg3_specs(n=192, seed=3):
    """192 images: side in {2048, 3072, 4096, 6144, 8192}, DWT levels 3..6,
    64x64 codeblocks for 70 % of images (else 32x32), 2 or 3 passes."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        side = int(rng.choice([2048, 3072, 4096, 6144, 8192]))
        out.append((side, side, int(rng.integers(3, 7)), int(rng.choice([2, 3])), 64 if rng.random() < 0.7 else 32))
    return out


def run_batched(args):
    """cfg3: the batched persistent form against one plain launch per image."""
    import torch
    import bpc_paco as bpc
    import bpc_synth

    specs = cfg3_specs(args.images)
    luts = {2: os.path.join(LUT_DIR, "2_coding_pass"), 3: os.path.join(LUT_DIR, "3_coding_pass")}
    tmp = torch.empty(8192 * 8192, dtype=torch.int32, device="cuda")
    d_in = []
    for k, (X, Y, lv, ps, cb) in enumerate(specs):
        d_in.append(bpc_synth.synthetic_coefficients_gpu(X, lv, 1000 + k, amp=30.0, nrect=max(30, X // 64),
                                                        tmp=tmp[:X * Y].view(Y, X)))
    del tmp
    torch.cuda.synchronize()
    total = sum(X * Y for (X, Y, _, _, _) in specs)
    b = bpc.Batch(specs, luts)
    compact = torch.empty(b.words, dtype=torch.int32, device="cuda")
    offs = torch.zeros(b.codeblocks + 1, dtype=torch.int64, device="cuda")
    out = [torch.empty_like(t) for t in d_in]
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    # autotune on a 24-image sub-batch, apply to the whole batch (--no-tune:
    # the default schedule, e.g. for profiling runs)
    if args.no_tune:
        tuned_us, sched, tuning = None, b.schedule(), b.tuning()
    else:
        sub = bpc.Batch(specs[:24], luts)
        sc = torch.empty(sub.words, dtype=torch.int32, device="cuda")
        so = torch.zeros(sub.codeblocks + 1, dtype=torch.int64, device="cuda")
        tuned_us = sub.tune(d_in[:24], sc, so, out[:24])
        sched = sub.schedule()
        tuning = sub.tuning()
        sub.close()
        del sc, so
    b.set_tuning(*tuning)
    b.set_schedule(*sched)
    stream = torch.cuda.current_stream()

    def batched_step(times=None):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        b.encode(d_in, compact, offs, st)
        e1.record(stream)
        b.decode(compact, offs, out, st)
        e2.record(stream)
        if times is not None:
            times.append((e0, e1, e2))

    for _ in range(max(args.warmup, 3)):
        batched_step()
    torch.cuda.synchronize()
    status = st.item()
    # bit-exactness: lossless where no codeblock overflowed; every image's
    # container equals the plain kernel's slot stream of the same image (the
    # plain kernel is the one the parity tests hold bit-exact to the oracle)
    lossless = sum(int(torch.equal(o, i)) for o, i in zip(out, d_in))
    offs_h = offs.cpu().numpy()
    checked = 0
    base = 0
    lut_chk = {}
    slot_chk = torch.empty(8192 * 8192, dtype=torch.int32, device="cuda")
    for k, (X, Y, lv, ps, cb) in enumerate(specs):
        ncb = (X // cb) * (Y // cb)
        if (ps, lv) not in lut_chk:
            lut_chk[(ps, lv)] = bpc.DeviceLut(luts[ps], ps, lv)
        sv = slot_chk[:X * Y]
        bpc.encode_device(d_in[k], sv, lut_chk[(ps, lv)], cb)
        slots = sv.view(ncb, cb * cb)
        sizes = torch.clamp((slots[:, 1:] != -1).sum(1) + 1, max=cb * cb)
        assert torch.equal(offs[base + 1:base + ncb + 1] - offs[base:base + ncb], sizes), f"image {k}: sizes differ"
        want = slots[torch.arange(cb * cb, device="cuda")[None, :] < sizes[:, None]]
        got = compact[int(offs_h[base]):int(offs_h[base + ncb])]
        assert torch.equal(got, want), f"image {k}: container differs from the plain stream"
        checked += ncb
        base += ncb
    for l in lut_chk.values():
        l.close()
    del slot_chk
    times = []
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            batched_step(times)
        torch.cuda.synchronize()
    te = sum(a.elapsed_time(b_) for a, b_, _ in times) / len(times) / 1e3
    td = sum(b_.elapsed_time(c_) for _, b_, c_ in times) / len(times) / 1e3
    # plain: one encode and one decode launch per image (slot stream)
    lut_dev = {}
    for (X, Y, lv, ps, cb) in specs:
        if (ps, lv) not in lut_dev:
            lut_dev[(ps, lv)] = bpc.DeviceLut(luts[ps], ps, lv)
    slot = torch.empty(8192 * 8192, dtype=torch.int32, device="cuda")

    def plain_step(times=None, spans=None):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k, (X, Y, lv, ps, cb) in enumerate(specs):
            sv = slot[:X * Y]
            if spans is not None:
                a = torch.cuda.Event(enable_timing=True)
                a.record(stream)
            bpc.encode_device(d_in[k], sv, lut_dev[(ps, lv)], cb)
            bpc.decode_device(sv, out[k], lut_dev[(ps, lv)], cb)
            if spans is not None:
                z = torch.cuda.Event(enable_timing=True)
                z.record(stream)
                spans.append((a, z))
        e1.record(stream)
        if times is not None:
            times.append((e0, e1))

    plain_step()
    torch.cuda.synchronize()
    pt = []
    for _ in range(max(1, args.steps // 2)):
        plain_step(pt)
    torch.cuda.synchronize()
    tp = sum(a.elapsed_time(b_) for a, b_ in pt) / len(pt) / 1e3
    # GPU busy and idle time of one plain step: the per-image encode+decode
    # spans against the whole step (the gaps are launch and host overhead)
    spans, one = [], []
    plain_step(one, spans)
    torch.cuda.synchronize()
    plain_busy = sum(a.elapsed_time(z) for a, z in spans) / 1e3
    plain_total = one[0][0].elapsed_time(one[0][1]) / 1e3
    value = 2 * total / (te + td) / 1e9
    peak, peak_kind = load_peaks()
    words = int(offs_h[-1])
    alg = 4.0 * total + 4.0 * words + 8.0 * (b.codeblocks + 1)  # compact form, per direction
    line = {
        "metric": METRIC, "value": value, "unit": "Gcoeff/s", "n_gpus": 1, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * (te + td), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (GPU generator + GPU 5/3 DWT)",
        "config": {"workload": f"cfg3 batch: {len(specs)} images, {total / 1e9:.2f} G coefficients, sides 2048-8192, "
                               f"levels 3-6, 64x64 (70%) / 32x32, 2/3 passes", "l2": "inputs >> L2",
                   "schedule": {"ctas_per_sm_enc": sched[0], "ctas_per_sm_dec": sched[1], "cbs_per_item": sched[2],
                                "graph": sched[3], "warps_per_cta_enc": tuning[0], "warps_per_cta_dec": tuning[1],
                                "cost_order_enc": tuning[2], "cost_order_dec": tuning[3],
                                "classes_in_sequence_enc": tuning[4], "classes_in_sequence_dec": tuning[5],
                                "tuned_us_24_images": tuned_us}},
        "encode_gcoeffs": total / te / 1e9, "decode_gcoeffs": total / td / 1e9,
        "plain_per_image_gcoeffs": 2 * total / tp / 1e9, "batched_over_plain": tp / (te + td),
        "plain_step_ms": 1e3 * plain_total, "plain_gpu_busy_ms": 1e3 * plain_busy,
        "plain_gpu_idle_ms_per_image": 1e3 * (plain_total - plain_busy) / len(specs),
        "compact_words": words, "compression": 4.0 * total / (4.0 * words),
        "status": status, "images_lossless": lossless, "codeblocks_checked_vs_plain_stream": checked,
        "gpu_launches": "4 persistent kernels + scan + gather per encode, 4 per decode (one CUDA graph each)",
        "roofline": {"bound": "hbm", "achieved": alg / max(te, td) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / max(te, td) / 1e9 / peak, "traffic": None, "peak_source": peak_kind},
        "clocks": clk.summary(),
    }
    for d in lut_dev.values():
        d.close()
    b.close()
    print(json.dumps(line))


def cfg4_specs(n=20000, seed=4):
    """n requests: 60 % encode / 40 % decode; side log-uniform in [2048, 8192]
    rounded to a multiple of 1024; DWT levels 3..6, 2 or 3 passes, 64x64
    codeblocks for 70 % (else 32x32), as in cfg3."""
    rng = np.random.default_rng(seed)
    side = np.exp(rng.uniform(np.log(2048), np.log(8192), n))
    side = np.clip(np.round(side / 1024) * 1024, 2048, 8192).astype(int)
    out = []
    for k in range(n):
        out.append((bpc_dir(rng.random() < 0.6), int(side[k]), int(rng.integers(3, 7)), int(rng.choice([2, 3])),
                    64 if rng.random() < 0.7 else 32))
    return out


def bpc_dir(encode: bool) -> int:
    return 0 if encode else 1  # BPC_CODE / BPC_DECODE


def run_served(args):
    """cfg4: a Poisson stream of encode/decode requests through the request
    server, at saturation and at 20/50/80/100 % of the saturated rate, against
    the plain form (the same server with one request on the GPU at a time,
    i.e. one launch per request back to back).  Every output is compared on
    the GPU with the one-request result of the same input."""
    import collections

    import torch
    import bpc_paco as bpc
    import bpc_synth

    reqs = cfg4_specs(args.requests)
    luts_dir = {2: os.path.join(LUT_DIR, "2_coding_pass"), 3: os.path.join(LUT_DIR, "3_coding_pass")}
    combos = sorted({(sd, lv, ps, cb) for (_, sd, lv, ps, cb) in reqs})
    lut_dev = {(ps, lv): bpc.DeviceLut(luts_dir[ps], ps, lv) for (_, lv, ps, _) in combos}
    # resident inputs: per combination one coefficient image, its stream (the
    # input of decode requests and the expected encode output) and, where the
    # stream is lossy (a codeblock overflowed its slot), the expected decode
    tmp = torch.empty(8192 * 8192, dtype=torch.int32, device="cuda")
    coef, strm, decd, cstat = {}, {}, {}, {}
    pool_bytes = 0
    for k, key in enumerate(combos):
        sd, lv, ps, cb = key
        x = bpc_synth.synthetic_coefficients_gpu(sd, lv, 4000 + k, amp=30.0, nrect=max(30, sd // 64),
                                                 tmp=tmp[:sd * sd].view(sd, sd))
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        s_ = torch.empty_like(x)
        bpc.encode_device(x, s_, lut_dev[(ps, lv)], cb, st)
        d_ = torch.empty_like(x)
        bpc.decode_device(s_, d_, lut_dev[(ps, lv)], cb, st)
        torch.cuda.synchronize()
        coef[key], strm[key], cstat[key] = x.view(-1), s_.view(-1), st.item()
        pool_bytes += 8 * x.numel()
        if not torch.equal(d_, x):
            decd[key] = d_.view(-1)
            pool_bytes += 4 * x.numel()
        else:
            del d_
    del tmp
    torch.cuda.synchronize()
    budget = int(args.budget_gb * 1e9) - pool_bytes  # resident inputs count against the 120 GB
    vs = torch.cuda.Stream()
    bad = torch.zeros(1, dtype=torch.int64, device="cuda")
    ncoef = np.array([sd * sd for (_, sd, _, _, _) in reqs], np.float64)

    def serve(srv, ids, rlist, rate, seed):
        n = len(rlist)
        if rate is None:
            arr = np.zeros(n)
        else:
            arr = np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, n))
        lat = np.zeros(n)
        stat = np.zeros(n, np.int64)
        tick = {}
        pending = collections.deque()
        i = done = 0
        t_last = 0.0
        t0 = time.perf_counter()
        while done < n:
            now = time.perf_counter() - t0
            while i < n and arr[i] <= now:
                d, sd, lv, ps, cb = rlist[i]
                key = (sd, lv, ps, cb)
                src = coef[key] if d == 0 else strm[key]
                t = srv.submit(d, src, ids[(ps, lv)], cb, shape=(sd, sd))
                assert t >= 0, t
                tick[t] = i
                i += 1
            wait = 1000 if i >= n else int(max(0.0, min(1e-3, arr[i] - (time.perf_counter() - t0))) * 1e6)
            for t, ptr, us, st in srv.poll(256, wait):
                k = tick.pop(t)
                assert st >= 0 and ptr, f"request {k} failed: {st}"
                lat[k], stat[k] = us, st
                done += 1
                t_last = time.perf_counter() - t0
                d, sd, lv, ps, cb = rlist[k]
                key = (sd, lv, ps, cb)
                want = strm[key] if d == 0 else decd.get(key, coef[key])
                view = bpc.as_tensor(ptr, sd * sd)
                with torch.cuda.stream(vs):
                    bad.add_(torch.ne(view, want).any())
                    ev = torch.cuda.Event()
                    ev.record(vs)
                pending.append((ev, ptr))
            while pending and pending[0][0].query():
                srv.release(pending.popleft()[1])
        vs.synchronize()
        while pending:
            srv.release(pending.popleft()[1])
        return lat, stat, t_last

    def summary(lat, stat, span):
        small = np.array([r[1] == 2048 for r in reqs])
        q = lambda a, p: float(np.percentile(a, p)) / 1e3
        return {"requests": len(reqs), "req_per_s": len(reqs) / span, "gcoeffs": float(ncoef.sum()) / span / 1e9,
                "p50_ms": q(lat, 50), "p99_ms": q(lat, 99), "p99_9_ms": q(lat, 99.9),
                "p50_ms_2048": q(lat[small], 50), "p99_ms_2048": q(lat[small], 99),
                "requests_with_status": int((stat != 0).sum())}

    result = {}
    with ClockSampler(0) as clk:
        for name, inflight in (("server", args.in_flight), ("plain", 1)):
            srv = bpc.Server(budget, inflight)
            ids = {key: srv.register_lut(l) for key, l in lut_dev.items()}
            # warm-up: every combination once, both directions
            warm = [(d, sd, lv, ps, cb) for (sd, lv, ps, cb) in combos for d in (0, 1)]
            serve(srv, ids, warm, None, 0)
            lat, stat, span = serve(srv, ids, reqs, None, 1)
            out = {"saturated": summary(lat, stat, span)}
            rate = len(reqs) / span
            loads = args.loads if name == "server" else [0.8]
            for f in loads:
                lat, stat, span = serve(srv, ids, reqs, f * rate, 10 + int(100 * f))
                out[f"load_{int(round(100 * f))}"] = dict(summary(lat, stat, span), offered_req_per_s=f * rate)
            srv.close()
            result[name] = out
    torch.cuda.synchronize()
    n_bad = int(bad.item())
    sat, plain = result["server"]["saturated"], result["plain"]["saturated"]
    line = {
        "metric": "served requests: Gcoeff/s and p50/p99 latency (bit-exact)", "value": sat["gcoeffs"],
        "unit": "Gcoeff/s", "n_gpus": 1, "steps": len(reqs), "warmup": 2 * len(combos), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (GPU generator + GPU 5/3 DWT)",
        "config": {"workload": f"cfg4: {len(reqs)} Poisson requests, 60/40 encode/decode, sides 2048-8192 "
                               f"log-uniform (multiples of 1024), levels 3-6, 2/3 passes, 64x64 (70%) / 32x32",
                   "budget_gb": args.budget_gb, "resident_inputs_gb": pool_bytes / 1e9,
                   "max_in_flight": args.in_flight, "combinations": len(combos), "l2": "inputs >> L2"},
        "server": result["server"], "plain": result["plain"],
        "server_over_plain_saturated": sat["req_per_s"] / plain["req_per_s"],
        "outputs_compared": len(reqs) * (len(args.loads) + 3), "outputs_differing": n_bad,
        "combinations_with_status": int(sum(1 for v in cstat.values() if v)),
        "gpu_launches": "1 coder launch + status memset/copy per request",
        "clocks": clk.summary(),
    }
    for l in lut_dev.values():
        l.close()
    print(json.dumps(line))


def run_ours(args, c):
    import torch
    import bpc_paco as bpc

    rank, world, local = dist_info()
    dist = world > 1
    if dist:
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local if dist else 0)
    torch.cuda.set_device(dev)
    img = make_input(c, rank_seed(rank))
    X = Y = c["side"]
    N = X * Y
    passes, levels, cb = c["passes"], c["levels"], c["cb"]
    lut = bpc.DeviceLut(os.path.join(LUT_DIR, f"{passes}_coding_pass"), passes, levels)
    stream = torch.cuda.current_stream()
    d_img = torch.from_numpy(img).to(dev)
    d_stream = torch.empty(N, dtype=torch.int32, device=dev)
    d_dec = torch.empty_like(d_img)
    d_status = torch.zeros(1, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    # work-ordered calls: images of more than two warp waves are coded heaviest
    # codeblocks first (two small planning kernels inside the timed call)
    sched = bpc.sched_buffer(X, Y, cb)

    def step(times=None):
        flush.fill_(1)
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        bpc.encode_device(d_img, d_stream, lut, cb, d_status, sched=sched)
        e1.record(stream)
        flush.fill_(2)
        e2.record(stream)
        bpc.decode_device(d_stream, d_dec, lut, cb, d_status, sched=sched)
        e3.record(stream)
        if times is not None:
            times.append((e0, e1, e2, e3))

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    # bit-exactness of this run's output (decode must return the input)
    assert torch.equal(d_dec, d_img), "decode did not return the input"
    assert d_status.item() == 0, f"status {d_status.item()}"

    times = []
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local if dist else 0) as clk:
        # the sampler polls every 50 ms: keep the GPU busy for a moment
        # before the timed region so that samples under load exist
        t_pre = time.perf_counter()
        while time.perf_counter() - t_pre < 0.3 and not (args.no_e2e or args.chain_only):  # profiling runs skip it
            step()
            torch.cuda.synchronize()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for _ in range(args.steps):
            step(times)
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
    if dist:
        tdist.barrier()
    te = sum(a.elapsed_time(b) for a, b, _, _ in times) / 1e3
    td = sum(c2.elapsed_time(d) for _, _, c2, d in times) / 1e3
    t_step = (te + td) / args.steps
    t_step = max_over_ranks(t_step, dev)
    value = 2 * N * world / t_step / 1e9

    # the serial chain: the top codeblock row coded alone as an X x cb image
    # (its codeblocks keep their subbands, since the subband of a codeblock of
    # the top row depends on x only); its LL codeblocks are the longest
    # lockstep chains of the whole image
    top = cb * X
    chain = {}
    probes = (("encode_ms", lambda: bpc.encode_device(d_img[:cb], d_stream[:top], lut, cb, d_status)),
              ("decode_ms", lambda: bpc.decode_device(d_stream[:top], d_dec[:cb], lut, cb, d_status)))
    if (cb >> levels) >= 1:  # else the top row's subbands would depend on y
        for name, fn in probes:
            chain[name] = 1e3 * _timed(fn, stream, flush, 10, 3)
    chain["what"] = f"top codeblock row alone ({X}x{cb}, {X // cb} codeblocks)" if chain else "n/a"
    if args.chain_only:
        if rank == 0:
            print(json.dumps({"chain": chain}))
        lut.close()
        return

    if args.no_e2e:
        lut.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "Gcoeff/s", "partial": "no e2e",
                              "encode_gcoeffs": N / (te / args.steps) / 1e9,
                              "decode_gcoeffs": N / (td / args.steps) / 1e9}))
        if dist:
            tdist.destroy_process_group()
        return

    # e2e through the C ABI with pinned host buffers (copies inside the timed region)
    h = torch.empty(N, dtype=torch.int32, pin_memory=True)
    hn = h.numpy()
    ref_stream = d_stream.cpu().numpy()
    e2e_t = []
    for k in range(max(args.warmup, 3) + args.steps):
        hn[:] = img.reshape(-1)
        t0 = time.perf_counter()
        st1 = bpc.lib().bpc_code_host(bpc.CODE, hn.ctypes.data, X, Y, bpc.ctypes.c_void_p(lut.ptr), lut.n,
                                      passes, levels, cb)
        t1 = time.perf_counter()
        if k == 0:
            assert np.array_equal(hn, ref_stream), "host-path stream differs from device-path stream"
        t2 = time.perf_counter()
        st2 = bpc.lib().bpc_code_host(bpc.DECODE, hn.ctypes.data, X, Y, bpc.ctypes.c_void_p(lut.ptr), lut.n,
                                      passes, levels, cb)
        t3 = time.perf_counter()
        assert st1 == 0 and st2 == 0
        if k >= max(args.warmup, 3):
            e2e_t.append((t1 - t0) + (t3 - t2))
    assert np.array_equal(hn.reshape(Y, X), img), "host-path decode differs"
    e2e_step = float(np.mean(e2e_t))
    e2e_step = max_over_ranks(e2e_step, dev)
    e2e = 2 * N * world / e2e_step / 1e9
    floor = max_over_ranks(copy_floor(N, dev), dev)

    peak, peak_kind = load_peaks()
    alg_bytes = 8.0 * N  # per launch: 4 B/coef in + 4 B/coef out (slot stream), encode and decode alike
    te1, td1 = te / args.steps, td / args.steps
    dom_t = max(te1, td1)
    dom = "decoder" if td1 >= te1 else "encoder"
    achieved = alg_bytes / dom_t / 1e9
    clocks = clk.summary()
    # issue roofline: warp instructions of one call of the dominant direction
    # (ncu capture of this workload; an isolated decode's two launches
    # together) over what the SMs can issue in the call's CUDA-event time at
    # the clock sampled during the run
    cnt = load_counters().get((args.config, dom))
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
    issue = None
    if cnt and mhz:
        peak_inst = sms * 4 * mhz * 1e6  # one warp instruction per SM sub-partition per cycle
        issue = {"warp_inst_per_call": cnt["warp_inst"], "achieved_ginst_s": cnt["warp_inst"] / dom_t / 1e9,
                 "peak_ginst_s": peak_inst / 1e9, "frac": cnt["warp_inst"] / dom_t / peak_inst, "sm_mhz": mhz,
                 "sms": sms, "source": "profiles/k_bpc_counters.txt"}
    line = {
        "metric": METRIC, "value": value, "unit": "Gcoeff/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * t_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator + 5/3 DWT)",
        "config": bench_config(args, c, world),
        "encode_gcoeffs": N / te1 / 1e9, "decode_gcoeffs": N / td1 / 1e9,
        "encode_ms": 1e3 * te1, "decode_ms": 1e3 * td1, "chain": chain,
        "e2e": {"value": e2e, "unit": "Gcoeff/s", "h2d_bytes_per_step": 2 * 4 * N, "d2h_bytes_per_step": 2 * 4 * N + 8,
                "ms_per_step": 1e3 * e2e_step, "copy_floor_ms": 1e3 * floor, "frac_of_floor": floor / e2e_step,
                "copy_floor": "pinned H2D + D2H of X*Y int32 each, both directions at once, per call, x2 calls"},
        "gpu_launches": args.steps * (launches_per_call(X, Y, cb, True, dev) + launches_per_call(X, Y, cb, False, dev)),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (cnt["dram_read"] + cnt["dram_write"]) if cnt else None, "peak_source": peak_kind,
                     "kernel": f"k_bpc {dom}", "issue": issue,
                     "note": "8 B/coefficient algorithmic; the coder is bound by SM integer issue and by the serial "
                             "chain of its heaviest codeblocks, not HBM; traffic and warp_inst from the ncu capture "
                             "of this workload (profiles/k_bpc_counters.txt)"},
        "clocks": clocks, "wall_s_timed": wall,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # baselines, after the timed region: the CPU restatement on the host
        # cores and the reference kernel rebuilt for this GPU (the timing bar)
        lut_np = bpc.load_luts_host(os.path.join(LUT_DIR, f"{passes}_coding_pass"), passes, levels)
        line["cpu_baseline"] = cpu_baseline(img, lut_np, c)
        if not args.no_ref_kernel:
            import time_ref
            rk = time_ref.time_reference_kernel(c, img, steps=min(args.steps, 10), warmup=3, flush=flush)
            line["ref_kernel"] = rk
            if "gcoeffs" in rk:
                line["vs_ref_kernel"] = value / rk["gcoeffs"]
                line["vs_ref_kernel_by_direction"] = {"encode": line["encode_gcoeffs"] / rk["encode_gcoeffs"],
                                                      "decode": line["decode_gcoeffs"] / rk["decode_gcoeffs"]}
    lut.close()
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def _timed(fn, stream, flush, steps, warmup):
    """Median device time (s) of fn() over `steps` runs after `warmup`, each
    preceded by an L2 flush, CUDA events on `stream`."""
    import torch
    ts = []
    for k in range(warmup + steps):
        flush.fill_(k & 255)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        if k >= warmup:
            ts.append(e0.elapsed_time(e1) / 1e3)
    return float(np.median(ts))


def run_dwt(args):
    """The GPU 5/3 DWT (bpc_dwt53_forward / _inverse) on cfg5's 16384x16384
    image, 5 levels.  Algorithmic bytes: every level reads and writes its
    region once for the row step and once for the column step (16 B per
    coefficient of the level), so 16 B x N x sum 4^-l per direction."""
    import torch
    import bpc_paco as bpc
    import bpc_synth
    c = CONFIGS["cfg5"]
    side, levels = c["side"], c["levels"]
    N = side * side
    img = bpc_synth.make_image_gpu(side, 1, c["amp"], c["nrect"]) - 128
    ref = img.clone()
    tmp = torch.empty_like(img)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    fwd = ref.clone()
    bpc.dwt53(fwd, levels, tmp=tmp)
    # each timed call transforms a fresh copy of its input; the copy is timed
    # alone and subtracted
    w = max(args.warmup, 3)
    tc = _timed(lambda: img.copy_(ref), stream, flush, args.steps, w)
    tf = _timed(lambda: (img.copy_(ref), bpc.dwt53(img, levels, tmp=tmp)), stream, flush, args.steps, w) - tc
    assert torch.equal(img, fwd), "forward differs between runs"
    ti = _timed(lambda: (img.copy_(fwd), bpc.dwt53(img, levels, inverse=True, tmp=tmp)), stream, flush, args.steps,
                w) - tc
    assert torch.equal(img, ref), "inverse(forward(x)) != x"
    alg = 16.0 * N * sum(4.0 ** -l for l in range(levels))
    peak, peak_kind = load_peaks()
    # e2e: pinned host image -> device, forward, -> host; and back through the inverse
    h = torch.empty(N, dtype=torch.int32, pin_memory=True)
    h.copy_(ref.view(-1))
    d = torch.empty_like(img)
    te = []
    for k in range(max(args.warmup, 3) + min(args.steps, 20)):
        t0 = time.perf_counter()
        d.view(-1).copy_(h, non_blocking=True)
        bpc.dwt53(d, levels, tmp=tmp)
        h.copy_(d.view(-1), non_blocking=True)
        d.view(-1).copy_(h, non_blocking=True)
        bpc.dwt53(d, levels, inverse=True, tmp=tmp)
        h.copy_(d.view(-1), non_blocking=True)
        torch.cuda.synchronize()
        if k >= max(args.warmup, 3):
            te.append(time.perf_counter() - t0)
    assert torch.equal(h.cuda().view(side, side), ref)
    line = {
        "metric": "5/3 DWT forward+inverse Gcoeff/s (lossless)", "value": 2 * N / (tf + ti) / 1e9,
        "unit": "Gcoeff/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": 1e3 * (tf + ti), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic (GPU generator)",
        "config": {"workload": f"{side}x{side} image, {levels}-level reversible CDF 5/3 DWT, forward then inverse",
                   "l2": "flushed (256 MiB write) before every timed call"},
        "forward_ms": 1e3 * tf, "inverse_ms": 1e3 * ti,
        "e2e": {"value": 2 * N / float(np.median(te)) / 1e9, "unit": "Gcoeff/s", "h2d_bytes_per_step": 8 * N,
                "d2h_bytes_per_step": 8 * N},
        "gpu_launches": "per level: 4 forward / 4 inverse kernels",
        "roofline": {"bound": "hbm", "achieved": alg / max(tf, ti) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / max(tf, ti) / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
                     "note": "16 B per coefficient and level (row step + column step, read + write)"},
    }
    print(json.dumps(line))


def run_train(args):
    """LUT training statistics (bpc_lut_stats) on the cfg2 image: the
    encoder's mask stage without its coder.  Algorithmic bytes: 4 B per
    coefficient read."""
    import torch
    import bpc_paco as bpc
    c = CONFIGS["cfg2"]
    img = make_input(c, 1)
    N = img.size
    d = torch.from_numpy(img).cuda()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    st = bpc.lut_stats(d, c["passes"], c["levels"], c["cb"])
    torch.cuda.synchronize()
    t = _timed(lambda: bpc.lut_stats(d, c["passes"], c["levels"], c["cb"], stats=st), stream, flush, args.steps,
               max(args.warmup, 3))
    n = st.cpu().numpy()
    peak, peak_kind = load_peaks()
    line = {
        "metric": "LUT training statistics Gcoeff/s", "value": N / t / 1e9, "unit": "Gcoeff/s", "n_gpus": 1,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * t, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator + 5/3 DWT)",
        "config": {"workload": workload_name(c) + ", symbol counts per LUT entry", "l2": "flushed before every call"},
        "symbols_counted_per_image": int(n[0::2].sum() // (args.steps + max(args.warmup, 3) + 1)),
        "gpu_launches": 1,
        "roofline": {"bound": "hbm", "achieved": 4.0 * N / t / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": 4.0 * N / t / 1e9 / peak, "traffic": None, "peak_source": peak_kind},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg2", choices=sorted(CONFIGS) + ["cfg3", "cfg4", "dwt", "train"])
    ap.add_argument("--images", type=int, default=192, help="cfg3: images per batch")
    ap.add_argument("--requests", type=int, default=20000, help="cfg4: requests per load level")
    ap.add_argument("--loads", type=float, nargs="+", default=[0.2, 0.5, 0.8, 1.0], help="cfg4: offered loads")
    ap.add_argument("--in-flight", type=int, default=8, help="cfg4: requests on the GPU at once")
    ap.add_argument("--budget-gb", type=float, default=120.0, help="cfg4: HBM admission budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="kernel timing only (profiling runs)")
    ap.add_argument("--no-ref-kernel", action="store_true", help="skip timing the rebuilt reference kernel")
    ap.add_argument("--chain-only", action="store_true", help="stop after timing the top codeblock row alone")
    ap.add_argument("--no-tune", action="store_true", help="cfg3: keep the default batch schedule")
    ap.add_argument("--ncu-import", help="print counter lines for profiles/k_bpc_counters.txt from ncu raw csv")
    ap.add_argument("--workload", default="cfg2", help="--ncu-import: workload name of the capture")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="--ncu-import: units of the workload over units of the captured case")
    args = ap.parse_args()
    if args.ncu_import:
        ncu_import(args.ncu_import, args.workload, args.scale)
        return
    if args.config in ("dwt", "train") and args.impl == "ours":
        (run_dwt if args.config == "dwt" else run_train)(args)
        return
    if args.config in ("cfg3", "cfg4", "dwt", "train"):
        if args.impl == "ours":
            (run_batched if args.config == "cfg3" else run_served)(args)
            return
        c = CONFIGS["cfg2"]
    else:
        c = CONFIGS[args.config]
    if args.impl == "reference":
        run_reference(args, c)
    else:
        run_ours(args, c)


if __name__ == "__main__":
    main()
