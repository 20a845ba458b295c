"""The multi-rank path of bench.py on CPU (gloo, world size 2): each rank codes
its own image (no data exchanged), the job time is the slowest rank's, and the
aggregate throughput counts every rank's coefficients."""
import os
import socket
import sys
import time

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT, lut_folder


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "cuda_bpc-paco_b200"))
    import torch.distributed as tdist
    from datetime import timedelta
    import bench
    import bpc_synth
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    img = bpc_synth.synthetic_coefficients(256, 5, bench.rank_seed(rank), amp=30, nrect=8)
    lut = oracle.load_luts(lut_folder(3), 3, 5)
    t0 = time.perf_counter()
    s = oracle.encode(img, lut, 3, 5, 64)
    dec = oracle.decode(s, img.shape, lut, 3, 5, 64)
    t = time.perf_counter() - t0 + 0.05 * rank  # ranks of different speed
    tmax = bench.max_over_ranks(t)
    out.put((rank, t, tmax, int(np.array_equal(dec, img)), int(img.sum())))
    tdist.barrier()
    tdist.destroy_process_group()


def test_two_ranks_shard_by_image_and_take_the_slowest():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, m0, ok0, s0), (r1, t1, m1, ok1, s1) = res
    assert ok0 and ok1                  # every rank's round trip is lossless
    assert s0 != s1                     # the ranks coded different images
    assert m0 == m1 == max(t0, t1)      # both report the slowest rank's time
    value = 2 * 256 * 256 * 2 / m0      # aggregate: all ranks' coefficients
    assert value < 2 * 256 * 256 * 2 / min(t0, t1)
