"""The request server: every result is the same alone and in the mix (bit-exact
against the one-request device entry points and the oracle), admission by the
memory budget in arrival order, and the host-side failure cases (oversized
request, cancellation, corrupted stream) ending with a status, never a hang."""
import time

import numpy as np
import pytest

import bpc_synth
from conftest import lut_folder

pytestmark = pytest.mark.gpu


def collect(srv, want, timeout_s=60.0):
    """Poll until `want` requests have finished; {ticket: (ptr, us, status)}."""
    got = {}
    t_end = time.time() + timeout_s
    while len(got) < want:
        assert time.time() < t_end, f"server stalled: {srv.state()}"
        for t, p, us, st in srv.poll(64, 2000):
            got[t] = (p, us, st)
    return got


@pytest.fixture(scope="module")
def luts(bpc):
    d = {p: bpc.DeviceLut(lut_folder(p), p, 5) for p in (2, 3)}
    yield d
    for l in d.values():
        l.close()


def alone(bpc, torch, direction, data, lut, cb):
    out = torch.empty_like(data)
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    f = bpc.encode_device if direction == bpc.CODE else bpc.decode_device
    f(data, out, lut, cb, st)
    torch.cuda.synchronize()
    return out, st.item()


def test_mixed_requests_match_alone(bpc, oracle_mod, luts):
    import torch
    rng = np.random.default_rng(5)
    cases = []
    for k in range(24):
        side = int(rng.choice([256, 512, 1024, 1536]))
        passes = int(rng.integers(2, 4))
        cb = 32 if k % 3 == 0 else 64
        levels = int(rng.integers(3, 6))
        img = bpc_synth.synthetic_coefficients(side, levels, 100 + k, amp=30, nrect=10)
        cases.append((passes, cb, levels, img))
    srv = bpc.Server(1 << 30, 6)
    try:
        ids = {p: srv.register_lut(luts[p]) for p in (2, 3)}
        reqs = []
        for passes, cb, levels, img in cases:
            d = torch.from_numpy(img).cuda()
            s_alone, st = alone(bpc, torch, bpc.CODE, d, luts[passes], cb)
            assert st == 0
            reqs.append((bpc.CODE, d, passes, cb, img.shape, s_alone))
            reqs.append((bpc.DECODE, s_alone, passes, cb, img.shape, d))
        order = rng.permutation(len(reqs))
        tickets = {}
        for i in order:
            dirn, inp, passes, cb, shape, _ = reqs[i]
            t = srv.submit(dirn, inp.view(-1), ids[passes], cb, shape=shape)
            assert t >= 0
            tickets[t] = i
        done = collect(srv, len(reqs))
        for t, (ptr, us, st) in done.items():
            dirn, inp, passes, cb, shape, want = reqs[tickets[t]]
            assert st == 0 and us > 0
            got = bpc.as_tensor(ptr, want.numel()).clone()
            assert torch.equal(got, want.view(-1)), f"request {tickets[t]} differs from its result alone"
            srv.release(ptr)
        # a sample of the streams against the oracle as well
        for passes, cb, levels, img in cases[:4]:
            lut_np = oracle_mod.load_luts(lut_folder(passes), passes, 5)
            want = oracle_mod.encode(img, lut_np, passes, 5, cb)
            d = torch.from_numpy(img).cuda()
            t = srv.submit(bpc.CODE, d, ids[passes], cb)
            (ptr, _, st), = collect(srv, 1).values()
            np.testing.assert_array_equal(bpc.as_tensor(ptr, img.size).cpu().numpy(), want)
            srv.release(ptr)
        assert srv.state()["bytes_used"] == 0
    finally:
        srv.close()


def test_large_requests_work_ordered(bpc, luts):
    """Requests of more than two warp waves run the work-ordered coder with its
    scratch beside the output in the arena: same words as the one-request
    raster-order calls, and the arena is empty again after release."""
    import torch
    d = bpc_synth.synthetic_coefficients_gpu(8192, 5, 17, amp=60.0, nrect=100)
    want, st = alone(bpc, torch, bpc.CODE, d, luts[3], 64)
    srv = bpc.Server(2 * d.numel() * 4 + (8 << 20), 2)
    try:
        lid = srv.register_lut(luts[3])
        t_enc = srv.submit(bpc.CODE, d.view(-1), lid, 64, shape=d.shape)
        t_dec = srv.submit(bpc.DECODE, want.view(-1), lid, 64, shape=d.shape)
        got = collect(srv, 2)
        ptr, _, s_enc = got[t_enc]
        assert s_enc == st
        assert torch.equal(bpc.as_tensor(ptr, d.numel()), want.view(-1))
        srv.release(ptr)
        ptr, _, s_dec = got[t_dec]
        dec_alone, s_alone = alone(bpc, torch, bpc.DECODE, want, luts[3], 64)
        assert s_dec == s_alone
        assert torch.equal(bpc.as_tensor(ptr, d.numel()), dec_alone.view(-1))
        srv.release(ptr)
        assert srv.state()["bytes_used"] == 0
    finally:
        srv.close()


def test_budget_admission_in_order(bpc, luts):
    import torch
    img = bpc_synth.synthetic_coefficients(1024, 5, 7, amp=30, nrect=10)
    d = torch.from_numpy(img).cuda()
    one = img.size * 4
    srv = bpc.Server(2 * one + 1024, 4)  # room for two outputs at a time
    try:
        lid = srv.register_lut(luts[2])
        tickets = [srv.submit(bpc.CODE, d, lid, 64) for _ in range(6)]
        assert tickets == sorted(tickets)
        finished = []
        ref = None
        while len(finished) < 6:
            st = srv.state()
            assert st["bytes_used"] <= 2 * one + 1024
            assert st["in_flight"] <= 2
            batch = srv.poll(8, 2000)
            for t, ptr, us, s in batch:
                assert s == 0
                out = bpc.as_tensor(ptr, img.size).clone()
                ref = out if ref is None else ref
                assert torch.equal(out, ref)
                finished.append(t)
                srv.release(ptr)  # frees room for the next queued request
        # first come, first served: with room for two outputs, the i-th
        # request to finish is one of the first i + 2 submitted (two admitted
        # requests run concurrently and may finish in either order)
        assert sorted(finished) == tickets
        assert all(t <= tickets[min(i + 1, 5)] for i, t in enumerate(finished))
    finally:
        srv.close()


def test_failures_end_with_a_status(bpc, luts):
    import torch
    img = bpc_synth.synthetic_coefficients(512, 5, 9, amp=30, nrect=10)
    d = torch.from_numpy(img).cuda()
    srv = bpc.Server(img.size * 4, 1)  # one output at a time
    try:
        lid = srv.register_lut(luts[3])
        big = torch.zeros(1024 * 1024, dtype=torch.int32, device="cuda")
        assert srv.submit(bpc.CODE, big, lid, 64, shape=(1024, 1024)) == bpc.ERR_TOO_LARGE
        assert srv.submit(bpc.CODE, d, 99, 64) == bpc.ERR_ARG
        t0 = srv.submit(bpc.CODE, d, lid, 64)
        t1 = srv.submit(bpc.CODE, d, lid, 64)  # waits: t0's output holds the budget
        time.sleep(0.05)
        assert srv.cancel(t1) == bpc.OK
        assert srv.cancel(t1) == bpc.ERR_ARG
        res = collect(srv, 2)
        assert res[t1][0] == 0 and res[t1][2] == bpc.ERR_CANCELLED
        ptr0, _, st0 = res[t0]
        assert st0 == 0
        stream = bpc.as_tensor(ptr0, img.size).clone()
        srv.release(ptr0)
        bad = stream.clone()
        bad[4096 * 3] = 40  # MSB word outside 0..32
        t2 = srv.submit(bpc.DECODE, bad, lid, 64, shape=img.shape)
        (ptr2, _, st2), = collect(srv, 1).values()
        assert st2 & bpc.ST_BAD_STREAM
        dec = bpc.as_tensor(ptr2, img.size).view(img.shape).cpu().numpy()
        srv.release(ptr2)
        ncbx = img.shape[1] // 64
        y0, x0 = (3 // ncbx) * 64, (3 % ncbx) * 64
        assert not dec[y0:y0 + 64, x0:x0 + 64].any()  # the bad codeblock decodes to zeros
        dec[y0:y0 + 64, x0:x0 + 64] = img[y0:y0 + 64, x0:x0 + 64]
        np.testing.assert_array_equal(dec, img)  # the others are intact
        assert t2 > t1
    finally:
        srv.close()
