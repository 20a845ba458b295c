"""Batched persistent form: mixed sizes, DWT levels, pass counts and codeblock
sizes in one call; the compact container equals, word for word, the MSB and
codewords of each image's slot stream from the oracle; decoding it returns
every image."""
import numpy as np
import pytest

import bpc_synth
from conftest import lut_folder

pytestmark = pytest.mark.gpu

IMAGES = [  # X, Y, levels, passes, cb
    (512, 512, 5, 3, 64),
    (256, 384, 3, 2, 32),
    (384, 256, 4, 3, 32),
    (512, 256, 6, 2, 64),
    (192, 192, 3, 3, 64),
    (256, 256, 6, 2, 32),
]


def make_inputs():
    imgs = []
    for k, (X, Y, lv, ps, cb) in enumerate(IMAGES):
        side = max(X, Y)
        img = bpc_synth.synthetic_coefficients(side, lv, 100 + k, amp=30)[:Y, :X]
        imgs.append(np.ascontiguousarray(img))
    return imgs


@pytest.fixture(scope="module")
def batch_setup(bpc, oracle_mod):
    import torch
    b = bpc.Batch(IMAGES, {2: lut_folder(2), 3: lut_folder(3)})
    imgs = make_inputs()
    want_words, want_dec, want_st = [], [], 0
    for img, (X, Y, lv, ps, cb) in zip(imgs, IMAGES):
        lut = oracle_mod.load_luts(lut_folder(ps), ps, lv)
        s, st = oracle_mod.encode(img, lut, ps, lv, cb, with_status=True)
        want_words += bpc.slots_to_compact(s, cb)
        # 6 levels with the 5-level tables leave zero probabilities: some
        # codeblocks overflow their slot (flagged); their decode is the oracle's
        want_dec.append(oracle_mod.decode(s, img.shape, lut, ps, lv, cb))
        want_st |= int(np.bitwise_or.reduce(st))
    d_in = [torch.from_numpy(i).cuda() for i in imgs]
    yield b, imgs, d_in, (want_words, want_dec, want_st)
    b.close()


def run_batch(b, d_in, torch):
    compact = torch.full((b.words,), 777, dtype=torch.int32, device="cuda")
    offs = torch.zeros(b.codeblocks + 1, dtype=torch.int64, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    b.encode(d_in, compact, offs, st)
    out = [torch.empty_like(t) for t in d_in]
    b.decode(compact, offs, out, st)
    torch.cuda.synchronize()
    return compact.cpu().numpy(), offs.cpu().numpy(), [o.cpu().numpy() for o in out], st.item()


@pytest.mark.parametrize("schedule,tuning", [
    (None, None), ((4, 7, 1, True), None), ((2, 3, 4, False), None), ((1, 2, 8, True), None),
    ((8, 14, 2, True), (2, 2, True, True, False, True)), ((2, 3, 4, True), (8, 8, True, False, True, False)),
    ((2, 3, 1, False), (4, 8, False, True, True, True))])
def test_batch_matches_oracle(batch_setup, schedule, tuning):
    """Every schedule (CTAs per SM, codeblocks per item, graph; warps per CTA
    and cost-ordered queues) gives the same container and decode."""
    import torch
    b, imgs, d_in, (want_words, want_dec, want_st) = batch_setup
    b.set_tuning(*(tuning or (4, 4, False, False, False, False)))
    if schedule:
        b.set_schedule(*schedule)
    for _ in range(2):  # second call replays the captured graph
        compact, offs, out, st = run_batch(b, d_in, torch)
        assert st == want_st
        assert offs[0] == 0 and len(offs) == len(want_words) + 1
        for g, w in enumerate(want_words):
            np.testing.assert_array_equal(compact[offs[g]:offs[g + 1]], w, err_msg=f"codeblock {g}")
        for o, d in zip(out, want_dec):
            np.testing.assert_array_equal(o, d)
        for o, i, (X, Y, lv, ps, cb) in zip(out, imgs, IMAGES):
            if lv <= 5:
                np.testing.assert_array_equal(o, i)


def test_batch_tune(batch_setup):
    import torch
    b, imgs, d_in, (want_words, want_dec, want_st) = batch_setup
    compact = torch.empty(b.words, dtype=torch.int32, device="cuda")
    offs = torch.zeros(b.codeblocks + 1, dtype=torch.int64, device="cuda")
    out = [torch.empty_like(t) for t in d_in]
    us = b.tune(d_in, compact, offs, out)
    assert us > 0
    ce, cd, per, graph = b.schedule()
    we, wd, _, _, _, _ = b.tuning()
    assert we in (2, 4, 8) and wd in (2, 4, 8)
    assert 1 <= ce * we <= 16 and 1 <= cd * wd <= 28 and per in (1, 2, 4, 8)
    compact, offs, out, st = run_batch(b, d_in, torch)
    for o, d in zip(out, want_dec):
        np.testing.assert_array_equal(o, d)
