"""The no-allocation encode (bpc_encode_compact_noalloc) against the
allocating batch encode of the same one-image batch.

Some callers of this codec may not allocate device memory while they code (a
fixed device budget already owned by their own pool, a stream an allocation
would stall, a host that only hands out device pointers); this entry point
serves them from a fixed scratch array inside the library.  Its output must be
exactly what the regular entry point produces, on two calls in a row (the
second call finds the first call's leftovers in the shared array).  The file
is named to run last so that a failure here cannot stop the rest of the GPU
suite."""
import numpy as np
import pytest

import bpc_synth
from conftest import lut_folder

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("passes,cb,side,levels", [(3, 64, 2048, 5), (2, 32, 1024, 4)])
def test_noalloc_matches_batch_encode(bpc, passes, cb, side, levels):
    import torch
    img = bpc_synth.synthetic_coefficients(side, levels, 31 + passes, amp=40)
    d_img = torch.from_numpy(img).cuda()
    # the regular (allocating) entry point: a one-image batch
    b = bpc.Batch([(side, side, levels, passes, cb)], {passes: lut_folder(passes)})
    ref_c = torch.full((b.words,), -7, dtype=torch.int32, device="cuda")
    ref_o = torch.zeros(b.codeblocks + 1, dtype=torch.int64, device="cuda")
    ref_s = torch.zeros(1, dtype=torch.int32, device="cuda")
    b.encode([d_img], ref_c, ref_o, ref_s)
    torch.cuda.synchronize()
    want_o = ref_o.cpu().numpy()
    want_c = ref_c.cpu().numpy()[:want_o[-1]]
    want_s = ref_s.item()
    b.close()
    lut = bpc.DeviceLut(lut_folder(passes), passes, levels)
    try:
        for call in range(2):
            c = torch.full((img.size,), 12345, dtype=torch.int32, device="cuda")
            o = torch.full((want_o.size,), -1, dtype=torch.int64, device="cuda")
            s = torch.zeros(1, dtype=torch.int32, device="cuda")
            rc = bpc.encode_compact_noalloc(d_img, c, o, lut, cb, s)
            torch.cuda.synchronize()
            assert rc == 0, f"call {call}: {bpc.status_string(rc)}"
            np.testing.assert_array_equal(o.cpu().numpy(), want_o, err_msg=f"offsets, call {call}")
            np.testing.assert_array_equal(c.cpu().numpy()[:want_o[-1]], want_c, err_msg=f"container, call {call}")
            assert s.item() == want_s
    finally:
        lut.close()


def test_noalloc_rejects_oversized_image(bpc):
    import torch
    lut = bpc.DeviceLut(lut_folder(2), 2, 5)
    try:
        big = torch.zeros((2048, 4096), dtype=torch.int32, device="cuda")
        c = torch.empty(16, dtype=torch.int32, device="cuda")
        o = torch.empty(16, dtype=torch.int64, device="cuda")
        assert bpc.encode_compact_noalloc(big, c, o, lut, 64) == bpc.ERR_TOO_LARGE
    finally:
        lut.close()
