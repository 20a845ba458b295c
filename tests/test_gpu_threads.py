"""Host threads coding at once through the device entry points, each with its
own stream and a LUT of another length (2-pass and 3-pass tables need
different shared memory), agree with the same calls made one at a time."""
import threading

import numpy as np
import pytest

import bpc_synth
from conftest import lut_folder

pytestmark = pytest.mark.gpu


def test_threads_with_different_luts(bpc):
    import torch
    side, levels, cb = 512, 5, 64
    img = bpc_synth.synthetic_coefficients(side, levels, 5, amp=40.0, nrect=20)
    luts = {p: bpc.DeviceLut(lut_folder(p), p, levels) for p in (2, 3)}
    try:
        d = torch.from_numpy(img).cuda()
        want, want_st = {}, {}
        for p, lut in luts.items():
            s = torch.empty_like(d)
            o = torch.empty_like(d)
            st = torch.zeros(1, dtype=torch.int32, device="cuda")
            bpc.encode_device(d, s, lut, cb, st)
            bpc.decode_device(s, o, lut, cb, st)
            torch.cuda.synchronize()
            want[p], want_st[p] = s.cpu().numpy(), st.item()
            assert want_st[p] != 0 or np.array_equal(o.cpu().numpy(), img)
        errors = []

        def worker(p, reps=40):
            try:
                stream = torch.cuda.Stream()
                s = torch.empty_like(d)
                o = torch.empty_like(d)
                st = torch.zeros(1, dtype=torch.int32, device="cuda")
                for _ in range(reps):
                    bpc.encode_device(d, s, luts[p], cb, st, cuda_stream=stream.cuda_stream)
                    bpc.decode_device(s, o, luts[p], cb, st, cuda_stream=stream.cuda_stream)
                stream.synchronize()
                if not np.array_equal(s.cpu().numpy(), want[p]):
                    errors.append(f"{p}-pass stream differs")
                if want_st[p] == 0 and not np.array_equal(o.cpu().numpy(), img):
                    errors.append(f"{p}-pass decode differs")
                if st.item() != want_st[p]:
                    errors.append(f"{p}-pass status {st.item()} against {want_st[p]}")
            except Exception as e:  # reported below, on the test's thread
                errors.append(repr(e))

        ts = [threading.Thread(target=worker, args=(p,)) for p in (2, 3, 2, 3)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        assert not errors, errors
    finally:
        for lut in luts.values():
            lut.close()
