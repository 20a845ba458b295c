"""Generate golden streams with the reference kernel itself, on a GPU box:

    make -C oracle ref            # in a container with the reference checkout
    python tests/golden/make_ref_golden.py OUT.npz    # on the GPU box

For each case it stores the input (int16 where it fits) and, per codeblock
slot, the reference's MSB word and codewords (the -1 fill is implied), so the
CPU oracle can be checked against the reference without a GPU
(tests/test_golden.py).  The cases cover both pass modes, all-zero codeblocks
(MSB = 32), codeblocks straddling subbands, a single-coefficient codeblock and
bitplane 15 (LUT reads past the loader's array).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "cuda_bpc-paco_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import bpc_synth  # noqa: E402
import oracle  # noqa: E402
import ref_run  # noqa: E402


def cases():
    out = {}
    out["synth256_a40"] = bpc_synth.synthetic_coefficients(256, 5, 3, amp=40)
    out["synth512_a20"] = bpc_synth.synthetic_coefficients(512, 5, 5, amp=20)
    mixed = bpc_synth.synthetic_coefficients(512, 5, 6, amp=40)
    mixed[256:, 256:] = 0  # all-zero codeblocks in the HH band of level 0
    mixed[300, 400] = -3  # one coefficient in an otherwise empty codeblock
    out["mixed512_zero"] = mixed
    out["straddle192x384"] = np.ascontiguousarray(bpc_synth.synthetic_coefficients(3072, 5, 21, amp=30)[:192, :384])
    lap = bpc_synth.laplacian_coefficients(256, 5, 4)
    lap[0, 0] = 40000
    out["laplace256_p15"] = lap
    return out


def main(path):
    res = {}
    for name, img in cases().items():
        for passes in (2, 3):
            lut = oracle.load_luts(os.path.join(HERE, "luts", f"{passes}_coding_pass"), passes, 5)
            s = ref_run.ref_encode(img, lut, passes).reshape(-1, 4096)
            n = (s[:, 1:] != -1).sum(1)
            words = np.concatenate([s[k, :1 + n[k]] for k in range(s.shape[0])])
            assert all((s[k, 1 + n[k]:] == -1).all() for k in range(s.shape[0]))
            res[f"{name}/p{passes}/count"] = n.astype(np.int32)
            res[f"{name}/p{passes}/words"] = words.astype(np.int32)
        res[f"{name}/input"] = img.astype(np.int16) if np.abs(img).max() < 32768 else img
    np.savez_compressed(path, **res)
    print("wrote", path, {k: v.shape for k, v in res.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "ref_golden.npz"))
