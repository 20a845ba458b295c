"""Regenerate the committed fixtures in tests/golden/ from the reference repo.

Run in a container that has the reference checkout (read-only):

    python tests/golden/make_fixtures.py /path/to/CUDA_BPC-PaCo

It writes
  * sample_headers.npy  -- (1024, 6) int32: file index, level, subband, MSBP,
    x0, y0 for every codeblock file of sample_image/sample_image.zip, placed
    as source/main_example.cu:71-179 (load_Data) places them;
  * sample_subset.npz   -- the 64x64 coefficient blocks of a subset of those
    codeblocks (all of levels 5..3 plus every 16th finer block) with their
    file indices, so a 2048x2048 image can be rebuilt on machines without the
    reference (the other codeblocks are left zero);
  * luts/{2,3}_coding_pass/*.txt -- the probability tables, byte-identical
    (the bitstream is defined by them; the codec cannot use other values);
  * lut_naive_{2,3}pass_L5.npy -- the tables placed directly at
    (group*15 + bitplane)*N + ctx with 64 in the planes a group does not list
    (except the last group): the layout load_LUTs must produce for these files
    if its fill rule's overwrite of the last listed plane changes nothing.
"""
from __future__ import annotations

import os
import shutil
import sys
import zipfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def sample_placement(X: int, Y: int, levels: int, cb: int):
    """(x0, y0) of codeblock file k in load_Data order (main_example.cu:71-179):
    the LL band first, then for level = levels..1 the HL, LH and HH bands, each
    in raster order of codeblocks."""
    pos = []
    sx, sy = X >> levels, Y >> levels
    for j in range(0, sy, cb):
        for i in range(0, sx, cb):
            pos.append((i, j))
    for lv in range(levels, 0, -1):
        sx, sy = X >> lv, Y >> lv
        for (ox, oy) in ((sx, 0), (0, sy), (sx, sy)):
            for j in range(0, sy, cb):
                for i in range(0, sx, cb):
                    pos.append((ox + i, oy + j))
    return pos


def read_sample(zip_path: str):
    z = zipfile.ZipFile(zip_path)
    heads, blocks = {}, {}
    for n in z.namelist():
        k = int(os.path.basename(n).split(".")[0])
        first, rest = z.read(n).decode().split("\n", 1)
        a = first.split()
        heads[k] = (int(a[0]), int(a[1]), int(a[3]))
        v = np.array(rest.split(), dtype=np.int32)
        assert v.size == 64 * 64
        blocks[k] = v.reshape(64, 64)
    return heads, blocks


def naive_lut(folder: str, passes: int, levels: int = 5, nbp: int = 15) -> np.ndarray:
    def rows(name, n):
        out = []
        for line in open(os.path.join(folder, name)):
            t = line.replace(":", " ").split()
            if t:
                out.append((int(t[2]), [int(v) for v in t[3:3 + n]]))
        return out

    secs = [("ref.txt", 1), ("sig.txt", 9), ("sign.txt", 4)]
    if passes == 3:
        secs += [("cp_sig.txt", 9), ("cp_sign.txt", 4)]
    parts = []
    for name, n in secs:
        size = 3 * nbp * n * levels + nbp * n
        sec = np.zeros(size, np.int32)
        groups = []
        prev = 10 ** 9
        for bp, vals in rows(name, n):
            if bp <= prev:
                groups.append({})
            prev = bp
            groups[-1][bp] = vals
        for g, planes in enumerate(groups):
            for bp in range(nbp):
                if bp in planes:
                    sec[(g * nbp + bp) * n:(g * nbp + bp) * n + n] = planes[bp]
                elif g + 1 < len(groups):
                    # planes a group does not list read 64 (p = 1/2), except in
                    # the last group, which nothing fills
                    sec[(g * nbp + bp) * n:(g * nbp + bp) * n + n] = 64
        parts.append(sec)
    return np.concatenate(parts)


def main(ref_root: str) -> None:
    heads, blocks = read_sample(os.path.join(ref_root, "sample_image", "sample_image.zip"))
    pos = sample_placement(2048, 2048, 5, 64)
    assert len(pos) == len(heads) == 1024
    tab = np.array([(k, heads[k][0], heads[k][1], heads[k][2], pos[k][0], pos[k][1]) for k in range(1024)],
                   np.int32)
    np.save(os.path.join(HERE, "sample_headers.npy"), tab)
    keep = list(range(64)) + list(range(64, 1024, 16))
    np.savez_compressed(os.path.join(HERE, "sample_subset.npz"), index=np.array(keep, np.int32),
                        blocks=np.stack([blocks[k] for k in keep]).astype(np.int16))
    for p in ("2_coding_pass", "3_coding_pass"):
        src = os.path.join(ref_root, "LUTs", p)
        dst = os.path.join(HERE, "luts", p)
        os.makedirs(dst, exist_ok=True)
        for f in sorted(os.listdir(src)):
            shutil.copyfile(os.path.join(src, f), os.path.join(dst, f))
        passes = int(p[0])
        np.save(os.path.join(HERE, f"lut_naive_{passes}pass_L5.npy"), naive_lut(src, passes))


def sample_image_from_subset() -> np.ndarray:
    """2048x2048 image holding the committed subset blocks at their sample
    positions, zeros elsewhere (those codeblocks are all-zero, MSB = 32)."""
    tab = np.load(os.path.join(HERE, "sample_headers.npy"))
    d = np.load(os.path.join(HERE, "sample_subset.npz"))
    img = np.zeros((2048, 2048), np.int32)
    for k, blk in zip(d["index"], d["blocks"]):
        x0, y0 = tab[k, 4], tab[k, 5]
        img[y0:y0 + 64, x0:x0 + 64] = blk
    return img


def sample_image_full(ref_root: str) -> np.ndarray:
    _, blocks = read_sample(os.path.join(ref_root, "sample_image", "sample_image.zip"))
    img = np.zeros((2048, 2048), np.int32)
    for k, (x0, y0) in enumerate(sample_placement(2048, 2048, 5, 64)):
        img[y0:y0 + 64, x0:x0 + 64] = blocks[k]
    return img


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BPC_REFERENCE_DIR", "/root/reference"))
