"""The request server's memory-budget allocator (bpc_arena.h), host code only:
a random sequence of allocations and releases against a byte-level model --
no overlap, first fit by address, every free neighbour merged, the whole
budget free again at the end.  Compiled here with g++; no GPU."""
import os
import subprocess

import numpy as np

from conftest import ROOT

DRIVER = r"""
#include <cstdio>
#include "bpc_arena.h"
int main() {
    bpc::Arena a;
    char op;
    unsigned long long x, y;
    while (std::scanf(" %c", &op) == 1) {
        if (op == 'i') { std::scanf("%llu", &x); a.init(x); }
        else if (op == 'a') {
            std::scanf("%llu", &x);
            size_t off = 0;
            if (a.alloc(x, &off)) std::printf("%zu\n", off); else std::printf("-1\n");
        } else if (op == 'r') { std::scanf("%llu %llu", &x, &y); a.release(x, y); }
        else if (op == 's') std::printf("%zu %zu %zu\n", a.used(), a.free_ranges(), a.largest_free());
        std::fflush(stdout);
    }
}
"""


def build(tmp_path):
    src = tmp_path / "arena_driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "arena_driver"
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "cuda_bpc-paco_b200", "csrc"),
                           str(src), "-o", str(exe)])
    return str(exe)


def first_fit(free, n):
    """Lowest offset with n free bytes (free ranges are kept merged, so this is
    the start of the first free range that is long enough)."""
    for i in range(len(free) - n + 1):
        if free[i:i + n].all():
            return i
    return -1


def test_random_alloc_release_matches_model(tmp_path):
    exe = build(tmp_path)
    rng = np.random.default_rng(11)
    size = 4096
    ops = [f"i {size}"]
    model = np.ones(size, bool)  # True = free
    live = []
    expected = []
    for _ in range(600):
        if live and rng.random() < 0.45:
            off, n = live.pop(int(rng.integers(len(live))))
            ops.append(f"r {off} {n}")
            model[off:off + n] = True
        else:
            n = int(rng.integers(1, 300))
            ops.append(f"a {n}")
            want = first_fit(model, n)
            expected.append(want)
            if want >= 0:
                model[want:want + n] = False
                live.append((want, n))
    for off, n in live:
        ops.append(f"r {off} {n}")
    ops.append("s")
    out = subprocess.run([exe], input="\n".join(ops) + "\n", capture_output=True, text=True, check=True).stdout
    lines = out.split()
    got = [int(v) for v in lines[:len(expected)]]
    assert got == expected
    used, ranges, largest = (int(v) for v in lines[len(expected):])
    assert (used, ranges, largest) == (0, 1, size)  # everything merged back into one range
