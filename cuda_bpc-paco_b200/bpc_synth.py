"""Seeded synthetic wavelet-coefficient inputs for the BPC-PaCo codec.

The reference ships one pre-transformed 2048x2048 sample and no generator; the
benchmark workloads are synthetic images of the shapes the benchmark names:

  * an 8-bit image: 4 random low-frequency sinusoids + Gaussian-blurred
    uniform noise (sigma 1.5, amplitude `amp`) + `nrect` sharp-edged constant
    rectangles, clipped to [0, 255];
  * a reversible CDF 5/3 integer lifting DWT (JPEG 2000 style, DC level shift
    by 128) with `levels` levels in Mallat layout: LL top-left, HL top-right
    (high-pass along x), LH bottom-left, HH bottom-right -- the layout the
    reference's subband finder assumes (source/BPC_PaCo.cu:84-111);
  * stored as a raster int32 array (two's complement; the coder converts to
    sign-magnitude internally).

Also an i.i.d. Laplacian coefficient field (scale 2**(level+3) per subband) for
the every-bitplane stress case.  Everything is numpy; it is input preparation,
not part of the coding path.
"""
from __future__ import annotations

import numpy as np


def _gauss_kernel(sigma: float) -> np.ndarray:
    r = int(np.ceil(4 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-(x * x) / (2 * sigma * sigma))
    return (k / k.sum()).astype(np.float32)


def _blur(a: np.ndarray, sigma: float) -> np.ndarray:
    k = _gauss_kernel(sigma)
    r = k.size // 2
    out = np.zeros_like(a)
    p = np.pad(a, ((0, 0), (r, r)), mode="reflect")
    for i, w in enumerate(k):
        out += w * p[:, i:i + a.shape[1]]
    p = np.pad(out, ((r, r), (0, 0)), mode="reflect")
    out2 = np.zeros_like(a)
    for i, w in enumerate(k):
        out2 += w * p[i:i + a.shape[0], :]
    return out2


def make_image(side: int, seed: int, amp: float = 20.0, nrect: int = 30, height: int | None = None) -> np.ndarray:
    """uint8 synthetic image (height x side)."""
    H = side if height is None else height
    W = side
    rng = np.random.default_rng(seed)
    y = np.arange(H, dtype=np.float32)[:, None]
    x = np.arange(W, dtype=np.float32)[None, :]
    img = np.full((H, W), 128.0, np.float32)
    for _ in range(4):
        a = rng.uniform(10.0, 35.0)
        fx = rng.uniform(0.3, 4.0) / W
        fy = rng.uniform(0.3, 4.0) / H
        ph = rng.uniform(0, 2 * np.pi)
        img += a * np.sin(2 * np.pi * (fx * x + fy * y) + ph).astype(np.float32)
    noise = rng.uniform(-amp, amp, size=(H, W)).astype(np.float32)
    img += _blur(noise, 1.5)
    for _ in range(nrect):
        w = int(rng.integers(max(2, W // 64), max(3, W // 5)))
        h = int(rng.integers(max(2, H // 64), max(3, H // 5)))
        x0 = int(rng.integers(0, W - w))
        y0 = int(rng.integers(0, H - h))
        img[y0:y0 + h, x0:x0 + w] += rng.uniform(-80.0, 80.0)
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def _fwd53_axis0(a: np.ndarray) -> np.ndarray:
    """One reversible 5/3 lifting step along axis 0 (even length); returns
    [low; high] stacked along axis 0."""
    n = a.shape[0]
    assert n % 2 == 0 and n >= 2
    even = a[0::2]
    odd = a[1::2]
    # symmetric extension: x[n] = x[n-2]
    even_next = np.concatenate([even[1:], even[-1:]], axis=0)
    d = odd - np.floor_divide(even + even_next, 2)
    d_prev = np.concatenate([d[:1], d[:-1]], axis=0)
    s = even + np.floor_divide(d_prev + d + 2, 4)
    return np.concatenate([s, d], axis=0)


def _inv53_axis0(a: np.ndarray) -> np.ndarray:
    n = a.shape[0]
    h = n // 2
    s = a[:h]
    d = a[h:]
    d_prev = np.concatenate([d[:1], d[:-1]], axis=0)
    even = s - np.floor_divide(d_prev + d + 2, 4)
    even_next = np.concatenate([even[1:], even[-1:]], axis=0)
    odd = d + np.floor_divide(even + even_next, 2)
    out = np.empty_like(a)
    out[0::2] = even
    out[1::2] = odd
    return out


def dwt53(img: np.ndarray, levels: int) -> np.ndarray:
    """Forward reversible CDF 5/3 DWT, Mallat layout, int32 output."""
    c = img.astype(np.int64) - 128
    H, W = c.shape
    for lv in range(levels):
        h, w = H >> lv, W >> lv
        sub = c[:h, :w]
        sub = _fwd53_axis0(sub.T).T  # rows: low | high along x
        sub = _fwd53_axis0(sub)  # columns: low over high along y
        c[:h, :w] = sub
    return c.astype(np.int32)


def idwt53(coef: np.ndarray, levels: int) -> np.ndarray:
    c = coef.astype(np.int64)
    H, W = c.shape
    for lv in reversed(range(levels)):
        h, w = H >> lv, W >> lv
        sub = c[:h, :w]
        sub = _inv53_axis0(sub)
        sub = _inv53_axis0(sub.T).T
        c[:h, :w] = sub
    return (c + 128).astype(np.int32)


def synthetic_coefficients(side: int, levels: int, seed: int, amp: float = 20.0, nrect: int = 30) -> np.ndarray:
    """Generator image -> 5/3 DWT -> int32 raster of coefficients."""
    return dwt53(make_image(side, seed, amp=amp, nrect=nrect), levels)


def laplacian_coefficients(side: int, levels: int, seed: int, max_plane: int = 15) -> np.ndarray:
    """i.i.d. Laplacian coefficients, scale 2**(level+3) per subband (level 0 =
    finest; LL uses level `levels`), magnitudes clipped below 2**(max_plane+1).
    The scale alone rarely reaches the top planes; laplacian_coefficients_gpu
    plants one top-plane coefficient per codeblock to make every codeblock
    code all of them."""
    rng = np.random.default_rng(seed)
    out = np.zeros((side, side), np.int64)
    for lv in range(levels):
        h = side >> (lv + 1)
        scale = 2.0 ** (lv + 3)
        for (y0, x0) in ((0, h), (h, 0), (h, h)):
            out[y0:y0 + h, x0:x0 + h] = np.rint(rng.laplace(0.0, scale, size=(h, h)))
    h = side >> levels
    out[:h, :h] = np.rint(rng.laplace(0.0, 2.0 ** (levels + 3), size=(h, h)))
    lim = (1 << (max_plane + 1)) - 1
    return np.clip(out, -lim, lim).astype(np.int32)


def make_image_gpu(side: int, seed: int, amp: float = 20.0, nrect: int = 30, device="cuda"):
    """The same kind of image as make_image, generated with torch on the GPU
    (its own RNG stream, so the pixels differ from make_image's): 4
    low-frequency sinusoids + blurred uniform noise + constant rectangles,
    clipped to [0, 255].  Returns an int32 tensor."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    H = W = side
    y = torch.arange(H, device=device, dtype=torch.float32)[:, None]
    x = torch.arange(W, device=device, dtype=torch.float32)[None, :]
    img = torch.full((H, W), 128.0, device=device)
    for _ in range(4):
        a, fx, fy, ph = (torch.rand(4, generator=g) * torch.tensor([25.0, 3.7, 3.7, 6.2832]) +
                         torch.tensor([10.0, 0.3, 0.3, 0.0])).tolist()
        img += a * torch.sin(2 * np.pi * (fx / W * x + fy / H * y) + ph)
    gg = torch.Generator(device=device).manual_seed(seed)
    noise = (torch.rand((1, 1, H, W), generator=gg, device=device) * 2 - 1) * amp
    k = torch.from_numpy(_gauss_kernel(1.5)).to(device)
    r = k.numel() // 2
    noise = torch.nn.functional.conv2d(torch.nn.functional.pad(noise, (r, r, 0, 0), mode="reflect"),
                                       k.view(1, 1, 1, -1))
    noise = torch.nn.functional.conv2d(torch.nn.functional.pad(noise, (0, 0, r, r), mode="reflect"),
                                       k.view(1, 1, -1, 1))
    img += noise[0, 0]
    rr = torch.rand((nrect, 5), generator=g).tolist()
    for (u0, u1, u2, u3, u4) in rr:
        w = int(max(2, W // 64) + u0 * (max(3, W // 5) - max(2, W // 64)))
        h = int(max(2, H // 64) + u1 * (max(3, H // 5) - max(2, H // 64)))
        x0 = int(u2 * (W - w))
        y0 = int(u3 * (H - h))
        img[y0:y0 + h, x0:x0 + w] += -80.0 + 160.0 * u4
    return torch.clamp(torch.round(img), 0, 255).to(torch.int32)


def synthetic_coefficients_gpu(side: int, levels: int, seed: int, amp: float = 20.0, nrect: int = 30, tmp=None):
    """make_image_gpu -> level shift -> 5/3 DWT on the GPU (bpc_dwt53_forward)."""
    import bpc_paco
    img = make_image_gpu(side, seed, amp, nrect) - 128
    bpc_paco.dwt53(img, levels, tmp=tmp)
    return img


def laplacian_coefficients_gpu(side: int, levels: int, seed: int, max_plane: int = 15, cb: int = 64,
                               device="cuda"):
    """The Laplacian field of laplacian_coefficients generated with torch on the
    GPU (its own RNG stream), plus, in every cb x cb codeblock, one coefficient
    at a random position with magnitude in [2**max_plane, 2**(max_plane+1))
    and a random sign: every codeblock then has MSB plane `max_plane` and codes
    all max_plane + 1 magnitude bitplanes.  Returns an int32 tensor."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    out = torch.empty((side, side), dtype=torch.float32, device=device)

    def lap(h, scale):
        u = torch.rand((h, h), generator=g, device=device) - 0.5
        return -scale * torch.sign(u) * torch.log1p(-2.0 * u.abs())

    for lv in range(levels):
        h = side >> (lv + 1)
        for (y0, x0) in ((0, h), (h, 0), (h, h)):
            out[y0:y0 + h, x0:x0 + h] = lap(h, 2.0 ** (lv + 3))
    h = side >> levels
    out[:h, :h] = lap(h, 2.0 ** (levels + 3))
    lim = (1 << (max_plane + 1)) - 1
    out = torch.clamp(torch.round(out), -lim, lim).to(torch.int32)
    n = side // cb
    pos = torch.randint(0, cb * cb, (n, n), generator=g, device=device)
    mag = torch.randint(1 << max_plane, 1 << (max_plane + 1), (n, n), generator=g, device=device, dtype=torch.int32)
    sgn = torch.randint(0, 2, (n, n), generator=g, device=device, dtype=torch.int32) * 2 - 1
    rows = (torch.arange(n, device=device)[:, None] * cb + pos // cb).reshape(-1)
    cols = (torch.arange(n, device=device)[None, :] * cb + pos % cb).reshape(-1)
    out[rows, cols] = (mag * sgn).reshape(-1)
    return out
