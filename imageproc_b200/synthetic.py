"""Seeded synthetic inputs for the template-matching workloads.

All randomness comes from numpy's PCG64 generator seeded explicitly, so a
(config, seed) pair always gives the same bytes on any machine with the same
numpy. The reference's own benches use a fixed pattern image
(`gray_bench_image`, src/utils.rs:671-680, pixel = x % 7 + y % 6); it is
provided as :func:`gray_bench_image`.

Workloads (image, template(s), mask):
  uniform_scene     512x512 i.i.d. U{0..255}; 16x16 crop + U{-4..4} noise
  blob_scene        1920x1080, 200 Gaussian blobs (sigma 5-80, amplitude
                    20-200) + U{-8..8} noise; 64x64 crop + brightness
                    U{-10..10}; mask Bernoulli(0.8) in {0,1}
  uneven_pairs      256 pairs, sides log-uniform 256..4096, template sides
                    U{8..128}, content as uniform_scene, method U{4}
  value_noise       3-octave value noise (lattice 64/16/4, weights
                    0.6/0.3/0.1) scaled to 0..255; 32x32 crops + U{-6..6}
  rect_scene        value noise + 500 axis-aligned rectangles of uniform
                    intensity; 48x48 crops + brightness U{-10..10} +
                    noise U{-6..6}
"""

from __future__ import annotations

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def clamp_u8(a) -> np.ndarray:
    return np.clip(np.rint(a), 0, 255).astype(np.uint8)


def gray_bench_image(width: int, height: int) -> np.ndarray:
    """The reference's bench image: pixel = x % 7 + y % 6."""
    x = np.arange(width) % 7
    y = np.arange(height) % 6
    return (y[:, None] + x[None, :]).astype(np.uint8)


def crop(image: np.ndarray, w: int, h: int, g: np.random.Generator):
    H, W = image.shape
    x = int(g.integers(0, W - w + 1))
    y = int(g.integers(0, H - h + 1))
    return image[y:y + h, x:x + w].astype(np.int32), (x, y)


def uniform_scene(W=512, H=512, tw=16, th=16, seed=0, noise=4):
    """512x512 U{0..255} image from `seed`; template = crop + U{-noise..noise}."""
    g = rng(seed)
    image = g.integers(0, 256, size=(H, W), dtype=np.uint8)
    t, loc = crop(image, tw, th, g)
    template = clamp_u8(t + g.integers(-noise, noise + 1, size=t.shape))
    return image, template, loc


def blob_scene(W=1920, H=1080, tw=64, th=64, seed=1, n_blobs=200, mask_p=0.8):
    g = rng(seed)
    acc = np.zeros((H, W), np.float64)
    for _ in range(n_blobs):
        cx, cy = g.uniform(0, W), g.uniform(0, H)
        sigma = g.uniform(5.0, 80.0)
        amp = g.uniform(20.0, 200.0)
        r = int(np.ceil(4 * sigma))
        x0, x1 = max(0, int(cx) - r), min(W, int(cx) + r + 1)
        y0, y1 = max(0, int(cy) - r), min(H, int(cy) + r + 1)
        xs = np.arange(x0, x1) - cx
        ys = np.arange(y0, y1) - cy
        gx = np.exp(-(xs * xs) / (2 * sigma * sigma))
        gy = np.exp(-(ys * ys) / (2 * sigma * sigma))
        acc[y0:y1, x0:x1] += amp * gy[:, None] * gx[None, :]
    image = clamp_u8(acc + g.integers(-8, 9, size=(H, W)))
    t, loc = crop(image, tw, th, g)
    template = clamp_u8(t + int(g.integers(-10, 11)))
    mask = (g.random((th, tw)) < mask_p).astype(np.uint8)
    return image, template, mask, loc


def value_noise(W, H, seed, lattices=(64, 16, 4), weights=(0.6, 0.3, 0.1), band=1024):
    """Multi-octave value noise in [0, 255] (u8): lattice values U[0,1),
    smoothstep-weighted bilinear interpolation, weighted octave sum."""
    g = rng(seed)
    grids = [g.random((H // L + 2, W // L + 2), dtype=np.float32) for L in lattices]
    out = np.empty((H, W), np.uint8)
    xs = np.arange(W)
    for y0 in range(0, H, band):
        y1 = min(H, y0 + band)
        ys = np.arange(y0, y1)
        acc = np.zeros((y1 - y0, W), np.float32)
        for grid, L, wt in zip(grids, lattices, weights):
            fx, fy = xs / L, ys / L
            ix, iy = fx.astype(np.int64), fy.astype(np.int64)
            tx, ty = (fx - ix).astype(np.float32), (fy - iy).astype(np.float32)
            sx, sy = tx * tx * (3 - 2 * tx), ty * ty * (3 - 2 * ty)
            g00 = grid[iy][:, ix]
            g01 = grid[iy][:, ix + 1]
            g10 = grid[iy + 1][:, ix]
            g11 = grid[iy + 1][:, ix + 1]
            top = g00 + (g01 - g00) * sx[None, :]
            bot = g10 + (g11 - g10) * sx[None, :]
            acc += wt * (top + (bot - top) * sy[:, None])
        out[y0:y1] = clamp_u8(acc * 255.0)
    return out


def value_noise_scene(W=4096, H=4096, n_templates=512, t=32, seed=4, noise=6):
    g = rng(seed + 1000)
    image = value_noise(W, H, seed)
    templates = np.empty((n_templates, t, t), np.uint8)
    locs = []
    for k in range(n_templates):
        c, loc = crop(image, t, t, g)
        templates[k] = clamp_u8(c + g.integers(-noise, noise + 1, size=c.shape))
        locs.append(loc)
    return image, templates, locs


def rect_scene(W=8192, H=8192, n_rects=500, n_templates=64, t=48, seed=5, max_side=256):
    """Value noise plus n_rects flat rectangles (sides U{8..max_side - 1},
    intensity U{0..255}) and n_templates t x t crops with a brightness offset
    in [-10, 10] and noise in [-6, 6]. With the default sides, 500 rectangles
    cover about 12 % of an 8192 x 8192 scene (sides up to 1024 would cover
    about 82 % and cut most templates from flat regions)."""
    g = rng(seed + 2000)
    image = value_noise(W, H, seed)
    for _ in range(n_rects):
        rw, rh = int(g.integers(8, max_side)), int(g.integers(8, max_side))
        x, y = int(g.integers(0, W - rw)), int(g.integers(0, H - rh))
        image[y:y + rh, x:x + rw] = np.uint8(g.integers(0, 256))
    templates = np.empty((n_templates, t, t), np.uint8)
    locs = []
    for k in range(n_templates):
        c, loc = crop(image, t, t, g)
        c = c + int(g.integers(-10, 11)) + g.integers(-6, 7, size=c.shape)
        templates[k] = clamp_u8(c)
        locs.append(loc)
    return image, templates, locs


def uneven_pairs(n=256, seed=3, lo=256, hi=4096, tmin=8, tmax=128):
    """List of (image, template, method) with per-pair seeds."""
    g = rng(seed)
    pairs = []
    for k in range(n):
        W = int(round(np.exp(g.uniform(np.log(lo), np.log(hi)))))
        H = int(round(np.exp(g.uniform(np.log(lo), np.log(hi)))))
        tw, th = int(g.integers(tmin, tmax + 1)), int(g.integers(tmin, tmax + 1))
        method = int(g.integers(0, 4))
        image, template, _ = uniform_scene(W, H, tw, th, seed=10_000 + k)
        pairs.append((image, template, method))
    return pairs
