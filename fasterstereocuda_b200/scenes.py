"""Seeded synthetic stereo pairs with the shapes and statistics of the benchmark configurations.

The published benchmark data (Cone, KITTI, Building) is not available here; these generators
stand in for it with the sizes, disparity ranges and textures the configurations describe.
Everything is a deterministic function of the seed (numpy PCG64).

    cone_like(seed)        450x375, 8 planar patches in [2,60], blurred noise + 6 gradient patches
    kitti_like(seed)       1242x375, ground plane 0->55 + 12 boxes in [5,50], 20% flat texture
    building_like(seed)    4800x3409, 5-octave fractal texture, 40 planes in [0,250]
    planar_pair(seed,w,h)  any size, planar scene as cone_like (batched configuration)
"""
from __future__ import annotations

import numpy as np
from scipy.ndimage import gaussian_filter


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _blurred_noise(rng, h, w, sigma=1.5):
    img = rng.uniform(0.0, 255.0, size=(h, w))
    img = gaussian_filter(img, sigma)
    lo, hi = img.min(), img.max()
    return (img - lo) / max(hi - lo, 1e-6) * 255.0


def _gradient_patches(rng, img, n):
    h, w = img.shape
    for _ in range(n):
        pw, ph = rng.integers(w // 10, w // 3), rng.integers(h // 10, h // 3)
        x0, y0 = rng.integers(0, w - pw), rng.integers(0, h - ph)
        gx, gy = rng.uniform(-2.0, 2.0, size=2)
        base = rng.uniform(40, 215)
        yy, xx = np.mgrid[0:ph, 0:pw]
        img[y0:y0 + ph, x0:x0 + pw] = 0.5 * img[y0:y0 + ph, x0:x0 + pw] + 0.5 * (base + gx * xx + gy * yy)
    return img


def _planar_disparity(rng, h, w, n_planes, lo, hi):
    """Voronoi partition into n_planes cells, each a plane clipped to [lo, hi]."""
    seeds = np.stack([rng.uniform(0, w, n_planes), rng.uniform(0, h, n_planes)], 1)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    best = np.full((h, w), np.inf)
    lab = np.zeros((h, w), np.int32)
    for i, (sx, sy) in enumerate(seeds):
        dist = (xx - sx) ** 2 + (yy - sy) ** 2
        m = dist < best
        best[m] = dist[m]
        lab[m] = i
    d = np.zeros((h, w))
    for i in range(n_planes):
        c = rng.uniform(lo, hi)
        a = rng.uniform(-0.3, 0.3) * (hi - lo) / max(w, 1)
        b = rng.uniform(-0.3, 0.3) * (hi - lo) / max(h, 1)
        m = lab == i
        d[m] = c + a * (xx[m] - seeds[i, 0]) + b * (yy[m] - seeds[i, 1])
    return np.clip(d, lo, hi)


def _warp_right(left, disp, rng, noise_sigma):
    """Right view: forward-splat left pixels to x - d (nearest surface wins), fill occlusion
    holes from the farther (background) neighbour, sample the left image there, add noise."""
    h, w = left.shape
    xs = np.arange(w)[None, :].repeat(h, 0)
    xr = np.rint(xs - disp).astype(np.int64)
    valid = (xr >= 0) & (xr < w)
    dr = np.full((h, w), -1.0)
    rows = np.arange(h)[:, None].repeat(w, 1)
    flat = rows[valid] * w + xr[valid]
    np.maximum.at(dr.reshape(-1), flat, disp[valid])
    # fill holes: nearest filled disparity to the left and to the right; take the smaller (background)
    filled = dr >= 0
    idx = np.where(filled, xs, -1)
    left_idx = np.maximum.accumulate(idx, axis=1)
    idx_r = np.where(filled, xs, w)
    right_idx = np.minimum.accumulate(idx_r[:, ::-1], axis=1)[:, ::-1]
    dl_ = np.where(left_idx >= 0, np.take_along_axis(dr, np.clip(left_idx, 0, w - 1), 1), np.inf)
    dr_ = np.where(right_idx < w, np.take_along_axis(dr, np.clip(right_idx, 0, w - 1), 1), np.inf)
    bg = np.minimum(dl_, dr_)
    bg[np.isinf(bg)] = 0.0
    dr = np.where(filled, dr, bg)
    src = np.clip(xs + dr, 0, w - 1)
    x0 = np.floor(src).astype(np.int64)
    x1 = np.minimum(x0 + 1, w - 1)
    f = src - x0
    right = (1 - f) * np.take_along_axis(left, x0, 1) + f * np.take_along_axis(left, x1, 1)
    right = right + rng.normal(0.0, noise_sigma, size=right.shape)
    return np.clip(np.rint(right), 0, 255).astype(np.uint8)


def planar_pair(seed: int, width: int, height: int, n_planes: int = 8, dmin: float = 2.0, dmax: float = 60.0,
                noise: float = 2.0):
    """Blurred noise + 6 gradient patches, piecewise-planar disparity, warped right view."""
    rng = _rng(seed)
    tex = _gradient_patches(rng, _blurred_noise(rng, height, width), 6)
    left = np.clip(np.rint(tex), 0, 255).astype(np.uint8)
    disp = _planar_disparity(rng, height, width, n_planes, dmin, dmax)
    right = _warp_right(left.astype(np.float64), disp, rng, noise)
    return left, right, disp.astype(np.float32)


def cone_like(seed: int = 0):
    """450x375, D=64 scene (first configuration)."""
    return planar_pair(seed, 450, 375)


def kitti_like(seed: int = 1, width: int = 1242, height: int = 375):
    """Driving-like scene: ground plane rising 0->55 toward the bottom rows plus 12 boxes in [5,50];
    blurred noise texture with 20% of the pixels in flat low-texture regions; N(0,3) noise."""
    rng = _rng(seed)
    tex = _blurred_noise(rng, height, width)
    # flat regions: random rectangles until ~20% of the pixels are flat
    flat = np.zeros((height, width), bool)
    while flat.mean() < 0.2:
        pw, ph = rng.integers(width // 40, width // 8), rng.integers(height // 40, height // 8)
        x0, y0 = rng.integers(0, width - pw), rng.integers(0, height - ph)
        flat[y0:y0 + ph, x0:x0 + pw] = True
    tex[flat] = gaussian_filter(tex, 6.0)[flat] * 0.2 + 100.0
    left = np.clip(np.rint(tex), 0, 255).astype(np.uint8)
    yy = np.arange(height, dtype=np.float64)[:, None]
    disp = np.repeat(55.0 * yy / max(height - 1, 1), width, 1)
    for _ in range(12):
        bw, bh = rng.integers(width // 30, width // 8), rng.integers(height // 12, height // 3)
        x0, y0 = rng.integers(0, width - bw), rng.integers(0, height - bh)
        disp[y0:y0 + bh, x0:x0 + bw] = np.maximum(disp[y0:y0 + bh, x0:x0 + bw], rng.uniform(5, 50))
    right = _warp_right(left.astype(np.float64), disp, rng, 3.0)
    return left, right, disp.astype(np.float32)


def building_like(seed: int = 2, width: int = 4800, height: int = 3409):
    """Large scene: 5 octaves of blurred noise, 40 planes in [0,250]."""
    rng = _rng(seed)
    tex = np.zeros((height, width))
    for o in range(5):
        tex += _blurred_noise(rng, height, width, sigma=1.0 * (2 ** o)) / (2 ** o)
    tex = (tex - tex.min()) / max(tex.max() - tex.min(), 1e-6) * 255.0
    left = np.clip(np.rint(tex), 0, 255).astype(np.uint8)
    disp = _planar_disparity(rng, height, width, 40, 0.0, 250.0)
    right = _warp_right(left.astype(np.float64), disp, rng, 2.0)
    return left, right, disp.astype(np.float32)


def batch_specs(seed: int = 3, n: int = 64):
    """(width, height, disparity range, scene seed) for the batched configuration."""
    rng = _rng(seed)
    out = []
    for i in range(n):
        w = int(rng.integers(320, 1921)) // 32 * 32
        h = int(rng.integers(240, 1081)) // 32 * 32
        d = int(rng.choice([64, 128]))
        out.append((w, h, d, 1000 + i))
    return out
