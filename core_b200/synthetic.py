"""Seeded synthetic interferograms for parity tests, the benchmark and users.

Data only: the solver, linking and filter paths do not import this module.

The reference ships no datasets for the unwrapper; its benchmark script builds
synthetic wrapped phase with Gaussian/turbulent signals, decorrelation noise
and NaN gaps (tests/test_unwrap_benchmark/test_unwrap_benchmark.py:37-303).
These generators restate the benchmark configurations named for this project
with fixed, documented draw orders so the same seed gives the same grid on any
machine (numpy.random.default_rng / PCG64 is platform independent):

G1  (`gen_g1`)   truth = 0.02 rad/px ramp along x + 8 Gaussians
                 (amplitude U[-40,40] rad, sigma U[50,300] px, centre U[0,H)xU[0,W))
                 + N(0, sigma_noise^2) noise (default 0.3); wrapped to (-pi, pi];
                 coherence U[0.3, 1.0]; 3 random ellipses whose union covers
                 5% +- 0.5% of the pixels are NaN in both phase and coherence.
G2  (`gen_g2`)   G1 plus a straight fault at a random angle through a point of the
                 central 40% of the grid, truth += 3*pi on one side, noise 0.6 rad,
                 coherence Beta(2,2) with values < 0.2 set to 0.05.
Stack (`gen_stack_meta`, `gen_stack_grid`)
                 64 G1 grids, rows U{1500..2600}, cols U{4000..7000},
                 noise sigma U[0.2, 0.8], grid i seeded with `seed * 1000 + i`.

Link scene (`gen_link_scene`)
                 n ellipses (centre U[0,H)xU[0,W), radii U[3, rmax]; with `holes`,
                 30% lose their inner half-radius ellipse) as the valid mask; a
                 smooth field plus N(0, noise^2), each 4-connected component shifted
                 by 2*pi*U{-2..2}; labels numbered by size (1 = largest) as the
                 unwrapper returns them.

Draw order (G1): 8 x (amp, sigma, cy, cx); noise[H,W]; coherence[H,W];
3 x (cy, cx, a0, b0, theta).  G2: 8 x (amp, sigma, cy, cx); fault (theta, py, px);
noise[H,W]; coherence Beta[H,W]; 3 x (cy, cx, a0, b0, theta).
"""
from __future__ import annotations

import numpy as np

NAN_FRACTION = 0.05
NAN_TOL = 0.005


def _gaussians(rng, H, W, n=8):
    y = np.arange(H, dtype=np.float64)
    x = np.arange(W, dtype=np.float64)
    out = np.zeros((H, W), dtype=np.float64)
    params = []
    for _ in range(n):
        amp = rng.uniform(-40.0, 40.0)
        sig = rng.uniform(50.0, 300.0)
        cy = rng.uniform(0.0, H)
        cx = rng.uniform(0.0, W)
        params.append((amp, sig, cy, cx))
    for amp, sig, cy, cx in params:
        gy = np.exp(-((y - cy) ** 2) / (2.0 * sig * sig))
        gx = np.exp(-((x - cx) ** 2) / (2.0 * sig * sig))
        out += amp * np.outer(gy, gx)
    return out


def _ellipse_params(rng, H, W, n=3):
    return [(rng.uniform(0.0, H), rng.uniform(0.0, W), rng.uniform(0.5, 1.5),
             rng.uniform(0.5, 1.5), rng.uniform(0.0, np.pi)) for _ in range(n)]


def _ellipse_mask(H, W, params, scale):
    """Union of rotated ellipses; semi-axes = scale * (a0, b0) * min(H, W) / 10."""
    mask = np.zeros((H, W), dtype=bool)
    base = min(H, W) / 10.0
    for cy, cx, a0, b0, th in params:
        a = max(scale * a0 * base, 1e-9)
        b = max(scale * b0 * base, 1e-9)
        r = max(a, b)
        y0, y1 = max(0, int(np.floor(cy - r))), min(H, int(np.ceil(cy + r)) + 1)
        x0, x1 = max(0, int(np.floor(cx - r))), min(W, int(np.ceil(cx + r)) + 1)
        if y0 >= y1 or x0 >= x1:
            continue
        yy = np.arange(y0, y1, dtype=np.float64)[:, None] - cy
        xx = np.arange(x0, x1, dtype=np.float64)[None, :] - cx
        c, s = np.cos(th), np.sin(th)
        u = xx * c + yy * s
        v = -xx * s + yy * c
        mask[y0:y1, x0:x1] |= (u / a) ** 2 + (v / b) ** 2 <= 1.0
    return mask


def _nan_mask(rng, H, W, frac=NAN_FRACTION):
    """Ellipse union scaled by bisection on a common radius factor to cover `frac`."""
    params = _ellipse_params(rng, H, W)
    lo, hi = 0.0, 1.0
    while _ellipse_mask(H, W, params, hi).mean() < frac and hi < 1e4:
        hi *= 2.0
    mask = _ellipse_mask(H, W, params, hi)
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        m = _ellipse_mask(H, W, params, mid)
        f = m.mean()
        if abs(f - frac) <= NAN_TOL * 0.5:
            mask = m
            break
        if f < frac:
            lo = mid
        else:
            hi = mid
            mask = m
    return mask


def _wrap(p):
    return np.arctan2(np.sin(p), np.cos(p))


def gen_g1(H, W=None, seed=0, noise=0.3, nan_fraction=NAN_FRACTION):
    """G1 grid. Returns (wrapped float32 [H,W] with NaN, coherence float32, truth float64)."""
    W = H if W is None else W
    rng = np.random.default_rng(seed)
    truth = _gaussians(rng, H, W)
    truth += 0.02 * np.arange(W, dtype=np.float64)[None, :]
    noisy = truth + rng.normal(0.0, noise, (H, W))
    coh = rng.uniform(0.3, 1.0, (H, W)).astype(np.float32)
    wrapped = _wrap(noisy).astype(np.float32)
    if nan_fraction > 0:
        m = _nan_mask(rng, H, W, nan_fraction)
        wrapped[m] = np.nan
        coh[m] = np.nan
    return wrapped, coh, truth


def gen_g2(H, W=None, seed=0, noise=0.6, nan_fraction=NAN_FRACTION):
    """G2 grid (G1 + 3*pi fault, noise 0.6, Beta(2,2) coherence)."""
    W = H if W is None else W
    rng = np.random.default_rng(seed)
    truth = _gaussians(rng, H, W)
    truth += 0.02 * np.arange(W, dtype=np.float64)[None, :]
    th = rng.uniform(0.0, np.pi)
    py = rng.uniform(0.3 * H, 0.7 * H)
    px = rng.uniform(0.3 * W, 0.7 * W)
    yy = np.arange(H, dtype=np.float64)[:, None] - py
    xx = np.arange(W, dtype=np.float64)[None, :] - px
    truth += 3.0 * np.pi * ((xx * np.sin(th) - yy * np.cos(th)) > 0.0)
    noisy = truth + rng.normal(0.0, noise, (H, W))
    coh = rng.beta(2.0, 2.0, (H, W))
    coh[coh < 0.2] = 0.05
    coh = coh.astype(np.float32)
    wrapped = _wrap(noisy).astype(np.float32)
    if nan_fraction > 0:
        m = _nan_mask(rng, H, W, nan_fraction)
        wrapped[m] = np.nan
        coh[m] = np.nan
    return wrapped, coh, truth


def gen_stack_meta(n=64, seed=0):
    """Per-grid (rows, cols, noise sigma, seed) of the uneven SBAS stack."""
    rng = np.random.default_rng(seed)
    meta = []
    for i in range(n):
        rows = int(rng.integers(1500, 2601))
        cols = int(rng.integers(4000, 7001))
        sig = float(rng.uniform(0.2, 0.8))
        meta.append((rows, cols, sig, seed * 1000 + i))
    return meta


def gen_stack_grid(meta_entry):
    rows, cols, sig, s = meta_entry
    return gen_g1(rows, cols, seed=s, noise=sig)


def gen_link_scene(H, W, n_blobs, seed=0, holes=False, noise=0.15, rmax=None):
    """Unwrapped phase with separately shifted components and their size-ordered uint16 labels."""
    from scipy import ndimage
    rng = np.random.default_rng(seed)
    valid = np.zeros((H, W), bool)
    for _ in range(n_blobs):
        cy, cx = rng.uniform(0, H), rng.uniform(0, W)
        ry, rx = rng.uniform(3, rmax or H / 8), rng.uniform(3, rmax or W / 8)
        y0, y1 = max(0, int(cy - ry) - 1), min(H, int(cy + ry) + 2)
        x0, x1 = max(0, int(cx - rx) - 1), min(W, int(cx + rx) + 2)
        yy, xx = np.mgrid[y0:y1, x0:x1]
        e = ((yy - cy) / ry) ** 2 + ((xx - cx) / rx) ** 2
        valid[y0:y1, x0:x1] |= e <= 1.0
        if holes and rng.random() < 0.3:
            valid[y0:y1, x0:x1] &= ~(e <= 0.25)
    lab, n = ndimage.label(valid, structure=[[0, 1, 0], [1, 1, 1], [0, 1, 0]])
    yy, xx = np.mgrid[:H, :W]
    truth = 0.03 * yy - 0.02 * xx + 2.0 * np.sin(xx / 37.0) * np.cos(yy / 53.0)
    shift = 2 * np.pi * rng.integers(-2, 3, n + 1)
    ph = np.where(valid, truth + shift[lab] + rng.normal(0, noise, (H, W)), np.nan).astype(np.float32)
    sizes = np.bincount(lab.ravel(), minlength=n + 1)
    order = sorted(range(1, n + 1), key=lambda L: (-sizes[L], -L))
    lut = np.zeros(n + 1, np.uint16)
    lut[order] = np.arange(1, n + 1)
    return ph, lut[lab]
