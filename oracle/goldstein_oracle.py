"""CPU restatement of insardev's Goldstein adaptive phase filter (GPU path).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
filter (`unw_goldstein_c64`); never by the product path.

Follows goldstein_pytorch (insardev/insardev/utils_goldstein.py:157-330), which
insardev dispatches to on CUDA devices (Batch.py:2023-2027):
  * triangular patch weight, separable, from a tent over half a patch (:198-203);
  * zero padding by psize - step plus what makes (size + pad - psize) a multiple
    of the step (:214-226); phase NaN -> 0, correlation NaN -> 0 (:229-230);
  * patches at stride step = psize // 2 (:240-243);
  * alpha = 1 - sum(wgt * corr) / sum(wgt) per patch (:259-262);
  * a patch counts when at least int(psize_y * psize_x * threshold) of its
    pixels are valid (:264-267);
  * F = fft2(patch); F *= max(|F|, 1e-10) ** alpha; ifft2 (:270-281);
  * weighted by wgt, invalid patches zeroed, overlap-added; divided by the
    number of valid patches covering the pixel (at least 1) (:283-307);
  * NaN where the input was NaN or no valid patch covers the pixel (:308-320).
The reference's numpy path (:12-154) divides by the summed weights instead;
the phase agrees, the magnitude differs by that factor.
"""
from __future__ import annotations

import numpy as np


def goldstein_weights(py, px):
    wx = 1.0 - np.abs(np.arange(px // 2) - (px / 2.0 - 1.0)) / (px / 2.0 - 1.0)
    wy = 1.0 - np.abs(np.arange(py // 2) - (py / 2.0 - 1.0)) / (py / 2.0 - 1.0)
    q = np.outer(wy, wx)
    return np.block([[q, np.flip(q, axis=1)], [np.flip(q, axis=0), np.flip(np.flip(q, axis=0), axis=1)]]).astype(
        np.float32)


def padded_shape(ny, nx, py, px):
    sy, sx = py // 2, px // 2
    pad_y, pad_x = py - sy, px - sx
    ey = (sy - ((ny + pad_y - py) % sy)) % sy
    ex = (sx - ((nx + pad_x - px) % sx)) % sx
    return ny + pad_y + ey, nx + pad_x + ex


def goldstein(phase, corr, py, px, threshold=0.5, dtype=np.float32):
    """Filtered complex array (complex64 for dtype float32), NaN as the reference."""
    phase = np.asarray(phase)
    corr = np.asarray(corr)
    ny, nx = phase.shape
    sy, sx = py // 2, px // 2
    nan_mask = np.isnan(phase)
    wgt = goldstein_weights(py, px).astype(dtype)
    wsum = wgt.sum(dtype=dtype)
    min_valid = int(py * px * threshold)
    H, W = padded_shape(ny, nx, py, px)
    ph = np.zeros((H, W), np.complex64 if dtype == np.float32 else np.complex128)
    ph[:ny, :nx] = np.where(nan_mask, 0, phase)
    cr = np.zeros((H, W), dtype)
    cr[:ny, :nx] = np.where(np.isnan(corr), 0, corr)
    valid = np.zeros((H, W), bool)
    valid[:ny, :nx] = ~nan_mask
    npy, npx = (H - py) // sy + 1, (W - px) // sx + 1
    ctype = ph.dtype
    out = np.zeros((H, W), ctype)
    cnt = np.zeros((H, W), dtype)
    for i in range(npy):
        for j in range(npx):
            y0, x0 = i * sy, j * sx
            patch = ph[y0:y0 + py, x0:x0 + px]
            alpha = dtype(1.0) - (wgt * cr[y0:y0 + py, x0:x0 + px]).sum(dtype=dtype) / wsum
            ok = valid[y0:y0 + py, x0:x0 + px].sum() >= min_valid
            if not ok:
                continue
            F = np.fft.fft2(patch).astype(ctype)
            mag = np.maximum(np.abs(F), dtype(1e-10)).astype(dtype)
            F = F * np.power(mag, alpha).astype(dtype)
            f = np.fft.ifft2(F).astype(ctype)
            out[y0:y0 + py, x0:x0 + px] += wgt * f
            cnt[y0:y0 + py, x0:x0 + px] += 1
    insufficient = cnt < 1e-6
    res = (out / np.maximum(cnt, 1))[:ny, :nx]
    res[nan_mask | insufficient[:ny, :nx]] = np.nan + 1j * np.nan
    return res.astype(ctype)
