"""CPU oracle: numpy restatement of insardev's DCT+IRLS L1 2-D phase unwrapper.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg may import this module, and only as the checker or as the
timed CPU baseline.  The product path (core_b200) never calls it.

It restates `irls_unwrap_2d` (insardev/insardev/utils_unwrap2d.py:1082-1766)
step by step with numpy / scipy, in either float32 (mirrors the reference's
float32 torch path) or float64 (the "FP64 run of the same algorithm" that
the error budget is measured against).  Each block cites the reference lines
it follows.  The DCT pair is scipy.fft.dct/idct type 2 with norm=None, which
is the same unnormalised DCT-II (X_k = 2 sum x_n cos(pi k (2n+1) / 2N)) and
exact inverse that the reference obtains from the third-party `torch_dct`
module (utils_unwrap2d.py:1334); the preconditioner only ever applies
idct(dct(.)/lambda), so any exact DCT-II / inverse pair is the same operator
up to rounding.

Parity pin: tests/golden/ holds outputs of the reference function itself, run
in a container where it imports (tests/golden/make_golden.py); the CPU test
suite checks this restatement against them.
"""
from __future__ import annotations

import os
import warnings

import numpy as np
import scipy.fft as sfft
import scipy.ndimage as ndi

_STRUCT4 = np.array([[0, 1, 0], [1, 1, 1], [0, 1, 0]], dtype=bool)


class OracleStats:
    """Iteration log: IRLS iterations run, CG iterations per IRLS iteration, last rel_change."""

    def __init__(self):
        self.irls_iters = 0
        self.cg_iters = []
        self.rel_change = []
        self.residual = []
        self.bbox = None


def _wrap(a):
    return np.arctan2(np.sin(a), np.cos(a))


def irls_unwrap_2d(phase, weight=None, device='cpu', max_iter=50, tol=1e-3,
                   cg_max_iter=20, cg_tol=1e-4, epsilon=1e-2, conncomp_size=30,
                   debug=False, *, dtype=np.float32, workers=None, stats=None,
                   return_raw=False):
    """Restatement of utils_unwrap2d.py:1082 with the same signature and outputs.

    Extra keyword-only arguments: `dtype` (np.float32 or np.float64),
    `workers` (scipy.fft threads), `stats` (an OracleStats to fill),
    `return_raw` (also return the solver output before post-processing, cropped).
    """
    dt = np.dtype(dtype)
    workers = workers or os.cpu_count()
    phase = np.asarray(phase)
    if phase.ndim != 2:                                               # :1170-1171
        raise ValueError(f"irls_unwrap_2d expects 2D phase array, got shape {phase.shape}")
    original_shape = phase.shape
    nan_mask = np.isnan(phase)                                        # :1198-1201
    if np.all(nan_mask):
        return np.full_like(phase, np.nan), np.zeros(phase.shape, dtype=np.uint16)

    valid_rows = np.any(~nan_mask, axis=1)                            # :1204-1209
    valid_cols = np.any(~nan_mask, axis=0)
    r0, r1 = int(np.argmax(valid_rows)), len(valid_rows) - int(np.argmax(valid_rows[::-1]))
    c0, c1 = int(np.argmax(valid_cols)), len(valid_cols) - int(np.argmax(valid_cols[::-1]))
    crop = (r1 - r0) < phase.shape[0] or (c1 - c0) < phase.shape[1]  # :1212-1220
    if crop:
        phase = phase[r0:r1, c0:c1]
        nan_mask = nan_mask[r0:r1, c0:c1]
        if weight is not None:
            weight = np.asarray(weight)[r0:r1, c0:c1]
    if stats is not None:
        stats.bbox = (r0, r1, c0, c1)
    H, W = phase.shape
    valid = ~nan_mask

    phi = np.where(nan_mask, 0.0, phase).astype(np.float32).astype(dt)  # :1229-1230, :1247
    if weight is not None:                                            # :1233-1241
        w = np.array(weight, dtype=np.asarray(weight).dtype, copy=True)
        w[np.isnan(w)] = 0.0
        w[nan_mask] = 0.0
        w = np.clip(w, 0.01, 1.0)
    else:
        w = np.subtract(1.0, nan_mask, dtype=np.float32)
    w = w.astype(np.float32).astype(dt)

    # wrapped forward differences, last column / row zero           # :1254-1262
    gx = np.zeros((H, W), dt)
    gy = np.zeros((H, W), dt)
    gx[:, :-1] = phi[:, 1:] - phi[:, :-1]
    gy[:-1, :] = phi[1:, :] - phi[:-1, :]
    gx = _wrap(gx).astype(dt)
    gy = _wrap(gy).astype(dt)

    # edge weights: mean of the two pixel weights, zero on invalid edges  # :1267-1275
    wx = np.zeros((H, W), dt)
    wy = np.zeros((H, W), dt)
    wx[:, :-1] = (w[:, :-1] + w[:, 1:]) / dt.type(2)
    wy[:-1, :] = (w[:-1, :] + w[1:, :]) / dt.type(2)
    wx[:, :-1] *= (valid[:, :-1] & valid[:, 1:]).astype(dt)
    wy[:-1, :] *= (valid[:-1, :] & valid[1:, :]).astype(dt)

    # eigenvalues of the Neumann Laplacian, in float64 then cast      # :1284-1289
    ci = np.cos(np.pi * np.arange(H, dtype=np.float64) / H)
    cj = np.cos(np.pi * np.arange(W, dtype=np.float64) / W)
    lam = (2 * ci[:, None] + 2 * cj[None, :] - 4).astype(dt)
    lam[0, 0] = 1.0
    eps_sq = dt.type(epsilon * epsilon)                              # :1311

    def dct2(x):                                                      # :1337-1350
        return sfft.dct(sfft.dct(x, type=2, axis=1, workers=workers), type=2, axis=0,
                        workers=workers).astype(dt, copy=False)

    def idct2(X):                                                     # :1352-1365
        return sfft.idct(sfft.idct(X, type=2, axis=0, workers=workers), type=2, axis=1,
                         workers=workers).astype(dt, copy=False)

    def apply_laplacian(x, wxi, wyi):                                 # :1367-1388
        dx = np.zeros((H, W), dt)
        dy = np.zeros((H, W), dt)
        dx[:, :-1] = x[:, 1:] - x[:, :-1]
        dy[:-1, :] = x[1:, :] - x[:-1, :]
        dx *= wxi
        dy *= wyi
        res = np.zeros((H, W), dt)
        res[:, 1:] -= dx[:, :-1]
        res[:, :-1] += dx[:, :-1]
        res[1:, :] -= dy[:-1, :]
        res[:-1, :] += dy[:-1, :]
        return -res

    def apply_preconditioner(r):                                      # :1390-1403
        t = dct2(r)
        t /= lam
        t = -t
        t[0, 0] = 0.0
        return idct2(t)

    def dot(a, b):
        return dt.type(np.dot(a.ravel(), b.ravel()))

    def conjugate_gradient(b, wxi, wyi, x, max_it, tol_cg):           # :1405-1474
        n_it = 0
        r = b - apply_laplacian(x, wxi, wyi)
        if not np.isfinite(r).all():
            return x, 0
        z = apply_preconditioner(r)
        p = z.copy()
        rz = dot(r, z)
        for i in range(max_it):
            n_it = i + 1
            Ap = apply_laplacian(p, wxi, wyi)
            pAp = dot(p, Ap)
            if abs(pAp) < 1e-15 or not np.isfinite(pAp):
                break
            alpha = dt.type(np.clip(rz / pAp, -1e6, 1e6))
            x = x + alpha * p
            r = r - alpha * Ap
            if not np.isfinite(x).all():
                break
            r_norm = np.sqrt(dot(r, r))
            if r_norm < tol_cg or not np.isfinite(r_norm):
                break
            z = apply_preconditioner(r)
            rz_new = dot(r, z)
            if abs(rz) < 1e-15:
                break
            beta = dt.type(np.clip(rz_new / rz, -1e6, 1e6))
            p = beta * p + z
            rz = rz_new
        return x, n_it

    # initial solution: unweighted-Laplacian pseudo-inverse of rho   # :1478-1513
    rho = np.zeros((H, W), dt)
    fx = wx[:, :-1] * gx[:, :-1]
    fy = wy[:-1, :] * gy[:-1, :]
    rho[:, 1:] += fx
    rho[:, :-1] -= fx
    rho[1:, :] += fy
    rho[:-1, :] -= fy
    u = apply_preconditioner(rho)
    u = np.nan_to_num(u, nan=0.0, posinf=0.0, neginf=0.0)
    vf = valid.astype(dt)
    vcount = vf.sum(dtype=np.float64)
    if vcount > 0:
        u = u - dt.type(np.dot(u.ravel(), vf.ravel()) / vcount)

    u_best = u.copy()                                                  # :1530-1531
    best = np.inf
    it = -1
    for it in range(max_iter):                                         # :1533-1626
        u_prev = u.copy()
        if vcount > 0:                                                 # :1539-1541
            u = u - dt.type(np.dot(u.ravel(), vf.ravel()) / vcount)
        rx = np.zeros((H, W), dt)                                      # :1544-1551
        ry = np.zeros((H, W), dt)
        rx[:, :-1] = u[:, 1:] - u[:, :-1]
        ry[:-1, :] = u[1:, :] - u[:-1, :]
        rx -= gx
        ry -= gy
        residual = float(dot(rx, rx) + dot(ry, ry))                    # :1555-1558
        if residual < best and np.isfinite(u).all():
            best = residual
            u_best = u.copy()
        with np.errstate(invalid='ignore', divide='ignore', over='ignore'):
            wxi = np.clip(wx / np.sqrt(rx * rx + eps_sq), 1e-6, 1e6).astype(dt)   # :1562-1574
            wyi = np.clip(wy / np.sqrt(ry * ry + eps_sq), 1e-6, 1e6).astype(dt)
        b = np.zeros((H, W), dt)                                       # :1577-1581
        bx = wxi[:, :-1] * gx[:, :-1]
        by = wyi[:-1, :] * gy[:-1, :]
        b[:, 1:] += bx
        b[:, :-1] -= bx
        b[1:, :] += by
        b[:-1, :] -= by
        u, cg_it = conjugate_gradient(b, wxi, wyi, u, cg_max_iter, cg_tol)   # :1593
        if stats is not None:
            stats.cg_iters.append(cg_it)
            stats.residual.append(residual)
        if not np.isfinite(u).all():                                   # :1600-1604
            u = u_best.copy()
            break
        diff = np.sqrt(dot(u_prev - u, u_prev - u))                    # :1607-1609
        norm_u = np.sqrt(dot(u, u)) + dt.type(1e-10)
        rel_change = float(diff / norm_u)
        if stats is not None:
            stats.rel_change.append(rel_change)
        if debug and it % 5 == 0:
            print(f'  IRLS iter {it}: rel_change = {rel_change:.2e}, residual = {residual:.2e}, cg_iters = {cg_it}')
        if rel_change < tol:                                           # :1623-1626
            break
    if stats is not None:
        stats.irls_iters = it + 1
    if not np.isfinite(u).all():                                       # :1629-1632
        u = u_best
    unwrapped = u.astype(np.float32)                                   # :1637
    raw = unwrapped.copy()

    if not np.isfinite(unwrapped[valid]).all():                        # :1659-1665
        nan_count = int(np.sum(~np.isfinite(unwrapped[valid])))
        warnings.warn(f'IRLS produced {nan_count}/{int(valid.sum())} NaN/inf values - '
                      'returning NaN for this component', RuntimeWarning)
        out = (np.full(original_shape, np.nan, dtype=np.float32),
               np.zeros(original_shape, dtype=np.uint16))
        return out + (raw,) if return_raw else out

    unwrapped[nan_mask] = np.nan                                       # :1668
    unwrapped = postprocess(unwrapped, phase, valid, conncomp_size)

    if crop:                                                           # :1750-1757
        res = np.full(original_shape, np.nan, dtype=np.float32)
        res[r0:r1, c0:c1] = unwrapped[0]
        cc = np.zeros(original_shape, dtype=np.uint16)
        cc[r0:r1, c0:c1] = unwrapped[1]
        out = (res, cc)
    else:
        out = unwrapped
    return out + (raw,) if return_raw else out


def postprocess(unwrapped, phase, valid, conncomp_size):
    """Median 2-pi shift, per-component circular-mean alignment, size-ranked labels.

    Follows utils_unwrap2d.py:1671-1746 and the numba kernels at :24-75.
    `unwrapped` is float32 with NaN at invalid pixels (modified in place).
    Size ties are ranked larger-label-first, i.e. a reversed stable ascending
    sort (the reference's np.argsort(...)[::-1] leaves tie order to numpy).
    """
    conncomp = np.zeros(unwrapped.shape, dtype=np.uint16)
    if not np.any(valid):
        return unwrapped, conncomp
    ph32 = np.asarray(phase)
    diff = unwrapped[valid] - ph32[valid]                              # :1671-1676
    k_values = np.round(diff / (2 * np.pi))
    k_median = np.median(k_values)
    unwrapped[valid] = unwrapped[valid] - k_median * 2 * np.pi

    labeled, n = ndi.label(valid, structure=_STRUCT4)                  # :1686-1690
    n_labels = n + 1
    lf = labeled.ravel()
    pin = ph32.ravel().astype(np.float32)
    pout = unwrapped.ravel().astype(np.float32)
    sel = lf > 0                                                        # :24-65
    sin_in = np.bincount(lf[sel], weights=np.sin(pin[sel]).astype(np.float64), minlength=n_labels)
    cos_in = np.bincount(lf[sel], weights=np.cos(pin[sel]).astype(np.float64), minlength=n_labels)
    sin_out = np.bincount(lf[sel], weights=np.sin(pout[sel]).astype(np.float64), minlength=n_labels)
    cos_out = np.bincount(lf[sel], weights=np.cos(pout[sel]).astype(np.float64), minlength=n_labels)
    counts = np.bincount(lf[sel], minlength=n_labels).astype(np.int64)
    cf = counts.astype(np.float64)                                     # :1706-1717
    cf[cf == 0] = 1
    in_mean = np.arctan2(sin_in / cf, cos_in / cf)
    out_mean = np.arctan2(sin_out / cf, cos_out / cf)
    d = in_mean - out_mean
    adj = np.arctan2(np.sin(d), np.cos(d))
    adj[0] = 0
    uf = unwrapped.ravel()                                             # :68-75
    uf[sel] = (uf[sel].astype(np.float64) + adj[lf[sel]]).astype(np.float32)
    sizes = counts[1:n_labels]                                         # :1722-1736
    order = np.lexsort((-np.arange(n), -sizes))  # size desc, then label desc
    old_to_new = np.zeros(n_labels, dtype=np.int64)
    new = 1
    for idx in order:
        if sizes[idx] >= conncomp_size:
            old_to_new[idx + 1] = new
            new += 1
    if new - 1 > 65535:
        raise OverflowError(f'{new - 1} components do not fit uint16 labels')
    conncomp = old_to_new[labeled].astype(np.uint16)                   # :1746
    return unwrapped, conncomp


def cycle_map(u, phase):
    """Integer 2-pi cycle count k = round((u - phase) / 2pi) on valid pixels (0 elsewhere)."""
    v = np.isfinite(phase) & np.isfinite(u)
    k = np.zeros(np.shape(u), dtype=np.int32)
    k[v] = np.round((u[v].astype(np.float64) - phase[v].astype(np.float64)) / (2 * np.pi)).astype(np.int32)
    return k
