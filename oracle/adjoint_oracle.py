"""FP64 oracle of the frozen-weight unwrap map and of its adjoint.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
adjoint (`unw_adjoint_f32`); never by the product path.

The differentiable map.  Given a forward solution u of the unwrapper
(insardev/insardev/utils_unwrap2d.py:1082-1766), freeze what is piecewise
constant or what the IRLS reweighting derived from u:
  * the valid mask, its 4-connected components and the median 2-pi shift k_med
    (utils_unwrap2d.py:1667-1690);
  * the IRLS scale s = 1 / sqrt(r^2 + eps^2), r = grad(u) - g, per edge
    (utils_unwrap2d.py:1560-1574);
then F(phase, weight) is
  g    = wrapped forward differences of the NaN-filled phase      (:1254-1262)
  wx   = (w_j + w_j+1)/2 on edges between valid pixels, w clipped (:1233-1275)
  wI   = clip(wx * s, 1e-6, 1e6)                                  (:1567-1574)
  u*   = A(wI)^+ b,  A = -div(wI grad), b = -div(wI g)            (:1367-1388, :1576-1581)
  out  = u* - 2 pi k_med + wrap(circmean(phase) - circmean(u*)) per component
                                                                  (:1667-1716)
on the bounding box of the valid pixels (:1204-1220), solved exactly (sparse
direct solve with one pixel pinned; the per-component alignment removes the
constant).  `adjoint` returns dL/dphase and dL/dweight of a loss whose
gradient with respect to `out` is G; `finite_difference` differentiates F
numerically for the check.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spl


def _wrap(a):
    return np.arctan2(np.sin(a), np.cos(a))


def _labels4(valid):
    """4-connected component labels 1..n of `valid` (0 elsewhere), raster order of first pixel."""
    H, W = valid.shape
    lab = np.zeros((H, W), np.int64)
    n = 0
    for i0 in range(H):
        for j0 in range(W):
            if valid[i0, j0] and lab[i0, j0] == 0:
                n += 1
                stack = [(i0, j0)]
                lab[i0, j0] = n
                while stack:
                    i, j = stack.pop()
                    for a, b in ((i - 1, j), (i + 1, j), (i, j - 1), (i, j + 1)):
                        if 0 <= a < H and 0 <= b < W and valid[a, b] and lab[a, b] == 0:
                            lab[a, b] = n
                            stack.append((a, b))
    return lab, n


class Frozen:
    """Frozen quantities of the map at a forward solution (all on the bbox crop)."""

    def __init__(self, phase, weight, u, epsilon=1e-2):
        phase = np.asarray(phase, np.float64)
        valid_full = np.isfinite(phase)
        rows = np.where(valid_full.any(1))[0]
        cols = np.where(valid_full.any(0))[0]
        self.crop = (rows[0], rows[-1] + 1, cols[0], cols[-1] + 1)
        r0, r1, c0, c1 = self.crop
        self.shape = phase.shape
        self.valid = valid_full[r0:r1, c0:c1]
        self.has_weight = weight is not None
        self.eps2 = float(epsilon) ** 2
        self.lab, self.nlab = _labels4(self.valid)
        ph = phase[r0:r1, c0:c1]
        uc = np.asarray(u, np.float64)[r0:r1, c0:c1]
        # frozen IRLS scale from the forward solution (NaN-filled where invalid)
        uf = np.where(self.valid, uc, 0.0)
        gx, gy = self._grads(np.where(self.valid, ph, 0.0))
        dux, duy = self._diff(uf)
        self.sx = 1.0 / np.sqrt((dux - gx) ** 2 + self.eps2)
        self.sy = 1.0 / np.sqrt((duy - gy) ** 2 + self.eps2)
        k = np.round((uc - ph) / (2 * np.pi))[self.valid]
        self.kmed = float(np.median(k))
        H, W = self.valid.shape
        self.Dx, self.Dy = self._diff_ops(H, W)

    # ---------------------------------------------------------------- pieces
    @staticmethod
    def _diff(x):
        dx = np.zeros_like(x)
        dy = np.zeros_like(x)
        dx[:, :-1] = x[:, 1:] - x[:, :-1]
        dy[:-1, :] = x[1:, :] - x[:-1, :]
        return dx, dy

    def _grads(self, pf):
        dx, dy = self._diff(pf)
        gx = _wrap(dx)
        gy = _wrap(dy)
        gx[:, -1] = 0.0
        gy[-1, :] = 0.0
        return gx, gy

    @staticmethod
    def _diff_ops(H, W):
        """Forward-difference operators (last column / row rows are zero), as sparse matrices."""
        n = H * W
        idx = np.arange(n).reshape(H, W)
        e = idx[:, :-1].ravel()
        Dx = sp.csr_matrix((np.r_[-np.ones(e.size), np.ones(e.size)], (np.r_[e, e], np.r_[e, e + 1])), shape=(n, n))
        e = idx[:-1, :].ravel()
        Dy = sp.csr_matrix((np.r_[-np.ones(e.size), np.ones(e.size)], (np.r_[e, e], np.r_[e, e + W])), shape=(n, n))
        return Dx, Dy

    def _weights(self, weight_crop):
        v = self.valid
        if self.has_weight:
            wf = np.where(np.isnan(weight_crop) | ~v, 0.0, weight_crop)
            wf = np.clip(wf, 0.01, 1.0)
        else:
            wf = v.astype(np.float64)
        wx = np.zeros_like(wf)
        wy = np.zeros_like(wf)
        wx[:, :-1] = (wf[:, :-1] + wf[:, 1:]) / 2 * (v[:, :-1] & v[:, 1:])
        wy[:-1, :] = (wf[:-1, :] + wf[1:, :]) / 2 * (v[:-1, :] & v[1:, :])
        return wx, wy

    def _system(self, ph_crop, w_crop):
        gx, gy = self._grads(np.where(self.valid, ph_crop, 0.0))
        wx, wy = self._weights(w_crop)
        wIx = np.clip(wx * self.sx, 1e-6, 1e6)
        wIy = np.clip(wy * self.sy, 1e-6, 1e6)
        A = (self.Dx.T @ sp.diags(wIx.ravel()) @ self.Dx + self.Dy.T @ sp.diags(wIy.ravel()) @ self.Dy).tocsc()
        b = self.Dx.T @ (wIx * gx).ravel() + self.Dy.T @ (wIy * gy).ravel()
        return A, b, gx, gy, wx, wy, wIx, wIy

    @staticmethod
    def _solve(A, b):
        """A^+ b up to a constant: pin the first unknown (the graph is connected)."""
        x = np.zeros(A.shape[0])
        x[1:] = spl.spsolve(A[1:, 1:].tocsc(), b[1:])
        return x

    def _post_terms(self, ph_crop, uc):
        """Per-component sums of sin/cos of phase and u, indexed by label."""
        v = self.valid
        L = self.lab[v]
        n = self.nlab + 1
        sp_ = np.bincount(L, np.sin(ph_crop[v]), n)
        cp_ = np.bincount(L, np.cos(ph_crop[v]), n)
        su = np.bincount(L, np.sin(uc[v]), n)
        cu = np.bincount(L, np.cos(uc[v]), n)
        return sp_, cp_, su, cu

    # ---------------------------------------------------------------- map
    def forward(self, phase, weight=None):
        """F(phase, weight): full-size float64 output, NaN where invalid."""
        r0, r1, c0, c1 = self.crop
        ph = np.asarray(phase, np.float64)[r0:r1, c0:c1]
        wc = None if weight is None else np.asarray(weight, np.float64)[r0:r1, c0:c1]
        A, b, *_ = self._system(ph, wc)
        H, W = self.valid.shape
        u = self._solve(A, b).reshape(H, W)
        sp_, cp_, su, cu = self._post_terms(ph, u)
        adj = _wrap(np.arctan2(sp_, cp_) - np.arctan2(su, cu))
        adj[0] = 0.0
        out = u - 2 * np.pi * self.kmed + adj[self.lab]
        full = np.full(self.shape, np.nan)
        full[r0:r1, c0:c1] = np.where(self.valid, out, np.nan)
        return full

    def adjoint(self, phase, weight, grad_out):
        """(dL/dphase, dL/dweight or None) for dL/dout = grad_out (full size; NaN-free where valid)."""
        r0, r1, c0, c1 = self.crop
        v = self.valid
        H, W = v.shape
        ph = np.asarray(phase, np.float64)[r0:r1, c0:c1]
        wc = None if weight is None else np.asarray(weight, np.float64)[r0:r1, c0:c1]
        G = np.where(v, np.asarray(grad_out, np.float64)[r0:r1, c0:c1], 0.0)
        A, b, gx, gy, wx, wy, wIx, wIy = self._system(ph, wc)
        u = self._solve(A, b).reshape(H, W)
        sp_, cp_, su, cu = self._post_terms(ph, u)
        S = np.bincount(self.lab[v], G[v], self.nlab + 1)
        Sc = S[self.lab]
        # through the alignment: d circmean(u)/du_q = (C cos u_q + S sin u_q) / (S^2 + C^2)
        with np.errstate(invalid="ignore", divide="ignore"):
            dthu = (cu[self.lab] * np.cos(u) + su[self.lab] * np.sin(u)) / (su[self.lab] ** 2 + cu[self.lab] ** 2)
        Gp = np.where(v, G - Sc * dthu, 0.0)
        lam = self._solve(A, Gp.ravel()).reshape(H, W)
        # dL/dphase: through g (A lambda) and through circmean(phase)
        Al = (A @ lam.ravel()).reshape(H, W)
        with np.errstate(invalid="ignore", divide="ignore"):
            dthp = (cp_[self.lab] * np.cos(ph) + sp_[self.lab] * np.sin(ph)) / (sp_[self.lab] ** 2 + cp_[self.lab] ** 2)
        gph = np.where(v, Al + Sc * dthp, 0.0)
        gphase = np.zeros(self.shape)
        gphase[r0:r1, c0:c1] = gph
        if weight is None:
            return gphase, None
        # dL/dwI = (D lambda) (g - D u); dwI/dwx = s where unclipped; wx = (w_p + w_q)/2
        dlx, dly = self._diff(lam)
        dux, duy = self._diff(u)
        gwx = dlx * (gx - dux) * self.sx * ((wx * self.sx > 1e-6) & (wx * self.sx < 1e6) & (wx > 0))
        gwy = dly * (gy - duy) * self.sy * ((wy * self.sy > 1e-6) & (wy * self.sy < 1e6) & (wy > 0))
        gw = np.zeros((H, W))
        gw[:, :-1] += 0.5 * gwx[:, :-1]
        gw[:, 1:] += 0.5 * gwx[:, :-1]
        gw[:-1, :] += 0.5 * gwy[:-1, :]
        gw[1:, :] += 0.5 * gwy[:-1, :]
        clip_ok = np.isfinite(wc) & (wc > 0.01) & (wc < 1.0) & v
        gw = np.where(clip_ok, gw, 0.0)
        gweight = np.zeros(self.shape)
        gweight[r0:r1, c0:c1] = gw
        return gphase, gweight

    def finite_difference_factored(self, phase, weight, grad_out, pixels, h=1e-4):
        """Central differences of L = sum(grad_out * F) with respect to the phase at the
        given (i, j) pixels, for grids too large for one sparse solve per evaluation.

        The frozen system matrix does not depend on the phase, so it is factorised once
        (sparse LU in symmetric mode, the first unknown pinned as in _solve).  Its
        right-hand side is affine in one pixel's phase over [-h, h] (the wrapped
        differences next to the pixel move by +-h and stay away from the wrap), so the
        two evaluations share one solve: u(phase +- h e_ij) = u* +- d with
        d = A^+ (b(phase + h e_ij) - b(phase - h e_ij)) / 2, and F(phase +- h e_ij) is the
        full map at those u and phases (alignment included).  L(+h) - L(-h) is summed
        from the output difference so that no two large sums are subtracted.
        """
        r0, r1, c0, c1 = self.crop
        v = self.valid
        H, W = v.shape
        ph = np.asarray(phase, np.float64)[r0:r1, c0:c1]
        wc = None if weight is None else np.asarray(weight, np.float64)[r0:r1, c0:c1]
        A, b, gx, gy, wx, wy, wIx, wIy = self._system(ph, wc)
        lu = spl.splu(A[1:, 1:].tocsc(), permc_spec="MMD_AT_PLUS_A", options=dict(SymmetricMode=True))

        def solve(rhs):
            x = np.zeros_like(rhs)
            x[1:] = lu.solve(rhs[1:])
            return x

        def rhs_of(phc):
            g1, g2 = self._grads(np.where(v, phc, 0.0))
            return self.Dx.T @ (wIx * g1).ravel() + self.Dy.T @ (wIy * g2).ravel()

        ustar = solve(b[:, None])[:, 0].reshape(H, W)
        G = np.where(v, np.asarray(grad_out, np.float64)[r0:r1, c0:c1], 0.0)
        loc = [(i - r0, j - c0) for i, j in pixels]
        cols = []
        for ii, jj in loc:
            a = ph.copy()
            a[ii, jj] += h
            m = ph.copy()
            m[ii, jj] -= h
            cols.append((rhs_of(a) - rhs_of(m)) / 2)
        D = solve(np.stack(cols, axis=1))
        res = []
        for k, (ii, jj) in enumerate(loc):
            d = D[:, k].reshape(H, W)
            adj = []
            for sgn in (1.0, -1.0):
                phs = ph.copy()
                phs[ii, jj] += sgn * h
                sp_, cp_, su, cu = self._post_terms(phs, ustar + sgn * d)
                a_ = _wrap(np.arctan2(sp_, cp_) - np.arctan2(su, cu))
                a_[0] = 0.0
                adj.append(a_)
            dout = 2 * d + (adj[0] - adj[1])[self.lab]
            res.append(float(np.sum(G[v] * dout[v])) / (2 * h))
        return np.array(res)

    def finite_difference(self, phase, weight, grad_out, pixels, h=1e-4, wrt="phase"):
        """Central differences of L = sum(grad_out * F) at the given (i, j) pixels."""
        phase = np.asarray(phase, np.float64)
        weight = None if weight is None else np.asarray(weight, np.float64)
        Gm = np.where(np.isfinite(grad_out), grad_out, 0.0)

        def loss(p, w):
            out = self.forward(p, w)
            return float(np.nansum(Gm * np.where(np.isfinite(out), out, 0.0)))

        res = []
        for i, j in pixels:
            if wrt == "phase":
                a = phase.copy(); a[i, j] += h
                c = phase.copy(); c[i, j] -= h
                res.append((loss(a, weight) - loss(c, weight)) / (2 * h))
            else:
                a = weight.copy(); a[i, j] += h
                c = weight.copy(); c[i, j] -= h
                res.append((loss(phase, a) - loss(phase, c)) / (2 * h))
        return np.array(res)


def fd_factored_job(args):
    """(phase, weight, u, grad_out, pixels, h) -> central differences at the pixels, from
    a fresh Frozen map at u; a process-pool task (one grid per task)."""
    phase, weight, u, grad_out, pixels, h = args
    return Frozen(phase, weight, u).finite_difference_factored(phase, weight, grad_out, pixels, h=h)
