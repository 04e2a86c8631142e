"""Autograd through an unrolled FP64 solve of the frozen-weight unwrap map.

TEST INFRASTRUCTURE ONLY: imported by tests/ as a second checker of the CUDA
adjoint (`unw_adjoint_f32`); never by the product path.

The same differentiated map as oracle/adjoint_oracle.py (`Frozen`): with the
IRLS scale of the forward solution, the valid mask, its components and the
median 2-pi shift held fixed, F(phase, weight) is the per-component aligned
solution of A(wI) u = b (insardev/insardev/utils_unwrap2d.py:1228-1290 for g and
the edge weights, :1560-1581 for wI and b, :1405-1474 for the PCG, :1667-1716 for
the alignment).  Here every step is a torch float64 operation on CPU tensors and
the solve is the reference's own algorithm, preconditioned CG with the DCT
Poisson preconditioner (:1390-1403), unrolled until the residual is below
`rtol` of the right-hand side: torch.autograd then differentiates through every
iteration, giving dL/dphase and dL/dweight without any hand-written adjoint.
The DCT is applied as dense DCT-II / DCT-III matrices, so the grids are small.
"""
from __future__ import annotations

import numpy as np
import torch

from oracle.adjoint_oracle import Frozen


def _dct_mats(n):
    """Unnormalised DCT-II matrix C[k][i] = 2 cos(pi k (2i+1) / 2n) and its inverse."""
    k = np.arange(n)[:, None]
    i = np.arange(n)[None, :]
    C = 2.0 * np.cos(np.pi * k * (2 * i + 1) / (2 * n))
    return torch.from_numpy(C), torch.from_numpy(np.linalg.inv(C))


class UnrolledMap:
    """F(phase, weight) at the frozen quantities of `Frozen(phase, weight, u)`."""

    def __init__(self, phase, weight, u, epsilon=1e-2):
        self.F = Frozen(phase, weight, u, epsilon=epsilon)
        F = self.F
        self.v = torch.from_numpy(F.valid)
        self.sx = torch.from_numpy(F.sx)
        self.sy = torch.from_numpy(F.sy)
        self.lab = torch.from_numpy(F.lab)
        H, W = F.valid.shape
        self.CH, self.CHi = _dct_mats(H)
        self.CW, self.CWi = _dct_mats(W)
        lam = (2 * np.cos(np.pi * np.arange(H) / H)[:, None] + 2 * np.cos(np.pi * np.arange(W) / W)[None, :] - 4)
        lam[0, 0] = 1.0
        self.inv_lam = torch.from_numpy(-1.0 / lam)
        self.inv_lam[0, 0] = 0.0

    @staticmethod
    def _wrap(a):
        return torch.atan2(torch.sin(a), torch.cos(a))

    def _grads(self, ph):
        gx = torch.zeros_like(ph)
        gy = torch.zeros_like(ph)
        gx[:, :-1] = self._wrap(ph[:, 1:] - ph[:, :-1])
        gy[:-1, :] = self._wrap(ph[1:, :] - ph[:-1, :])
        return gx, gy

    def _edge_weights(self, w):
        v = self.v
        if w is None:
            wf = v.to(torch.float64)
        else:
            wf = torch.where(torch.isnan(w) | ~v, torch.zeros_like(w), w)
            wf = torch.clamp(wf, 0.01, 1.0)
        wx = torch.zeros_like(wf)
        wy = torch.zeros_like(wf)
        wx[:, :-1] = (wf[:, :-1] + wf[:, 1:]) / 2 * (v[:, :-1] & v[:, 1:])
        wy[:-1, :] = (wf[:-1, :] + wf[1:, :]) / 2 * (v[:-1, :] & v[1:, :])
        return wx, wy

    @staticmethod
    def _div(ex, ey):
        """D^T applied to edge fields: (D^T e)_q = e_{q-1} - e_q per axis."""
        out = torch.zeros_like(ex)
        out[:, :-1] = out[:, :-1] - ex[:, :-1]
        out[:, 1:] = out[:, 1:] + ex[:, :-1]
        out[:-1, :] = out[:-1, :] - ey[:-1, :]
        out[1:, :] = out[1:, :] + ey[:-1, :]
        return out

    def _apply_A(self, x, wIx, wIy):
        dx = torch.zeros_like(x)
        dy = torch.zeros_like(x)
        dx[:, :-1] = x[:, 1:] - x[:, :-1]
        dy[:-1, :] = x[1:, :] - x[:-1, :]
        return self._div(wIx * dx, wIy * dy)

    def _precond(self, r):
        """idct2(-dct2(r) / lambda) with the zero mode removed."""
        X = self.CH @ r @ self.CW.T
        return self.CHi @ (X * self.inv_lam) @ self.CWi.T

    def forward(self, phase_t, weight_t, rtol=1e-13, max_iter=20000):
        """Full-size float64 output (NaN outside the valid pixels) and the PCG iteration count."""
        F = self.F
        r0, r1, c0, c1 = F.crop
        ph = torch.where(self.v, phase_t[r0:r1, c0:c1], torch.zeros((), dtype=torch.float64))
        w = None if weight_t is None else weight_t[r0:r1, c0:c1]
        gx, gy = self._grads(ph)
        wx, wy = self._edge_weights(w)
        wIx = torch.clamp(wx * self.sx, 1e-6, 1e6)
        wIy = torch.clamp(wy * self.sy, 1e-6, 1e6)
        b = self._div(wIx * gx, wIy * gy)
        # PCG from x = 0 (utils_unwrap2d.py:1405-1474), unrolled
        x = torch.zeros_like(b)
        r = b
        z = self._precond(r)
        p = z
        rz = (r * z).sum()
        bn = torch.linalg.norm(b.detach())
        it = 0
        while it < max_iter and float(torch.linalg.norm(r.detach())) > rtol * float(bn):
            Ap = self._apply_A(p, wIx, wIy)
            alpha = rz / (p * Ap).sum()
            x = x + alpha * p
            r = r - alpha * Ap
            z = self._precond(r)
            rz_new = (r * z).sum()
            p = z + (rz_new / rz) * p
            rz = rz_new
            it += 1
        # per-component circular-mean alignment (utils_unwrap2d.py:1694-1716)
        v = self.v
        L = self.lab[v]
        n = F.nlab + 1
        zeros = torch.zeros(n, dtype=torch.float64)
        sp_ = zeros.index_add(0, L, torch.sin(ph[v]))
        cp_ = zeros.index_add(0, L, torch.cos(ph[v]))
        su = zeros.index_add(0, L, torch.sin(x[v]))
        cu = zeros.index_add(0, L, torch.cos(x[v]))
        adj = self._wrap(torch.atan2(sp_, cp_) - torch.atan2(su, cu))
        adj = torch.cat([torch.zeros(1, dtype=torch.float64), adj[1:]])
        out = x - 2 * np.pi * F.kmed + adj[self.lab]
        full = torch.full(F.shape, float("nan"), dtype=torch.float64)
        full[r0:r1, c0:c1] = torch.where(v, out, torch.full_like(out, float("nan")))
        return full, it

    def gradients(self, phase, weight, grad_out, rtol=1e-13):
        """(dL/dphase, dL/dweight or None, PCG iterations) of L = sum(grad_out * F) by autograd."""
        pt = torch.tensor(np.asarray(phase, np.float64), requires_grad=True)
        wt = None if weight is None else torch.tensor(np.asarray(weight, np.float64), requires_grad=True)
        out, it = self.forward(pt, wt, rtol=rtol)
        G = torch.from_numpy(np.where(np.isfinite(grad_out), grad_out, 0.0).astype(np.float64))
        fin = torch.isfinite(out)
        loss = (G[fin] * out[fin]).sum()
        loss.backward()
        gp = pt.grad.numpy().copy()
        gp[~np.isfinite(np.asarray(phase))] = 0.0
        gw = None
        if wt is not None:
            gw = wt.grad.numpy().copy()
            gw[~np.isfinite(np.asarray(phase))] = 0.0
        return gp, gw, it
