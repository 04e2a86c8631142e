"""The differentiable unwrap at the size of the differentiable-unwrap configuration:
a batch of 16 G1 grids of 1024 x 1024 through core_b200.irls_unwrap_2d_diff, the loss
being the L2 distance of the unwrapped phase to the true phase; the backward pass's
gradient with respect to the wrapped phase is checked against float64 central finite
differences (h = 1e-4) of the frozen-weight map on 256 random pixels (16 per grid),
within 1e-4 of the largest finite difference.

The finite differences run on the CPU (oracle/adjoint_oracle.py,
Frozen.finite_difference_factored: one sparse factorisation of each grid's frozen
system, one solve per pixel), one grid per worker of a spawned process pool.  The
reference has no differentiable path; the map differentiated is the unwrap of
utils_unwrap2d.py:1533-1626 with its final IRLS scale, mask, components and median
shift held at the forward solution.
"""
import multiprocessing as mp
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import core_b200  # noqa: E402
from core_b200.synthetic import gen_g1  # noqa: E402
from oracle.adjoint_oracle import fd_factored_job  # noqa: E402

B, N, PIX, H_FD = 16, 1024, 16, 1e-4


def test_config5_batch_gradients_match_float64_finite_differences():
    dev = torch.device("cuda", 0)
    grids = [gen_g1(N, N, seed=k) for k in range(B)]
    pt = torch.from_numpy(np.stack([g[0] for g in grids])).to(dev).requires_grad_(True)
    ct = torch.from_numpy(np.stack([g[1] for g in grids])).to(dev)
    tt = torch.from_numpy(np.stack([g[2] for g in grids]).astype(np.float32)).to(dev)
    u, cc = core_b200.irls_unwrap_2d_diff(pt, ct, adjoint_cg_max_iter=3000, adjoint_cg_tol=1e-6)
    v = torch.isfinite(u)
    loss = 0.5 * (u[v] - tt[v]).pow(2).sum()
    loss.backward()
    grad = pt.grad.cpu().numpy()
    un = u.detach().cpu().numpy()
    G = np.where(np.isfinite(un), un - np.stack([g[2] for g in grids]), np.nan)
    rng = np.random.default_rng(5)
    jobs, picks = [], []
    for b, (p, c, _) in enumerate(grids):
        vb = np.isfinite(p)
        # pixels whose four wrapped neighbour differences stay away from the wrap over +-h
        far = lambda a: np.abs(np.angle(np.exp(1j * a))) < np.pi - 1e-2
        dx, dy = np.roll(p, -1, 1) - p, np.roll(p, -1, 0) - p
        ok = vb & far(dx) & far(dy) & far(np.roll(dx, 1, 1)) & far(np.roll(dy, 1, 0))
        cand = np.argwhere(ok)
        pix = [tuple(map(int, x)) for x in cand[rng.choice(len(cand), PIX, replace=False)]]
        picks.append(pix)
        jobs.append((p, c, un[b], G[b], pix, H_FD))
    workers = max(1, min(8, (os.cpu_count() or 2) // 2))
    with mp.get_context("spawn").Pool(workers) as pool:
        fds = pool.map(fd_factored_job, jobs)
    fd = np.concatenate(fds)
    ad = np.array([grad[b][i, j] for b, pix in enumerate(picks) for i, j in pix])
    assert fd.size == B * PIX == 256
    err = np.abs(ad - fd).max() / np.abs(fd).max()
    assert err <= 1e-4, err
