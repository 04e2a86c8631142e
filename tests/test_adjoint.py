"""Frozen-weight adjoint (unw_adjoint_f32, core_b200.irls_unwrap_2d_diff).

The FP64 oracle (oracle/adjoint_oracle.py) restates the differentiated map
and its adjoint; the CPU tests pin the oracle's adjoint against central finite
differences of the map itself, the GPU tests compare the CUDA adjoint with the
oracle's (and with finite differences) on the same inputs and the same
forward solution.

Tolerances, relative to the largest gradient: oracle vs finite differences
1e-4 (h = 1e-5 phase, 1e-6 weight); oracle vs torch autograd through the unrolled
float64 PCG solve of the same map (oracle/adjoint_unrolled.py) 1e-6; CUDA
(float32 PCG solves to 1e-6 relative residual, float64 refinement of u*) vs the
oracle, vs the unrolled autograd and vs finite differences 1e-4.
"""
import numpy as np
import pytest

from oracle.adjoint_oracle import Frozen
from core_b200.synthetic import gen_g1
from oracle.irls_oracle import irls_unwrap_2d as oracle_unwrap


def _split_nan(p, c):
    """A NaN column band that splits the grid into two components, plus the generator's blobs."""
    p = p.copy(); c = c.copy()
    W = p.shape[1]
    p[:, W // 2:W // 2 + 2] = np.nan
    c[:, W // 2:W // 2 + 2] = np.nan
    return p, c


def _case(kind, H=24, W=28, seed=3):
    p, c, t = gen_g1(H, W, seed=seed, noise=1.2, nan_fraction=0.0 if kind == "full" else 0.05)
    if kind == "split":
        p, c = _split_nan(p, c)
    return p, c


def _relerr(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("kind", ["full", "nan", "split"])
def test_oracle_adjoint_matches_finite_differences(kind):
    p, c = _case(kind)
    u, _ = oracle_unwrap(p, c, dtype=np.float64)
    F = Frozen(p, c, u)
    v = np.isfinite(p)
    rng = np.random.default_rng(1)
    G = np.where(v, rng.standard_normal(p.shape), np.nan)
    gp, gw = F.adjoint(p, c, G)
    pix = [tuple(x) for x in np.argwhere(v)[rng.choice(v.sum(), 24, replace=False)]]
    fdp = F.finite_difference(p, c, G, pix, h=1e-5)
    fdw = F.finite_difference(p, c, G, pix, h=1e-6, wrt="weight")
    assert _relerr(np.array([gp[i, j] for i, j in pix]), fdp) <= 1e-4
    assert _relerr(np.array([gw[i, j] for i, j in pix]), fdw) <= 1e-4
    assert (gp[~v] == 0).all() and (gw[~v] == 0).all()
    if kind == "split":
        assert F.nlab >= 2


def test_factored_finite_differences_match_plain_ones():
    """The large-grid FD evaluator (one factorisation, one solve per pixel) against the
    plain one (one sparse solve per map evaluation) and the oracle adjoint."""
    p, c, _ = gen_g1(40, 48, seed=5, noise=1.0)
    u, _ = oracle_unwrap(p, c, dtype=np.float64)
    F = Frozen(p, c, u)
    v = np.isfinite(p)
    rng = np.random.default_rng(3)
    G = np.where(v, rng.standard_normal(p.shape), np.nan)
    pix = [tuple(x) for x in np.argwhere(v)[rng.choice(v.sum(), 12, replace=False)]]
    a = F.finite_difference(p, c, G, pix, h=1e-5)
    b = F.finite_difference_factored(p, c, G, pix, h=1e-4)
    gp, _ = F.adjoint(p, c, G)
    assert _relerr(b, a) <= 1e-6
    assert _relerr(np.array([gp[i, j] for i, j in pix]), b) <= 1e-6


@pytest.mark.parametrize("kind", ["full", "nan", "split"])
def test_unrolled_fp64_autograd_matches_oracle_adjoint(kind):
    """torch autograd through the unrolled float64 PCG solve of the same frozen map
    (oracle/adjoint_unrolled.py) against the oracle's hand-written adjoint (exact sparse
    solves): two independent derivations of dL/dphase and dL/dweight."""
    from oracle.adjoint_unrolled import UnrolledMap
    p, c = _case(kind, H=40, W=48, seed=5)
    u, _ = oracle_unwrap(p, c)
    v = np.isfinite(p)
    rng = np.random.default_rng(2)
    G = np.where(v, rng.standard_normal(p.shape), np.nan)
    op, ow = Frozen(p, c, u).adjoint(p, c, G)
    gp, gw, iters = UnrolledMap(p, c, u).gradients(p, c, G)
    assert 0 < iters < 20000
    assert _relerr(gp, op) <= 1e-6
    assert _relerr(gw, ow) <= 1e-6


# ------------------------------------------------------------------ GPU
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["full", "nan", "split"])
def test_cuda_adjoint_matches_oracle(kind):
    torch = _gpu()
    import core_b200
    p, c = _case(kind, H=40, W=48, seed=5)
    dev = torch.device("cuda", 0)
    u, _ = core_b200.irls_unwrap_2d(p, c)
    v = np.isfinite(p)
    rng = np.random.default_rng(2)
    G = np.where(v, rng.standard_normal(p.shape), np.nan).astype(np.float32)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    gph, gw, st = core_b200.irls_adjoint(T(p), T(c), T(u), T(G), cg_max_iter=3000, cg_tol=1e-6)
    gph, gw = gph.cpu().numpy(), gw.cpu().numpy()
    assert st["adjoint_rel_residual"] <= 1e-6 and not st["numeric_warning"]
    F = Frozen(p, c, u)
    op, ow = F.adjoint(p, c, G)
    assert (gph[~v] == 0).all() and (gw[~v] == 0).all()
    assert _relerr(gph, op) <= 1e-4, _relerr(gph, op)
    assert _relerr(gw, ow) <= 1e-4, _relerr(gw, ow)
    pix = [tuple(x) for x in np.argwhere(v)[rng.choice(v.sum(), 16, replace=False)]]
    fdp = F.finite_difference(p, c, G, pix, h=1e-5)
    assert _relerr(np.array([gph[i, j] for i, j in pix]), fdp) <= 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["full", "nan", "split"])
def test_cuda_adjoint_matches_unrolled_fp64_autograd(kind):
    """The CUDA adjoint against torch autograd through an unrolled float64 PCG solve of
    the frozen map (no hand-written adjoint on the reference side), within 1e-4 of the
    largest gradient."""
    torch = _gpu()
    import core_b200
    from oracle.adjoint_unrolled import UnrolledMap
    p, c = _case(kind, H=40, W=48, seed=5)
    dev = torch.device("cuda", 0)
    u, _ = core_b200.irls_unwrap_2d(p, c)
    v = np.isfinite(p)
    rng = np.random.default_rng(4)
    G = np.where(v, rng.standard_normal(p.shape), np.nan).astype(np.float32)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    gph, gw, st = core_b200.irls_adjoint(T(p), T(c), T(u), T(np.nan_to_num(G)), cg_max_iter=3000, cg_tol=1e-6)
    ap, aw, _ = UnrolledMap(p, c, u).gradients(p, c, G)
    assert _relerr(gph.cpu().numpy(), ap) <= 1e-4
    assert _relerr(gw.cpu().numpy(), aw) <= 1e-4


@pytest.mark.gpu
def test_adjoint_batch_matches_single_calls():
    """unw_adjoint_batch over grids of one shape with different masks (one split into
    two components, one all NaN) against one unw_adjoint_f32 call per grid."""
    torch = _gpu()
    import core_b200
    dev = torch.device("cuda", 0)
    cases = [_case("full", H=40, W=48, seed=5), _case("nan", H=40, W=48, seed=6), _case("split", H=40, W=48, seed=7)]
    allnan = (np.full((40, 48), np.nan, np.float32), np.full((40, 48), 0.5, np.float32))
    cases.append(allnan)
    ps = np.stack([c[0] for c in cases]).astype(np.float32)
    cs = np.stack([c[1] for c in cases]).astype(np.float32)
    us = np.stack([core_b200.irls_unwrap_2d(p, c)[0] for p, c in cases]).astype(np.float32)
    rng = np.random.default_rng(9)
    G = np.where(np.isfinite(us), rng.standard_normal(us.shape), 0.0).astype(np.float32)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    gph, gw, sts = core_b200.irls_adjoint_batch(T(ps), T(cs), T(us), T(G))
    assert len(sts) == 4
    for b in range(4):
        g1, w1, s1 = core_b200.irls_adjoint(T(ps[b]), T(cs[b]), T(us[b]), T(G[b]))
        np.testing.assert_array_equal(gph[b].cpu().numpy(), g1.cpu().numpy())
        np.testing.assert_array_equal(gw[b].cpu().numpy(), w1.cpu().numpy())
        assert sts[b]["adjoint_cg_iters"] == s1["adjoint_cg_iters"]
    assert (gph[3] == 0).all() and (gw[3] == 0).all()


@pytest.mark.gpu
def test_autograd_function_backward():
    torch = _gpu()
    import core_b200
    p, c, truth = gen_g1(64, 72, seed=7, noise=1.0)
    dev = torch.device("cuda", 0)
    pt = torch.from_numpy(p).to(dev).requires_grad_(True)
    ct = torch.from_numpy(c).to(dev).requires_grad_(True)
    tt = torch.from_numpy(truth.astype(np.float32)).to(dev)
    u, cc = core_b200.irls_unwrap_2d_diff(pt, ct)
    v = torch.isfinite(u)
    loss = 0.5 * (u[v] - tt[v]).pow(2).sum()
    loss.backward()
    assert pt.grad is not None and ct.grad is not None
    assert torch.isfinite(pt.grad).all() and torch.isfinite(ct.grad).all()
    assert (pt.grad[~v] == 0).all()
    # the same gradients through the direct call
    G = torch.where(v, u - tt, torch.zeros_like(u)).detach()
    gph, gw, _ = core_b200.irls_adjoint(pt.detach(), ct.detach(), u.detach(), G)
    assert torch.allclose(pt.grad, gph, rtol=0, atol=1e-6 * float(gph.abs().max()))
    assert torch.allclose(ct.grad, gw, rtol=0, atol=1e-6 * float(gw.abs().max()) + 1e-30)


@pytest.mark.gpu
def test_autograd_batch_matches_single_grids():
    torch = _gpu()
    import core_b200
    dev = torch.device("cuda", 0)
    ps, cs, ts = zip(*[gen_g1(48, 56, seed=s, noise=1.0) for s in (21, 22, 23)])
    pt = torch.from_numpy(np.stack(ps)).to(dev).requires_grad_(True)
    ct = torch.from_numpy(np.stack(cs)).to(dev).requires_grad_(True)
    tt = torch.from_numpy(np.stack(ts).astype(np.float32)).to(dev)
    u, cc = core_b200.irls_unwrap_2d_diff(pt, ct)
    assert u.shape == pt.shape and cc.shape == pt.shape
    v = torch.isfinite(u)
    (0.5 * (u[v] - tt[v]).pow(2).sum()).backward()
    for b in range(3):
        p1 = pt[b].detach().clone().requires_grad_(True)
        c1 = ct[b].detach().clone().requires_grad_(True)
        u1, _ = core_b200.irls_unwrap_2d_diff(p1, c1)
        v1 = torch.isfinite(u1)
        (0.5 * (u1[v1] - tt[b][v1]).pow(2).sum()).backward()
        assert torch.allclose(u[b], u1, equal_nan=True)
        assert torch.allclose(pt.grad[b], p1.grad, rtol=0, atol=1e-6 * float(p1.grad.abs().max()))
        assert torch.allclose(ct.grad[b], c1.grad, rtol=0, atol=1e-6 * float(c1.grad.abs().max()) + 1e-30)
