"""Differentiable unwrap: a torch.autograd.Function over the B200 solver.

The forward pass is `irls_unwrap_2d` on CUDA tensors.  The backward pass calls
`unw_adjoint_f32` (one grid) or `unw_adjoint_batch` (a (B, H, W) batch, one launch
sequence for all grids): gradients of the unwrap with the forward solution's IRLS
scale, valid mask, components and median 2-pi shift held fixed (the frozen
final IRLS system of insardev/insardev/utils_unwrap2d.py:1529-1626 and the
alignment of :1667-1716), through an implicit adjoint solve with the same
DCT-preconditioned PCG.  The reference has no differentiable path.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .irls import _torch, irls_unwrap_2d, irls_unwrap_2d_batch, make_params


def irls_adjoint(phase, weight, u, grad_u, *, cg_max_iter=1000, cg_tol=1e-6, epsilon=1e-2, need_weight=True):
    """dL/dphase (and dL/dweight) for dL/du = grad_u at the forward output u.

    All arrays are CUDA float32 tensors of one shape.  cg_tol is relative to the
    initial residual of each of the two PCG solves.  Returns (grad_phase,
    grad_weight or None, stats dict).
    """
    torch = _torch()
    lib = _lib.load()
    dev = phase.device
    H, W = int(phase.shape[0]), int(phase.shape[1])
    f32 = lambda t: t.detach().to(device=dev, dtype=torch.float32).contiguous()
    ph, uu, gu = f32(phase), f32(u), f32(grad_u)
    wt = f32(weight) if weight is not None else None
    gph = torch.empty((H, W), dtype=torch.float32, device=dev)
    gw = torch.empty((H, W), dtype=torch.float32, device=dev) if (wt is not None and need_weight) else None
    ws = torch.empty(lib.unw_adjoint_workspace_bytes(H, W), dtype=torch.uint8, device=dev)
    prm = make_params(cg_max_iter=cg_max_iter, cg_tol=cg_tol, epsilon=epsilon)
    st = _lib.UnwStats()
    with torch.cuda.device(dev):
        rc = lib.unw_adjoint_f32(ph.data_ptr(), W, wt.data_ptr() if wt is not None else None, W, H, W,
                                 C.byref(prm), uu.data_ptr(), W, gu.data_ptr(), W, gph.data_ptr(), W,
                                 gw.data_ptr() if gw is not None else None, W, ws.data_ptr(), ws.numel(),
                                 C.byref(st), torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(rc, "unw_adjoint_f32")
    return gph, gw, _adj_stats(st, rc)


def _adj_stats(st, rc):
    return {"refine_cg_iters": int(st.cg_iters[0]), "adjoint_cg_iters": int(st.cg_iters[1]),
            "refine_pass_cg_iters": [int(st.cg_iters[2 + k]) for k in range(3)],
            "refine_rel_residual": float(st.resid_rel),
            "adjoint_rel_residual": float(st.rel_change), "status": int(st.status), "numeric_warning": rc == 1}


def irls_adjoint_batch(phase, weight, u, grad_u, *, cg_max_iter=1000, cg_tol=1e-6, epsilon=1e-2,
                       need_weight=True):
    """`irls_adjoint` for a (B, H, W) batch through one `unw_adjoint_batch` call.

    Returns (grad_phase (B, H, W), grad_weight (B, H, W) or None, list of per-grid stats).
    """
    torch = _torch()
    lib = _lib.load()
    dev = phase.device
    nb, H, W = (int(x) for x in phase.shape)
    f32 = lambda t: t.detach().to(device=dev, dtype=torch.float32).contiguous()
    ph, uu, gu = f32(phase), f32(u), f32(grad_u)
    wt = f32(weight) if weight is not None else None
    gph = torch.empty((nb, H, W), dtype=torch.float32, device=dev)
    gw = torch.empty((nb, H, W), dtype=torch.float32, device=dev) if (wt is not None and need_weight) else None
    grids = (_lib.UnwAdjGrid * nb)()
    for b in range(nb):
        grids[b] = _lib.UnwAdjGrid(ph[b].data_ptr(), W, wt[b].data_ptr() if wt is not None else None, W, H, W,
                                   uu[b].data_ptr(), W, gu[b].data_ptr(), W, gph[b].data_ptr(), W,
                                   gw[b].data_ptr() if gw is not None else None, W)
    Hs, Ws = (C.c_int64 * nb)(*([H] * nb)), (C.c_int64 * nb)(*([W] * nb))
    ws = torch.empty(lib.unw_adjoint_batch_workspace_bytes(nb, Hs, Ws), dtype=torch.uint8, device=dev)
    prm = make_params(cg_max_iter=cg_max_iter, cg_tol=cg_tol, epsilon=epsilon)
    sts = (_lib.UnwStats * nb)()
    with torch.cuda.device(dev):
        rc = lib.unw_adjoint_batch(nb, grids, C.byref(prm), ws.data_ptr(), ws.numel(), sts,
                                   torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(rc, "unw_adjoint_batch")
    return gph, gw, [_adj_stats(sts[b], rc) for b in range(nb)]


def _make_function():
    torch = _torch()

    class _Fn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, phase, weight, kw, akw):
            if phase.ndim == 3:
                # a batch of grids: one batched forward solve (each grid on its own tests)
                ws = None if weight is None else list(weight)
                res = irls_unwrap_2d_batch(list(phase), ws, **kw)
                u = torch.stack([r[0] for r in res])
                # labels stacked as int16, then reinterpreted
                cc = torch.stack([r[1].view(torch.int16) for r in res]).view(res[0][1].dtype)
            else:
                u, cc = irls_unwrap_2d(phase, weight, **kw)
            ctx.save_for_backward(phase, weight if weight is not None else phase.new_empty(0), u)
            ctx.has_weight = weight is not None
            ctx.akw = akw
            ctx.mark_non_differentiable(cc)
            return u, cc

        @staticmethod
        def backward(ctx, grad_u, grad_cc):
            phase, weight, u = ctx.saved_tensors
            need_w = ctx.has_weight and ctx.needs_input_grad[1]
            if phase.ndim == 3:
                w = weight if ctx.has_weight else None
                gph, gw, _ = irls_adjoint_batch(phase, w, u, grad_u, need_weight=need_w, **ctx.akw)
                return gph, (gw if need_w else None), None, None
            w = weight if ctx.has_weight else None
            gph, gw, _ = irls_adjoint(phase, w, u, grad_u, need_weight=need_w, **ctx.akw)
            return gph, gw, None, None

    return _Fn


_FN = None


def irls_unwrap_2d_diff(phase, weight=None, max_iter=50, tol=1e-3, cg_max_iter=20, cg_tol=1e-4, epsilon=1e-2,
                        conncomp_size=30, *, adjoint_cg_max_iter=1000, adjoint_cg_tol=1e-6):
    """`irls_unwrap_2d` on CUDA tensors with gradients for phase and weight.

    phase (and weight): one (H, W) grid or a (B, H, W) batch (one batched forward
    solve; one batched adjoint in the backward pass).
    Returns (u, conncomp); u carries autograd history (conncomp does not).
    adjoint_cg_max_iter / adjoint_cg_tol control the backward pass's PCG solves
    (tolerance relative to each solve's initial residual).
    """
    global _FN
    torch = _torch()
    if not (isinstance(phase, torch.Tensor) and phase.is_cuda):
        raise ValueError("irls_unwrap_2d_diff takes CUDA tensors")
    if phase.ndim not in (2, 3):
        raise ValueError(f"irls_unwrap_2d_diff expects (H, W) or (B, H, W), got {tuple(phase.shape)}")
    if _FN is None:
        _FN = _make_function()
    kw = dict(max_iter=max_iter, tol=tol, cg_max_iter=cg_max_iter, cg_tol=cg_tol, epsilon=epsilon,
              conncomp_size=conncomp_size)
    akw = dict(cg_max_iter=adjoint_cg_max_iter, cg_tol=adjoint_cg_tol, epsilon=epsilon)
    return _FN.apply(phase, weight, kw, akw)
