"""Goldstein adaptive phase filter on the B200 (`unw_goldstein_c64`).

Drop-in for insardev's GPU filter path goldstein_pytorch
(insardev/insardev/utils_goldstein.py:157-330), which insardev's Batch filter
dispatches to on CUDA devices (Batch.py:2023-2027): same arguments, same
complex64 result (NaN where the input is NaN or no valid patch covers a pixel).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .irls import _np_to_device, _torch, resolve_device


def goldstein(phase, corr, psize_y=32, psize_x=None, threshold=0.5, device='auto'):
    """Filter complex64 `phase` with coherence `corr` (numpy or CUDA tensors).

    psize_y / psize_x: patch size (powers of two in [4, 64]; psize_x defaults to
    psize_y; a dict {'y': .., 'x': ..} is accepted for psize_y as in Batch.py:2009-2012).
    Returns the same kind of array as the input (numpy complex64 or a CUDA tensor).
    """
    torch = _torch()
    if isinstance(psize_y, dict):
        psize_y, psize_x = int(psize_y['y']), int(psize_y['x'])
    psize_x = psize_y if psize_x is None else int(psize_x)
    psize_y = int(psize_y)
    is_torch = isinstance(phase, torch.Tensor)
    if phase.ndim != 2 or tuple(corr.shape) != tuple(phase.shape):
        raise ValueError(f"goldstein expects 2-D phase and corr of one shape, got {tuple(phase.shape)}, "
                         f"{tuple(corr.shape)}")
    dev = resolve_device(device, phase)
    lib = _lib.load()
    H, W = int(phase.shape[0]), int(phase.shape[1])
    with torch.cuda.device(dev):
        if is_torch:
            ph = phase.to(device=dev, dtype=torch.complex64).contiguous()
            cr = corr.to(device=dev, dtype=torch.float32).contiguous()
        else:
            ph = _np_to_device(np.ascontiguousarray(phase, np.complex64), dev)
            cr = _np_to_device(np.ascontiguousarray(corr, np.float32), dev)
        out = torch.empty((H, W), dtype=torch.complex64, device=dev)
        nb = lib.unw_goldstein_workspace_bytes(H, W, psize_y, psize_x)
        if nb == 0:
            raise NotImplementedError(f"goldstein: patch sizes must be powers of two in [4, 64], "
                                      f"got {psize_y} x {psize_x}")
        ws = torch.empty(nb, dtype=torch.uint8, device=dev)
        rc = lib.unw_goldstein_c64(ph.data_ptr(), W, cr.data_ptr(), W, H, W, psize_y, psize_x, float(threshold),
                                   out.data_ptr(), W, ws.data_ptr(), ws.numel(),
                                   torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(rc, "unw_goldstein_c64")
    if is_torch and phase.is_cuda:
        return out
    return out.cpu().numpy()
