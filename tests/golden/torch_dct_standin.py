"""Stand-in for the third-party `torch_dct` module (not installed in this image).

Used only by make_golden.py to run the reference unwrapper.  The reference calls
`torch_dct.dct(x)` / `torch_dct.idct(X)` with norm=None along the last dimension
(insardev/insardev/utils_unwrap2d.py:1334-1365).  This restates the published
algorithm (Makhoul 1980, "A fast cosine transform in one and two dimensions"):
DCT-II X_k = 2 sum_n x_n cos(pi k (2n+1) / 2N) through one length-N FFT of the
even/odd-reordered sequence, and its exact inverse.
"""
import math

import torch


def dct(x, norm=None):
    if norm is not None:
        raise NotImplementedError("only norm=None is used by the unwrapper")
    N = x.shape[-1]
    v = torch.cat([x[..., ::2], x[..., 1::2].flip([-1])], dim=-1)
    V = torch.fft.fft(v, dim=-1)
    k = torch.arange(N, dtype=x.dtype, device=x.device) * (-math.pi / (2 * N))
    return 2 * (V.real * torch.cos(k) - V.imag * torch.sin(k))


def idct(X, norm=None):
    if norm is not None:
        raise NotImplementedError("only norm=None is used by the unwrapper")
    N = X.shape[-1]
    k = torch.arange(N, dtype=X.dtype, device=X.device) * (math.pi / (2 * N))
    Xr = X / 2
    Xm = torch.cat([torch.zeros_like(Xr[..., :1]), Xr.flip([-1])[..., :-1]], dim=-1)  # X_{N-k}, X_N = 0
    re = Xr * torch.cos(k) + Xm * torch.sin(k)
    im = Xr * torch.sin(k) - Xm * torch.cos(k)
    v = torch.fft.ifft(torch.complex(re, im), dim=-1).real
    x = torch.empty_like(v)
    h = (N + 1) // 2
    x[..., ::2] = v[..., :h]
    x[..., 1::2] = v[..., h:].flip([-1])
    return x
