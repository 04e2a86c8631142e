"""Drop-in replacement for insardev's `irls_unwrap_2d` on NVIDIA B200 GPUs.

`irls_unwrap_2d` keeps the reference signature, argument meaning, output
conventions and error behaviour of insardev/insardev/utils_unwrap2d.py:1082:

* `phase` 2-D float array (NaN = invalid), numpy or torch (CPU or CUDA);
  non-contiguous views are accepted;
* `weight` same shape or None (NaN allowed; clipped to [0.01, 1] after NaN
  zeroing, like :1233-1238);
* returns `(unwrapped float32 [H,W] with NaN where invalid,
  conncomp uint16 [H,W], 0 = invalid/small, 1 = largest, ...)`, numpy arrays
  for numpy input, torch tensors on the device for CUDA tensor input;
* `ValueError` for non-2-D input; all-NaN input -> (NaN, zeros); a
  non-finite solution -> `RuntimeWarning` and (NaN, zeros).

The solve runs entirely in libunwrap_b200.so (hand-written sm_100a kernels);
PyTorch only provides device memory and the stream.  A `device` that names the
host or another accelerator (insardev's stack pipeline passes 'cpu' when its
dask workers advertise no GPU) runs on the current CUDA device; the stats
record the request.  There is no CPU fallback: without a CUDA device the call
raises.
"""
from __future__ import annotations

import ctypes as C
import threading
import warnings

import numpy as np

from . import _lib

FN_DEFAULTS = dict(max_iter=50, tol=1e-3, cg_max_iter=20, cg_tol=1e-4, epsilon=1e-2, conncomp_size=30)


def _torch():
    import torch
    return torch


def resolve_device(device, phase=None):
    """The CUDA torch.device a call runs on.

    'auto' / None -> the device of a CUDA tensor input, else the current CUDA
    device; 'cuda' / 'cuda:N' / torch.device('cuda', N) -> that device.  A host
    or other accelerator request ('cpu', 'mps', 'tpu', ...) also runs on the
    current CUDA device: insardev's stack pipeline passes the device it
    resolved from its dask worker resources (Stack_unwrap2d.py:834-835, passed
    on at :65), which is 'cpu' whenever the workers advertise no GPU, and this
    implementation has only the CUDA path.  With no CUDA device visible the
    call raises RuntimeError (there is no CPU fallback).
    """
    torch = _torch()
    if isinstance(phase, torch.Tensor) and phase.is_cuda and device in ("auto", None):
        return phase.device
    dev = None
    if device not in ("auto", None):
        try:
            dev = torch.device(device) if not isinstance(device, torch.device) else device
        except (RuntimeError, TypeError):
            dev = None  # e.g. 'tpu': not a torch device type here
        if dev is not None and dev.type != "cuda":
            dev = None
    if dev is None:
        if not torch.cuda.is_available():
            raise RuntimeError("core_b200.irls_unwrap_2d needs a CUDA GPU; none is visible")
        if isinstance(phase, torch.Tensor) and phase.is_cuda:
            return phase.device
        return torch.device("cuda", torch.cuda.current_device())
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


PRECISIONS = ("plain", "mixed")
COL_PASSES = ("auto", "tc", "fft")


def precision_flags(precision="plain", col_pass="auto"):
    """UNW_F_* bits of the precision keywords.

    precision='plain'  float32 FFT DCTs throughout (the reference's arithmetic);
    precision='mixed'  for grids of at most 1024 rows the column DCT / scaling /
                       inverse DCT of the preconditioner may run as split-precision
                       bf16 products on the tensor cores: col_pass='auto' lets the
                       autotuner time both on the first call for a shape, 'tc' / 'fft'
                       force one; the stats report the path and the float64 residual of
                       the final weighted system.
    """
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}, got {precision!r}")
    if col_pass not in COL_PASSES:
        raise ValueError(f"col_pass must be one of {COL_PASSES}, got {col_pass!r}")
    if precision == "plain":
        return 0
    return _lib.UNW_F_MIXED | {"auto": 0, "tc": _lib.UNW_F_COL_TC, "fft": _lib.UNW_F_COL_FFT}[col_pass]


def make_params(max_iter=50, tol=1e-3, cg_max_iter=20, cg_tol=1e-4, epsilon=1e-2, conncomp_size=30,
                congruent=False, check_every=1, fixed_iters=False, precision="plain", col_pass="auto"):
    p = _lib.UnwParams()
    p.max_iter = int(max_iter)
    p.tol = float(tol)
    p.cg_max_iter = int(cg_max_iter)
    p.cg_tol = float(cg_tol)
    p.epsilon = float(epsilon)
    p.conncomp_size = int(conncomp_size)
    p.flags = ((_lib.UNW_F_CONGRUENT if congruent else 0) | (_lib.UNW_F_FIXED_ITERS if fixed_iters else 0)
               | precision_flags(precision, col_pass))
    p.check_every = int(check_every)
    return p


# Host inputs of at least this many bytes go to the device through pinned staging.
_STAGE_MIN_BYTES = 4 << 20
# Bytes per staged chunk.
_STAGE_CHUNK_BYTES = 8 << 20


def _staged_h2d(src, dev):
    """Host tensor (contiguous, pageable) -> device, through pinned staging.

    A copy from pageable memory goes through the driver's own bounce buffers at a
    fraction of the link speed (two 4096 x 4096 float32 arrays: 12.3 ms on a B200
    host).  Here each 8 MB chunk is copied into a pinned buffer by the host (torch's
    multi-threaded copy) and then sent with an asynchronous copy on the current
    stream, so the host copy of one chunk overlaps the transfer of the previous one
    (3.3 ms for the same two arrays).  Work enqueued later on the current stream sees
    the data; the pinned buffer returns to torch's host caching allocator, which keeps
    it from reuse until the copies that read it have completed.
    """
    torch = _torch()
    flat = src.reshape(-1)
    n = flat.numel()
    out = torch.empty(n, dtype=src.dtype, device=dev)
    stage = torch.empty(n, dtype=src.dtype, pin_memory=True)
    step = max(1, _STAGE_CHUNK_BYTES // flat.element_size())
    for o in range(0, n, step):
        e = min(n, o + step)
        stage[o:e].copy_(flat[o:e])
        out[o:e].copy_(stage[o:e], non_blocking=True)
    return out.view(src.shape)


def _np_to_device(arr, dev):
    """Contiguous numpy array -> CUDA tensor of the same dtype (pinned staging when large).

    Call with `dev` current."""
    torch = _torch()
    t = torch.from_numpy(arr)
    return _staged_h2d(t, dev) if arr.nbytes >= _STAGE_MIN_BYTES else t.to(dev)


def _to_device_f32(a, dev):
    """Contiguous float32 CUDA tensor from numpy / torch input (copies only when needed).

    Call with `dev` current (its current stream is the one the solver uses).
    """
    torch = _torch()
    if isinstance(a, torch.Tensor):
        if a.device.type == "cpu" and not a.is_pinned() and a.numel() * 4 >= _STAGE_MIN_BYTES:
            return _staged_h2d(a.to(torch.float32).contiguous(), dev)
        t = a.to(device=dev, dtype=torch.float32, non_blocking=a.device.type == "cpu" and a.is_pinned())
        return t.contiguous()
    return _np_to_device(np.ascontiguousarray(a, dtype=np.float32), dev)


class _Workspace:
    """Per-device workspace cache (the caching allocator would also reuse it)."""

    def __init__(self):
        self.buf = {}

    def get(self, dev, nbytes):
        torch = _torch()
        key = (dev.type, dev.index)
        b = self.buf.get(key)
        if b is None or b.numel() < nbytes:
            self.buf.pop(key, None)
            b = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
            self.buf[key] = b
        return b


_WS_LOCAL = threading.local()


def _to_host(pairs, dev):
    """Device (u, cc) pairs -> numpy (float32, uint16) arrays.

    The copies go into pinned host tensors (torch's host caching allocator
    recycles them once the caller drops the arrays, which keep their tensor
    alive), so the device-to-host transfer runs at full link speed instead of
    through the driver's pageable staging path.
    """
    torch = _torch()
    hs = []
    for ou, oc in pairs:
        hu = torch.empty(ou.shape, dtype=ou.dtype, pin_memory=True)
        hc = torch.empty(oc.shape, dtype=oc.dtype, pin_memory=True)
        hu.copy_(ou, non_blocking=True)
        hc.copy_(oc, non_blocking=True)
        hs.append((hu, hc))
    torch.cuda.current_stream(dev).synchronize()
    return [(hu.numpy(), hc.numpy().view(np.uint16)) for hu, hc in hs]


def _ws():
    if not hasattr(_WS_LOCAL, "ws"):
        _WS_LOCAL.ws = _Workspace()
    return _WS_LOCAL.ws


def irls_unwrap_2d(phase, weight=None, device='auto', max_iter=50, tol=1e-3,
                   cg_max_iter=20, cg_tol=1e-4, epsilon=1e-2, conncomp_size=30, debug=False,
                   *, congruent=False, return_stats=False, check_every=1, fixed_iters=False,
                   precision="plain", col_pass="auto"):
    """Unwrap 2-D phase with the DCT-preconditioned IRLS L1 solver on a B200.

    Same parameters and outputs as the reference (utils_unwrap2d.py:1082-1083).
    Keyword-only extras (defaults keep the reference behaviour):
      congruent     return phase + 2*pi*round((u - phase)/2pi) instead of u
      return_stats  also return a dict of iteration counts and status bits
      check_every   IRLS iterations enqueued between device->host convergence reads
      fixed_iters   run exactly max_iter x cg_max_iter iterations (tol / cg_tol stop
                    tests off, numerical breaks kept): identical work for timing
      precision     'plain' (float32 FFT DCTs) or 'mixed' (tensor-core column pass for
                    grids of <= 1024 rows where the autotuner finds it faster)
      col_pass      with precision='mixed': 'auto', or force 'tc' / 'fft'
    """
    torch = _torch()
    is_torch = isinstance(phase, torch.Tensor)
    if phase.ndim != 2:
        raise ValueError(f"irls_unwrap_2d expects 2D phase array, got shape {tuple(phase.shape)}")
    dev = resolve_device(device, phase)
    lib = _lib.load()
    H, W = int(phase.shape[0]), int(phase.shape[1])
    with torch.cuda.device(dev):
        ph = _to_device_f32(phase, dev)
        wt = _to_device_f32(weight, dev) if weight is not None else None
        if wt is not None and tuple(wt.shape) != (H, W):
            raise ValueError(f"weight shape {tuple(wt.shape)} differs from phase shape {(H, W)}")
        out_u = torch.empty((H, W), dtype=torch.float32, device=dev)
        out_cc = torch.empty((H, W), dtype=torch.int16, device=dev)
        nbytes = lib.unw_workspace_bytes(H, W)
        ws = _ws().get(dev, nbytes)
        st = _lib.UnwStats()
        prm = make_params(max_iter, tol, cg_max_iter, cg_tol, epsilon, conncomp_size, congruent, check_every,
                          fixed_iters, precision, col_pass)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = lib.unw_solve_f32(ph.data_ptr(), W, wt.data_ptr() if wt is not None else None, W, H, W,
                               C.byref(prm), out_u.data_ptr(), W, out_cc.data_ptr(), W,
                               ws.data_ptr(), ws.numel(), C.byref(st), stream)
        _lib.check(rc, "unw_solve_f32")
    stats = st.as_dict()
    stats["device"] = str(dev)
    stats["device_requested"] = str(device)
    if debug:
        _print_debug(H, W, stats)
    if st.status & _lib.UNW_S_ALL_NAN:
        # utils_unwrap2d.py:1200-1201 returns full_like(phase, nan) in the input dtype
        if is_torch:
            res = (torch.full_like(phase, float("nan")), torch.zeros((H, W), dtype=torch.int16, device=phase.device))
        else:
            res = (np.full_like(phase, np.nan), np.zeros((H, W), dtype=np.uint16))
        return res + (stats,) if return_stats else res
    if rc == _lib.UNW_W_NUMERIC:
        warnings.warn("IRLS produced NaN/inf values - returning NaN for this component", RuntimeWarning)
    if is_torch and phase.is_cuda:
        res = (out_u, out_cc.view(torch.uint16) if hasattr(torch, "uint16") else out_cc)
    else:
        res = _to_host([(out_u, out_cc)], dev)[0]
    return res + (stats,) if return_stats else res


def irls_unwrap_2d_batch(phases, weights=None, device='auto', max_iter=50, tol=1e-3, cg_max_iter=20,
                         cg_tol=1e-4, epsilon=1e-2, conncomp_size=30, debug=False, *, congruent=False,
                         return_stats=False, check_every=1, fixed_iters=False, precision="plain",
                         col_pass="auto"):
    """Unwrap a list of independent grids (any sizes) in one batched launch sequence.

    Each grid converges on its own test, exactly as if `irls_unwrap_2d` had been
    called on it alone.  Returns a list of (unwrapped, conncomp) tuples.
    """
    torch = _torch()
    phases = list(phases)
    n = len(phases)
    if n == 0:
        return []
    weights = [None] * n if weights is None else list(weights)
    if len(weights) != n:
        raise ValueError("weights must match phases")
    for p in phases:
        if p.ndim != 2:
            raise ValueError(f"irls_unwrap_2d expects 2D phase array, got shape {tuple(p.shape)}")
    dev = resolve_device(device, phases[0])
    lib = _lib.load()
    grids = (_lib.UnwGrid * n)()
    keep = []
    outs = []
    Hs = (C.c_int64 * n)()
    Ws = (C.c_int64 * n)()
    with torch.cuda.device(dev):
        for g, (p, w) in enumerate(zip(phases, weights)):
            H, W = int(p.shape[0]), int(p.shape[1])
            ph = _to_device_f32(p, dev)
            wt = _to_device_f32(w, dev) if w is not None else None
            ou = torch.empty((H, W), dtype=torch.float32, device=dev)
            oc = torch.empty((H, W), dtype=torch.int16, device=dev)
            keep += [ph, wt]
            outs.append((ou, oc))
            grids[g].phase = ph.data_ptr()
            grids[g].phase_pitch = W
            grids[g].weight = wt.data_ptr() if wt is not None else None
            grids[g].weight_pitch = W
            grids[g].H = H
            grids[g].W = W
            grids[g].out_u = ou.data_ptr()
            grids[g].out_u_pitch = W
            grids[g].out_cc = oc.data_ptr()
            grids[g].out_cc_pitch = W
            Hs[g] = H
            Ws[g] = W
        nbytes = lib.unw_batch_workspace_bytes(n, Hs, Ws)
        ws = _ws().get(dev, nbytes)
        sts = (_lib.UnwStats * n)()
        prm = make_params(max_iter, tol, cg_max_iter, cg_tol, epsilon, conncomp_size, congruent, check_every,
                          fixed_iters, precision, col_pass)
        rc = lib.unw_solve_batch(n, grids, C.byref(prm), ws.data_ptr(), ws.numel(), sts,
                                 torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(rc, "unw_solve_batch")
    res = []
    host_idx = [g for g in range(n) if not (isinstance(phases[g], torch.Tensor) and phases[g].is_cuda)
                and not (sts[g].status & _lib.UNW_S_ALL_NAN)]
    host = dict(zip(host_idx, _to_host([outs[g] for g in host_idx], dev))) if host_idx else {}
    for g in range(n):
        st = sts[g]
        p = phases[g]
        is_torch = isinstance(p, torch.Tensor)
        ou, oc = outs[g]
        if debug:
            _print_debug(int(p.shape[0]), int(p.shape[1]), st.as_dict())
        if st.status & _lib.UNW_S_ALL_NAN:
            r = ((torch.full_like(p, float("nan")), torch.zeros_like(oc)) if is_torch
                 else (np.full_like(p, np.nan), np.zeros(p.shape, dtype=np.uint16)))
        else:
            if st.status & _lib.UNW_S_NONFINITE_OUT:
                warnings.warn("IRLS produced NaN/inf values - returning NaN for this component", RuntimeWarning)
            r = ((ou, oc.view(torch.uint16) if hasattr(torch, "uint16") else oc) if is_torch and p.is_cuda
                 else host[g])
        res.append(r + (st.as_dict(),) if return_stats else r)
    return res


def _print_debug(H, W, s):
    r0, r1, c0, c1 = s["bbox"]
    if s.get("device_requested") not in (None, "auto", "None", s.get("device")):
        print(f"  device {s['device_requested']!r} requested: solved on {s['device']}")
    print(f"  Cropped to bbox [{r0}:{r1}, {c0}:{c1}] = {r1 - r0}x{c1 - c0} (from {H}x{W})")
    for i, cg in enumerate(s["cg_iters"]):
        if i % 5 == 0:
            print(f"  IRLS iter {i}: cg_iters = {cg}")
    print(f"  IRLS iters: {s['irls_iters']} iterations, rel_change = {s['rel_change']:.2e}, "
          f"best residual = {s['best_residual']:.3e}")
    print(f"  conncomp: {s['n_components']} kept of {s['n_labels']}")
