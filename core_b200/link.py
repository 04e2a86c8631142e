"""Component linking on the GPU: integer 2-pi offsets between components.

Drop-in for the linking step of insardev's `Stack.unwrap2d` (conncomp=False):
`_link_2d` (insardev/insardev/Stack_unwrap2d.py:325-407) with
`find_component_connections_fast` (utils_unwrap2d.py:195-444) and
`connect_components_ilp_fast` (utils_unwrap2d.py:886-1040).

The geometry runs in `unw_link_pairs_f32` on the device (components, border
pixels, hulls, neighbour ranking, closest pixels, blocking, window means); the
greedy choice of connections, the integer program and the reachability test
run here; `unw_link_apply_f32` writes the result on the device.  Lattice
geometry stands in for the reference's cv2 contours and shapely measures:
boundary = border pixels (the cv2 contour points), polygon = their convex hull,
distances between pixel centres; components in one row or column have no
contour polygon in the reference and take no part here either.

The integer program is the reference's: minimise sum w |k_i - k_j - k_offset|
over integers k in [-100, 100] with k_0 = 0, w = int(1000 * weight); the
reference hands it to OR-Tools CP-SAT (60 s limit), here to an exact native
solver (`unw_link_offsets`: steepest descent over unit moves, each a minimum
cut), and of the optimal assignments the one with the least sum |k| is
returned.  The reference
adds k_i * 2 pi to component i with k_i - k_j = round((mean_i - mean_j) / 2pi),
which moves the components apart by the measured offset; `sign='aligned'`
solves k_j - k_i = k_offset instead and brings them together (the convention
of the reference's older connect_components_ilp, utils_unwrap2d.py:846-857).
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time

import numpy as np

from . import _lib
from .irls import _np_to_device, _torch, resolve_device


class _LinkWorkspace:
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


_TLS = threading.local()


def _ws():
    if not hasattr(_TLS, "ws"):
        _TLS.ws = _LinkWorkspace()
    return _TLS.ws


def solve_offsets(n, edges, sign="reference"):
    """Integer offsets (k_0 = 0) minimising sum w |s (k_i - k_j) - off|, then sum |k| (exact, native).

    edges: sequence of (i, j, k_offset, int weight).  s = 1 for sign='reference', -1 for 'aligned'.
    """
    m = len(edges)
    k = np.zeros(n, np.int32)
    if n < 2 or m == 0:
        return k.astype(np.int64)
    e = np.asarray(edges, np.int64).reshape(m, 4)
    ei = np.ascontiguousarray(e[:, 0], np.int32)
    ej = np.ascontiguousarray(e[:, 1], np.int32)
    off = np.ascontiguousarray(e[:, 2], np.int32)
    w = np.ascontiguousarray(e[:, 3], np.int64)
    rc = _lib.load().unw_link_offsets(n, m, ei.ctypes.data, ej.ctypes.data, off.ctypes.data, w.ctypes.data,
                                      1 if sign == "reference" else -1, k.ctypes.data)
    _lib.check(rc, "unw_link_offsets")
    return k.astype(np.int64)


def _reachable_from_first(n, edges):
    adj = [[] for _ in range(n)]
    for i, j, _, _ in edges:
        adj[i].append(j)
        adj[j].append(i)
    seen = np.zeros(n, bool)
    seen[0] = True
    stack = [0]
    while stack:
        v = stack.pop()
        for u in adj[v]:
            if not seen[u]:
                seen[u] = True
                stack.append(u)
    return seen


def _device_labels(conncomp, dev, H, W):
    torch = _torch()
    if isinstance(conncomp, torch.Tensor):
        t = conncomp
        if t.dtype not in (torch.int16, getattr(torch, "uint16", torch.int16)):
            if int(t.max()) > 65535 or int(t.min()) < 0:
                raise ValueError("conncomp labels must lie in [0, 65535]")
            t = t.to(torch.int32).to(torch.int16) if int(t.max()) < 32768 else \
                torch.from_numpy(t.cpu().numpy().astype(np.uint16).view(np.int16))
        t = t.to(dev, non_blocking=t.device.type == "cpu" and t.is_pinned()).contiguous()
    else:
        a = np.asarray(conncomp)
        if a.dtype != np.uint16:
            if a.size and (a.max() > 65535 or a.min() < 0):
                raise ValueError("conncomp labels must lie in [0, 65535]")
            a = a.astype(np.uint16)
        t = _np_to_device(np.ascontiguousarray(a).view(np.int16), dev)
    if tuple(t.shape) != (H, W):
        raise ValueError(f"conncomp shape {tuple(t.shape)} differs from phase shape {(H, W)}")
    return t


def _device_pairs(ph, lab, min_size, K, window, dev, stream):
    """unw_link_pairs_f32 on device tensors: (labels, sizes, pair array, pair count, workspace)."""
    lib = _lib.load()
    H, W = int(ph.shape[0]), int(ph.shape[1])
    prm = _lib.UnwLinkParams(min_size, K, window, 0)
    ws = _ws().get(dev, lib.unw_link_workspace_bytes(H, W, min_size))
    ncomp, npair = C.c_int32(0), C.c_int32(0)
    ccap, pcap = 1024, 1024 * max(K, 1)
    # A call that finds its output arrays too small reports the counts it reached: first the
    # components, then (on the next call) the candidate pairs, so at most three calls.
    for attempt in range(3):
        clab = np.zeros(ccap, np.int64)
        csz = np.zeros(ccap, np.int64)
        cfl = np.zeros(ccap, np.int32)
        pairs = (_lib.UnwLinkPair * max(pcap, 1))()
        rc = lib.unw_link_pairs_f32(ph.data_ptr(), W, lab.data_ptr() if lab is not None else None, W, H, W,
                                    C.byref(prm), clab.ctypes.data, csz.ctypes.data, cfl.ctypes.data, ccap,
                                    C.byref(ncomp), pairs, pcap, C.byref(npair), ws.data_ptr(), ws.numel(), stream)
        if rc == _lib.UNW_E_WORKSPACE and (ncomp.value > ccap or npair.value > pcap) and attempt < 2:
            # each component adds at most K candidate pairs: size for that (bounded) once n is known
            bound = min(ncomp.value * max(K, 1), 1 << 24)
            ccap, pcap = max(ccap, ncomp.value), max(pcap, npair.value, bound)
            continue
        _lib.check(rc, "unw_link_pairs_f32")
        break
    n = ncomp.value
    if n > len(clab) or npair.value > len(pairs):
        raise RuntimeError("unw_link_pairs_f32: output arrays not filled")
    return clab[:n].copy(), csz[:n].copy(), pairs, npair.value, ws


def _edge_weights(conns, sizes):
    """(i, j, k_offset, int(1000 * weight)) per connection (utils_unwrap2d.py:917-931, :956-962)."""
    edges = []
    for ci, cj, _, _, dist, k_off, conf, _ in conns:
        size_weight = np.sqrt(min(sizes[ci], sizes[cj]))
        weight = conf * size_weight / (np.sqrt(dist) + 1.0)
        edges.append((ci, cj, int(k_off), int(weight * 1000)))
    return edges


def link_components(phase, conncomp=None, conncomp_size=100, conncomp_gap=None, conncomp_linksize=5,
                    conncomp_linkcount=30, debug=False, *, device='auto', sign='reference', return_info=False):
    """Link separately unwrapped components by integer 2-pi offsets (`_link_2d`, Stack_unwrap2d.py:325-407).

    phase      unwrapped phase (H, W) or (1, H, W), NaN = invalid; numpy or torch (CUDA tensors stay on device)
    conncomp   IRLS labels of the same shape (components taken in label order), or None: 4-connected
               components of the non-NaN pixels, largest first
    Components below max(conncomp_size, 4) pixels are set to NaN (labelled ones; label 0 is kept).
    Keyword-only extras: device, sign ('reference' or 'aligned'), return_info (also return a dict with
    components, connections, offsets and host timings).
    """
    torch = _torch()
    if sign not in ("reference", "aligned"):
        raise ValueError("sign must be 'reference' or 'aligned'")
    if not 0 <= int(conncomp_linksize) <= 31:
        raise ValueError("conncomp_linksize must lie in [0, 31] (windows of at most 31 x 31 pixels)")
    is_torch = isinstance(phase, torch.Tensor)
    squeeze = phase.ndim == 3 and phase.shape[0] == 1
    ph2 = phase[0] if squeeze else phase
    cc2 = None if conncomp is None else (conncomp[0] if conncomp.ndim == 3 and conncomp.shape[0] == 1 else conncomp)
    if ph2.ndim != 2:
        raise ValueError(f"link_components expects a 2D phase array, got shape {tuple(phase.shape)}")
    H, W = int(ph2.shape[0]), int(ph2.shape[1])
    dev = resolve_device(device, ph2)
    info = {"components": np.zeros(0, np.int64), "sizes": np.zeros(0, np.int64), "connections": [],
            "k": np.zeros(0, np.int64)}

    def finish(out_t):
        if is_torch and phase.is_cuda:
            res = out_t
        else:
            # through a pinned host block (torch's host caching allocator recycles it)
            host = torch.empty(out_t.shape, dtype=out_t.dtype, pin_memory=True)
            host.copy_(out_t, non_blocking=True)
            torch.cuda.current_stream(out_t.device).synchronize()
            res = host if is_torch else host.numpy()
        if squeeze:
            res = res[None]
        return (res, info) if return_info else res

    with torch.cuda.device(dev):
        if is_torch:
            ph = ph2.to(device=dev, dtype=torch.float32,
                        non_blocking=ph2.device.type == "cpu" and ph2.is_pinned()).contiguous()
        else:
            ph = _np_to_device(np.ascontiguousarray(ph2, dtype=np.float32), dev)
        if bool(torch.isnan(ph).all()):
            return finish(ph.clone())
        lab = _device_labels(cc2, dev, H, W) if cc2 is not None else None
        min_size = max(int(conncomp_size), 4)
        K = int(conncomp_linkcount)
        stream = torch.cuda.current_stream(dev).cuda_stream
        t0 = time.perf_counter()
        clab, csz, pairs, npair, ws = _device_pairs(ph, lab, min_size, K, int(conncomp_linksize), dev, stream)
        n = len(clab)
        t1 = time.perf_counter()
        info["components"], info["sizes"] = clab, csz
        k = np.zeros(n, np.int32)
        t2 = t1
        if n >= 2:
            conns = _greedy_connections(pairs, npair, K, conncomp_gap)
            info["connections"] = conns
            t2 = time.perf_counter()
            if conns:
                edges = _edge_weights(conns, csz)
                kk = solve_offsets(n, edges, sign)
                kk[~_reachable_from_first(n, edges)] = 0
                k = kk.astype(np.int32)
        info["k"] = k.astype(np.int64)
        if debug:
            print(f"link: {n} components, {len(info['connections'])} connections, "
                  f"{int(np.count_nonzero(k))} offsets applied")
        t3 = time.perf_counter()
        out = torch.empty((H, W), dtype=torch.float32, device=dev)
        rc = _lib.load().unw_link_apply_f32(ph.data_ptr(), W, H, W, k.ctypes.data, n, out.data_ptr(), W,
                                            ws.data_ptr(), ws.numel(), min_size, stream)
        _lib.check(rc, "unw_link_apply_f32")
        info["timing_ms"] = {"geometry": 1e3 * (t1 - t0), "greedy": 1e3 * (t2 - t1), "offsets": 1e3 * (t3 - t2),
                             "apply": 1e3 * (time.perf_counter() - t3)}
    return finish(out)


def _greedy_connections(pairs, npair, max_neighbors, gap):
    """Connections in order of distance under the per-component cap (utils_unwrap2d.py:335-444).

    Filter, sort and the float32 offset arithmetic run on whole columns (numpy float32 arrays round
    each operation as the reference's numpy float32 scalars do); only the cap walk is a loop.
    """
    if npair == 0:
        return []
    P = np.ctypeslib.as_array(pairs, shape=(len(pairs),))[:npair]
    dist = np.sqrt(P["d2"].astype(np.float64))
    keep = P["blocked"] == 0
    if gap is not None:
        keep &= ~(dist > gap)
    idx = np.nonzero(keep)[0]
    ci, cj = P["comp_i"][idx].astype(np.int64), P["comp_j"][idx].astype(np.int64)
    order = np.lexsort((cj, ci, dist[idx]))
    idx, ci, cj = idx[order], ci[order], cj[order]
    mi, mj = P["mean_i"][idx], P["mean_j"][idx]
    usable = (P["n_i"][idx] > 0) & (P["n_j"][idx] > 0) & ~np.isnan(mi) & ~np.isnan(mj)
    delta = mi - mj                                            # float32
    q = delta / (2 * np.pi)                                    # float32 / Python float -> float32
    k_off = np.round(q)                                        # half to even, float32
    fractional = q - k_off                                     # float32 - float32
    confidence = np.maximum(np.float32(0), np.float32(1.0) - np.float32(2) * np.abs(fractional))
    conns = []
    count = {}
    ci_l, cj_l, use_l = ci.tolist(), cj.tolist(), usable.tolist()
    yi, xi, yj, xj = (P[f][idx].tolist() for f in ("yi", "xi", "yj", "xj"))
    dl, kl = dist[idx].tolist(), np.where(usable, k_off, 0).astype(np.int64).tolist()
    conf_l, delta_l, pos_l = list(confidence), list(delta), (confidence > 0).tolist()   # numpy float32 scalars
    for t in range(len(ci_l)):
        i, j = ci_l[t], cj_l[t]
        if count.get(i, 0) >= max_neighbors or count.get(j, 0) >= max_neighbors or not use_l[t]:
            continue
        conns.append((i, j, (yi[t], xi[t]), (yj[t], xj[t]), dl[t], kl[t], conf_l[t] if pos_l[t] else 0, delta_l[t]))
        count[i] = count.get(i, 0) + 1
        count[j] = count.get(j, 0) + 1
    return conns


def find_component_connections_fast(labeled_array, phase, components, conncomp_gap=None, max_neighbors=30,
                                    n_neighbors=5, *, device='auto'):
    """Same signature and result as utils_unwrap2d.find_component_connections_fast (:195-444).

    labeled_array  int labels (0 = invalid); components: the reference's list of dicts ('label', 'size',
    'slices'), in the order whose indices the connections use.  Returns
    [(comp_i, comp_j, (row_i, col_i), (row_j, col_j), distance, k_offset, confidence, delta)].
    """
    torch = _torch()
    n = len(components)
    if n < 2:
        return []
    if n > 65535:
        raise OverflowError("more than 65535 components")
    labeled_array = np.asarray(labeled_array)
    lut = np.zeros(int(labeled_array.max()) + 1, np.uint16)
    for c, comp in enumerate(components):
        lut[comp["label"]] = c + 1
    lab16 = lut[labeled_array]
    ph2 = np.asarray(phase, np.float32)
    dev = resolve_device(device, None)
    with torch.cuda.device(dev):
        ph = _np_to_device(np.ascontiguousarray(ph2), dev)
        lab = _np_to_device(np.ascontiguousarray(lab16).view(np.int16), dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _, _, pairs, npair, _ = _device_pairs(ph, lab, 1, int(max_neighbors), int(n_neighbors), dev, stream)
    return _greedy_connections(pairs, npair, int(max_neighbors), conncomp_gap)


def connect_components_ilp_fast(unwrapped, labeled_array, components, connections, max_time=60.0, debug=False):
    """Same signature and result as utils_unwrap2d.connect_components_ilp_fast (:886-1040).

    The integer program goes to the exact native solver (max_time is accepted and unused: the solve
    is exact and fast); offsets reach only components connected to the first; float32 updates as the
    reference's `result[labels == L] += k * 2 * np.pi`.
    """
    n = len(components)
    if n < 2 or len(connections) == 0:
        return unwrapped.copy()
    sizes = [int(c["size"]) for c in components]
    edges = _edge_weights(connections, sizes)
    k = solve_offsets(n, edges)
    k[~_reachable_from_first(n, edges)] = 0
    result = unwrapped.copy()
    labeled_array = np.asarray(labeled_array)
    # a Python float added to the array: rounded to the array's dtype, added in that dtype
    shift = np.zeros(int(labeled_array.max()) + 1, result.dtype)
    for i, comp in enumerate(components):
        if k[i] != 0:
            shift[comp["label"]] = int(k[i]) * 2 * np.pi
    add = shift[labeled_array]
    moved = add != 0
    result[moved] = result[moved] + add[moved]
    if debug:
        print(f"  Applied 2pi offsets to {int(np.count_nonzero(k))}/{n} components")
    return result


def unwrap2d_link(phase, conncomp_size=10_000, conncomp_gap=None, conncomp_linksize=5, conncomp_linkcount=30,
                  debug=False, *, device='auto'):
    """Stack.unwrap2d_link (Stack_unwrap2d.py:460-523) on numpy / torch arrays: link the components of
    already unwrapped phase, labels from the valid mask.  phase (H, W) or (n, H, W)."""
    if conncomp_linksize > conncomp_size:
        raise ValueError(
            f'conncomp_linksize ({conncomp_linksize}) cannot be greater than conncomp_size ({conncomp_size}). '
            f'Components must have at least conncomp_linksize pixels for reliable offset estimation.')
    kw = dict(conncomp_size=conncomp_size, conncomp_gap=conncomp_gap, conncomp_linksize=conncomp_linksize,
              conncomp_linkcount=conncomp_linkcount, debug=debug, device=device)
    if phase.ndim == 2:
        return link_components(phase, None, **kw)
    torch = _torch()
    outs = [link_components(phase[i], None, **kw) for i in range(phase.shape[0])]
    return torch.stack(outs) if isinstance(phase, torch.Tensor) else np.stack(outs)


def unwrap2d(phase, weight=None, conncomp=False, conncomp_size=1000, conncomp_gap=None, conncomp_linksize=5,
             conncomp_linkcount=30, device='auto', debug=False, **kwargs):
    """IRLS unwrap then component linking (Stack.unwrap2d, Stack_unwrap2d.py:525-640), on numpy / torch arrays.

    phase (H, W) or (n, H, W).  kwargs go to the unwrapper with the Stack defaults of unwrap2d_irls
    (Stack_unwrap2d.py:753-755: max_iter=50, tol=1e-2, cg_max_iter=10, cg_tol=1e-3, epsilon=1e-2).
    conncomp=True returns (unwrapped, labels) without linking.
    """
    from .irls import irls_unwrap_2d_batch
    if not conncomp and conncomp_linksize > conncomp_size:
        raise ValueError(
            f'conncomp_linksize ({conncomp_linksize}) cannot be greater than conncomp_size ({conncomp_size}). '
            f'Components must have at least conncomp_linksize pixels for reliable offset estimation.')
    kw = dict(max_iter=50, tol=1e-2, cg_max_iter=10, cg_tol=1e-3, epsilon=1e-2)
    kw.update(kwargs)
    torch = _torch()
    if isinstance(phase, torch.Tensor):
        phase = phase.detach().cpu().numpy()
    if isinstance(weight, torch.Tensor):
        weight = weight.detach().cpu().numpy()
    a = np.asarray(phase, np.float32)
    single = a.ndim == 2
    stack = a[None] if single else a
    if weight is None:
        ws = None
    else:
        w = np.asarray(weight, np.float32)
        ws = list(w[None] if w.ndim == 2 else w)
    res = irls_unwrap_2d_batch(list(stack), ws, device=device, conncomp_size=conncomp_size, debug=debug, **kw)
    u = np.stack([r[0] for r in res])
    cc = np.stack([r[1] for r in res])
    if conncomp:
        return (u[0], cc[0]) if single else (u, cc)
    out = np.stack([link_components(u[i], cc[i], conncomp_size=conncomp_size, conncomp_gap=conncomp_gap,
                                    conncomp_linksize=conncomp_linksize, conncomp_linkcount=conncomp_linkcount,
                                    debug=debug, device=device) for i in range(len(u))])
    return out[0] if single else out
