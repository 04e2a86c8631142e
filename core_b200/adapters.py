"""Drop-in task adapters and the tiled overlap unwrap, on numpy blocks.

The reference wraps `irls_unwrap_2d` in per-block functions that dask calls
(insardev/insardev/Stack_unwrap2d.py:32-130) and builds the tiled unwrap on
`da.map_overlap` (Stack_unwrap2d.py:992-1136).  These functions keep those
signatures and return shapes but solve on the GPU, and where the reference
loops over the slices of a block they solve the slices in one batched call.
xarray/dask objects are not handled here: the functions take and return the
numpy blocks dask would pass.
"""
from __future__ import annotations

import numpy as np

from .irls import irls_unwrap_2d, irls_unwrap_2d_batch


def _unpack(params_tuple):
    device, max_iter, tol, cg_max_iter, cg_tol, epsilon, conncomp_size, debug, _sem = params_tuple
    dev = 'auto' if str(device) in ('cpu', 'mps', 'tpu', 'auto') else device
    return dev, dict(max_iter=max_iter, tol=tol, cg_max_iter=cg_max_iter, cg_tol=cg_tol, epsilon=epsilon,
                     conncomp_size=conncomp_size, debug=debug)


def _irls_process_chunk_with_tuple(phase_chunk, weight_chunk, params_tuple):
    """Stack_unwrap2d.py:32-71: (1, y, x) or (y, x) block -> ((1, y, x) unwrapped, (1, y, x) conncomp)."""
    dev, kw = _unpack(params_tuple)
    if phase_chunk.ndim == 3:
        phase_2d = phase_chunk[0]
        weight_2d = weight_chunk[0] if weight_chunk is not None else None
    elif phase_chunk.ndim == 2:
        phase_2d, weight_2d = phase_chunk, weight_chunk
    else:
        raise ValueError(f"Expected 2D or 3D phase_chunk, got shape {phase_chunk.shape}")
    if np.all(np.isnan(phase_2d)):
        return phase_2d.astype(np.float32)[np.newaxis], np.zeros_like(phase_2d, dtype=np.uint16)[np.newaxis]
    u, cc = irls_unwrap_2d(phase_2d, weight_2d, device=dev, **kw)
    return u[np.newaxis], cc[np.newaxis]


def _irls_process_no_weight(phase_chunk, params_tuple):
    """Stack_unwrap2d.py:74-77: unwrapped phase only."""
    return _irls_process_chunk_with_tuple(phase_chunk, None, params_tuple)[0]


def _irls_process_with_weight(phase_chunk, weight_chunk, params_tuple):
    """Stack_unwrap2d.py:80-84."""
    return _irls_process_chunk_with_tuple(phase_chunk, weight_chunk, params_tuple)[0]


def _stacked(u, cc):
    return np.stack([u[0].astype(np.float32), cc[0].astype(np.float32)], axis=0)[np.newaxis]


def _irls_process_no_weight_conncomp(phase_chunk, params_tuple):
    """Stack_unwrap2d.py:86-91: returns (1, 2, y, x) = (unwrapped, conncomp as float32)."""
    return _stacked(*_irls_process_chunk_with_tuple(phase_chunk, None, params_tuple))


def _irls_process_with_weight_conncomp(phase_chunk, weight_chunk, params_tuple):
    """Stack_unwrap2d.py:94-99."""
    return _stacked(*_irls_process_chunk_with_tuple(phase_chunk, weight_chunk, params_tuple))


def _irls_overlap_kernel(phase_block, weight_or_params, params_tuple=None):
    """Stack_unwrap2d.py:102-130: unwrap every (y, x) slice of a (n, y, x) block.

    The reference loops over the slices one GPU call at a time; here all
    non-empty slices go through one batched solve.  All-NaN slices pass
    through as float32.
    """
    if params_tuple is None:
        params_tuple, weight_block = weight_or_params, None
    else:
        weight_block = weight_or_params
    dev, kw = _unpack(params_tuple)
    out = [None] * phase_block.shape[0]
    todo = []
    for i in range(phase_block.shape[0]):
        if np.all(np.isnan(phase_block[i])):
            out[i] = phase_block[i].astype(np.float32)
        else:
            todo.append(i)
    if todo:
        ws = None if weight_block is None else [weight_block[i] for i in todo]
        res = irls_unwrap_2d_batch([phase_block[i] for i in todo], ws, device=dev, **kw)
        for i, (u, _cc) in zip(todo, res):
            out[i] = u
    return np.stack(out)


def _depth(overlap, chunk):
    """Stack_unwrap2d.py:1091-1092: fraction of the first chunk or pixels, at least 1."""
    return max(1, int(overlap * chunk) if isinstance(overlap, float) else int(overlap))


def _axis_chunks(n, c):
    """Chunk sizes along one axis: an int gives regular chunks (the last one smaller)."""
    if isinstance(c, (tuple, list)):
        sizes = [int(v) for v in c]
        if sum(sizes) != n or min(sizes) < 1:
            raise ValueError(f"chunk sizes {tuple(sizes)} do not cover an axis of {n}")
        return sizes
    c = max(1, min(int(c), n))
    return [min(c, n - s) for s in range(0, n, c)]


def _merge_small(sizes, depth):
    """Fold chunks smaller than the overlap depth into their left neighbour.

    `da.map_overlap` needs every chunk to be at least as deep as the overlap and
    rechunks the array when one is not; with regular chunks only the trailing
    one can be smaller, and folding it into its neighbour is that rechunk.
    """
    out = []
    for c in sizes:
        if out and (c < depth or out[-1] < depth):
            out[-1] += c
        else:
            out.append(c)
    return out


def overlap_tiles(H, W, chunks, overlap):
    """Tile geometry of the tiled unwrap.

    Returns (depth_y, depth_x, tiles) with tiles a list of
    (y0, y1, x0, x1, ey0, ey1, ex0, ex1): the chunk [y0:y1, x0:x1] and the
    halo'd block [ey0:ey1, ex0:ex1] that is solved for it (boundary='none':
    no halo beyond the raster edge).
    """
    if overlap is None:
        ov_y, ov_x = 0, 0
    elif isinstance(overlap, tuple):
        ov_y, ov_x = overlap
    else:
        ov_y, ov_x = overlap, overlap
    ys, xs = _axis_chunks(H, chunks[0]), _axis_chunks(W, chunks[1])
    dy, dx = _depth(ov_y, ys[0]), _depth(ov_x, xs[0])
    ys, xs = _merge_small(ys, dy), _merge_small(xs, dx)
    tiles = []
    y0 = 0
    for cy in ys:
        x0 = 0
        for cx in xs:
            y1, x1 = y0 + cy, x0 + cx
            tiles.append((y0, y1, x0, x1, max(0, y0 - dy), min(H, y1 + dy), max(0, x0 - dx), min(W, x1 + dx)))
            x0 = x1
        y0 += cy
    return dy, dx, tiles


def unwrap2d_chunk(phase, weight=None, chunks=(1024, 1024), overlap=None, device='auto', debug=False,
                   **kwargs):
    """Tiled unwrap with overlap, the numpy form of Stack_unwrap2d.py:992-1136.

    phase   (y, x) or (pair, y, x) float array, NaN = invalid
    weight  optional array of the same shape
    chunks  (cy, cx): ints for regular chunks, or tuples of chunk sizes per axis
    overlap None, float (fraction of the first chunk), int (pixels) or a (y, x) tuple
    kwargs  max_iter, tol, cg_max_iter, cg_tol, epsilon, conncomp_size with the
            defaults of the reference method (50, 1e-2, 10, 1e-3, 1e-2, 30)

    Every chunk is extended by the overlap depth towards its neighbours (not
    beyond the raster edge), unwrapped on its own, and trimmed back, as
    `da.map_overlap(..., boundary='none')` does; every pair is unwrapped on its
    own.  All tiles of all pairs are solved in one batched call.  Returns
    float32 unwrapped phase of the input shape (all-NaN tiles stay NaN).
    """
    p = np.asarray(phase)
    squeeze = p.ndim == 2
    if p.ndim not in (2, 3):
        raise ValueError(f"unwrap2d_chunk expects 2D or 3D phase, got shape {p.shape}")
    w = None if weight is None else np.asarray(weight)
    if w is not None and w.shape != p.shape:
        raise ValueError(f"weight shape {w.shape} differs from phase shape {p.shape}")
    if squeeze:
        p = p[np.newaxis]
        w = None if w is None else w[np.newaxis]
    kw = dict(max_iter=kwargs.get('max_iter', 50), tol=kwargs.get('tol', 1e-2),
              cg_max_iter=kwargs.get('cg_max_iter', 10), cg_tol=kwargs.get('cg_tol', 1e-3),
              epsilon=kwargs.get('epsilon', 1e-2), conncomp_size=kwargs.get('conncomp_size', 30))
    _, H, W = p.shape
    dy, dx, tiles = overlap_tiles(H, W, chunks, overlap)
    if debug:
        print(f"unwrap2d_chunk: depth=({dy},{dx}), {len(tiles)} tiles x {p.shape[0]} pairs")
    jobs, phs, wts = [], [], []
    for s in range(p.shape[0]):
        for k, (_, _, _, _, ey0, ey1, ex0, ex1) in enumerate(tiles):
            blk = p[s, ey0:ey1, ex0:ex1]
            if np.all(np.isnan(blk)):
                continue
            jobs.append((s, k))
            phs.append(blk)
            if w is not None:
                wts.append(w[s, ey0:ey1, ex0:ex1])
    out = np.full(p.shape, np.nan, dtype=np.float32)
    if jobs:
        res = irls_unwrap_2d_batch(phs, wts if w is not None else None, device=device, debug=debug, **kw)
        for (s, k), (u, _cc) in zip(jobs, res):
            y0, y1, x0, x1, ey0, ey1, ex0, ex1 = tiles[k]
            out[s, y0:y1, x0:x1] = u[y0 - ey0:y1 - ey0, x0 - ex0:x1 - ex0]
    return out[0] if squeeze else out
