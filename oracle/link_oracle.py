"""CPU restatement of insardev's component linking (2-pi offsets between components).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
linking path (`unw_link_*`, `core_b200.link_components`); never by the product.

Follows the reference path taken by `Stack.unwrap2d(..., conncomp=False)`:
  * `_link_2d` (insardev/insardev/Stack_unwrap2d.py:325-407): components from
    the IRLS labels (label order, size >= max(conncomp_size, 4)) or from a
    4-connected labelling of the valid mask (size order, utils_unwrap2d.py:78-121);
    pixels of labelled components below the size are set to NaN;
  * `find_component_connections_fast` (utils_unwrap2d.py:195-444);
  * `connect_components_ilp_fast` (utils_unwrap2d.py:886-1040).

Raster geometry.  The reference traces each component with cv2.findContours
and measures with shapely.  Here the same quantities are stated on the pixel
lattice:
  * boundary of a component = its border pixels (a pixel of the component with
    a 4-neighbour outside it or outside the raster): exactly the union of the
    cv2 contour points (RETR_TREE, CHAIN_APPROX_NONE), checked in tests;
  * a component whose pixels lie in one row or one column has a cv2 contour of
    fewer than 3 points (CHAIN_APPROX_SIMPLE), which the reference skips
    (:240-241): it has no boundary and takes part in no connection;
  * component polygon = convex hull of its border pixel centres (:285-290);
  * distances are Euclidean between pixel centres (boundaries: closest pair of
    border pixels; polygons: exact convex-polygon distance, 0 when they meet);
  * a connection is blocked when its segment meets (closed) the convex hull
    of a third component (:335-346).
Not reproduced: shapely's make_valid drops zero-area contour pieces (one-pixel
spurs and necks) from the boundary; here every border pixel counts.  Ties are
broken deterministically where the reference leaves them to STRtree and set
order: neighbours by (distance, index), closest pairs by (d^2, y_i, x_i, y_j,
x_j), connections by (distance, comp_i, comp_j).

Integer offsets.  The reference minimises sum w |k_i - k_j - k_offset| with
CP-SAT (k_0 = 0, k in [-100, 100], w = int(1000 * weight)); OR-Tools is absent
here, so `solve_offsets` states the same program for scipy's HiGHS MILP and,
among optimal assignments, returns the one with the least sum |k| (CP-SAT
returns an unspecified optimum).  `sign='aligned'` solves k_j - k_i =
k_offset instead (the convention of the older connect_components_ilp,
utils_unwrap2d.py:846-857), which removes the measured offset instead of
adding it.
"""
from __future__ import annotations

import math
import warnings

import numpy as np

STRUCT4 = np.array([[0, 1, 0], [1, 1, 1], [0, 1, 0]], dtype=bool)
TWO_PI = 2 * np.pi


# ---------------------------------------------------------------------- components
def components_from_labels(conncomp, min_size):
    """IRLS labels -> (labeled int32, component labels in label order, sizes). Stack_unwrap2d.py:345-357."""
    labeled = np.asarray(conncomp).astype(np.int32)
    n_total = int(labeled.max()) if labeled.size else 0
    sizes = np.bincount(labeled.ravel(), minlength=n_total + 1)
    comps = [L for L in range(1, n_total + 1) if sizes[L] >= min_size]
    return labeled, comps, sizes


def components_from_mask(valid, min_size):
    """4-connected labels of the valid mask, components by size (ties: larger label first). :78-121."""
    from scipy import ndimage
    labeled, n = ndimage.label(valid, structure=STRUCT4)
    labeled = labeled.astype(np.int32)
    sizes = np.bincount(labeled.ravel(), minlength=n + 1)
    order = sorted(range(1, n + 1), key=lambda L: (-int(sizes[L]), -L))
    comps = [L for L in order if sizes[L] >= min_size]
    return labeled, comps, sizes


def border_points(labeled, label):
    """Border pixels (y, x) of one component, raster order."""
    full = labeled == label
    pad = np.pad(full, 1)
    core = pad[1:-1, 1:-1] & pad[:-2, 1:-1] & pad[2:, 1:-1] & pad[1:-1, :-2] & pad[1:-1, 2:]
    ys, xs = np.nonzero(full & ~core)
    return np.stack([ys, xs], 1).astype(np.int64)


def convex_hull(pts_yx):
    """Convex hull of integer (y, x) points as (x, y) vertices, counter-clockwise, no collinear vertices."""
    pts = sorted({(int(x), int(y)) for y, x in pts_yx})
    if len(pts) <= 2:
        return pts

    def cross(o, a, b):
        return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])

    lower, upper = [], []
    for p in pts:
        while len(lower) >= 2 and cross(lower[-2], lower[-1], p) <= 0:
            lower.pop()
        lower.append(p)
    for p in reversed(pts):
        while len(upper) >= 2 and cross(upper[-2], upper[-1], p) <= 0:
            upper.pop()
        upper.append(p)
    return lower[:-1] + upper[:-1]


def _cross(o, a, b):
    return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])


def point_segment_distance(p, a, b):
    """Distance from integer point p to segment ab, (x, y) tuples, in float64 (one fixed formula)."""
    dx, dy = b[0] - a[0], b[1] - a[1]
    t = (p[0] - a[0]) * dx + (p[1] - a[1]) * dy
    if t <= 0:
        return math.sqrt(float((p[0] - a[0]) ** 2 + (p[1] - a[1]) ** 2))
    L2 = dx * dx + dy * dy
    if t >= L2:
        return math.sqrt(float((p[0] - b[0]) ** 2 + (p[1] - b[1]) ** 2))
    return abs(float(_cross(a, b, p))) / math.sqrt(float(L2))


def _separated(P, Q):
    """True if an edge line of counter-clockwise polygon P has every vertex of Q strictly outside."""
    n = len(P)
    for k in range(n):
        a, b = P[k], P[(k + 1) % n]
        if all(_cross(a, b, q) < 0 for q in Q):
            return True
    return False


def hull_distance(P, Q):
    """Distance between two convex polygons (>= 3 vertices each), 0 when they meet."""
    if not (_separated(P, Q) or _separated(Q, P)):
        return 0.0
    d = math.inf
    for A, B in ((P, Q), (Q, P)):
        m = len(B)
        for p in A:
            for k in range(m):
                d = min(d, point_segment_distance(p, B[k], B[(k + 1) % m]))
    return d


def segment_meets_hull(p, q, H):
    """Closed segment pq meets closed convex polygon H (separating-axis test, exact integers)."""
    if _separated(H, [p, q]):
        return False
    s = [_cross(p, q, h) for h in H]
    if all(v > 0 for v in s) or all(v < 0 for v in s):
        return False
    return True


def nearest_pair(Bi, Bj):
    """Closest pair between two (y, x) point sets: (d2, yi, xi, yj, xj), ties lexicographic."""
    best = None
    step = max(1, 4_000_000 // max(1, len(Bj)))
    for s in range(0, len(Bi), step):
        a = Bi[s:s + step]
        d2 = ((a[:, None, 0] - Bj[None, :, 0]) ** 2 + (a[:, None, 1] - Bj[None, :, 1]) ** 2)
        m = int(d2.min())
        if best is not None and m > best[0]:
            continue
        ii, jj = np.nonzero(d2 == m)
        cands = sorted(zip(a[ii, 0].tolist(), a[ii, 1].tolist(), Bj[jj, 0].tolist(), Bj[jj, 1].tolist()))
        c = (m,) + tuple(cands[0])
        if best is None or c < best:
            best = c
    return best


def window_mean(phase, labeled, label, cy, cx, half):
    """np.nanmean of the window values of one component (utils_unwrap2d.py:403-414); None if empty/NaN."""
    H, W = phase.shape
    y0, y1 = max(0, cy - half), min(H, cy + half + 1)
    x0, x1 = max(0, cx - half), min(W, cx + half + 1)
    vals = phase[y0:y1, x0:x1][labeled[y0:y1, x0:x1] == label]
    if len(vals) == 0:
        return None
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        m = np.nanmean(vals)
    if np.isnan(m):
        return None
    return m


# ---------------------------------------------------------------------- connections
class Geometry:
    """Per-component border pixels and hulls (components with a boundary only)."""

    def __init__(self, labeled, comps):
        self.border = []
        self.hull = []
        for L in comps:
            b = border_points(labeled, L)
            ys, xs = b[:, 0], b[:, 1]
            if ys.min() == ys.max() or xs.min() == xs.max():
                self.border.append(None)      # straight line: contour < 3 points (:240-241)
                self.hull.append(None)
            else:
                self.border.append(b)
                self.hull.append(convex_hull(b))


def candidate_pairs(geom, max_neighbors):
    """Unordered component pairs from each component's nearest polygons (:308-332)."""
    n = len(geom.hull)
    valid = [i for i in range(n) if geom.hull[i] is not None]
    pairs = set()
    for i in valid:
        nb = sorted(((hull_distance(geom.hull[i], geom.hull[j]), j) for j in valid if j != i))
        for _, j in nb[:max_neighbors]:
            pairs.add((min(i, j), max(i, j)))
    return sorted(pairs)


def find_connections(labeled, phase, comps, sizes, conncomp_gap=None, max_neighbors=30, n_neighbors=5,
                     geom=None):
    """Connections (ci, cj, (yi, xi), (yj, xj), dist, k_offset, confidence, delta). :195-444."""
    n = len(comps)
    if n < 2:
        return []
    geom = geom or Geometry(labeled, comps)
    valid = []
    for i, j in candidate_pairs(geom, max_neighbors):
        d2, yi, xi, yj, xj = nearest_pair(geom.border[i], geom.border[j])
        dist = math.sqrt(float(d2))
        if conncomp_gap is not None and dist > conncomp_gap:
            continue
        p, q = (xi, yi), (xj, yj)
        blocked = any(k != i and k != j and geom.hull[k] is not None and segment_meets_hull(p, q, geom.hull[k])
                      for k in range(n))
        if not blocked:
            valid.append((dist, i, j, (yi, xi), (yj, xj)))
    valid.sort(key=lambda v: (v[0], v[1], v[2]))
    conns = []
    count = [0] * n
    half = n_neighbors // 2
    for dist, i, j, pi, pj in valid:
        if count[i] >= max_neighbors or count[j] >= max_neighbors:
            continue
        mi = window_mean(phase, labeled, comps[i], pi[0], pi[1], half)
        mj = window_mean(phase, labeled, comps[j], pj[0], pj[1], half)
        if mi is None or mj is None:
            continue
        delta = mi - mj
        k_offset = int(np.round(delta / (2 * np.pi)))
        fractional = (delta / (2 * np.pi)) - k_offset
        confidence = max(0, 1.0 - 2 * abs(fractional))
        conns.append((i, j, pi, pj, dist, k_offset, confidence, delta))
        count[i] += 1
        count[j] += 1
    return conns


# ---------------------------------------------------------------------- offsets
def edge_weights(conns, comp_sizes):
    """(ci, cj, k_offset, int weight) per connection (utils_unwrap2d.py:917-931, :956-962)."""
    out = []
    for ci, cj, _, _, dist, k_off, conf, _ in conns:
        size_weight = np.sqrt(min(comp_sizes[ci], comp_sizes[cj]))
        weight = conf * size_weight / (np.sqrt(dist) + 1.0)
        out.append((ci, cj, int(k_off), int(weight * 1000)))
    return out


def solve_offsets(n, edges, sign="reference", time_limit=60.0):
    """Integer offsets per component (k_0 = 0), or None if the program has no solution."""
    from scipy.optimize import Bounds, LinearConstraint, milp
    from scipy.sparse import coo_matrix
    m = len(edges)
    if n < 2 or m == 0:
        return np.zeros(n, np.int64)
    s = 1 if sign == "reference" else -1
    # variables: k (n), a (m, |diff|), t (n, |k|)
    nv = 2 * n + m
    rows, cols, vals, lo, hi = [], [], [], [], []
    r = 0
    for e, (i, j, off, _) in enumerate(edges):
        # diff = s*(k_i - k_j) - off;  a >= diff, a >= -diff
        for sg in (1, -1):
            rows += [r, r, r]
            cols += [i, j, n + e]
            vals += [-sg * s, sg * s, 1.0]
            lo.append(-sg * off)
            hi.append(np.inf)
            r += 1
    for i in range(n):
        for sg in (1, -1):
            rows += [r, r]
            cols += [i, n + m + i]
            vals += [-sg, 1.0]
            lo.append(0.0)
            hi.append(np.inf)
            r += 1
    A = coo_matrix((vals, (rows, cols)), shape=(r, nv)).tocsr()
    lb = np.r_[np.full(n, -100.0), np.zeros(m), np.zeros(n)]
    ub = np.r_[np.full(n, 100.0), np.full(m, 200.0), np.full(n, 100.0)]
    lb[0] = ub[0] = 0.0
    w = np.array([e[3] for e in edges], np.float64)
    c1 = np.r_[np.zeros(n), w, np.zeros(n)]
    opts = {"time_limit": float(time_limit)}
    integ = np.r_[np.ones(n), np.zeros(m), np.zeros(n)]
    res = milp(c1, constraints=[LinearConstraint(A, lo, hi)], bounds=Bounds(lb, ub), integrality=integ,
               options=opts)
    if res.x is None:
        return None
    best = round(float(res.fun))
    c2 = np.r_[np.zeros(n + m), np.ones(n)]
    A2 = coo_matrix(c1.reshape(1, -1))
    res2 = milp(c2, constraints=[LinearConstraint(A, lo, hi), LinearConstraint(A2, -np.inf, best + 0.5)],
                bounds=Bounds(lb, ub), integrality=integ, options=opts)
    x = res2.x if res2.x is not None else res.x
    return np.round(x[:n]).astype(np.int64)


def reachable_from_first(n, edges):
    """Components reachable from component 0 over the connections (utils_unwrap2d.py:989-1009)."""
    adj = [set() for _ in range(n)]
    for i, j, _, _ in edges:
        adj[i].add(j)
        adj[j].add(i)
    seen = {0}
    stack = [0]
    while stack:
        v = stack.pop()
        for u in adj[v]:
            if u not in seen:
                seen.add(u)
                stack.append(u)
    return seen


# ---------------------------------------------------------------------- whole path
def link(phase, conncomp=None, conncomp_size=100, conncomp_gap=None, conncomp_linksize=5,
         conncomp_linkcount=30, sign="reference", return_info=False):
    """Linked phase (float32), as `_link_2d` returns it (Stack_unwrap2d.py:325-407)."""
    phase = np.asarray(phase, np.float32)
    info = {"components": [], "connections": [], "k": np.zeros(0, np.int64)}
    valid = ~np.isnan(phase)
    if not valid.any():
        return (phase, info) if return_info else phase
    min_size = max(conncomp_size, 4)
    if conncomp is not None:
        labeled, comps, sizes = components_from_labels(conncomp, min_size)
    else:
        labeled, comps, sizes = components_from_mask(valid, min_size)
    linked = np.isin(labeled, np.array(comps, np.int32)) | (labeled == 0)
    ph = phase.copy()
    ph[~linked] = np.nan
    info["components"] = list(comps)
    if len(comps) < 2:
        return (ph, info) if return_info else ph
    conns = find_connections(labeled, ph, comps, sizes, conncomp_gap, conncomp_linkcount, conncomp_linksize)
    info["connections"] = conns
    if not conns:
        return (ph, info) if return_info else ph
    comp_sizes = [int(sizes[L]) for L in comps]
    edges = edge_weights(conns, comp_sizes)
    k = solve_offsets(len(comps), edges, sign)
    if k is None:
        return (ph, info) if return_info else ph
    reach = reachable_from_first(len(comps), edges)
    for i in range(len(comps)):
        if i not in reach:
            k[i] = 0
    info["k"] = k
    out = ph.copy()
    for i, L in enumerate(comps):
        if k[i] != 0:
            # a Python float added to a float32 array stays float32 (:1014-1018)
            out[labeled == L] += int(k[i]) * 2 * np.pi
    return (out, info) if return_info else out
