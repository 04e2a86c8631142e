"""Generate component-linking golden fixtures by running the reference linking code.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_link_golden.py --ref <insardev checkout> (or INSARDEV_REF=<checkout>)

The reference functions `find_component_connections_fast` and
`connect_components_ilp_fast` (insardev/insardev/utils_unwrap2d.py:195-444,
:886-1040) run unmodified, loaded as in make_golden.py.  They call cv2 (present)
for the contours, and shapely and OR-Tools, which are absent here; those two are
replaced by small stand-in modules defined below:

  * geometry on the pixel lattice: a contour polygon's boundary is the set of
    lattice points on its closed polyline (the cv2 CHAIN_APPROX_SIMPLE vertices
    joined by their horizontal, vertical or diagonal runs); the union of a
    component's boundaries has as convex hull scipy's qhull hull; distances,
    nearest points and intersection tests are exact on those point sets and
    polygons, with ties broken by index / lexicographic (x, y) order;
  * CP-SAT: the model the reference builds is solved by enumerating every
    assignment in a box around zero; the optimum with the least sum |k| is
    returned and the script refuses a case whose optimum is not unique.

The `_link_2d` wrapper (Stack_unwrap2d.py:325-407) sits inside a method that
needs xarray and dask; its few steps (component list, NaN filter, the two
calls) are restated in `link_2d` below.  Outputs: `.npz` fixtures `lk_*.npz`
next to this script.  Nothing at test time reads the reference tree.
"""
from __future__ import annotations

import argparse
import itertools
import math
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)


# ---------------------------------------------------------------------- stand-in shapely
def _cross(o, a, b):
    return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])


def _pseg(p, a, b):
    dx, dy = b[0] - a[0], b[1] - a[1]
    t = (p[0] - a[0]) * dx + (p[1] - a[1]) * dy
    if t <= 0:
        return math.sqrt(float((p[0] - a[0]) ** 2 + (p[1] - a[1]) ** 2))
    L2 = dx * dx + dy * dy
    if t >= L2:
        return math.sqrt(float((p[0] - b[0]) ** 2 + (p[1] - b[1]) ** 2))
    return abs(float(_cross(a, b, p))) / math.sqrt(float(L2))


def _on_seg(p, a, b):
    return (_cross(a, b, p) == 0 and min(a[0], b[0]) <= p[0] <= max(a[0], b[0])
            and min(a[1], b[1]) <= p[1] <= max(a[1], b[1]))


def _seg_meet(a, b, c, d):
    d1, d2 = _cross(c, d, a), _cross(c, d, b)
    d3, d4 = _cross(a, b, c), _cross(a, b, d)
    if ((d1 > 0 and d2 < 0) or (d1 < 0 and d2 > 0)) and ((d3 > 0 and d4 < 0) or (d3 < 0 and d4 > 0)):
        return True
    return _on_seg(a, c, d) or _on_seg(b, c, d) or _on_seg(c, a, b) or _on_seg(d, a, b)


def _inside(p, V):
    n = len(V)
    return all(_cross(V[k], V[(k + 1) % n], p) >= 0 for k in range(n))


def _edges(V):
    return [(V[k], V[(k + 1) % len(V)]) for k in range(len(V))]


class _Geom:
    geom_type = "Geometry"

    def envelope(self):
        raise NotImplementedError


class _Point(_Geom):
    geom_type = "Point"

    def __init__(self, x, y):
        self.x, self.y = x, y

    def distance(self, o):
        return math.sqrt(float((self.x - o.x) ** 2 + (self.y - o.y) ** 2))


class _PtSet(_Geom):
    """A boundary: lattice points (x, y)."""
    geom_type = "LinearRing"

    def __init__(self, pts):
        self.pts = np.array(sorted(set(map(tuple, np.asarray(pts).tolist()))), np.int64).reshape(-1, 2)
        self.length = float(len(self.pts))
        self.centroid = _Point(*self.pts.mean(0)) if len(self.pts) else None

    def envelope(self):
        return (*self.pts.min(0), *self.pts.max(0))

    def _closest(self, o):
        d2 = ((self.pts[:, None, 0] - o.pts[None, :, 0]) ** 2 + (self.pts[:, None, 1] - o.pts[None, :, 1]) ** 2)
        m = int(d2.min())
        ii, jj = np.nonzero(d2 == m)
        # lexicographic over (y_self, x_self, y_other, x_other)
        c = min(zip(self.pts[ii, 1].tolist(), self.pts[ii, 0].tolist(), o.pts[jj, 1].tolist(), o.pts[jj, 0].tolist()))
        return m, c

    def distance(self, o):
        return math.sqrt(float(self._closest(o)[0]))

    @property
    def convex_hull(self):
        from scipy.spatial import ConvexHull
        h = ConvexHull(self.pts.astype(np.float64))
        return _Hull([tuple(int(v) for v in self.pts[k]) for k in h.vertices])


class _Hull(_Geom):
    geom_type = "Polygon"

    def __init__(self, verts):
        self.V = verts                      # counter-clockwise (qhull order in 2-D)

    def envelope(self):
        xs = [v[0] for v in self.V]
        ys = [v[1] for v in self.V]
        return (min(xs), min(ys), max(xs), max(ys))

    def buffer(self, d):
        x0, y0, x1, y1 = self.envelope()
        return _Box((x0 - d, y0 - d, x1 + d, y1 + d))

    def distance(self, o):
        A, B = self.V, o.V
        if any(_inside(p, B) for p in A) or any(_inside(q, A) for q in B):
            return 0.0
        if any(_seg_meet(a, b, c, d) for a, b in _edges(A) for c, d in _edges(B)):
            return 0.0
        return min(min(_pseg(p, c, d) for p in A for c, d in _edges(B)),
                   min(_pseg(q, a, b) for q in B for a, b in _edges(A)))

    def meets_segment(self, s):
        if _inside(s.p, self.V) or _inside(s.q, self.V):
            return True
        return any(_seg_meet(s.p, s.q, c, d) for c, d in _edges(self.V))


class _Box(_Geom):
    def __init__(self, env):
        self.env = env

    def envelope(self):
        return self.env


class _Seg(_Geom):
    geom_type = "LineString"

    def __init__(self, pts):
        a, b = pts
        self.p = (int(a.x), int(a.y))
        self.q = (int(b.x), int(b.y))

    def envelope(self):
        return (min(self.p[0], self.q[0]), min(self.p[1], self.q[1]), max(self.p[0], self.q[0]),
                max(self.p[1], self.q[1]))


class Polygon(_Geom):
    geom_type = "Polygon"
    is_valid = True

    def __init__(self, pts):
        pts = np.asarray(pts, np.int64)
        ring = []
        for k in range(len(pts)):
            a, b = pts[k], pts[(k + 1) % len(pts)]
            dx, dy = int(b[0] - a[0]), int(b[1] - a[1])
            n = max(abs(dx), abs(dy))
            assert dx == 0 or dy == 0 or abs(dx) == abs(dy), "CHAIN_APPROX_SIMPLE run"
            for t in range(max(n, 1)):
                ring.append((int(a[0]) + t * np.sign(dx), int(a[1]) + t * np.sign(dy)))
        self.boundary = _PtSet(ring)


def _make_valid(p):
    return p


class STRtree:
    def __init__(self, geoms):
        self.geoms = list(geoms)

    def query(self, g, predicate=None):
        out = []
        if predicate is None:
            x0, y0, x1, y1 = g.envelope()
            for k, h in enumerate(self.geoms):
                a0, b0, a1, b1 = h.envelope()
                if a0 <= x1 and x0 <= a1 and b0 <= y1 and y0 <= b1:
                    out.append(k)
        else:
            assert predicate == "intersects" and isinstance(g, _Seg)
            out = [k for k, h in enumerate(self.geoms) if h.meets_segment(g)]
        return np.array(out, np.int64)

    def nearest(self, g):
        d = [g.distance(h) for h in self.geoms]
        return int(np.argmin(d))


def _nearest_points(a, b):
    _, (ya, xa, yb, xb) = a._closest(b)
    return _Point(xa, ya), _Point(xb, yb)


def _unary_union(geoms):
    return _PtSet(np.concatenate([g.pts for g in geoms]))


def install_shapely():
    sh = types.ModuleType("shapely")
    sh.make_valid = _make_valid
    geo = types.ModuleType("shapely.geometry")
    geo.Polygon, geo.LinearRing, geo.LineString, geo.box = Polygon, _PtSet, _Seg, None
    st = types.ModuleType("shapely.strtree")
    st.STRtree = STRtree
    ops = types.ModuleType("shapely.ops")
    ops.nearest_points, ops.unary_union = _nearest_points, _unary_union
    sh.geometry, sh.strtree, sh.ops = geo, st, ops
    sys.modules.update({"shapely": sh, "shapely.geometry": geo, "shapely.strtree": st, "shapely.ops": ops})


# ---------------------------------------------------------------------- stand-in CP-SAT
class _Expr:
    def __init__(self, terms=None, const=0):
        self.terms = dict(terms or {})
        self.const = const

    @staticmethod
    def of(v):
        return v if isinstance(v, _Expr) else _Expr({}, v)

    def __add__(self, o):
        o = _Expr.of(o)
        t = dict(self.terms)
        for k, c in o.terms.items():
            t[k] = t.get(k, 0) + c
        return _Expr(t, self.const + o.const)

    __radd__ = __add__

    def __neg__(self):
        return _Expr({k: -c for k, c in self.terms.items()}, -self.const)

    def __sub__(self, o):
        return self + (-_Expr.of(o))

    def __rsub__(self, o):
        return _Expr.of(o) + (-self)

    def __mul__(self, c):
        return _Expr({k: c * v for k, v in self.terms.items()}, c * self.const)

    __rmul__ = __mul__

    def __eq__(self, o):
        return ("eq", self, _Expr.of(o))

    __hash__ = object.__hash__


class _Var(_Expr):
    def __init__(self, model, lb, ub, name):
        super().__init__({len(model.vars): 1}, 0)
        self.idx, self.lb, self.ub, self.name = len(model.vars), lb, ub, name
        model.vars.append(self)


class CpModel:
    def __init__(self):
        self.vars, self.eqs, self.abs = [], [], []
        self.obj = None

    def NewIntVar(self, lb, ub, name):
        return _Var(self, lb, ub, name)

    def Add(self, ct):
        self.eqs.append(ct)

    def AddAbsEquality(self, a, d):
        self.abs.append((a, d))

    def Minimize(self, e):
        self.obj = e


class _Params:
    max_time_in_seconds = 0.0


class CpSolver:
    LAST = None

    def __init__(self):
        self.parameters = _Params()

    def Solve(self, m):
        kv = [v for v in m.vars if v.name.startswith("k_")]
        n = len(kv)
        fixed = {}
        defs = {}
        for _, lhs, rhs in m.eqs:
            (vi,), = [tuple(lhs.terms)]
            if rhs.terms:
                defs[vi] = rhs                     # diff = k_i - k_j - off
            else:
                fixed[vi] = rhs.const
        free = [v.idx for v in kv if v.idx not in fixed]
        offs = [abs(r.const) for r in defs.values()]
        R = max(2, int(sum(offs)))
        assert (2 * R + 1) ** len(free) <= 3_000_000, "case too large for enumeration"
        grid = np.array(list(itertools.product(range(-R, R + 1), repeat=len(free))), np.int64).reshape(-1, len(free))
        val = np.zeros((len(grid), len(m.vars)), np.int64)
        for c, vi in enumerate(free):
            val[:, vi] = grid[:, c]
        for vi, c in fixed.items():
            val[:, vi] = c
        for vi, e in defs.items():
            val[:, vi] = e.const + sum(coef * val[:, k] for k, coef in e.terms.items())
        for a, d in m.abs:
            val[:, a.idx] = np.abs(val[:, d.idx])
        obj = m.obj.const + sum(coef * val[:, k] for k, coef in m.obj.terms.items())
        sec = np.abs(val[:, [v.idx for v in kv]]).sum(1)
        best = obj.min()
        cand = np.nonzero(obj == best)[0]
        s2 = sec[cand]
        win = cand[s2 == s2.min()]
        assert len(win) == 1, "optimum not unique under (objective, sum |k|)"
        kvals = val[win[0], [v.idx for v in kv]]
        assert np.abs(kvals).max(initial=0) < R, "optimum on the enumeration box"
        self.sol = val[win[0]]
        CpSolver.LAST = kvals
        return 4

    def Value(self, v):
        return int(self.sol[v.idx])


def install_ortools():
    cp = types.ModuleType("ortools.sat.python.cp_model")
    cp.CpModel, cp.CpSolver, cp.OPTIMAL, cp.FEASIBLE = CpModel, CpSolver, 4, 2
    mods = {"ortools": types.ModuleType("ortools"), "ortools.sat": types.ModuleType("ortools.sat"),
            "ortools.sat.python": types.ModuleType("ortools.sat.python"), "ortools.sat.python.cp_model": cp}
    mods["ortools.sat.python"].cp_model = cp
    sys.modules.update(mods)


# ---------------------------------------------------------------------- reference loading and wrapper
def load_reference(ref_root):
    from make_golden import load_reference as load_unwrapper
    load_unwrapper(ref_root)
    return sys.modules["insardev.utils_unwrap2d"]


def link_2d(U, phase_2d, conncomp_2d, conncomp_size, conncomp_gap, linksize, linkcount):
    """Stack_unwrap2d.py:325-407 (`_link_2d`), steps restated; returns (result, components, connections)."""
    from scipy import ndimage
    CpSolver.LAST = None
    valid_mask = ~np.isnan(phase_2d)
    if not np.any(valid_mask):
        return phase_2d, [], []
    min_size = max(conncomp_size, 4)
    if conncomp_2d is not None:
        labeled = conncomp_2d.astype(np.int32)
        n_total = int(labeled.max())
        sizes = np.bincount(labeled.ravel(), minlength=n_total + 1)
        slices = ndimage.find_objects(labeled)
        components = [{'label': i, 'size': sizes[i], 'slices': slices[i - 1] if i > 0 and i <= len(slices) else None}
                      for i in range(1, n_total + 1)
                      if sizes[i] >= min_size and (i <= len(slices) and slices[i - 1] is not None)]
    else:
        labeled, components, n_total, sizes = U.get_connected_components(valid_mask, min_size)
    linked_labels = np.array([c['label'] for c in components])
    is_linked = np.isin(labeled, linked_labels) | (labeled == 0)
    phase_2d = phase_2d.copy()
    phase_2d[~is_linked] = np.nan
    if len(components) < 2:
        return phase_2d, components, []
    connections = U.find_component_connections_fast(labeled, phase_2d, components, conncomp_gap=conncomp_gap,
                                                     max_neighbors=linkcount, n_neighbors=linksize)
    if len(connections) == 0:
        return phase_2d, components, []
    result = U.connect_components_ilp_fast(phase_2d, labeled, components, connections, max_time=60.0)
    return result, components, connections


# ---------------------------------------------------------------------- scenes
def _ellipse(H, W, cy, cx, ry, rx):
    yy, xx = np.mgrid[:H, :W]
    return ((yy - cy) / ry) ** 2 + ((xx - cx) / rx) ** 2 <= 1.0


def scene(kind, seed):
    rng = np.random.default_rng(seed)
    H, W = {"blobs": (72, 96), "row": (40, 110), "holes": (80, 80), "many": (96, 128), "lines": (60, 70)}[kind]
    mask_parts = []
    if kind == "blobs":
        for _ in range(6):
            mask_parts.append(_ellipse(H, W, rng.uniform(8, H - 8), rng.uniform(8, W - 8), rng.uniform(4, 11),
                                       rng.uniform(4, 14)))
    elif kind == "row":
        for cx in (14, 52, 92):
            mask_parts.append(_ellipse(H, W, 20 + rng.uniform(-2, 2), cx, rng.uniform(8, 15), rng.uniform(8, 14)))
    elif kind == "holes":
        ring = _ellipse(H, W, 40, 40, 30, 30) & ~_ellipse(H, W, 40, 40, 17, 17)
        mask_parts += [ring, _ellipse(H, W, 40, 40, 9, 9), _ellipse(H, W, 8, 72, 6, 6)]
    elif kind == "many":
        for _ in range(9):
            mask_parts.append(_ellipse(H, W, rng.uniform(6, H - 6), rng.uniform(6, W - 6), rng.uniform(3, 9),
                                       rng.uniform(3, 12)))
    elif kind == "lines":
        mask_parts.append(_ellipse(H, W, 20, 20, 12, 14))
        mask_parts.append(_ellipse(H, W, 42, 50, 10, 12))
        line = np.zeros((H, W), bool)
        line[52, 5:40] = True                     # straight one-pixel line: no contour polygon
        mask_parts.append(line)
    valid = np.zeros((H, W), bool)
    for m in mask_parts:
        valid |= m
    from scipy import ndimage
    lab, n = ndimage.label(valid, structure=[[0, 1, 0], [1, 1, 1], [0, 1, 0]])
    yy, xx = np.mgrid[:H, :W]
    truth = 0.08 * yy - 0.05 * xx + 1.5 * np.sin(xx / 17.0) * np.cos(yy / 23.0)
    comp_shift = np.zeros(n + 1)
    for L in range(1, n + 1):
        comp_shift[L] = 2 * np.pi * rng.integers(-1, 2)
    ph = truth + comp_shift[lab] + rng.normal(0, 0.15, (H, W))
    ph = np.where(valid, ph, np.nan).astype(np.float32)
    sizes = np.bincount(lab.ravel(), minlength=n + 1)
    order = sorted(range(1, n + 1), key=lambda L: -sizes[L])
    assert len(set(sizes[1:].tolist())) == n, "component size tie"
    cc = np.zeros((H, W), np.uint16)
    for r, L in enumerate(order, 1):
        cc[lab == L] = r
    return ph, cc


CASES = [
    # name, scene, seed, use_conncomp, conncomp_size, gap, linksize, linkcount
    ("lk_blobs_cc", "blobs", 11, True, 30, None, 5, 30),
    ("lk_blobs_mask", "blobs", 12, False, 30, None, 5, 30),
    ("lk_many_cap1", "many", 13, True, 30, None, 5, 1),
    ("lk_row_blocked", "row", 21, True, 30, None, 5, 30),
    ("lk_holes", "holes", 31, True, 30, None, 7, 30),
    ("lk_many_gap", "many", 41, False, 40, 17.0, 5, 30),
    ("lk_many_cap2", "many", 42, True, 60, None, 3, 2),
    ("lk_lines", "lines", 51, True, 20, None, 5, 30),
]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("INSARDEV_REF"), required="INSARDEV_REF" not in os.environ,
                    help="root of the insardev source checkout (default: $INSARDEV_REF)")
    a = ap.parse_args()
    install_shapely()
    install_ortools()
    U = load_reference(a.ref)
    for name, kind, seed0, use_cc, csize, gap, lsize, lcount in CASES:
        # the first seed from seed0 whose scene has distinct component sizes and a unique optimum
        for seed in range(seed0, seed0 + 50):
            try:
                ph, cc = scene(kind, seed)
                res, comps, conns = link_2d(U, ph, cc if use_cc else None, csize, gap, lsize, lcount)
                break
            except AssertionError:
                continue
        else:
            raise RuntimeError(f"{name}: no usable seed")
        carr = np.array([(c[0], c[1], c[2][0], c[2][1], c[3][0], c[3][1], c[4], c[5], float(c[6]), float(c[7]))
                         for c in conns], np.float64).reshape(-1, 10)
        k = np.zeros(0, np.int64) if CpSolver.LAST is None else np.asarray(CpSolver.LAST, np.int64)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), phase=ph, conncomp=cc, use_conncomp=use_cc,
                            params=np.array([csize, -1.0 if gap is None else gap, lsize, lcount], np.float64),
                            comp_labels=np.array([c['label'] for c in comps], np.int64), connections=carr,
                            k_solver=k, out=res.astype(np.float32))
        print(name, "seed", seed, ph.shape, "components", len(comps), "connections", len(conns), "k", k.tolist())


if __name__ == "__main__":
    main()
