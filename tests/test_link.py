"""Component linking (insardev/insardev/utils_unwrap2d.py:195-444, :886-1040; Stack_unwrap2d.py:325-407).

Golden fixtures: the reference's own linking functions run with stand-in
geometry and CP-SAT modules (tests/golden/make_link_golden.py).  CPU tests pin
the oracle to them and pin its primitives (border pixels against cv2 contours,
hulls against qhull, the integer program against enumeration); GPU tests
compare the CUDA path with the fixtures and the oracle.  The bar is exact:
identical connection lists (indices, pixels, distances, window means) and
bit-identical output rasters.
"""
import glob
import itertools
import os

import numpy as np
import pytest

from conftest import REPO
from oracle import link_oracle as O

GOLD = sorted(glob.glob(os.path.join(REPO, "tests", "golden", "lk_*.npz")))
IDS = [os.path.basename(p)[:-4] for p in GOLD]


def load(path):
    d = np.load(path)
    csize, gap, lsize, lcount = d["params"]
    return dict(phase=d["phase"], conncomp=d["conncomp"] if bool(d["use_conncomp"]) else None,
                conncomp_size=int(csize), conncomp_gap=None if gap < 0 else float(gap),
                conncomp_linksize=int(lsize), conncomp_linkcount=int(lcount)), d


def conn_array(conns):
    return np.array([(c[0], c[1], c[2][0], c[2][1], c[3][0], c[3][1], c[4], c[5], float(c[6]), float(c[7]))
                     for c in conns], np.float64).reshape(-1, 10)


def same_raster(a, b):
    na = np.isnan(a)
    return np.array_equal(na, np.isnan(b)) and np.array_equal(a[~na], b[~na])


def test_fixtures_present():
    assert len(GOLD) >= 8


@pytest.mark.parametrize("path", GOLD, ids=IDS)
def test_oracle_matches_reference_fixture(path):
    kw, d = load(path)
    out, info = O.link(return_info=True, **kw)
    np.testing.assert_array_equal(conn_array(info["connections"]), d["connections"])
    assert same_raster(out, d["out"])


def _random_labels(rng, H, W, p):
    from scipy import ndimage
    m = ndimage.binary_opening(rng.random((H, W)) < p) if rng.random() < 0.5 else rng.random((H, W)) < p
    lab, n = ndimage.label(m, structure=O.STRUCT4)
    return lab, n


def test_border_pixels_equal_cv2_contours():
    cv2 = pytest.importorskip("cv2")
    from scipy import ndimage
    rng = np.random.default_rng(0)
    for _ in range(60):
        H, W = rng.integers(5, 40, 2)
        lab, n = _random_labels(rng, H, W, rng.uniform(0.4, 0.8))
        for L in range(1, n + 1):
            sl = ndimage.find_objects(lab)[L - 1]
            cs, _ = cv2.findContours((lab[sl] == L).astype(np.uint8), cv2.RETR_TREE, cv2.CHAIN_APPROX_NONE)
            pts = {(int(y) + sl[0].start, int(x) + sl[1].start) for c in cs for x, y in c.reshape(-1, 2)}
            assert {tuple(p) for p in O.border_points(lab, L).tolist()} == pts


def test_short_contours_are_straight_lines():
    """The reference skips contours of < 3 points (utils_unwrap2d.py:240-241): one-row / one-column components."""
    cv2 = pytest.importorskip("cv2")
    from scipy import ndimage
    rng = np.random.default_rng(1)
    for _ in range(60):
        H, W = rng.integers(5, 40, 2)
        lab, n = _random_labels(rng, H, W, rng.uniform(0.3, 0.8))
        for L in range(1, n + 1):
            sl = ndimage.find_objects(lab)[L - 1]
            cm = (lab[sl] == L).astype(np.uint8)
            cs, _ = cv2.findContours(cm, cv2.RETR_TREE, cv2.CHAIN_APPROX_SIMPLE)
            short = any(len(c) < 3 for c in cs)
            assert short == (cm.shape[0] == 1 or cm.shape[1] == 1)


def test_hull_matches_qhull():
    from scipy.spatial import ConvexHull
    rng = np.random.default_rng(2)
    for _ in range(100):
        pts = rng.integers(0, 50, (rng.integers(3, 60), 2))
        if np.linalg.matrix_rank(pts - pts[0]) < 2:
            continue
        h = O.convex_hull(pts)
        q = ConvexHull(pts[:, ::-1].astype(float))
        assert set(h) == {tuple(int(v) for v in pts[k, ::-1]) for k in q.vertices}
        n = len(h)
        assert all(O._cross(h[k], h[(k + 1) % n], h[(k + 2) % n]) > 0 for k in range(n))


def test_hull_distance_against_dense_sampling():
    rng = np.random.default_rng(3)
    for _ in range(40):
        A = O.convex_hull(rng.integers(0, 30, (8, 2)))
        B = O.convex_hull(rng.integers(0, 30, (8, 2)) + rng.integers(-20, 20, 2))
        if len(A) < 3 or len(B) < 3:
            continue
        d = O.hull_distance(A, B)

        def edge_pts(V):
            t = np.linspace(0, 1, 200)[:, None]
            return np.concatenate([np.array(V[k]) * (1 - t) + np.array(V[(k + 1) % len(V)]) * t
                                   for k in range(len(V))])
        ea, eb = edge_pts(A), edge_pts(B)
        dd = np.sqrt(((ea[:, None] - eb[None]) ** 2).sum(-1)).min()
        if d > 0:
            assert abs(dd - d) <= 0.2
        else:
            # meeting: a vertex of one inside the other, or boundaries within sampling resolution
            assert dd <= 0.2 or any(all(O._cross(B[k], B[(k + 1) % len(B)], p) >= 0 for k in range(len(B)))
                                    for p in A) or any(all(O._cross(A[k], A[(k + 1) % len(A)], q) >= 0
                                                           for k in range(len(A))) for q in B)


def _enumerate(n, edges, sign, R=4):
    best = None
    s = 1 if sign == "reference" else -1
    for ks in itertools.product(range(-R, R + 1), repeat=n - 1):
        k = (0,) + ks
        obj = sum(w * abs(s * (k[i] - k[j]) - off) for i, j, off, w in edges)
        key = (obj, sum(abs(v) for v in k))
        if best is None or key < best[0]:
            best = (key, [k])
        elif key == best[0]:
            best[1].append(k)
    return best


@pytest.mark.parametrize("sign", ["reference", "aligned"])
def test_offsets_program_matches_enumeration(sign):
    rng = np.random.default_rng(4)
    checked = 0
    for _ in range(40):
        n = int(rng.integers(2, 6))
        m = int(rng.integers(1, 8))
        edges = []
        for _ in range(m):
            i, j = sorted(rng.choice(n, 2, replace=False).tolist())
            edges.append((i, j, int(rng.integers(-1, 2)), int(rng.integers(0, 3000))))
        (obj, sec), sols = _enumerate(n, edges, sign)
        from core_b200.link import solve_offsets as native
        s = 1 if sign == "reference" else -1
        for k in (O.solve_offsets(n, edges, sign), native(n, edges, sign)):
            got = sum(w * abs(s * (k[i] - k[j]) - off) for i, j, off, w in edges)
            assert got == obj and int(np.abs(k).sum()) == sec
            if len(sols) == 1:
                assert tuple(k.tolist()) == sols[0]
        checked += len(sols) == 1
    assert checked >= 20


def test_native_offsets_match_milp_on_large_programs():
    """The library's exact solver (unw_link_offsets, no GPU) against the oracle's HiGHS MILP."""
    from core_b200.link import solve_offsets as native
    rng = np.random.default_rng(5)
    for n, m in ((40, 150), (200, 900)):
        edges = []
        while len(edges) < m:
            i, j = (int(v) for v in rng.integers(0, n, 2))
            if i != j:
                edges.append((min(i, j), max(i, j), int(rng.integers(-3, 4)), int(rng.integers(0, 2_000_000))))
        for sign in ("reference", "aligned"):
            np.testing.assert_array_equal(native(n, edges, sign), O.solve_offsets(n, edges, sign))


def test_aligned_sign_removes_offsets():
    """With sign='aligned' three shifted blobs come back to one level; the reference sign does not."""
    H, W = 40, 100
    yy, xx = np.mgrid[:H, :W]
    truth = (0.02 * xx).astype(np.float32)
    ph = np.full((H, W), np.nan, np.float32)
    for x0, m in ((5, 0), (38, 1), (71, -1)):
        sl = (slice(10, 30), slice(x0, x0 + 24))
        ph[sl] = truth[sl] + np.float32(2 * np.pi * m)
    fixed = O.link(ph, conncomp_size=10, sign="aligned")
    v = ~np.isnan(fixed)
    # aligned to the first (largest) component: one constant 2-pi multiple everywhere
    assert np.ptp(fixed[v] - truth[v]) < 1e-4
    ref = O.link(ph, conncomp_size=10)
    assert np.ptp(ref[v] - truth[v]) > 6.0


# ------------------------------------------------------------------ GPU
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _scene(seed, H, W, n_blobs, holes=False, noise=0.15, rmax=None):
    from core_b200.synthetic import gen_link_scene
    return gen_link_scene(H, W, n_blobs, seed=seed, holes=holes, noise=noise, rmax=rmax)


def _check_cuda_vs(kw, ref_conns, ref_out):
    import core_b200
    out, info = core_b200.link_components(return_info=True, **kw)
    assert out.dtype == np.float32 and out.shape == kw["phase"].shape
    np.testing.assert_array_equal(conn_array(info["connections"]), ref_conns)
    assert same_raster(out, ref_out)
    return info


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLD, ids=IDS)
def test_cuda_matches_reference_fixture(path):
    _gpu()
    kw, d = load(path)
    _check_cuda_vs(kw, d["connections"], d["out"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLD, ids=IDS)
def test_reference_signature_dropins_match_fixture(path):
    """find_component_connections_fast / connect_components_ilp_fast with the reference's signatures,
    driven through the _link_2d steps (Stack_unwrap2d.py:345-407)."""
    _gpu()
    from core_b200 import link as L
    kw, d = load(path)
    ph, cc = kw["phase"], kw["conncomp"]
    min_size = max(kw["conncomp_size"], 4)
    if cc is not None:
        labeled, comps, sizes = O.components_from_labels(cc, min_size)
    else:
        labeled, comps, sizes = O.components_from_mask(~np.isnan(ph), min_size)
    dicts = [{"label": lab, "size": sizes[lab], "slices": None} for lab in comps]
    ph2 = ph.copy()
    ph2[~(np.isin(labeled, comps) | (labeled == 0))] = np.nan
    conns = L.find_component_connections_fast(labeled, ph2, dicts, kw["conncomp_gap"], kw["conncomp_linkcount"],
                                              kw["conncomp_linksize"]) if len(comps) >= 2 else []
    np.testing.assert_array_equal(conn_array(conns), d["connections"])
    out = L.connect_components_ilp_fast(ph2, labeled, dicts, conns)
    assert same_raster(out, d["out"])


CASES = [
    # seed, H, W, blobs, holes, use labels, conncomp_size, gap, linksize, linkcount
    (101, 160, 200, 14, False, True, 30, None, 5, 30),
    (102, 160, 200, 14, True, False, 30, None, 5, 30),
    (103, 200, 180, 24, True, True, 20, None, 5, 2),
    (104, 220, 260, 30, False, False, 40, 15.0, 7, 3),
    (105, 128, 333, 18, True, True, 10, 25.0, 3, 1),
    (106, 300, 301, 40, True, True, 60, None, 9, 4),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[str(c[0]) for c in CASES])
def test_cuda_matches_oracle(case):
    _gpu()
    seed, H, W, nb, holes, use_cc, csize, gap, lsize, lcount = case
    ph, cc = _scene(seed, H, W, nb, holes)
    kw = dict(phase=ph, conncomp=cc if use_cc else None, conncomp_size=csize, conncomp_gap=gap,
              conncomp_linksize=lsize, conncomp_linkcount=lcount)
    ref, rinfo = O.link(return_info=True, **kw)
    info = _check_cuda_vs(kw, conn_array(rinfo["connections"]), ref)
    assert len(info["components"]) == len(rinfo["components"])
    if not use_cc:
        assert list(info["sizes"]) == [int((np.asarray(O.components_from_mask(~np.isnan(ph), max(csize, 4))[0])
                                             == L).sum()) for L in rinfo["components"]]


@pytest.mark.gpu
@pytest.mark.parametrize("sign", ["reference", "aligned"])
def test_cuda_sign_and_tensor_io(sign):
    torch = _gpu()
    import core_b200
    ph, cc = _scene(107, 150, 170, 12, False)
    ref = O.link(ph, cc, conncomp_size=30, sign=sign)
    dev = torch.device("cuda", 0)
    t = core_b200.link_components(torch.from_numpy(ph).to(dev), torch.from_numpy(cc.astype(np.int32)).to(dev),
                                  conncomp_size=30, sign=sign)
    assert t.is_cuda and t.dtype == torch.float32
    assert same_raster(t.cpu().numpy(), ref)
    out3 = core_b200.link_components(ph[None], cc[None], conncomp_size=30, sign=sign)
    assert out3.shape == (1,) + ph.shape and same_raster(out3[0], ref)


@pytest.mark.gpu
def test_cuda_edge_cases():
    _gpu()
    import core_b200
    allnan = np.full((20, 30), np.nan, np.float32)
    assert np.isnan(core_b200.link_components(allnan)).all()
    one = np.zeros((20, 30), np.float32)
    assert same_raster(core_b200.link_components(one), one)
    # a small labelled component is removed, label 0 pixels are kept
    ph, cc = _scene(108, 80, 90, 6, False)
    cc2 = cc.copy()
    cc2[cc == cc.max()] = 0
    for kw in (dict(conncomp=cc2, conncomp_size=10 ** 6), dict(conncomp=cc, conncomp_size=50)):
        out = core_b200.link_components(ph, **kw)
        assert same_raster(out, O.link(ph, **kw))


@pytest.mark.gpu
def test_unwrap2d_links_irls_components():
    _gpu()
    import core_b200
    ph, _ = _scene(109, 180, 240, 12, False, noise=0.3)
    wrapped = np.angle(np.exp(1j * ph.astype(np.float64))).astype(np.float32)
    wrapped[np.isnan(ph)] = np.nan
    u, cc = core_b200.unwrap2d(wrapped, conncomp=True, conncomp_size=50)
    out = core_b200.unwrap2d(wrapped, conncomp_size=50)
    assert same_raster(out, O.link(u, cc, conncomp_size=50))
    stack = core_b200.unwrap2d(np.stack([wrapped, wrapped]), conncomp_size=50)
    assert stack.shape == (2,) + wrapped.shape and same_raster(stack[1], out)
    with pytest.raises(ValueError):
        core_b200.unwrap2d(wrapped, conncomp_size=4, conncomp_linksize=5)


@pytest.mark.gpu
def test_cuda_large_grid_properties():
    """2048^2 with a few hundred components: each component moves by one 2-pi multiple, the first stays."""
    _gpu()
    import core_b200
    ph, cc = _scene(110, 2048, 2048, 600, True, rmax=45)
    out, info = core_b200.link_components(ph, cc, conncomp_size=200, return_info=True)
    comps = info["components"]
    assert len(comps) > 50 and len(info["connections"]) > len(comps) // 2
    d = (out.astype(np.float64) - ph) / (2 * np.pi)
    for c, L in enumerate(comps[:60]):
        m = cc == L
        kd = np.unique(np.round(d[m]))
        assert len(kd) == 1 and kd[0] == info["k"][c]
        assert np.abs(d[m] - kd[0]).max() < 1e-5
    assert info["k"][0] == 0
    small = (cc > 0) & ~np.isin(cc, comps)
    assert np.isnan(out[small]).all()


EDGE = [
    # name, kwargs for the scene and link, transformed labels
    ("window0", dict(conncomp_linksize=0), None),
    ("window1", dict(conncomp_linksize=1), None),
    ("window31", dict(conncomp_linksize=31), None),
    ("k_all", dict(conncomp_linkcount=1000), None),
    ("k0", dict(conncomp_linkcount=0), None),
    ("gap0", dict(conncomp_gap=0.0), None),
    ("label_gaps", dict(), "gaps"),
    ("edges", dict(), "edges"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,mode", EDGE, ids=[e[0] for e in EDGE])
def test_cuda_edge_parameters_match_oracle(name, kw, mode):
    _gpu()
    import core_b200
    ph, cc = _scene(111, 140, 190, 16, True)
    if mode == "gaps":                      # label values with holes in the numbering
        cc = np.where(cc > 0, cc * 3 + 7, 0).astype(np.uint16)
    if mode == "edges":                     # components cut by every raster edge
        ph, cc = ph[20:120, 30:160].copy(), cc[20:120, 30:160].copy()
        from scipy import ndimage
        lab, n = ndimage.label(cc > 0, structure=O.STRUCT4)
        sizes = np.bincount(lab.ravel(), minlength=n + 1)
        order = sorted(range(1, n + 1), key=lambda L: (-sizes[L], -L))
        lut = np.zeros(n + 1, np.uint16)
        lut[order] = np.arange(1, n + 1)
        cc = lut[lab]
        ph[cc == 0] = np.nan
    args = dict(conncomp_size=20)
    args.update(kw)
    for labels in (cc, None):
        ref, rinfo = O.link(ph, labels, return_info=True, **args)
        out, info = core_b200.link_components(ph, labels, return_info=True, **args)
        np.testing.assert_array_equal(conn_array(info["connections"]), conn_array(rinfo["connections"]))
        assert same_raster(out, ref)


@pytest.mark.gpu
def test_unwrap2d_link_stack_and_validation():
    _gpu()
    import core_b200
    a, _ = _scene(112, 120, 150, 12, False)
    b, _ = _scene(113, 120, 150, 12, True)
    out = core_b200.unwrap2d_link(np.stack([a, b]), conncomp_size=40)
    for k, ph in enumerate((a, b)):
        assert same_raster(out[k], O.link(ph, None, conncomp_size=40))
    with pytest.raises(ValueError):
        core_b200.unwrap2d_link(a, conncomp_size=4, conncomp_linksize=5)


@pytest.mark.gpu
def test_cuda_lines_only_and_single_component():
    """Straight-line components take no part (no contour polygon); one component: NaN filter only."""
    _gpu()
    import core_b200
    ph = np.full((40, 60), np.nan, np.float32)
    ph[5, 2:50] = 1.0
    ph[20, 3:58] = 2.0
    ph[30:39, 10] = 3.0
    for labels in (None,):
        out, info = core_b200.link_components(ph, labels, conncomp_size=5, return_info=True)
        assert len(info["components"]) == 3 and info["connections"] == []
        assert same_raster(out, ph)
    blob = np.full((30, 30), np.nan, np.float32)
    blob[5:20, 5:20] = 0.5
    blob[25, 25] = 9.0                      # a one-pixel component below the size: NaN
    out = core_b200.link_components(blob, conncomp_size=10)
    ref = O.link(blob, conncomp_size=10)
    assert same_raster(out, ref) and np.isnan(out[25, 25])


@pytest.mark.gpu
@pytest.mark.parametrize("prob,K", [(0.5, 30), (0.4, 30), (0.5, 3), (0.6, 5)])
def test_cuda_noisy_mask_matches_oracle(prob, K):
    """Dense random masks: many small interleaved components, most hulls overlapping."""
    _gpu()
    import core_b200
    rng = np.random.default_rng(int(prob * 100) + K)
    valid = rng.random((60, 80)) < prob
    ph = np.where(valid, rng.normal(0, 1, (60, 80)), np.nan).astype(np.float32)
    ref, rinfo = O.link(ph, None, conncomp_size=4, conncomp_linkcount=K, return_info=True)
    out, info = core_b200.link_components(ph, None, conncomp_size=4, conncomp_linkcount=K, return_info=True)
    assert len(info["components"]) == len(rinfo["components"])
    np.testing.assert_array_equal(conn_array(info["connections"]), conn_array(rinfo["connections"]))
    assert same_raster(out, ref)


@pytest.mark.gpu
def test_cuda_many_components_fill_the_pair_arrays():
    """Thousands of components: more components and candidate pairs than the first output arrays
    hold, so the host call is repeated with larger arrays; the 4-connected components and the
    candidate pairs must come back complete (checked on a sample against the oracle's geometry)."""
    _gpu()
    import core_b200
    from core_b200 import link as L
    import torch
    rng = np.random.default_rng(3)
    valid = rng.random((512, 512)) < 0.5
    ph = np.where(valid, rng.normal(0, 1, (512, 512)), np.nan).astype(np.float32)
    dev = torch.device("cuda", 0)
    t = torch.from_numpy(ph).to(dev)
    clab, csz, pairs, npair, _ = L._device_pairs(t, None, 4, 30, 5, dev, torch.cuda.current_stream(dev).cuda_stream)
    labeled, comps, sizes = O.components_from_mask(valid, 4)
    assert len(clab) == len(comps) > 1024
    assert list(csz) == [int(sizes[c]) for c in comps]
    P = np.ctypeslib.as_array(pairs, shape=(len(pairs),))[:npair]
    assert npair > 1024 * 30 and (P["comp_i"] < P["comp_j"]).all() and (P["d2"] > 0).all()
    for k in rng.choice(npair, 40, replace=False):
        i, j = int(P["comp_i"][k]), int(P["comp_j"][k])
        d2, yi, xi, yj, xj = O.nearest_pair(O.border_points(labeled, comps[i]), O.border_points(labeled, comps[j]))
        assert (int(P["d2"][k]), int(P["yi"][k]), int(P["xi"][k]), int(P["yj"][k]), int(P["xj"][k])) == \
            (d2, yi, xi, yj, xj)
    out, info = core_b200.link_components(ph, None, conncomp_size=4, return_info=True)
    assert len(info["connections"]) > 0
