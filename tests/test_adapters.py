"""Task adapters and the tiled overlap unwrap (insardev/insardev/Stack_unwrap2d.py:32-130, :992-1136).

CPU tests cover the tile geometry and the stitching with the solver replaced
by a stand-in that labels every pixel with the tile it was solved in; the GPU
tests solve for real and compare each trimmed tile with a separate solve of
its halo'd block and with the oracle.
"""
import numpy as np
import pytest

from core_b200 import adapters
from core_b200.adapters import overlap_tiles, unwrap2d_chunk

PARAMS = ('cuda', 50, 1e-3, 20, 1e-4, 1e-2, 30, False, 1)


# ------------------------------------------------------------------ geometry (CPU)
@pytest.mark.parametrize("H,W,chunks,overlap", [
    (300, 260, (128, 128), 0.25), (300, 260, (128, 100), 16), (64, 64, (64, 64), None),
    (513, 77, (128, 32), (0.1, 5)), (1000, 1000, (300, 300), 150), (90, 90, ((30, 60), (45, 45)), 8),
])
def test_tiles_partition_raster(H, W, chunks, overlap):
    dy, dx, tiles = overlap_tiles(H, W, chunks, overlap)
    cover = np.zeros((H, W), np.int32)
    for y0, y1, x0, x1, ey0, ey1, ex0, ex1 in tiles:
        cover[y0:y1, x0:x1] += 1
        assert ey0 == max(0, y0 - dy) and ey1 == min(H, y1 + dy)
        assert ex0 == max(0, x0 - dx) and ex1 == min(W, x1 + dx)
        assert y1 - y0 >= min(dy, H) and x1 - x0 >= min(dx, W)
    assert (cover == 1).all()


def test_depth_rules():
    # Stack_unwrap2d.py:1091-1092: float = fraction of the first chunk, int = pixels, >= 1
    assert overlap_tiles(256, 256, (128, 64), 0.25)[:2] == (32, 16)
    assert overlap_tiles(256, 256, (128, 64), 7)[:2] == (7, 7)
    assert overlap_tiles(256, 256, (128, 64), (3, 0.5))[:2] == (3, 32)
    assert overlap_tiles(256, 256, (128, 64), None)[:2] == (1, 1)
    assert overlap_tiles(256, 256, (128, 64), 0.001)[:2] == (1, 1)


def test_small_trailing_chunk_merged():
    _, _, tiles = overlap_tiles(1000, 64, (300, 64), 150)
    assert [(t[0], t[1]) for t in tiles] == [(0, 300), (300, 600), (600, 1000)]
    _, _, tiles = overlap_tiles(1000, 64, (300, 64), 100)
    assert [(t[0], t[1]) for t in tiles] == [(0, 300), (300, 600), (600, 900), (900, 1000)]


def test_bad_chunk_tuple_rejected():
    with pytest.raises(ValueError):
        overlap_tiles(90, 90, ((30, 50), (45, 45)), 4)


def _fake_batch(calls):
    def fake(phases, weights=None, device='auto', **kw):
        calls.append((len(phases), None if weights is None else len(weights), kw))
        out = []
        for i, p in enumerate(phases):
            u = np.where(np.isnan(p), np.nan, float(len(calls) * 1000 + i)).astype(np.float32)
            out.append((u, np.zeros(p.shape, np.uint16)))
        return out
    return fake


def test_stitching_trims_every_halo(monkeypatch):
    calls = []
    monkeypatch.setattr(adapters, "irls_unwrap_2d_batch", _fake_batch(calls))
    rng = np.random.default_rng(0)
    p = rng.uniform(-np.pi, np.pi, (2, 100, 90))
    p[1, :60, :55] = np.nan                      # one all-NaN halo'd block in the second pair
    out = unwrap2d_chunk(p, chunks=(50, 45), overlap=10, max_iter=7)
    assert out.shape == p.shape and out.dtype == np.float32
    assert len(calls) == 1 and calls[0][0] == 7 and calls[0][2]["max_iter"] == 7
    assert calls[0][2]["tol"] == 1e-2 and calls[0][2]["cg_max_iter"] == 10     # method defaults
    assert np.isnan(out[1, :50, :45]).all()
    # each chunk carries the single value its own solve produced
    k = 0
    for s in range(2):
        for y0 in (0, 50):
            for x0 in (0, 45):
                blk = out[s, y0:y0 + 50, x0:x0 + 45]
                if s == 1 and y0 == 0 and x0 == 0:
                    continue
                v = np.isfinite(p[s, y0:y0 + 50, x0:x0 + 45])
                assert (blk[v] == 1000 + k).all() and np.isnan(blk[~v]).all()
                k += 1


def test_overlap_kernel_and_chunk_adapters(monkeypatch):
    calls = []
    monkeypatch.setattr(adapters, "irls_unwrap_2d_batch", _fake_batch(calls))
    monkeypatch.setattr(adapters, "irls_unwrap_2d",
                        lambda p, w=None, **kw: (np.zeros(p.shape, np.float32) + 3, np.ones(p.shape, np.uint16)))
    blk = np.random.default_rng(1).uniform(-3, 3, (3, 20, 24))
    blk[1] = np.nan
    out = adapters._irls_overlap_kernel(blk, PARAMS)
    assert out.shape == blk.shape and out.dtype == np.float32 and np.isnan(out[1]).all()
    assert calls[-1][0] == 2 and calls[-1][1] is None
    adapters._irls_overlap_kernel(blk, np.ones_like(blk), PARAMS)
    assert calls[-1][1] == 2
    u = adapters._irls_process_no_weight(blk[:1], PARAMS)
    assert u.shape == (1, 20, 24) and (u == 3).all()
    st = adapters._irls_process_with_weight_conncomp(blk[0], np.ones((20, 24)), PARAMS)
    assert st.shape == (1, 2, 20, 24) and st.dtype == np.float32 and (st[0, 1] == 1).all()
    u, cc = adapters._irls_process_chunk_with_tuple(blk[1:2], None, PARAMS)
    assert np.isnan(u).all() and (cc == 0).all() and cc.dtype == np.uint16
    with pytest.raises(ValueError):
        adapters._irls_process_chunk_with_tuple(blk[None], None, PARAMS)


# ------------------------------------------------------------------ GPU
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.gpu
def test_tiled_unwrap_equals_per_tile_solves():
    _gpu()
    import core_b200
    from core_b200.synthetic import gen_g1
    p, c, _ = gen_g1(300, 260, seed=31)
    w = np.stack([c, c])
    ps = np.stack([p, gen_g1(300, 260, seed=32)[0]])
    kw = dict(max_iter=30, tol=1e-3, cg_max_iter=20, cg_tol=1e-4)
    out = core_b200.unwrap2d_chunk(ps, w, chunks=(128, 128), overlap=0.25, **kw)
    _, _, tiles = overlap_tiles(300, 260, (128, 128), 0.25)
    for s in range(2):
        for y0, y1, x0, x1, ey0, ey1, ex0, ex1 in tiles:
            u, _ = core_b200.irls_unwrap_2d(ps[s, ey0:ey1, ex0:ex1], w[s, ey0:ey1, ex0:ex1], **kw)
            ref = u[y0 - ey0:y1 - ey0, x0 - ex0:x1 - ex0]
            got = out[s, y0:y1, x0:x1]
            assert (np.isnan(ref) == np.isnan(got)).all()
            v = np.isfinite(ref)
            assert np.abs(got[v] - ref[v]).max() <= 1e-4


@pytest.mark.gpu
def test_tiled_unwrap_matches_oracle_per_tile():
    _gpu()
    import core_b200
    from core_b200.synthetic import gen_g1
    from oracle.irls_oracle import cycle_map, irls_unwrap_2d as oracle_unwrap
    p, c, _ = gen_g1(200, 180, seed=33)
    out = core_b200.unwrap2d_chunk(p, c, chunks=(100, 90), overlap=12)
    _, _, tiles = overlap_tiles(200, 180, (100, 90), 12)
    for y0, y1, x0, x1, ey0, ey1, ex0, ex1 in tiles:
        uo, _ = oracle_unwrap(p[ey0:ey1, ex0:ex1], c[ey0:ey1, ex0:ex1], max_iter=50, tol=1e-2,
                              cg_max_iter=10, cg_tol=1e-3)
        ref = uo[y0 - ey0:y1 - ey0, x0 - ex0:x1 - ex0]
        got = out[y0:y1, x0:x1]
        ph = p[y0:y1, x0:x1]
        v = np.isfinite(ph)
        assert (np.isnan(ref) == np.isnan(got)).all()
        assert (cycle_map(got, ph) == cycle_map(ref, ph))[v].mean() >= 0.9999
        e = (got.astype(np.float64) - ref)[v]
        assert np.sqrt(np.mean((e - e.mean()) ** 2)) <= 1e-3


@pytest.mark.gpu
def test_overlap_kernel_matches_single_solves():
    _gpu()
    import core_b200
    from core_b200.synthetic import gen_g1, gen_g2
    blk = np.stack([gen_g1(96, 112, seed=41)[0], np.full((96, 112), np.nan), gen_g2(96, 112, seed=42)[0]])
    out = adapters._irls_overlap_kernel(blk, PARAMS)
    assert np.isnan(out[1]).all()
    for i in (0, 2):
        u, _ = core_b200.irls_unwrap_2d(blk[i], None, max_iter=50, tol=1e-3, cg_max_iter=20, cg_tol=1e-4)
        v = np.isfinite(u)
        assert (np.isnan(u) == np.isnan(out[i])).all()
        assert np.abs(out[i][v] - u[v]).max() <= 1e-4
