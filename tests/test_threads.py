"""Concurrent calls from several host threads (the reference is called from dask
worker threads, Stack_unwrap2d.py:20,63): each call owns its workspace and its
capture stream, so results equal the serial ones bit for bit."""
import concurrent.futures as cf

import numpy as np
import pytest


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _same(a, b):
    na = np.isnan(a)
    return np.array_equal(na, np.isnan(b)) and np.array_equal(a[~na], b[~na])


@pytest.mark.gpu
def test_unwrap_from_threads_equals_serial():
    _gpu()
    import core_b200
    from core_b200.synthetic import gen_g1, gen_g2
    inputs = [gen_g1(256 + 32 * k, 300 - 16 * k, seed=k) for k in range(3)] + [gen_g2(384, seed=5)]
    serial = [core_b200.irls_unwrap_2d(p, c) for p, c, _ in inputs]
    with cf.ThreadPoolExecutor(4) as ex:
        for _ in range(2):
            got = list(ex.map(lambda t: core_b200.irls_unwrap_2d(t[0], t[1]), inputs))
            for (u, cc), (us, ccs) in zip(got, serial):
                assert _same(u, us) and np.array_equal(cc, ccs)


@pytest.mark.gpu
def test_link_and_filter_from_threads_equal_serial():
    _gpu()
    import core_b200
    from core_b200.synthetic import gen_g1, gen_link_scene
    scenes = [gen_link_scene(200 + 20 * k, 240, 20, seed=k, holes=k % 2 == 1) for k in range(4)]
    serial = [core_b200.link_components(ph, cc, conncomp_size=30) for ph, cc in scenes]
    p, c, _ = gen_g1(200, 180, seed=7)
    z = np.exp(1j * p.astype(np.float64)).astype(np.complex64)
    z[np.isnan(p)] = np.nan
    gs = core_b200.goldstein(z, c, 32)
    with cf.ThreadPoolExecutor(5) as ex:
        futs = [ex.submit(core_b200.link_components, ph, cc, conncomp_size=30) for ph, cc in scenes]
        fg = ex.submit(core_b200.goldstein, z, c, 32)
        for f, ref in zip(futs, serial):
            assert _same(f.result(), ref)
        assert _same(fg.result(), gs)
