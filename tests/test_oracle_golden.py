"""The numpy oracle against outputs of the reference unwrapper itself (tests/golden).

The fixtures were produced by tests/golden/make_golden.py, which runs
insardev/insardev/utils_unwrap2d.py:irls_unwrap_2d; this pins the oracle
before any GPU result is compared with it.
"""
import numpy as np
import pytest

from conftest import load_golden, small_golden_names
from core_b200.synthetic import gen_g1, gen_g2
from oracle.irls_oracle import OracleStats, cycle_map, irls_unwrap_2d


@pytest.mark.parametrize("name", small_golden_names())
def test_oracle_matches_reference(name):
    d = load_golden(name)
    p = d["phase"]
    dt = np.float64 if str(d["precision"]) == "fp64" else np.float32
    st = OracleStats()
    u, cc = irls_unwrap_2d(p, d["w"], dtype=dt, stats=st, **d["kw"])
    ur, ccr = d["u"], d["cc"]
    assert u.dtype == np.float32 and cc.dtype == np.uint16
    assert u.shape == p.shape and cc.shape == p.shape
    assert (np.isnan(u) == np.isnan(ur)).all()
    assert (cc == ccr).all()
    v = np.isfinite(p)
    if not v.any():
        return
    assert st.irls_iters == int(d["iters"])
    assert (cycle_map(u, p) == cycle_map(ur, p))[v].all()
    v &= np.isfinite(ur)  # an infinite input phase leaves its component NaN
    if not v.any():
        return
    e = (u - ur)[v].astype(np.float64)
    rms = np.sqrt(np.mean((e - e.mean()) ** 2))
    assert rms <= (1e-6 if dt == np.float64 else 1e-4)


def test_generators_reproduce_fixture_inputs():
    d = load_golden("g1_64_fn")
    p, c, _ = gen_g1(64, seed=1)
    np.testing.assert_array_equal(p, d["phase"])
    np.testing.assert_array_equal(c, d["w"])
    d = load_golden("g2_128_fn")
    p, c, _ = gen_g2(128, seed=4)
    np.testing.assert_array_equal(p, d["phase"])


def test_generator_nan_fraction():
    for seed in range(3):
        p, c, _ = gen_g1(256, 192, seed=seed)
        f = np.isnan(p).mean()
        assert 0.045 <= f <= 0.055
        assert (np.isnan(p) == np.isnan(c)).all()
        assert np.nanmax(np.abs(p)) <= np.pi + 1e-6


def test_oracle_fp32_vs_fp64_cycle_map():
    d32, d64 = load_golden("g2_128_fn"), load_golden("g2_128_fn_fp64")
    p = d32["phase"]
    v = np.isfinite(p)
    assert (cycle_map(d32["u"], p) == cycle_map(d64["u"], p))[v].mean() >= 0.9999
