"""Goldstein adaptive filter (insardev/insardev/utils_goldstein.py:157-330, the GPU path).

Golden fixtures: the reference's own goldstein_pytorch run on the CPU torch
device (tests/golden/make_goldstein_golden.py).  CPU tests pin the oracle to
them; GPU tests compare the CUDA filter with the fixtures and the oracle.
Tolerance: NaN positions identical; max |out - ref| <= 2e-5 * max |ref|
(float32 FFTs of different association orders).
"""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from conftest import REPO
from oracle.goldstein_oracle import goldstein as oracle_goldstein

GOLD = sorted(glob.glob(os.path.join(REPO, "tests", "golden", "gs_*.npz")))


def _load(path):
    d = np.load(path)
    py, px = (int(v) for v in d["psize"])
    return d["phase"], d["corr"], py, px, float(d["threshold"]), d["out"]


def _close(out, ref, tol):
    nm = np.isnan(ref)
    assert (np.isnan(out) == nm).all()
    if (~nm).any():
        err = np.abs(out[~nm] - ref[~nm]).max() / np.abs(ref[~nm]).max()
        assert err <= tol, err


def test_fixtures_present():
    assert len(GOLD) >= 5


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_oracle_matches_reference_fixture(path):
    z, corr, py, px, thr, ref = _load(path)
    _close(oracle_goldstein(z, corr, py, px, thr), ref, 2e-6)


def test_goldstein_rejects_bad_args_without_gpu():
    from core_b200 import _lib
    lib = _lib.load()
    assert lib.unw_goldstein_workspace_bytes(64, 64, 32, 32) > 64 * 64 * 12
    assert lib.unw_goldstein_workspace_bytes(64, 64, 24, 32) == 0
    assert lib.unw_goldstein_workspace_bytes(64, 64, 128, 32) == 0
    f = C.c_void_p(0x10000)
    rc = lib.unw_goldstein_c64(None, 8, f, 8, 8, 8, 4, 4, 0.5, f, 8, f, 1 << 30, None)
    assert rc == _lib.UNW_E_ARG
    rc = lib.unw_goldstein_c64(f, 8, f, 8, 8, 8, 6, 4, 0.5, f, 8, f, 1 << 30, None)
    assert rc == _lib.UNW_E_UNSUPPORTED
    rc = lib.unw_goldstein_c64(f, 8, f, 8, 8, 8, 4, 4, 1.5, f, 8, f, 1 << 30, None)
    assert rc == _lib.UNW_E_ARG
    rc = lib.unw_goldstein_c64(f, 8, f, 8, 8, 8, 4, 4, 0.5, f, 8, f, 16, None)
    assert rc == _lib.UNW_E_WORKSPACE


# ------------------------------------------------------------------ GPU
def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_cuda_matches_reference_fixture(path):
    _gpu()
    import core_b200
    z, corr, py, px, thr, ref = _load(path)
    out = core_b200.goldstein(z, corr, py, px, threshold=thr)
    assert out.dtype == np.complex64 and out.shape == z.shape
    _close(out, ref, 2e-5)


@pytest.mark.gpu
def test_cuda_matches_oracle_larger_and_tensor_io():
    torch = _gpu()
    import core_b200
    from core_b200.synthetic import gen_g1
    p, c, _ = gen_g1(300, 257, seed=9, noise=0.7)
    z = np.exp(1j * p.astype(np.float64)).astype(np.complex64)
    z[np.isnan(p)] = np.nan
    ref = oracle_goldstein(z, c, 32, 32, 0.5)
    out = core_b200.goldstein(z, c, {"y": 32, "x": 32})
    _close(out, ref, 2e-5)
    dev = torch.device("cuda", 0)
    t = core_b200.goldstein(torch.from_numpy(z).to(dev), torch.from_numpy(c).to(dev), 32)
    assert t.is_cuda and t.dtype == torch.complex64
    np.testing.assert_array_equal(t.cpu().numpy(), out)   # deterministic
