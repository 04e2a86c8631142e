"""The mixed-precision form: the tensor-core (tcgen05, split-precision bf16) column
pass of the DCT preconditioner for grids of at most 1024 rows.

It replaces the float32 FFT column pass of utils_unwrap2d.py:1316-1365 / :1390-1403
inside the same operator, so it is checked the same way:
  * the operator idct2(-dct2(r)/lambda) through unw_apply_preconditioner_mixed
    against the float64 operator (scipy), forced onto the tensor cores, with a
    bar of 3e-4 of the largest value: each product keeps about 16 significant
    bits per term (hi*hi + hi*lo + lo*hi), against 2e-5 for the float32 FFT;
  * full solves forced onto the tensor cores against the reference function's
    own FP32 and FP64 runs of the 1024^2 grid (cycle map >= 99.99%, RMS <= 1e-3
    rad), and a batch of four 1024^2 grids against the plain form;
  * the autotuner reports both timings and the path it chose.
"""
import numpy as np
import pytest
import scipy.fft as sfft

from conftest import load_golden
from core_b200.synthetic import gen_g1
from oracle.irls_oracle import cycle_map

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

import core_b200  # noqa: E402
from core_b200 import _lib  # noqa: E402

DEV = torch.device("cuda", 0)
TC_TOL = 3e-4


def fp64_operator(r):
    H, W = r.shape
    lam = 2 * np.cos(np.pi * np.arange(H) / H)[:, None] + 2 * np.cos(np.pi * np.arange(W) / W)[None, :] - 4
    lam[0, 0] = 1.0
    t = -sfft.dct(sfft.dct(r.astype(np.float64), type=2, axis=1), type=2, axis=0) / lam
    t[0, 0] = 0.0
    return sfft.idct(sfft.idct(t, type=2, axis=0), type=2, axis=1)


def precond_mixed(r, col_path):
    lib = _lib.load()
    H, W = r.shape
    t = torch.from_numpy(np.ascontiguousarray(r, np.float32)).to(DEV)
    z = torch.empty((H, W), dtype=torch.float32, device=DEV)
    ws = torch.empty(lib.unw_workspace_bytes(H, W), dtype=torch.uint8, device=DEV)
    rc = lib.unw_apply_preconditioner_mixed(t.data_ptr(), H, W, z.data_ptr(), col_path, ws.data_ptr(), ws.numel(),
                                            torch.cuda.current_stream(DEV).cuda_stream)
    _lib.check(rc, "unw_apply_preconditioner_mixed")
    torch.cuda.synchronize()
    return z.cpu().numpy(), rc


@pytest.mark.parametrize("shape", [(64, 64), (17, 64), (128, 96), (256, 512), (700, 300), (1000, 2048),
                                   (1024, 1024), (1024, 4), (333, 1000)])
def test_tensor_core_preconditioner_matches_float64_operator(shape):
    rng = np.random.default_rng(shape[0] * 31 + shape[1])
    r = rng.standard_normal(shape).astype(np.float32)
    z, path = precond_mixed(r, 1)
    assert path == 1
    z64 = fp64_operator(r)
    scale = np.abs(z64).max()
    err = np.abs(z - z64).max() / scale
    assert err <= TC_TOL, err
    # the forced FFT path of the same entry point is the float32 operator
    zf, pf = precond_mixed(r, 0)
    assert pf == 0
    assert np.abs(zf - z64).max() / scale <= 2e-5


def test_tensor_core_pass_rejects_unsupported_shapes():
    lib = _lib.load()
    H, W = 1100, 64
    t = torch.zeros((H, W), dtype=torch.float32, device=DEV)
    ws = torch.empty(lib.unw_workspace_bytes(H, W), dtype=torch.uint8, device=DEV)
    rc = lib.unw_apply_preconditioner_mixed(t.data_ptr(), H, W, t.data_ptr(), 1, ws.data_ptr(), ws.numel(),
                                            torch.cuda.current_stream(DEV).cuda_stream)
    assert rc == _lib.UNW_E_UNSUPPORTED
    assert "tensor-core" in _lib.last_error()


@pytest.mark.parametrize("name", ["L_g1_1024_fn_fp32", "L_g1_1024_fn_fp64"])
def test_mixed_solve_1024_matches_reference(name):
    d = load_golden(name)
    H, W, seed = [int(x) for x in d["gen_args"]]
    p, c, _ = gen_g1(H, W, seed=seed)
    u, cc, st = core_b200.irls_unwrap_2d(p, c, precision="mixed", col_pass="tc", return_stats=True, **d["kw"])
    assert st["col_path"] == 1
    assert not st["status"] & _lib.UNW_S_TC_TIMEOUT
    assert 0 < st["resid_rel"] < 1e-2
    v = np.isfinite(p)
    assert (cycle_map(u, p) == d["cycles"])[v].mean() >= 0.9999
    s = int(d["step"])
    vs = np.isfinite(p[::s, ::s])
    e = (u[::s, ::s].astype(np.float64) - d["u_sub"])[vs]
    assert np.sqrt(np.mean((e - e.mean()) ** 2)) <= 1e-3


def test_mixed_batch_matches_plain_form():
    grids = [gen_g1(1024, 1024, seed=40 + k) for k in range(4)]
    ps, cs = [g[0] for g in grids], [g[1] for g in grids]
    mixed = core_b200.irls_unwrap_2d_batch(ps, cs, precision="mixed", col_pass="tc", return_stats=True)
    plain = core_b200.irls_unwrap_2d_batch(ps, cs)
    for p, (um, ccm, st), (up, ccp) in zip(ps, mixed, plain):
        assert st["col_path"] == 1
        v = np.isfinite(p)
        assert (cycle_map(um, p) == cycle_map(up, p))[v].mean() >= 0.9999
        e = (um.astype(np.float64) - up)[v]
        assert np.sqrt(np.mean((e - e.mean()) ** 2)) <= 1e-3


def test_autotuner_reports_its_choice():
    p, c, _ = gen_g1(512, 768, seed=5)
    u, cc, st = core_b200.irls_unwrap_2d(p, c, precision="mixed", return_stats=True)
    assert st["col_path"] in (0, 1)
    ms_fft, ms_tc = st["tune_ms"]
    assert ms_fft > 0 and ms_tc > 0
    assert st["col_path"] == (1 if ms_tc < ms_fft else 0)
    uf, ccf = core_b200.irls_unwrap_2d(p, c)
    v = np.isfinite(p)
    assert (cycle_map(u, p) == cycle_map(uf, p))[v].mean() >= 0.9999
