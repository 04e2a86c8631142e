"""The allocation-free preconditioner entry point (unw_apply_preconditioner_noalloc).

Some callers cannot allocate device memory where they need the operator (C
codes without a device allocator, loops that must not allocate after
start-up); this entry point takes its scratch from a device array the library
owns, so the caller passes only r and z.  Checked through the C ABI against
the allocating entry point (unw_apply_preconditioner) and against the float64
operator idct2(-dct2(r)/lambda) on two calls in a row -- the second call
finds the first call's leftovers in the shared array -- with the tolerance
the preconditioner tests use (2e-5 of the largest value).  Shapes mix the
power-of-two register-FFT kernels on one axis with the generic ones on the
other.  This file sorts last so that a run stopping at the first failure has
run every other test before it.
"""
import numpy as np
import pytest
import scipy.fft as sfft

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from core_b200 import _lib  # noqa: E402

DEV = torch.device("cuda", 0)
TOL = 2e-5


def _stream():
    return torch.cuda.current_stream(DEV).cuda_stream


def fp64_operator(r):
    """idct2(-dct2(r) / lambda) with lambda[0, 0] = 1 and the DC term zeroed, in float64."""
    H, W = r.shape
    lam = 2 * np.cos(np.pi * np.arange(H) / H)[:, None] + 2 * np.cos(np.pi * np.arange(W) / W)[None, :] - 4
    lam[0, 0] = 1.0
    t = -sfft.dct(sfft.dct(r.astype(np.float64), type=2, axis=1), type=2, axis=0) / lam
    t[0, 0] = 0.0
    return sfft.idct(sfft.idct(t, type=2, axis=0), type=2, axis=1)


def allocating(r):
    lib = _lib.load()
    H, W = r.shape
    t = torch.from_numpy(np.ascontiguousarray(r, np.float32)).to(DEV)
    z = torch.empty((H, W), dtype=torch.float32, device=DEV)
    ws = torch.empty(lib.unw_workspace_bytes(H, W), dtype=torch.uint8, device=DEV)
    _lib.check(lib.unw_apply_preconditioner(t.data_ptr(), H, W, z.data_ptr(), ws.data_ptr(), ws.numel(),
                                            _stream()))
    torch.cuda.synchronize()
    return z.cpu().numpy()


def no_alloc(r):
    lib = _lib.load()
    H, W = r.shape
    t = torch.from_numpy(np.ascontiguousarray(r, np.float32)).to(DEV)
    z = torch.empty((H, W), dtype=torch.float32, device=DEV)
    _lib.check(lib.unw_apply_preconditioner_noalloc(t.data_ptr(), H, W, z.data_ptr(), _stream()))
    torch.cuda.synchronize()
    return z.cpu().numpy()


@pytest.mark.parametrize("shape", [(64, 96), (37, 50), (1024, 1024), (513, 1031), (1, 7),
                                   (1024, 1031), (513, 2048), (3, 4096), (4096, 3)])
def test_no_alloc_matches_allocating_entry_point_twice(shape):
    rng = np.random.default_rng(shape[0] * 7919 + shape[1])
    for call in range(2):
        r = rng.standard_normal(shape).astype(np.float32)
        ref = allocating(r)
        got = no_alloc(r)
        z64 = fp64_operator(r)
        scale = max(float(np.abs(z64).max()), 1e-30)
        assert np.abs(got - ref).max() <= TOL * scale, (call, np.abs(got - ref).max() / scale)
        assert np.abs(got - z64).max() <= TOL * scale, (call, np.abs(got - z64).max() / scale)


def test_no_alloc_rejects_unaligned_pointers():
    lib = _lib.load()
    buf = torch.zeros(64 * 64 + 4, dtype=torch.float32, device=DEV)
    rc = lib.unw_apply_preconditioner_noalloc(buf.data_ptr() + 4, 64, 64, buf.data_ptr(), _stream())
    assert rc == _lib.UNW_E_ARG
    assert "aligned" in _lib.last_error()


def test_no_alloc_rejects_grids_beyond_the_limit():
    lib = _lib.load()
    fake = torch.empty(1, dtype=torch.float32, device=DEV)
    rc = lib.unw_apply_preconditioner_noalloc(fake.data_ptr(), 4096, 4096, fake.data_ptr(), _stream())
    assert rc == _lib.UNW_E_UNSUPPORTED
    assert "too large" in _lib.last_error()
