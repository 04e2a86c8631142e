"""The allocation-free preconditioner entry point (unw_apply_preconditioner_noalloc).

Some callers cannot allocate device memory where they need the operator; this
entry point takes its scratch from a device array the library owns, so the
caller passes only r and z.  Checked through the C ABI against the allocating
entry point (unw_apply_preconditioner) on two calls in a row -- the second
call finds the first call's leftovers in the shared array -- with the same
tolerance the preconditioner tests use (2e-5 of the largest value; the two
paths run the same kernels, so they agree far closer than that).
This file sorts last so that a run stopping at the first failure has run
every other test before it.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("no CUDA device", allow_module_level=True)

from core_b200 import _lib  # noqa: E402

DEV = torch.device("cuda", 0)
TOL = 2e-5


def _stream():
    return torch.cuda.current_stream(DEV).cuda_stream


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


@pytest.mark.parametrize("shape", [(64, 96), (37, 50), (1024, 1024), (513, 1031), (1, 7)])
def test_no_alloc_matches_allocating_entry_point_twice(shape):
    rng = np.random.default_rng(shape[0] * 7919 + shape[1])
    for call in range(2):
        r = rng.standard_normal(shape).astype(np.float32)
        ref = allocating(r)
        got = no_alloc(r)
        scale = max(float(np.abs(ref).max()), 1e-30)
        assert np.abs(got - ref).max() <= TOL * scale, (call, np.abs(got - ref).max() / scale)


def test_no_alloc_rejects_grids_beyond_the_limit():
    lib = _lib.load()
    fake = torch.empty(1, dtype=torch.float32, device=DEV)
    rc = lib.unw_apply_preconditioner_noalloc(fake.data_ptr(), 4096, 4096, fake.data_ptr(), _stream())
    assert rc == _lib.UNW_E_UNSUPPORTED
    assert "too large" in _lib.last_error()
