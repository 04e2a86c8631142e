"""C ABI: the library loads without a GPU, exports every symbol the header
declares, sizes workspaces, and rejects bad arguments before any CUDA call."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import REPO
from core_b200 import _lib

HEADER = os.path.join(REPO, "include", "unwrap_b200.h")


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"UNW_API\s+[\w\s\*]+?\b(unw_\w+)\s*\(", txt)))


def test_header_declares_expected_entry_points():
    syms = header_symbols()
    for s in ("unw_solve_f32", "unw_solve_batch", "unw_workspace_bytes", "unw_last_error",
              "unw_apply_laplacian", "unw_apply_preconditioner", "unw_setup_gradients"):
        assert s in syms


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    for s in header_symbols():
        assert hasattr(lib, s), s
        assert s in _lib.SIGNATURES, s
    assert lib.unw_abi_version() == 2


def test_workspace_bytes_monotone_and_sane():
    lib = _lib.load()
    a = lib.unw_workspace_bytes(1024, 1024)
    b = lib.unw_workspace_bytes(4096, 4096)
    assert 0 < a < b
    # about 16 float arrays + masks per pixel, well under 100 B/px
    assert 60 * 4096 * 4096 < b < 100 * 4096 * 4096
    assert lib.unw_workspace_bytes(0, 5) == 0
    H = (C.c_int64 * 2)(100, 200)
    W = (C.c_int64 * 2)(300, 50)
    both = lib.unw_batch_workspace_bytes(2, H, W)
    assert both >= lib.unw_workspace_bytes(100, 300) + lib.unw_workspace_bytes(200, 50) - 4096


def test_solve_rejects_bad_args_without_gpu():
    lib = _lib.load()
    prm = _lib.UnwParams(50, 1e-3, 20, 1e-4, 1e-2, 30, 0, 1)
    fake = C.c_void_p(0x10000)
    rc = lib.unw_solve_f32(None, 8, None, 8, 8, 8, C.byref(prm), fake, 8, fake, 8, fake, 1 << 30, None, None)
    assert rc == _lib.UNW_E_ARG and "null" in _lib.last_error()
    rc = lib.unw_solve_f32(fake, 4, None, 8, 8, 8, C.byref(prm), fake, 8, fake, 8, fake, 1 << 30, None, None)
    assert rc == _lib.UNW_E_ARG and "pitch" in _lib.last_error()
    rc = lib.unw_solve_f32(fake, 8, None, 8, 8, 8, C.byref(prm), fake, 8, fake, 8, fake, 16, None, None)
    assert rc == _lib.UNW_E_WORKSPACE
    bad = _lib.UnwParams(-1, 1e-3, 20, 1e-4, 1e-2, 30, 0, 1)
    rc = lib.unw_solve_f32(fake, 8, None, 8, 8, 8, C.byref(bad), fake, 8, fake, 8, fake, 1 << 30, None, None)
    assert rc == _lib.UNW_E_ARG
    with pytest.raises(ValueError):
        _lib.check(_lib.UNW_E_ARG)
    with pytest.raises(OverflowError):
        _lib.check(_lib.UNW_E_OVERFLOW)


def test_python_boundary_validation_without_gpu():
    import core_b200
    with pytest.raises(ValueError):
        core_b200.irls_unwrap_2d(np.zeros((2, 3, 4), np.float32))


def test_host_device_requests_run_on_the_cuda_device(monkeypatch):
    """insardev's stack pipeline passes the device it resolved from its dask workers
    (Stack_unwrap2d.py:834-835, then :65), 'cpu' when they advertise no GPU: the
    drop-in runs such calls on the current CUDA device instead of failing, and
    raises RuntimeError when no CUDA device is visible (no CPU fallback)."""
    import torch

    from core_b200.irls import resolve_device
    monkeypatch.setattr(torch.cuda, "is_available", lambda: True)
    monkeypatch.setattr(torch.cuda, "current_device", lambda: 3)
    for req in ("cpu", "mps", "tpu", "auto", None, torch.device("cpu")):
        assert resolve_device(req) == torch.device("cuda", 3), req
    assert resolve_device("cuda:1") == torch.device("cuda", 1)
    assert resolve_device("cuda") == torch.device("cuda", 3)
    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    for req in ("cpu", "auto"):
        with pytest.raises(RuntimeError):
            resolve_device(req)
    import core_b200
    with pytest.raises(RuntimeError):
        core_b200.irls_unwrap_2d(np.zeros((4, 4), np.float32), device="cpu")


def test_adjoint_rejects_bad_args_without_gpu():
    lib = _lib.load()
    prm = _lib.UnwParams(50, 1e-3, 200, 1e-6, 1e-2, 30, 0, 1)
    f = C.c_void_p(0x10000)
    big = 1 << 40
    assert lib.unw_adjoint_workspace_bytes(64, 64) > lib.unw_workspace_bytes(64, 64)
    assert lib.unw_adjoint_workspace_bytes(0, 64) == 0
    call = lambda *a: lib.unw_adjoint_f32(*a)
    rc = call(None, 8, None, 8, 8, 8, C.byref(prm), f, 8, f, 8, f, 8, None, 8, f, big, None, None)
    assert rc == _lib.UNW_E_ARG and "null" in _lib.last_error()
    rc = call(f, 8, None, 8, 8, 8, C.byref(prm), f, 4, f, 8, f, 8, None, 8, f, big, None, None)
    assert rc == _lib.UNW_E_ARG and "pitch" in _lib.last_error()
    rc = call(f, 8, None, 8, 8, 8, C.byref(prm), f, 8, f, 8, f, 8, f, 8, f, big, None, None)
    assert rc == _lib.UNW_E_ARG and "weight" in _lib.last_error()
    rel0 = _lib.UnwParams(50, 1e-3, 200, 0.0, 1e-2, 30, 0, 1)
    rc = call(f, 8, None, 8, 8, 8, C.byref(rel0), f, 8, f, 8, f, 8, None, 8, f, big, None, None)
    assert rc == _lib.UNW_E_ARG and "relative" in _lib.last_error()
    rc = call(f, 8, None, 8, 8, 8, C.byref(prm), f, 8, f, 8, f, 8, None, 8, f, 64, None, None)
    assert rc == _lib.UNW_E_WORKSPACE


def test_link_entries_reject_bad_args_without_gpu():
    lib = _lib.load()
    assert lib.unw_link_workspace_bytes(4096, 4096, 1000) > 4096 * 4096 * 24
    assert lib.unw_link_workspace_bytes(70000, 10, 4) == 0          # sides above 65535
    assert C.sizeof(_lib.UnwLinkPair) == 64
    f = C.c_void_p(0x10000)
    prm = _lib.UnwLinkParams(30, 30, 5, 0)
    n1, n2 = C.c_int32(0), C.c_int32(0)
    rc = lib.unw_link_pairs_f32(None, 8, None, 8, 8, 8, C.byref(prm), None, None, None, 0, C.byref(n1), None, 0,
                                C.byref(n2), f, 1 << 30, None)
    assert rc == _lib.UNW_E_ARG
    rc = lib.unw_link_pairs_f32(f, 4, None, 8, 8, 8, C.byref(prm), None, None, None, 0, C.byref(n1), None, 0,
                                C.byref(n2), f, 1 << 30, None)
    assert rc == _lib.UNW_E_ARG                                      # pitch below width
    bad = _lib.UnwLinkParams(30, 30, 40, 0)                          # window above 31
    rc = lib.unw_link_pairs_f32(f, 8, None, 8, 8, 8, C.byref(bad), None, None, None, 0, C.byref(n1), None, 0,
                                C.byref(n2), f, 1 << 30, None)
    assert rc == _lib.UNW_E_ARG
    rc = lib.unw_link_pairs_f32(f, 8, None, 8, 8, 8, C.byref(prm), None, None, None, 0, C.byref(n1), None, 0,
                                C.byref(n2), f, 16, None)
    assert rc == _lib.UNW_E_WORKSPACE
    k = (C.c_int32 * 2)(0, 1)
    assert lib.unw_link_apply_f32(None, 8, 8, 8, k, 2, f, 8, f, 1 << 30, 30, None) == _lib.UNW_E_ARG
    assert lib.unw_link_apply_f32(f, 8, 8, 8, k, 2, f, 8, f, 16, 30, None) == _lib.UNW_E_WORKSPACE


def test_link_offsets_host_solver_without_gpu():
    """unw_link_offsets is host code: it runs here.  Two components joined by one edge."""
    lib = _lib.load()
    ei, ej, off = (C.c_int32 * 1)(0), (C.c_int32 * 1)(1), (C.c_int32 * 1)(2)
    w = (C.c_int64 * 1)(500)
    k = (C.c_int32 * 2)()
    assert lib.unw_link_offsets(2, 1, ei, ej, off, w, 1, k) == _lib.UNW_OK
    assert list(k) == [0, -2]                    # k_0 - k_1 = 2 (reference sign)
    assert lib.unw_link_offsets(2, 1, ei, ej, off, w, -1, k) == _lib.UNW_OK
    assert list(k) == [0, 2]                     # k_1 - k_0 = 2
    bad = (C.c_int32 * 1)(5)
    assert lib.unw_link_offsets(2, 1, ei, bad, off, w, 1, k) == _lib.UNW_E_ARG
