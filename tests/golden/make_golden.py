"""Generate golden fixtures by running the reference unwrapper itself.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_golden.py --ref <insardev checkout> (or INSARDEV_REF=<checkout>) [--large]

It imports `insardev/insardev/utils_unwrap2d.py` through a synthetic `insardev`
package with two shims: a stub `insardev.BatchCore` (the function imports it
unconditionally at utils_unwrap2d.py:1165; the real package __init__ needs
xarray/dask) and `torch_dct_standin` registered as `torch_dct` (the third-party
DCT module is not installed).  NUMBA_CACHE_DIR is pointed at a scratch
directory so that numba writes nothing into the reference tree.

An FP64 variant of the same function is made by substituting only the two dtype
lines (`dtype = torch.float32`, `np_dtype = np.float32`, :1192-1193) in a scratch
copy of the module.

`--stack` runs members 0-2 of the 64-grid uneven stack (rows 1500-2600, cols
4000-7000, gen_stack_meta(64, 0)).

Outputs: small `.npz` fixtures next to this script holding inputs, parameters,
the reference's (unwrapped, conncomp) and its IRLS iteration count.  Grids of
1024^2 and above store the full 2-pi cycle map (int16) plus the unwrapped phase
on a sub-sampled lattice, to keep the files small.  Nothing at test time reads
the reference tree: tests only read these fixtures.
"""
from __future__ import annotations

import argparse
import contextlib
import io
import os
import re
import sys
import tempfile
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from core_b200.synthetic import gen_g1, gen_g2  # noqa: E402

FN_DEFAULTS = dict(max_iter=50, tol=1e-3, cg_max_iter=20, cg_tol=1e-4, epsilon=1e-2, conncomp_size=30)
API_DEFAULTS = dict(max_iter=50, tol=1e-2, cg_max_iter=10, cg_tol=1e-3, epsilon=1e-2, conncomp_size=30)


def load_reference(ref_root):
    scratch = tempfile.mkdtemp(prefix="unw_golden_")
    os.environ["NUMBA_CACHE_DIR"] = os.path.join(scratch, "numba")
    import torch
    import torch_dct_standin
    sys.modules["torch_dct"] = torch_dct_standin
    pkg_dir = os.path.join(ref_root, "insardev", "insardev")
    pkg = types.ModuleType("insardev")
    pkg.__path__ = [pkg_dir, scratch]
    sys.modules["insardev"] = pkg
    bc = types.ModuleType("insardev.BatchCore")

    class BatchCore:
        @staticmethod
        def _get_torch_device(device="auto", debug=False):
            return torch.device("cpu")

    bc.BatchCore = BatchCore
    sys.modules["insardev.BatchCore"] = bc
    import importlib
    ref32 = importlib.import_module("insardev.utils_unwrap2d")
    src = open(os.path.join(pkg_dir, "utils_unwrap2d.py")).read()
    n1 = src.count("dtype = torch.float32")
    n2 = src.count("np_dtype = np.float32")
    assert n1 == 1 and n2 == 1, (n1, n2)
    src64 = src.replace("dtype = torch.float32", "dtype = torch.float64").replace(
        "np_dtype = np.float32", "np_dtype = np.float64")
    with open(os.path.join(scratch, "utils_unwrap2d_fp64.py"), "w") as f:
        f.write(src64)
    ref64 = importlib.import_module("insardev.utils_unwrap2d_fp64")
    return ref32.irls_unwrap_2d, ref64.irls_unwrap_2d


def run_ref(fn, phase, weight, params):
    buf = io.StringIO()
    t0 = time.time()
    with contextlib.redirect_stdout(buf):
        u, cc = fn(phase, weight, device="cpu", debug=True, **params)
    dt = time.time() - t0
    m = re.search(r"IRLS iters:.*\((\d+) iterations\)", buf.getvalue())
    iters = int(m.group(1)) if m else -1
    return u, cc, iters, dt


def cases_small():
    out = []
    p, c, _ = gen_g1(64, seed=1)
    out.append(("g1_64_fn", p, c, FN_DEFAULTS))
    p, c, _ = gen_g1(96, 80, seed=2)
    out.append(("g1_96x80_api", p, c, API_DEFAULTS))
    p, c, _ = gen_g1(75, 61, seed=3)
    out.append(("g1_75x61_fn", p, c, FN_DEFAULTS))
    p, c, _ = gen_g2(128, seed=4)
    out.append(("g2_128_fn", p, c, FN_DEFAULTS))
    p, c, _ = gen_g1(128, seed=5)
    out.append(("g1_128_fixed", p, c, dict(FN_DEFAULTS, max_iter=4, tol=0.0, cg_max_iter=8, cg_tol=0.0)))
    p, c, _ = gen_g1(64, seed=6)
    out.append(("g1_64_noweight", p, None, FN_DEFAULTS))
    # crop + components: NaN border rows/cols, a NaN wall, isolated specks
    p, c, _ = gen_g1(80, 90, seed=7, nan_fraction=0.0)
    p[:5, :] = np.nan
    p[:, 84:] = np.nan
    p[:, 30:33] = np.nan
    p[60:63, 33:84] = np.nan
    rng = np.random.default_rng(77)
    for _ in range(40):
        y, x = rng.integers(5, 80), rng.integers(33, 84)
        p[max(5, y - 2):y + 3, max(33, x - 2):x + 3] = np.nan
    p[70, 10] = 0.5
    p[69, 9:12] = np.nan
    p[71, 9:12] = np.nan
    p[70, 9] = np.nan
    p[70, 11] = np.nan
    c = c.copy()
    c[np.isnan(p)] = np.nan
    out.append(("edge_crop_components", p, c, dict(FN_DEFAULTS, conncomp_size=10)))
    # weight quirks: NaN weight on valid phase, weights outside [0.01, 1]
    p, c, _ = gen_g1(48, 56, seed=8)
    c = c.astype(np.float32).copy()
    rng = np.random.default_rng(88)
    sel = rng.random(c.shape)
    c[sel < 0.05] = np.nan
    c[(sel >= 0.05) & (sel < 0.1)] = 3.0
    c[(sel >= 0.1) & (sel < 0.15)] = -1.0
    c[(sel >= 0.15) & (sel < 0.2)] = 1e-4
    out.append(("weight_quirks", p, c, FN_DEFAULTS))
    # tiny and degenerate shapes
    rng = np.random.default_rng(9)
    for (h, w) in [(1, 7), (5, 1), (3, 5), (2, 2), (1, 1), (17, 3)]:
        ph = rng.uniform(-np.pi, np.pi, (h, w)).astype(np.float32)
        wt = rng.uniform(0.3, 1.0, (h, w)).astype(np.float32)
        out.append((f"tiny_{h}x{w}", ph, wt, dict(FN_DEFAULTS, conncomp_size=1)))
    ph = np.full((8, 8), np.nan, np.float32)
    out.append(("all_nan", ph, None, FN_DEFAULTS))
    # non-finite phase on valid pixels: wrap(inf) = NaN gradients reach the DCT
    # initial solve (zero-filled, utils_unwrap2d.py:1498-1502), the IRLS weights
    # and the PCG start (non-finite residual, :1418-1419), and the circular means
    # of the component that holds the pixel
    p, c, _ = gen_g1(64, 72, seed=10)
    p[10, 10] = np.inf
    p[40, 50] = -np.inf
    out.append(("nonfinite_phase", p, c, FN_DEFAULTS))
    # the same with the infinite pixel cut off from the rest (its own 1-pixel component)
    p, c, _ = gen_g1(48, 40, seed=11, nan_fraction=0.0)
    p[19:22, 19:22] = np.nan
    p[20, 20] = np.inf
    c = c.copy()
    c[np.isnan(p)] = np.nan
    out.append(("nonfinite_isolated", p, c, dict(FN_DEFAULTS, conncomp_size=5)))
    return out


def save_full(name, phase, weight, params, u, cc, iters, secs, precision):
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"), phase=phase,
        weight=weight if weight is not None else np.zeros((0,), np.float32),
        has_weight=np.array(weight is not None), u=u, cc=cc, iters=np.array(iters),
        params=np.array([params[k] for k in ("max_iter", "tol", "cg_max_iter", "cg_tol", "epsilon", "conncomp_size")],
                        dtype=np.float64),
        precision=np.array(precision), seconds=np.array(secs))


def save_large(name, gen, gen_args, params, phase, u, cc, iters, secs, precision, step, cycles=True):
    """Large grids: regenerate inputs from (gen, gen_args); store cycle map + sub-sampled u
    (without the cycle map when `cycles` is false)."""
    v = np.isfinite(phase) & np.isfinite(u)
    k = np.zeros(phase.shape, np.int16)
    k[v] = np.round((u[v].astype(np.float64) - phase[v].astype(np.float64)) / (2 * np.pi)).astype(np.int16)
    extra = dict(cycles=k) if cycles else {}
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"), gen=np.array(gen), gen_args=np.array(gen_args, dtype=np.int64),
        step=np.array(step), u_sub=u[::step, ::step], cc_sub=cc[::step, ::step], **extra,
        cc_hist=np.bincount(cc.ravel().astype(np.int64)), iters=np.array(iters),
        params=np.array([params[k2] for k2 in ("max_iter", "tol", "cg_max_iter", "cg_tol", "epsilon", "conncomp_size")],
                        dtype=np.float64),
        precision=np.array(precision), seconds=np.array(secs))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("INSARDEV_REF"), required="INSARDEV_REF" not in os.environ,
                    help="root of the insardev source checkout (default: $INSARDEV_REF)")
    ap.add_argument("--large", action="store_true", help="also the 1024^2 grids")
    ap.add_argument("--xlarge", action="store_true", help="also the 4096^2 fault grid (~8 min)")
    ap.add_argument("--xlarge64", action="store_true",
                    help="FP64 runs at full size: the 4096^2 fault grid and the G1 grid at 2048^2 and 4096^2")
    ap.add_argument("--stack", action="store_true",
                    help="members 0, 1, 2 of the 64-grid uneven stack (gen_stack_meta(64, 0)): FP32 run "
                         "(cycle map + lattice) and FP64 run (lattice)")
    ap.add_argument("--only", default=None)
    ap.add_argument("--no-small", action="store_true", help="skip the small fixtures")
    a = ap.parse_args()
    f32, f64 = load_reference(a.ref)
    if not (a.no_small or (a.only and a.only.startswith("L"))):
        for name, p, c, params in cases_small():
            if a.only and a.only != name:
                continue
            u, cc, it, s = run_ref(f32, p, c, params)
            save_full(name, p, c, params, u, cc, it, s, "fp32")
            print(f"{name}: iters={it} {s:.2f}s")
            if name in ("g1_64_fn", "g2_128_fn", "g1_128_fixed", "g1_75x61_fn"):
                u, cc, it, s = run_ref(f64, p, c, params)
                save_full(name + "_fp64", p, c, params, u, cc, it, s, "fp64")
                print(f"{name}_fp64: iters={it} {s:.2f}s")
    if a.large:
        p, c, _ = gen_g1(1024, seed=0)
        for prec, fn in (("fp32", f32), ("fp64", f64)):
            u, cc, it, s = run_ref(fn, p, c, FN_DEFAULTS)
            save_large(f"L_g1_1024_fn_{prec}", "g1", (1024, 1024, 0), FN_DEFAULTS, p, u, cc, it, s, prec, 4)
            print(f"L_g1_1024_fn_{prec}: iters={it} {s:.2f}s")
        u, cc, it, s = run_ref(f32, p, c, API_DEFAULTS)
        save_large("L_g1_1024_api_fp32", "g1", (1024, 1024, 0), API_DEFAULTS, p, u, cc, it, s, "fp32", 4)
        print(f"L_g1_1024_api_fp32: iters={it} {s:.2f}s")
    if a.xlarge:
        p, c, _ = gen_g2(4096, seed=0)
        u, cc, it, s = run_ref(f32, p, c, FN_DEFAULTS)
        save_large("L_g2_4096_fn_fp32", "g2", (4096, 4096, 0), FN_DEFAULTS, p, u, cc, it, s, "fp32", 16)
        print(f"L_g2_4096_fn_fp32: iters={it} {s:.2f}s")
    if a.stack:
        stack_fixtures(f32, f64)
    if a.xlarge64:
        for name, gen, args, step in (("L_g1_2048_fn_fp64", "g1", (2048, 2048, 0), 8),
                                      ("L_g2_4096_fn_fp64", "g2", (4096, 4096, 0), 16),
                                      ("L_g1_4096_fn_fp64", "g1", (4096, 4096, 0), 16)):
            if a.only and a.only != name:
                continue
            p, c, _ = gen_g1(args[0], args[1], seed=args[2]) if gen == "g1" else gen_g2(args[0], seed=args[2])
            u, cc, it, s = run_ref(f64, p, c, FN_DEFAULTS)
            save_large(name, gen, args, FN_DEFAULTS, p, u, cc, it, s, "fp64", step)
            print(f"{name}: iters={it} {s:.2f}s", flush=True)


def stack_fixtures(f32, f64):
    from core_b200.synthetic import gen_stack_grid, gen_stack_meta
    meta = gen_stack_meta(64, seed=0)
    for m in (0, 1, 2):
        p, c, _ = gen_stack_grid(meta[m])
        for prec, fn in (("fp32", f32), ("fp64", f64)):
            u, cc, it, s = run_ref(fn, p, c, FN_DEFAULTS)
            save_large(f"L_stack{m}_fn_{prec}", "stack", (64, 0, m), FN_DEFAULTS, p, u, cc, it, s, prec, 8,
                       cycles=prec == "fp32")
            print(f"L_stack{m}_fn_{prec} {p.shape}: iters={it} {s:.2f}s", flush=True)


if __name__ == "__main__":
    main()
