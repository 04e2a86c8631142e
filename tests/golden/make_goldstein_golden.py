"""Generate Goldstein-filter golden fixtures by running the reference filter itself.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_goldstein_golden.py --ref <insardev checkout> (or INSARDEV_REF=<checkout>)

It loads `insardev/insardev/utils_goldstein.py` as a plain module (its
functions import numpy and torch only) and runs `goldstein_pytorch` on the CPU
torch device: the code path insardev takes on CUDA devices
(insardev/insardev/Batch.py:2023-2027), executed here without a GPU.  The
fixtures hold the complex64 input, the float32 correlation, the patch sizes,
the threshold and the reference output.  Nothing at test time reads the
reference tree.
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from core_b200.synthetic import gen_g1  # noqa: E402


def load_reference(ref_root):
    path = os.path.join(ref_root, "insardev", "insardev", "utils_goldstein.py")
    spec = importlib.util.spec_from_file_location("ref_utils_goldstein", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


CASES = [
    # name, H, W, psize_y, psize_x, threshold, seed, nan_fraction
    ("gs_64x80_p16", 64, 80, 16, 16, 0.5, 1, 0.0),
    ("gs_100x123_p32_nan", 100, 123, 32, 32, 0.5, 2, 0.05),
    ("gs_97x61_p8x16", 97, 61, 8, 16, 0.5, 3, 0.05),
    ("gs_130x140_p64_thr", 130, 140, 64, 64, 0.8, 4, 0.05),
    ("gs_40x33_p4", 40, 33, 4, 4, 0.25, 5, 0.0),
]


def make_case(H, W, seed, nan_fraction):
    import torch  # noqa: F401
    p, c, _ = gen_g1(H, W, seed=seed, noise=0.8, nan_fraction=nan_fraction)
    rng = np.random.default_rng(seed + 100)
    amp = rng.uniform(0.5, 2.0, size=(H, W))
    z = (amp * np.exp(1j * p.astype(np.float64))).astype(np.complex64)
    z[np.isnan(p)] = np.nan + 1j * np.nan
    corr = c.astype(np.float32)
    corr[rng.random((H, W)) < 0.02] = np.nan   # correlation NaNs where the phase is valid
    return z, corr


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("INSARDEV_REF"), required="INSARDEV_REF" not in os.environ,
                    help="root of the insardev source checkout (default: $INSARDEV_REF)")
    a = ap.parse_args()
    import torch
    ref = load_reference(a.ref)
    for name, H, W, py, px, thr, seed, nanf in CASES:
        z, corr = make_case(H, W, seed, nanf)
        out = ref.goldstein_pytorch(z.copy(), corr.copy(), py, px, torch.device("cpu"), threshold=thr)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), phase=z, corr=corr, psize=np.array([py, px]),
                            threshold=np.float32(thr), out=out)
        print(name, z.shape, "nan out", int(np.isnan(out).sum()))


if __name__ == "__main__":
    main()
