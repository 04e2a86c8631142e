import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def load_golden(name):
    import numpy as np
    d = np.load(os.path.join(GOLDEN, name if name.endswith(".npz") else name + ".npz"))
    out = {k: d[k] for k in d.files}
    mi, tol, cgi, cgt, eps, ccs = out["params"]
    out["kw"] = dict(max_iter=int(mi), tol=float(tol), cg_max_iter=int(cgi), cg_tol=float(cgt),
                     epsilon=float(eps), conncomp_size=int(ccs))
    if "has_weight" in out:
        out["w"] = out["weight"] if bool(out["has_weight"]) else None
    return out


def small_golden_names():
    """Unwrapper fixtures (L_* are the large ones; gs_* and lk_* belong to the filter and the linking)."""
    return sorted(f[:-4] for f in os.listdir(GOLDEN)
                  if f.endswith(".npz") and not f.startswith(("L_", "gs_", "lk_")))


@pytest.fixture
def golden():
    return load_golden
