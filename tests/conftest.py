"""Shared test configuration: the ``gpu`` marker and helpers to load golden fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA device (B200)")


def load_golden(name):
    """Returns (hfmIn dict, reference outputs dict, extras dict) of a fixture."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    params, out, extra = {}, {}, {}
    for k in z.files:
        v = z[k]
        if k.startswith("in_"):
            key = k[3:]
            if v.dtype.kind in "US":
                params[key] = str(v)
            elif v.ndim == 0:
                params[key] = float(v)
            else:
                params[key] = v
        elif k.startswith("out_"):
            out[k[4:]] = v
        else:
            extra[k] = v
    return params, out, extra


GOLDEN_SOLVES = ["riemann2_64", "riemann2_48_seeds", "riemann3_16_walls", "reedsshepp2_32x24",
                 "reedsshepp2_24x16_walls", "elastica2_24x16", "rsf2_32x24", "rsf2_24x16_walls"]
GOLDEN_STENCILS = ["selling2_32", "selling2_dual_24", "selling3_10"]


@pytest.fixture(scope="session")
def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
