import glob
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path through the C ABI)")


SCHEME_PREFIXES = ("incremental_", "warm_")
EXPLICIT_PREFIX = "explicit_"
FLIP_PREFIX = "flip_relabel_"
BC_PREFIX = "bc_"
LIMIT_PREFIX = "limit_"  # fixtures of scenes outside an equivalence, read by the tests that show the limit


def golden_names():
    """The Chorin fixtures (one solve from zero)."""
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))
    return [n for n in names
            if not n.startswith(SCHEME_PREFIXES + (EXPLICIT_PREFIX, FLIP_PREFIX, BC_PREFIX, LIMIT_PREFIX))]


def explicit_golden_names():
    """The fixtures of the EXPLICIT method's own SOR pressure step and projection."""
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))
    return [n for n in names if n.startswith(EXPLICIT_PREFIX)]


def flip_golden_names():
    """The fixtures of FLIP's re-labelling from particles followed by the Chorin step."""
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))
    return [n for n in names if n.startswith(FLIP_PREFIX)]


def bc_golden_names():
    """The fixtures of the boundary-condition replay (EnforceVelocityBC + EnforcePressureBC)."""
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))
    return [n for n in names if n.startswith(BC_PREFIX)]


def scheme_golden_names():
    """The fixtures with a previous step: the incremental scheme and the Chorin warm start."""
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))
    return [n for n in names if n.startswith(SCHEME_PREFIXES)]


def load_golden(name):
    """A fixture plus its case, rebuilt from the stored builder name and arguments."""
    from nereus_cfd_b200 import workloads as W

    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    case = getattr(W, meta["builder"])(**meta["kwargs"])
    return case, meta, z


def cuda_ok():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def nb():
    """The B200 library through its C ABI; GPU tests only."""
    if not cuda_ok():
        pytest.skip("no CUDA device")
    from nereus_cfd_b200 import capi

    return capi.load()
