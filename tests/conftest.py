import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["uniform3d", "periodic3d", "periodic_demo", "uniform6d", "clustered2d",
                "tiny_k_gt_n"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (sm_100a) and libckd.so")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
    g = {k: z[k] for k in z.files}
    g["boxsize"] = None if g["boxsize"].size == 0 else g["boxsize"]
    g["leaf"] = int(g["leaf"])
    g["k"] = int(g["k"])
    g["radius"] = float(g["radius"])
    return g


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build_library()
    return O


@pytest.fixture(scope="session")
def gpu():
    """The product package, with libckd.so loaded and a B200 present (fails loudly
    otherwise: GPU tests never fall back to the CPU)."""
    import torch
    import cosmokdtree_b200 as ck
    from cosmokdtree_b200 import _lib
    assert torch.cuda.is_available(), "GPU test requires CUDA"
    major, _ = torch.cuda.get_device_capability(0)
    assert major == 10, "GPU tests need a B200 (sm_100)"
    _lib.load()
    return ck
