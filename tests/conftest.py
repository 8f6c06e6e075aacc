import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "first_gpu_run: a GPU path whose first run on a B200 is still to come; "
                                       "collected after every other test")


def pytest_collection_modifyitems(config, items):
    """Tests of paths that have not run on a GPU yet go after the established
    ones (stable order otherwise), so that under -x a failure among them
    leaves every established test already run; the allocation-free entry
    point's file (test_zz_no_alloc.py) stays the very last."""
    def rank(it):
        if os.path.basename(str(it.fspath)) == "test_zz_no_alloc.py":
            return 2
        return 1 if it.get_closest_marker("first_gpu_run") is not None else 0

    items[:] = sorted(items, key=rank)


@pytest.fixture
def golden():
    import numpy as np

    def load(name):
        return np.load(os.path.join(GOLDEN, name), allow_pickle=False)

    return load


def has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
