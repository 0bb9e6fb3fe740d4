import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not _has_gpu():
        pytest.fail("this test needs a CUDA GPU")
    return 0


def bit_equal(a, b) -> bool:
    """Equal element by element, bit for bit, except that +0/-0 compare equal
    and NaN equals NaN."""
    import numpy as np

    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    return bool(same.all())


def first_mismatch(a, b):
    import numpy as np

    a = np.asarray(a)
    b = np.asarray(b)
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    idx = np.argwhere(bad)
    if len(idx) == 0:
        return None
    t = tuple(idx[0])
    return dict(count=int(bad.sum()), index=t, got=float(a[t]), want=float(b[t]))
