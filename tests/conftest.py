import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a) and the built library")
    config.addinivalue_line("markers", "slow: larger CPU cases")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    out = {}
    for name in ("sift_ref", "sift_cv2", "match_ref"):
        with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
            out[name] = {k: z[k] for k in z.files}
    return out


@pytest.fixture(scope="session")
def match_golden():
    """The camera-geometry and pair-worker fixture (tests/golden/make_match_pair.py)."""
    import numpy as np
    with np.load(os.path.join(GOLDEN, "match_pair.npz")) as z:
        return {k: z[k] for k in z.files}
