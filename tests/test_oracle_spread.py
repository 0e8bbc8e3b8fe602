"""The oracle's grid-spread selection (oracle/features_ref.py) against the reference's own
features._spread on the committed fixtures (tests/golden/make_spread.py): identical index lists in
both tie modes, and the stable response order of features.py:126, on uniform, clustered and
border-crossing keypoints with distinct and heavily tied responses."""
import os

import numpy as np
import pytest

from oracle.features_ref import spread

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "spread.npz")


@pytest.fixture(scope="module")
def fixture():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


def test_oracle_spread_matches_reference(fixture):
    z = fixture
    for k in range(int(z["n_cases"])):
        x, y, r = z["c%d/x" % k], z["c%d/y" % k], z["c%d/resp" % k]
        W, H, n = (int(v) for v in z["c%d/wh_n" % k])
        for stable in (True, False):
            got = spread(x, y, r, W, H, n, stable=stable)
            np.testing.assert_array_equal(got, z["c%d/sel" % k], err_msg="case %d stable=%s" % (k, stable))
        got = spread(x, y, r, W, H, n)
        np.testing.assert_array_equal(got[np.argsort(-r[got], kind="stable")], z["c%d/sorted" % k])
