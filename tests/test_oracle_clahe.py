"""The CLAHE oracle (oracle/clahe_ref.py) reproduces OpenCV's output bit for bit on the golden
fixtures (tests/golden/make_clahe.py): tile sides that are and are not multiples of the tile
count, another clip limit and tile grid, and no clipping."""
import os

import numpy as np

from oracle import clahe_ref

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "clahe.npz")


def test_clahe_oracle_matches_opencv():
    with np.load(GOLDEN) as z:
        names = [k[:-4] for k in z.files if k.endswith("/img")]
        assert len(names) >= 6
        for n in names:
            clip, tx, ty = z[n + "/params"]
            np.testing.assert_array_equal(clahe_ref.clahe(z[n + "/img"], clip, (int(tx), int(ty))), z[n + "/out"],
                                          err_msg=n)
