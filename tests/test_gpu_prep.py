"""Device CLAHE (the contrast equalisation of features.prepare) through the C ABI: identical to
OpenCV's output on the golden fixtures and to the oracle at the bench's image size, on strided
input and on images smaller than the tile grid."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "clahe.npz")


def test_clahe_matches_opencv_fixtures():
    from fieldstitch_b200 import features
    with np.load(GOLDEN) as z:
        for n in [k[:-4] for k in z.files if k.endswith("/img")]:
            clip, tx, ty = z[n + "/params"]
            np.testing.assert_array_equal(features.clahe(z[n + "/img"], clip, (int(tx), int(ty))), z[n + "/out"],
                                          err_msg=n)


@pytest.mark.parametrize("hw", [(1978, 2640), (1001, 1333), (8, 24), (7, 7), (3, 40)])
def test_clahe_matches_oracle(hw):
    from fieldstitch_b200 import features, synth
    from oracle import clahe_ref
    img = synth.synth_image(*hw, 12)
    ref = clahe_ref.clahe(img)
    np.testing.assert_array_equal(features.clahe(img), ref)
    strided = np.zeros((hw[0], hw[1] + 13), np.uint8)
    strided[:, 5:5 + hw[1]] = img
    np.testing.assert_array_equal(features.clahe(strided[:, 5:5 + hw[1]]), ref)


def test_clahe_rejects_bad_tile_grids():
    from fieldstitch_b200 import features
    for tiles in ((0, 8), (17, 16)):
        with pytest.raises(RuntimeError):
            features.clahe(np.zeros((64, 64), np.uint8), 2.0, tiles)
