"""Grid-spread keypoint selection (features._spread, app/planesite/features.py:38-57) on the
device against the oracle's restatement: identical index lists, in _spread's order and after the
stable response sort of features.py:126, including runs of equal responses across cells, points
on and beyond the image border, one-cell clusters and inputs of several chunks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(rng, n, W, H, mode, ties):
    if mode == "uniform":
        x, y = rng.uniform(0, W, n), rng.uniform(0, H, n)
    elif mode == "cluster":
        x, y = rng.uniform(0, W / 6, n), rng.uniform(0, H / 4, n)
    else:
        x, y = rng.uniform(-5, W + 5, n), rng.uniform(-5, H + 5, n)
    if ties:
        r = rng.integers(1, 20, n).astype(np.float32)
    else:
        r = rng.uniform(0.01, 1.0, n).astype(np.float32)
    return x.astype(np.float32), y.astype(np.float32), np.sort(r)[::-1].copy()


@pytest.mark.parametrize("mode", ["uniform", "cluster", "border"])
@pytest.mark.parametrize("ties", [False, True])
def test_spread_matches_oracle(mode, ties):
    from fieldstitch_b200 import features
    from oracle.features_ref import spread
    rng = np.random.default_rng(7 if ties else 8)
    for n, nfeat in [(1, 1), (50, 10), (500, 108), (3000, 1000), (4000, 3999), (12000, 5000), (20000, 300),
                     (35200, 16000), (70000, 20000)]:
        W, H = int(rng.integers(100, 3000)), int(rng.integers(100, 3000))
        x, y, r = _case(rng, n, W, H, mode, ties)
        want = spread(x, y, r, W, H, nfeat)
        got = features.spread_arrays(x, y, r, W, H, nfeat)
        np.testing.assert_array_equal(got, want, err_msg="%s n=%d nfeat=%d" % (mode, n, nfeat))
        want_r = want[np.argsort(-r[want], kind="stable")]
        got_r = features.spread_arrays(x, y, r, W, H, nfeat, response_order=True)
        np.testing.assert_array_equal(got_r, want_r, err_msg="%s n=%d nfeat=%d" % (mode, n, nfeat))


def test_spread_edges_and_reference_signature():
    from fieldstitch_b200 import features
    from oracle.features_ref import spread
    rng = np.random.default_rng(3)
    x, y, r = _case(rng, 400, 640, 480, "uniform", True)
    assert len(features.spread_arrays(x, y, r, 640, 480, 0)) == 0
    assert len(features.spread_arrays(x[:0], y[:0], r[:0], 640, 480, 10)) == 0
    np.testing.assert_array_equal(features.spread_arrays(x, y, r, 640, 480, 400), np.arange(400))

    class KP:
        def __init__(self, px, py, resp):
            self.pt, self.response = (float(px), float(py)), float(resp)
    kps = [KP(a, b, c) for a, b, c in zip(x, y, r)]
    assert features._spread(kps, 640, 480, 150) == spread(x, y, r, 640, 480, 150).tolist()
    assert features._spread(kps, 640, 480, 1000) == list(range(400))
    with pytest.raises(RuntimeError):
        features.spread_arrays(x, y, r[::-1].copy(), 640, 480, 100)   # not response-descending


def test_sift_gpu_selection_is_spread_of_detect(golden):
    """The selection inside fsb_sift_features equals the oracle's spread + stable response sort
    of the device's own detection (max_kp = int(2.2 nfeat)): the same keypoints in the same order."""
    from fieldstitch_b200 import features, gsift
    from oracle.features_ref import spread
    g = golden["sift_ref"]
    for case in ["s240x320_c04", "s200x264_c015"]:
        img = g[case + "/img"]
        for nfeat in [40, 150, 400]:
            kps, _ = gsift.detect(img, max_kp=int(nfeat * 2.2))
            h, w = img.shape[:2]
            xy, _, resp = features.sift_gpu_u8(img, nfeat)
            if len(kps["x"]) < 10:
                assert len(xy) == 0
                continue
            sel = spread(kps["x"], kps["y"], kps["response"], w, h, nfeat)
            sel = sel[np.argsort(-kps["response"][sel], kind="stable")]
            np.testing.assert_array_equal(xy, np.c_[kps["x"][sel], kps["y"][sel]].astype(np.float32))
            np.testing.assert_array_equal(resp, kps["response"][sel])


def test_spread_matches_reference_fixtures():
    """The device selection against the reference's own _spread outputs (tests/golden/spread.npz),
    in _spread's order and after the stable response sort."""
    import os
    from fieldstitch_b200 import features
    with np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "spread.npz")) as z:
        for k in range(int(z["n_cases"])):
            x, y, r = z["c%d/x" % k], z["c%d/y" % k], z["c%d/resp" % k]
            W, H, n = (int(v) for v in z["c%d/wh_n" % k])
            np.testing.assert_array_equal(features.spread_arrays(x, y, r, W, H, n), z["c%d/sel" % k])
            np.testing.assert_array_equal(features.spread_arrays(x, y, r, W, H, n, response_order=True),
                                          z["c%d/sorted" % k])
