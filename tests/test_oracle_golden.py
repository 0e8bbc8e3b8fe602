"""The CPU oracle reproduces the reference's outputs stored in tests/golden (bit for bit)."""
import numpy as np
import pytest

from oracle import features_ref, gsift_ref, matching_ref

SIFT = ["s240x320_c04", "s200x264_c015", "s97x131_c04"]


@pytest.mark.parametrize("case", SIFT)
def test_detect_describe_match_reference(golden, case):
    g = golden["sift_ref"]
    img = g[case + "/img"]
    contrast, edge, max_kp, _ = g[case + "/params"]
    kps, st = gsift_ref.detect(img, max_kp=int(max_kp), contrast=float(contrast), edge=float(edge))
    for k in ("x", "y", "size", "angle", "response", "octave", "layer"):
        np.testing.assert_array_equal(kps[k], g[case + "/kp_" + k], err_msg=k)
    desc = gsift_ref.describe(st, kps, np.arange(len(kps["x"])))
    np.testing.assert_array_equal(desc, g[case + "/desc"])


@pytest.mark.parametrize("case", SIFT)
def test_sift_gpu_sequence_and_rootsift(golden, case):
    g = golden["sift_ref"]
    img = g[case + "/img"]
    nfeat = int(g[case + "/params"][3])
    xy, desc, resp = features_ref.sift_gpu_ref(img, nfeat, stable=False)
    np.testing.assert_array_equal(xy, g[case + "/sg_xy"])
    np.testing.assert_array_equal(resp, g[case + "/sg_resp"])
    np.testing.assert_array_equal(desc, g[case + "/sg_desc"])
    np.testing.assert_array_equal(features_ref.rootsift_u8(desc), g[case + "/sg_u8"])


def test_flat_image_has_no_keypoints(golden):
    kps, _ = gsift_ref.detect(golden["sift_ref"]["flat/img"])
    assert len(kps["x"]) == int(golden["sift_ref"]["flat/n"]) == 0


@pytest.mark.parametrize("case", ["bf_400x380", "bf_257x300", "bf_2x2"])
def test_ratio_match_bf(golden, case):
    g = golden["match_ref"]
    q, t = matching_ref.ratio_match_bf(g[case + "/a"].astype(np.float32), g[case + "/b"].astype(np.float32),
                                       float(g[case + "/ratio"]))
    np.testing.assert_array_equal(q, g[case + "/q"])
    np.testing.assert_array_equal(t, g[case + "/t"])


def test_unique(golden):
    g = golden["match_ref"]
    q, t = matching_ref.unique(g["uniq/q"], g["uniq/t"], g["uniq/dd"])
    np.testing.assert_array_equal(q, g["uniq/uq"])
    np.testing.assert_array_equal(t, g["uniq/ut"])


@pytest.mark.parametrize("case", ["g_600_k16", "g_600_k2", "g_600_k1", "g_500_all"])
def test_guided(golden, case):
    g = golden["match_ref"]
    radius, kc, ratio, W, H = g[case + "/args"]
    fa, fb = g[case + "/a"].astype(np.float32), g[case + "/b"].astype(np.float32)
    A = {"und": g[case + "/ua"], "desc": fa, "wh": (W, H)}
    B = {"und": g[case + "/ub"], "desc": fb, "wh": (W, H)}
    q, t = matching_ref.guided(A, B, g[case + "/Hm"], radius, int(kc), ratio)
    np.testing.assert_array_equal(q, g[case + "/q"])
    np.testing.assert_array_equal(t, g[case + "/t"])


def test_cv2_fixture_agrees_with_oracle_statistically(golden):
    """OpenCV SIFT (the reference CPU extractor) and the gsift oracle find mostly the same
    keypoints: >= 90 % of oracle keypoints have an OpenCV keypoint within 0.05 px."""
    from scipy.spatial import cKDTree
    g, c = golden["sift_ref"], golden["sift_cv2"]
    for case in ("s240x320_c04", "s200x264_c015"):
        ox = np.c_[g[case + "/kp_x"], g[case + "/kp_y"]]
        d, _ = cKDTree(c[case + "/xy"]).query(ox)
        assert (d < 0.05).mean() > 0.9, case
