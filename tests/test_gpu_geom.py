"""Camera geometry and the pair worker on the device against the reference's outputs
(tests/golden/make_match_pair.py): keypoint undistortion, the ground-plane prior and
matching.match_pair on a synthetic two-view scene."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PARAMS = {"prior_tol": 0.18, "ransac_thr": 1.0, "min_inliers": 20, "ratio": 0.8, "checks": 48, "use_prior": True,
          "guided": True, "n_coarse": 1000, "guided_radius": 0.03, "guided_k": 16}


def test_undistort_pixels(match_golden):
    """float64, the reference's operation order without fused multiply-add: equal to the
    reference's NumPy result to the last bits (1e-9 px bound written here)."""
    from fieldstitch_b200 import matching
    g = match_golden
    for k, want in zip(g["und/k"], g["und/out"]):
        got = matching.undistort_pixels(g["und/uv"], k)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-9)
    assert matching.undistort_pixels(np.zeros((0, 2)), g["und/k"][1]).shape == (0, 2)


def test_predict_ground(match_golden):
    from fieldstitch_b200 import matching
    g = match_golden
    K, R, C = g["ctx/K"], g["ctx/R"], g["ctx/C"]
    pred, ok = matching.predict_ground(g["pred/u"], K[0], R[0], C[0], K[1], R[1], C[1], 0.0)
    np.testing.assert_array_equal(ok, g["pred/ok"])
    np.testing.assert_allclose(pred, g["pred/pred"], rtol=0, atol=1e-7)
    # a camera looking up (the plane behind it) is flagged, as in the reference
    up = np.eye(3)
    p2, ok2 = matching.predict_ground(np.array([[320.0, 240.0]]), K[0], up, C[0], K[1], R[1], C[1], 0.0)
    assert not ok2[0]


def _context(g, tmp, **over):
    for i in (0, 1):
        np.savez(os.path.join(tmp, "%d.npz" % i), xy=g["f%d/xy" % i], desc=g["f%d/desc" % i],
                 resp=g["f%d/resp" % i], red_wh=g["f%d/red_wh" % i])
    c = {"feat_dir": str(tmp), "W": [640, 640], "H": [480, 480], "K": list(g["ctx/K"]), "dist": list(g["ctx/dist"]),
         "R": list(g["ctx/R"]), "C": list(g["ctx/C"]), "zg": [0.0, 0.0], "has_rot": [True, True]}
    c.update(PARAMS)
    c.update(over)
    return c


@pytest.mark.parametrize("case,over", [("guided", {}), ("noprior", {"use_prior": False})])
def test_match_pair_guided_path_equals_reference(match_golden, tmp_path, case, over):
    """Coarse exhaustive match -> prior filter -> RANSAC homography -> guided match -> fundamental
    verification: the device matchers return the reference's candidate sets exactly, so the
    OpenCV fits downstream see the same inputs and the outputs are identical."""
    from fieldstitch_b200 import matching
    g = match_golden
    matching.set_context(_context(g, tmp_path, **over))
    i, j, q, t, sim, n_in = matching.match_pair((0, 1))
    assert (i, j) == (0, 1)
    assert n_in == int(g[case + "/n_in"])
    np.testing.assert_array_equal(q, g[case + "/q"])
    np.testing.assert_array_equal(t, g[case + "/t"])
    np.testing.assert_allclose(np.array(sim), g[case + "/sim"], rtol=0, atol=1e-9)


def test_match_pair_fallback_close_to_reference(match_golden, tmp_path):
    """Guided stage off: the exhaustive fallback is the exact ratio test where the reference
    uses a FLANN kd-forest (approximate neighbours), so the verified sets agree closely, not
    exactly."""
    from fieldstitch_b200 import matching
    g = match_golden
    matching.set_context(_context(g, tmp_path, guided=False))
    _, _, q, t, sim, n_in = matching.match_pair((0, 1))
    ref = set(zip(g["fallback/q"].tolist(), g["fallback/t"].tolist()))
    got = set(zip(q.tolist(), t.tolist()))
    assert abs(n_in - int(g["fallback/n_in"])) <= 0.05 * int(g["fallback/n_in"])
    assert len(ref & got) >= 0.9 * len(ref)
    np.testing.assert_allclose(np.array(sim)[:2], g["fallback/sim"][:2], atol=2e-3)


def test_match_pair_too_few_features(match_golden, tmp_path):
    from fieldstitch_b200 import matching
    g = match_golden
    c = _context(g, tmp_path)
    np.savez(os.path.join(tmp_path, "1.npz"), xy=g["f1/xy"][:20], desc=g["f1/desc"][:20], resp=g["f1/resp"][:20],
             red_wh=g["f1/red_wh"])
    matching.set_context(c)
    assert matching.match_pair((0, 1)) == (0, 1, None, None, None, 0)
