"""The geometry oracle (oracle/geom_ref.py) against the reference's own outputs on the golden
scene: undistortion and the ground-plane prior reproduce them exactly (same NumPy expressions)."""
import numpy as np

from oracle import geom_ref


def test_undistort_matches_reference(match_golden):
    g = match_golden
    for k, want in zip(g["und/k"], g["und/out"]):
        np.testing.assert_array_equal(geom_ref.undistort_pixels(g["und/uv"], tuple(k)), want)


def test_predict_matches_reference(match_golden):
    g = match_golden
    K, R, C = g["ctx/K"], g["ctx/R"], g["ctx/C"]
    pred, ok = geom_ref.predict_ground(g["pred/u"], K[0], R[0], C[0], K[1], R[1], C[1], 0.0)
    np.testing.assert_array_equal(ok, g["pred/ok"])
    np.testing.assert_allclose(pred, g["pred/pred"], rtol=0, atol=1e-9)


def test_fixture_scene_is_consistent(match_golden):
    """The guided path of the reference found a well-supported pair (the scene is not degenerate)."""
    g = match_golden
    assert int(g["guided/n_in"]) >= 200
    assert abs(np.degrees(g["guided/sim"][0]) + 4.0) < 0.2
