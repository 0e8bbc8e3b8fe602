"""The synthetic flight of the config-5 workload (CPU parts): lawnmower poses, true frame-to-frame
homographies and the reference pipeline's GNSS neighbour pairs (app/planesite/pipeline.py:452-476)."""
import numpy as np

from fieldstitch_b200 import synth


def test_lawnmower_grid_and_overlaps():
    p = synth.lawnmower(5)
    assert p.shape == (400, 4)
    # along-track spacing 20 % of the frame height, across-track 30 % of the width
    assert np.allclose(np.abs(p[1, 1] - p[0, 1]), 0.2 * 1978)
    assert np.allclose(p[20, 0] - p[0, 0], 0.3 * 2640)
    # serpentine: the second line is flown back at 180 deg
    assert abs(np.degrees(p[0, 2])) <= 3.0 and abs(np.degrees(p[20, 2]) - 180.0) <= 3.0
    assert np.all(np.abs(p[:, 3] - 1.0) <= 0.02)
    # every frame lies inside the 20000 x 16000 terrain
    for pose in p:
        M = synth.frame_to_terrain(pose)
        c = np.array([[0, 0, 1], [2639, 0, 1], [0, 1977, 1], [2639, 1977, 1]], np.float64) @ M.T
        assert c[:, 0].min() >= 0 and c[:, 0].max() <= 19999 and c[:, 1].min() >= 0 and c[:, 1].max() <= 15999


def test_frame_homographies_compose():
    p = synth.lawnmower(5)
    H01, H12, H02 = synth.frame_homography(p[0], p[1]), synth.frame_homography(p[1], p[2]), \
        synth.frame_homography(p[0], p[2])
    np.testing.assert_allclose(H12 @ H01, H02, atol=1e-9)
    np.testing.assert_allclose(synth.frame_homography(p[1], p[0]) @ H01, np.eye(3), atol=1e-12)
    # a point of frame 0 lands on the same terrain point through frame 1
    x = np.array([[100.0, 200.0]])
    t0 = synth.apply_homography(synth.frame_to_terrain(p[0]), x)
    t1 = synth.apply_homography(synth.frame_to_terrain(p[1]), synth.apply_homography(H01, x))
    np.testing.assert_allclose(t0, t1, atol=1e-9)


def test_gnss_pairs_follow_the_pipeline_rule():
    p = synth.lawnmower(5)
    pairs = synth.gnss_pairs(p, sigma=15.0, seed=1)
    assert 2800 <= len(pairs) <= 3600, len(pairs)
    assert pairs == sorted(set(pairs)) and all(i < j for i, j in pairs)
    # consecutive frames in flight order are paired; frames more than 2 x the long footprint apart are not
    assert all((i, i + 1) in set(pairs) for i in range(399))
    d = np.array([np.hypot(*(p[i, :2] - p[j, :2])) for i, j in pairs])
    assert d.max() < 2 * 1320 + 100
    # the 16-neighbour cap: no frame has more than 16 + 2 * 2 partners from its own query
    deg = np.bincount(np.array(pairs).ravel(), minlength=400)
    assert deg.max() <= 2 * 16 + 4
