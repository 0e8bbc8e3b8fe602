"""Device RANSAC homographies (the stage-1 fit of matching.match_pair) through the C ABI, against
the ground truth of seeded synthetic pairs and against OpenCV's cv2.findHomography (the
reference's call). Random samples differ from OpenCV's, so the comparison is statistical: inlier
masks agree on >= 97 % of correspondences, fitted homographies reproject the true inliers within
1 px of the truth (median)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

THR = 0.012 * 2640


def _problem(seed, n, outliers, noise=0.7):
    rng = np.random.default_rng(seed)
    a, s = rng.uniform(-0.2, 0.2), rng.uniform(0.9, 1.1)
    H = np.array([[s * np.cos(a), -s * np.sin(a), rng.uniform(-200, 200)],
                  [s * np.sin(a), s * np.cos(a), rng.uniform(-200, 200)],
                  [rng.uniform(-3e-5, 3e-5), rng.uniform(-3e-5, 3e-5), 1.0]])
    src = np.c_[rng.uniform(0, 2640, n), rng.uniform(0, 1978, n)]
    p = np.c_[src, np.ones(n)] @ H.T
    dst = p[:, :2] / p[:, 2:] + rng.normal(0, noise, (n, 2))
    bad = rng.random(n) < outliers
    dst[bad] = np.c_[rng.uniform(0, 2640, bad.sum()), rng.uniform(0, 1978, bad.sum())]
    return src, dst, H, ~bad


def _reproj(H, src):
    p = np.c_[src, np.ones(len(src))] @ H.T
    return p[:, :2] / p[:, 2:]


def test_homography_batch_against_truth_and_opencv():
    import cv2
    from fieldstitch_b200 import matching
    sizes = [(40, 0.0), (300, 0.3), (1000, 0.45), (2500, 0.2), (120, 0.5), (4000, 0.35)]
    probs = [_problem(10 + k, n, f) for k, (n, f) in enumerate(sizes)]
    res = matching.find_homography_batch([(s, d) for s, d, _, _ in probs], THR)
    for (src, dst, Ht, truth), (H, mask) in zip(probs, res):
        assert H is not None and mask.shape == (len(src), 1)
        m = mask.ravel().astype(bool)
        err = np.linalg.norm(_reproj(H, src[truth]) - _reproj(Ht, src[truth]), axis=1)
        assert np.median(err) < 1.0, np.median(err)
        assert (m & truth).sum() >= 0.97 * truth.sum()
        assert (m & truth).sum() >= 0.97 * m.sum()
        Hc, mc = cv2.findHomography(src, dst, cv2.RANSAC, THR)
        assert (m == mc.ravel().astype(bool)).mean() >= 0.97


def test_homography_deterministic_and_degenerate():
    from fieldstitch_b200 import matching
    src, dst, _, _ = _problem(3, 500, 0.3)
    a = matching.find_homography(src, dst, THR, seed=5)
    b = matching.find_homography(src, dst, THR, seed=5)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    H, m = matching.find_homography(src[:3], dst[:3], THR)
    assert H is None and m.shape == (3, 1) and not m.any()
    assert matching.find_homography_batch([], THR) == []


def test_match_pair_with_device_ransac(match_golden, tmp_path):
    """The pair worker with the device RANSAC in stage 1: the homography only seeds the guided
    search, so the verified matches stay those of the reference (>= 95 % shared)."""
    from fieldstitch_b200 import matching
    from test_gpu_geom import _context
    g = match_golden
    matching.set_context(_context(g, tmp_path, ransac="device"))
    _, _, q, t, sim, n_in = matching.match_pair((0, 1))
    ref = set(zip(g["guided/q"].tolist(), g["guided/t"].tolist()))
    got = set(zip(q.tolist(), t.tolist()))
    assert len(ref & got) >= 0.95 * len(ref) and abs(n_in - int(g["guided/n_in"])) <= 0.05 * int(g["guided/n_in"])


def _two_view(seed, n, outliers, noise=0.25):
    """A seeded two-view scene with relief (points 0-30 m above ground, cameras at 100 m, 20 m
    apart, a few degrees of relative rotation), pixel correspondences with noise and outliers."""
    rng = np.random.default_rng(seed)
    f, cx, cy = 2000.0, 1320.0, 989.0
    K = np.array([[f, 0, cx], [0, f, cy], [0, 0, 1.0]])

    def rot(ax, ay, az):
        Rx = np.array([[1, 0, 0], [0, np.cos(ax), -np.sin(ax)], [0, np.sin(ax), np.cos(ax)]])
        Ry = np.array([[np.cos(ay), 0, np.sin(ay)], [0, 1, 0], [-np.sin(ay), 0, np.cos(ay)]])
        Rz = np.array([[np.cos(az), -np.sin(az), 0], [np.sin(az), np.cos(az), 0], [0, 0, 1]])
        return Rz @ Ry @ Rx

    X = np.c_[rng.uniform(-60, 60, n), rng.uniform(-45, 45, n), rng.uniform(0, 30, n)]
    R1, C1 = rot(np.pi, 0, 0), np.array([0.0, 0.0, 100.0])
    R2 = rot(np.pi + rng.uniform(-0.05, 0.05), rng.uniform(-0.05, 0.05), rng.uniform(-0.1, 0.1))
    C2 = np.array([rng.uniform(15, 25), rng.uniform(-5, 5), 100.0 + rng.uniform(-3, 3)])

    def proj(R, C):
        p = (K @ (R @ (X - C).T)).T
        return p[:, :2] / p[:, 2:]

    a = proj(R1, C1) + rng.normal(0, noise, (n, 2))
    b = proj(R2, C2) + rng.normal(0, noise, (n, 2))
    bad = rng.random(n) < outliers
    b[bad] = np.c_[rng.uniform(0, 2640, bad.sum()), rng.uniform(0, 1978, bad.sum())]
    return a, b, ~bad


def _epi_dist(F, a, b):
    """max of the two point-to-epipolar-line distances (pixels)"""
    ha, hb = np.c_[a, np.ones(len(a))], np.c_[b, np.ones(len(b))]
    l2, l1 = ha @ F.T, hb @ F
    e = np.abs((hb * l2).sum(1))
    return np.maximum(e / np.hypot(l2[:, 0], l2[:, 1]), e / np.hypot(l1[:, 0], l1[:, 1]))


def test_fundamental_batch_against_truth_and_opencv():
    """matching._verify's fundamental fit (cv2.findFundamentalMat with USAC_MAGSAC): the device's
    masks keep >= 97 % of the true inliers with >= 97 % precision and agree with OpenCV's masks on
    >= 97 % of correspondences; the true inliers lie within the threshold of the fitted F."""
    import cv2
    from fieldstitch_b200 import matching
    thr = 1.0
    sizes = [(60, 0.0), (400, 0.3), (1500, 0.45), (3000, 0.2), (200, 0.5), (5000, 0.35)]
    probs = [_two_view(40 + k, n, f) for k, (n, f) in enumerate(sizes)]
    res = matching.find_fundamental_batch([(a, b) for a, b, _ in probs], thr)
    agree = []
    for (a, b, truth), (F, mask) in zip(probs, res):
        assert F is not None and mask.shape == (len(a), 1)
        m = mask.ravel().astype(bool)
        assert (m & truth).sum() >= 0.97 * truth.sum(), ((m & truth).sum(), truth.sum())
        assert (m & truth).sum() >= 0.97 * m.sum()
        assert np.median(_epi_dist(F, a[truth], b[truth])) < thr
        Fc, mc = cv2.findFundamentalMat(a.astype(np.float32), b.astype(np.float32), cv2.USAC_MAGSAC, thr, 0.999, 10000)
        agree.append((m == mc.ravel().astype(bool)).mean())
    print("\n[fundamental] mask agreement with OpenCV USAC_MAGSAC per pair:", ["%.4f" % v for v in agree])
    assert min(agree) >= 0.97, agree


def test_fundamental_deterministic_and_degenerate():
    from fieldstitch_b200 import matching
    a, b, _ = _two_view(7, 500, 0.3)
    x = matching.find_fundamental(a, b, 1.0, seed=9)
    y = matching.find_fundamental(a, b, 1.0, seed=9)
    np.testing.assert_array_equal(x[0], y[0])
    np.testing.assert_array_equal(x[1], y[1])
    F, m = matching.find_fundamental(a[:7], b[:7], 1.0)
    assert F is None and m.shape == (7, 1) and not m.any()
    assert matching.find_fundamental_batch([], 1.0) == []
