"""Parity of the CUDA matchers (through the C ABI) with the reference fixtures and the oracle:
match lists must be identical (integer/index work, bit-exact bar)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def m():
    import fieldstitch_b200 as f
    f.context(0)
    return f.matching


@pytest.mark.parametrize("case", ["bf_400x380", "bf_257x300", "bf_2x2"])
def test_bf_matches_reference_fixture(m, golden, case):
    g = golden["match_ref"]
    q, t = m._ratio_match_bf(g[case + "/a"].astype(np.float32), g[case + "/b"].astype(np.float32),
                             float(g[case + "/ratio"]))
    np.testing.assert_array_equal(q, g[case + "/q"])
    np.testing.assert_array_equal(t, g[case + "/t"])


@pytest.mark.parametrize("na,nb,seed,ratio", [(3000, 2500, 1, 0.8), (1000, 4097, 2, 0.85), (129, 131, 3, 0.7),
                                              (2, 5000, 4, 0.9), (5000, 2, 5, 0.8)])
def test_bf_matches_oracle(m, na, nb, seed, ratio):
    from fieldstitch_b200 import synth
    from oracle import matching_ref
    a, b, _ = synth.synth_descriptors(na, nb, seed)
    q, t = m._ratio_match_bf(a, b, ratio)
    q2, t2 = matching_ref.ratio_match_bf(a.astype(np.float32), b.astype(np.float32), ratio)
    np.testing.assert_array_equal(q, q2)
    np.testing.assert_array_equal(t, t2)


def test_bf_ties_and_duplicates(m):
    """Duplicate rows in B make the best distance tie: the reference's ratio test rejects them."""
    from oracle import matching_ref
    rng = np.random.default_rng(9)
    a = rng.integers(0, 40, (300, 128)).astype(np.uint8)
    b = np.concatenate([a[:100], a[:100], rng.integers(0, 40, (50, 128)).astype(np.uint8)])
    for ratio in (0.8, 0.99):
        q, t = m._ratio_match_bf(a, b, ratio)
        q2, t2 = matching_ref.ratio_match_bf(a.astype(np.float32), b.astype(np.float32), ratio)
        np.testing.assert_array_equal(q, q2)
        np.testing.assert_array_equal(t, t2)


def test_unique_matches_reference_fixture(m, golden):
    g = golden["match_ref"]
    q, t = m._unique(g["uniq/q"], g["uniq/t"], g["uniq/dd"])
    np.testing.assert_array_equal(q, g["uniq/uq"])
    np.testing.assert_array_equal(t, g["uniq/ut"])


def test_unique_random_against_oracle(m):
    from oracle import matching_ref
    rng = np.random.default_rng(3)
    for n in (1, 2, 17, 5000):
        q = rng.integers(0, 10 ** 6, n)
        t = rng.integers(-50, 50, n)
        dd = rng.integers(0, 20, n).astype(np.float32)
        dd[rng.random(n) < 0.1] = -1.5
        a = m._unique(q, t, dd)
        b = matching_ref.unique(q, t, dd)
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])


@pytest.mark.parametrize("case", ["g_600_k16", "g_600_k2", "g_600_k1", "g_500_all"])
def test_guided_matches_reference_fixture(m, golden, case):
    g = golden["match_ref"]
    radius, kc, ratio, W, H = g[case + "/args"]
    A = {"und": g[case + "/ua"], "desc": g[case + "/a"].astype(np.float32), "wh": (W, H)}
    B = {"und": g[case + "/ub"], "desc": g[case + "/b"].astype(np.float32), "wh": (W, H)}
    q, t = m._guided(A, B, g[case + "/Hm"], radius, int(kc), ratio)
    np.testing.assert_array_equal(q, g[case + "/q"])
    np.testing.assert_array_equal(t, g[case + "/t"])


@pytest.mark.parametrize("n,kc,radius,seed", [(4000, None, 40.0, 1), (4000, 16, 40.0, 2), (3000, 1, 25.0, 3),
                                              (2000, None, 0.5, 4), (3000, 64, 80.0, 5)])
def test_guided_matches_oracle(m, n, kc, radius, seed):
    from fieldstitch_b200 import synth
    from oracle import matching_ref
    rng = np.random.default_rng(seed)
    a, b, truth = synth.synth_descriptors(n, n, seed, true_frac=0.5)
    W, H = 2640.0, 1978.0
    ua = np.c_[rng.uniform(0, W, n), rng.uniform(0, H, n)]
    ub = np.c_[rng.uniform(0, W, n), rng.uniform(0, H, n)]
    hit = truth >= 0
    Hm = synth.random_homography(rng, int(H), int(W))
    ub[hit] = synth.apply_homography(Hm, ua[truth[hit]])
    pred = synth.apply_homography(Hm, ua) + rng.normal(0, 15.0, (n, 2))
    q, t = m.guided_from_pred(pred, a, ub, b, (W, H), radius, kc, 0.85)
    q2, t2 = matching_ref.guided_from_pred(pred, a, ub, b, (W, H), radius, kc, 0.85)
    np.testing.assert_array_equal(q, q2)
    np.testing.assert_array_equal(t, t2)
    assert kc is not None or radius < 1 or len(q) > 0.2 * n


def test_guided_edge_cases(m):
    a = np.zeros((3, 128), np.uint8)
    q, t = m.guided_from_pred(np.full((3, 2), -1e9), a, np.zeros((3, 2)), a, (100, 100), 10.0, None, 0.8)
    assert len(q) == 0
    q, t = m.guided_from_pred(np.zeros((3, 2)), a, np.zeros((0, 2)), np.zeros((0, 128), np.uint8), (100, 100), 10.0,
                              None, 0.8)
    assert len(q) == 0


def test_perspective_matches_cv2(m):
    import cv2
    rng = np.random.default_rng(0)
    from fieldstitch_b200 import synth
    for s in range(3):
        H = synth.random_homography(rng, 1978, 2640)
        H[2, :2] = rng.normal(0, 1e-4, 2)
        xy = rng.uniform(-100, 2700, (5000, 2))
        want = cv2.perspectiveTransform(xy.reshape(-1, 1, 2), H).reshape(-1, 2)
        got = m.perspective(xy, H)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-9)
