"""Device track building (recon.build_tracks) through the C ABI: the reference's output on the
golden graphs, and the oracle's on a pipeline-sized random graph (400 photos, about 0.5 M
matches), both exactly."""
import numpy as np
import pytest

from test_oracle_recon import golden_graphs

pytestmark = pytest.mark.gpu


def test_tracks_match_reference_fixtures():
    from fieldstitch_b200 import recon
    for g in golden_graphs():
        tid, img, feat, n = recon.build_tracks(g["pairs"], g["nfeat"], len(g["nfeat"]))
        assert n == int(g["n"])
        for a, b in ((tid, g["tid"]), (img, g["img"]), (feat, g["feat"])):
            np.testing.assert_array_equal(a, b)


def test_tracks_match_oracle_large():
    from fieldstitch_b200 import recon
    from oracle import recon_ref
    rng = np.random.default_rng(5)
    n_img = 400
    nfeat = rng.integers(500, 3000, n_img)
    pairs = []
    for _ in range(3000):
        i, j = rng.choice(n_img, 2, replace=False)
        m = int(rng.integers(20, 300))
        pairs.append((int(i), int(j), rng.integers(0, nfeat[i], m), rng.integers(0, nfeat[j], m)))
    for _ in range(20000):   # consistent chains over neighbouring photos
        p0 = int(rng.integers(0, n_img - 6))
        ph = p0 + np.sort(rng.choice(6, int(rng.integers(2, 6)), replace=False))
        fs = [int(rng.integers(0, nfeat[p])) for p in ph]
        for a in range(len(ph) - 1):
            pairs.append((int(ph[a]), int(ph[a + 1]), np.array([fs[a]]), np.array([fs[a + 1]])))
    want = recon_ref.build_tracks(pairs, nfeat, n_img)
    got = recon.build_tracks(pairs, nfeat, n_img)
    assert got[3] == want[3] and want[3] > 1000
    for a, b in zip(got[:3], want[:3]):
        np.testing.assert_array_equal(a, b)


def test_tracks_empty_inputs():
    from fieldstitch_b200 import recon
    z = np.zeros(0, np.int64)
    for pairs in ([], [(0, 1, z, z)]):
        tid, img, feat, n = recon.build_tracks(pairs, [10, 10], 2)
        assert n == 0 and len(tid) == len(img) == len(feat) == 0
