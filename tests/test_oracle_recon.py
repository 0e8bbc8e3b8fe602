"""The track oracle (oracle/recon_ref.py) reproduces the reference's recon.build_tracks on the
golden match graphs (tests/golden/make_tracks.py): rejected components, self-matches, photos
without features."""
import os

import numpy as np

from oracle import recon_ref

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tracks.npz")


def golden_graphs():
    with np.load(GOLDEN) as z:
        out = []
        k = 0
        while "g%d/nfeat" % k in z.files:
            g = {n: z["g%d/%s" % (k, n)] for n in ("nfeat", "pi", "pj", "len", "q", "t", "tid", "img", "feat", "n")}
            cuts = np.cumsum(g["len"])[:-1]
            g["pairs"] = [(int(a), int(b), q, t) for a, b, q, t in
                          zip(g["pi"], g["pj"], np.split(g["q"], cuts), np.split(g["t"], cuts))]
            out.append(g)
            k += 1
    return out


def test_tracks_oracle_matches_reference():
    gs = golden_graphs()
    assert len(gs) == 3
    for g in gs:
        tid, img, feat, n = recon_ref.build_tracks(g["pairs"], g["nfeat"], len(g["nfeat"]))
        assert n == int(g["n"])
        for a, b in ((tid, g["tid"]), (img, g["img"]), (feat, g["feat"])):
            np.testing.assert_array_equal(a, b)
