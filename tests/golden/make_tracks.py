"""Golden track fixtures: the reference's recon.build_tracks on seeded synthetic match graphs.

    python tests/golden/make_tracks.py <path to the reference's app directory>

Graphs: photos with random feature counts (some zero), pairs of random verified matches plus
chains of true tracks across several photos, some joined so that a component holds two features
of one photo (rejected by the reference), self-matches and repeated matches. Writes tracks.npz
next to this script; nothing at test time reads the reference tree.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def graph(seed, n_img, n_pairs, n_chains):
    rng = np.random.default_rng(seed)
    nfeat = rng.integers(0, 400, n_img)
    nfeat[rng.integers(0, n_img)] = 0
    pairs = []
    have = np.flatnonzero(nfeat > 0)
    for _ in range(n_pairs):
        i, j = rng.choice(have, 2, replace=False)
        m = int(rng.integers(0, 60))
        q = rng.integers(0, nfeat[i], m).astype(np.int32)
        t = rng.integers(0, nfeat[j], m).astype(np.int32)
        pairs.append((int(i), int(j), q, t))
    for _ in range(n_chains):   # a feature seen in several photos, matched consecutively
        ph = rng.choice(have, int(rng.integers(2, min(6, len(have)) + 1)), replace=False)
        fs = [int(rng.integers(0, nfeat[p])) for p in ph]
        for a in range(len(ph) - 1):
            pairs.append((int(ph[a]), int(ph[a + 1]), np.array([fs[a]], np.int32), np.array([fs[a + 1]], np.int32)))
    i = int(have[0])
    pairs.append((i, i, np.array([0, 1], np.int32), np.array([0, 1], np.int32)))   # self-matches
    return nfeat, pairs


def main(app_dir):
    sys.path.insert(0, app_dir)
    # recon imports the geodesy module, which needs pyproj (absent here and unused by build_tracks):
    # a stand-in module lets the reference's recon import unchanged
    import types
    for name in ("pyproj",):
        try:
            __import__(name)
        except ImportError:
            sys.modules[name] = types.SimpleNamespace(Transformer=None, CRS=None)
    from planesite import recon
    out = {}
    for k, (seed, n_img, n_pairs, n_chains) in enumerate(((1, 6, 8, 20), (2, 30, 80, 300), (3, 12, 0, 40))):
        nfeat, pairs = graph(seed, n_img, n_pairs, n_chains)
        tid, img, feat, n = recon.build_tracks(pairs, nfeat, n_img)
        out["g%d/nfeat" % k] = nfeat
        out["g%d/pi" % k] = np.array([p[0] for p in pairs], np.int32)
        out["g%d/pj" % k] = np.array([p[1] for p in pairs], np.int32)
        out["g%d/len" % k] = np.array([len(p[2]) for p in pairs], np.int64)
        out["g%d/q" % k] = np.concatenate([p[2] for p in pairs]).astype(np.int32)
        out["g%d/t" % k] = np.concatenate([p[3] for p in pairs]).astype(np.int32)
        out["g%d/tid" % k], out["g%d/img" % k], out["g%d/feat" % k] = tid, img, feat
        out["g%d/n" % k] = np.array(n)
        print("graph", k, "observations", len(tid), "tracks", n)
    np.savez_compressed(os.path.join(HERE, "tracks.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_tracks.py <path to the reference's app directory>")
    main(sys.argv[1])
