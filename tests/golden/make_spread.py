"""Golden grid-spread fixtures: the reference's features._spread (and the stable response sort that
follows it in features.py:126) on seeded keypoint lists in detect's order (responses descending).

    python tests/golden/make_spread.py <path to the reference's app directory>

Cases: uniform, clustered (few cells) and border-crossing positions; distinct responses and
heavily tied ones (a handful of values), n below, near and far above the cap. Writes spread.npz
next to this script; nothing at test time reads the reference tree.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = [  # (n, nfeat, mode, ties)
    (60, 100, "uniform", False), (500, 108, "uniform", False), (3000, 1000, "cluster", False),
    (4000, 3999, "border", False), (12000, 5000, "uniform", False), (20000, 300, "cluster", False),
    (3000, 1000, "uniform", True), (12000, 5000, "border", True), (6000, 2000, "cluster", True),
]


def keypoints(rng, n, W, H, mode, ties):
    if mode == "uniform":
        x, y = rng.uniform(0, W, n), rng.uniform(0, H, n)
    elif mode == "cluster":
        x, y = rng.uniform(0, W / 6, n), rng.uniform(0, H / 4, n)
    else:
        x, y = rng.uniform(-5, W + 5, n), rng.uniform(-5, H + 5, n)
    r = rng.integers(1, 12, n).astype(np.float32) * np.float32(0.01) if ties else \
        rng.uniform(0.01, 1.0, n).astype(np.float32)
    return x.astype(np.float32), y.astype(np.float32), np.sort(r)[::-1].copy()


def main(app_dir):
    sys.path.insert(0, app_dir)
    from planesite import features
    rng = np.random.default_rng(2024)
    out = {}
    for k, (n, nfeat, mode, ties) in enumerate(CASES):
        W, H = int(rng.integers(300, 3000)), int(rng.integers(300, 3000))
        x, y, r = keypoints(rng, n, W, H, mode, ties)
        kps = [features._KP(float(a), float(b), float(c)) for a, b, c in zip(x, y, r)]
        sel = np.array(features._spread(kps, W, H, nfeat), np.int64)
        out["c%d/x" % k], out["c%d/y" % k], out["c%d/resp" % k] = x, y, r
        out["c%d/wh_n" % k] = np.array([W, H, nfeat], np.int64)
        out["c%d/sel" % k] = sel
        out["c%d/sorted" % k] = sel[np.argsort(-r[sel], kind="stable")]
        print("case", k, n, nfeat, mode, "ties" if ties else "", "selected", len(sel))
    out["n_cases"] = np.array(len(CASES))
    np.savez_compressed(os.path.join(HERE, "spread.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_spread.py <path to the reference's app directory>")
    main(sys.argv[1])
