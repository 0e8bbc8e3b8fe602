"""Golden fixtures for the matching stage's camera geometry and pair worker.

Run in the build container, where the reference source tree is available:

    python tests/golden/make_match_pair.py <path to the reference's app directory>

It imports PlaneSite's camera.undistort_pixels, matching._predict and matching.match_pair and runs
them on a seeded synthetic two-view scene: a nadir camera pair over flat ground (the second view
shifted and yawed; its image is the first warped by the induced ground-plane homography), feature
files written by the reference's own CPU extractor and writer (features.sift_cpu, features._save).
Writes match_pair.npz next to this script; nothing at test time reads the reference tree.
"""
import math
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fieldstitch_b200 import synth  # noqa: E402
from oracle import geom_ref  # noqa: E402

W, H, F = 640, 480, 600.0


def nadir(yaw_deg):
    """World-to-camera rotation of a camera looking straight down (image x = world x, image y =
    -world y), turned by yaw about the vertical."""
    a = math.radians(yaw_deg)
    rz = np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]])
    return np.diag([1.0, -1.0, -1.0]) @ rz


def scene():
    K = np.array([[F, 0, 320.0], [0, F, 240.0], [0, 0, 1]])
    R = [nadir(0.0), nadir(4.0)]
    C = [np.array([0.0, 0.0, 120.0]), np.array([9.0, 4.0, 120.0])]
    dist = np.array([-0.02, 0.004, 0.0005, -0.0003, 0.0])
    return K, R, C, dist


def images(K, R, C):
    import cv2
    a = synth.synth_image(H, W, 4242)
    corners = np.array([[0, 0], [W - 1, 0], [W - 1, H - 1], [0, H - 1]], np.float64)
    pj, _ = geom_ref.predict_ground(corners, K, R[0], C[0], K, R[1], C[1], 0.0)
    Hm = cv2.getPerspectiveTransform(corners.astype(np.float32), pj.astype(np.float32))
    b = cv2.warpPerspective(a, Hm, (W, H), flags=cv2.INTER_LINEAR, borderMode=cv2.BORDER_REFLECT)
    rng = np.random.default_rng(7)
    b = np.clip(b.astype(np.float64) + rng.normal(0, 2.0, b.shape), 0, 255).astype(np.uint8)
    return a, b


def main(app_dir):
    sys.path.insert(0, app_dir)
    from planesite import camera, features, matching

    out = {}
    rng = np.random.default_rng(99)
    # undistortion: three parameter sets (none, mild, strong), points around and beyond the frame
    uv = np.c_[rng.uniform(-60, W + 60, 600), rng.uniform(-60, H + 60, 600)]
    ks = np.array([[F, 320, 240, 0, 0, 0, 0, 0], [F, 320, 240, -0.02, 0.004, 0.0005, -0.0003, 0],
                   [800, 300, 250, -0.3, 0.1, 0.002, -0.001, -0.01]], np.float64)
    out["und/uv"] = uv
    out["und/k"] = ks
    out["und/out"] = np.stack([camera.undistort_pixels(uv, tuple(k)) for k in ks])

    K, R, C, dist = scene()
    a, b = images(K, R, C)
    tmp = tempfile.mkdtemp(prefix="fsb_match_pair_")
    for i, img in enumerate((a, b)):
        xy, desc, resp, _ = features.sift_cpu(img, 1200)
        features._save(os.path.join(tmp, "%d.npz" % i), xy, desc, resp, W, H)
        with np.load(os.path.join(tmp, "%d.npz" % i)) as z:
            for k in ("xy", "desc", "resp", "red_wh"):
                out["f%d/%s" % (i, k)] = z[k]
    ctx = {"feat_dir": tmp, "W": [W, W], "H": [H, H], "K": [K, K], "dist": [dist, dist], "R": R, "C": C,
           "zg": [0.0, 0.0], "has_rot": [True, True], "prior_tol": 0.18, "ransac_thr": 1.0, "min_inliers": 20,
           "ratio": 0.8, "checks": 48, "use_prior": True, "guided": True, "n_coarse": 1000, "guided_radius": 0.03,
           "guided_k": 16}
    out["ctx/K"] = np.stack([K, K])
    out["ctx/dist"] = np.stack([dist, dist])
    out["ctx/R"] = np.stack(R)
    out["ctx/C"] = np.stack(C)

    # the prior, on undistorted keypoints of image 0
    matching._CTX = ctx
    matching._CACHE.clear()
    u0 = matching._get(0)["und"]
    pred, ok = matching._predict(u0, 0, 1)
    out["pred/u"] = u0
    out["pred/pred"] = pred
    out["pred/ok"] = ok

    # the pair worker: guided path, exhaustive fallback (guided off), no prior
    for name, over in (("guided", {}), ("fallback", {"guided": False}), ("noprior", {"use_prior": False})):
        c = dict(ctx, **over)
        matching._CTX = c
        matching._CACHE.clear()
        i, j, q, t, sim, n_in = matching.match_pair((0, 1))
        out[name + "/n_in"] = np.array(n_in)
        out[name + "/q"] = np.zeros(0, np.int32) if q is None else q
        out[name + "/t"] = np.zeros(0, np.int32) if t is None else t
        out[name + "/sim"] = np.full(4, np.nan) if sim is None or isinstance(sim[0], str) else np.array(sim)
        print(name, "n_in", n_in, "matches", 0 if q is None else len(q), "sim", sim)
    for f in os.listdir(tmp):
        os.remove(os.path.join(tmp, f))
    os.rmdir(tmp)
    np.savez_compressed(os.path.join(HERE, "match_pair.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_match_pair.py <path to the reference's app directory>")
    main(sys.argv[1])
