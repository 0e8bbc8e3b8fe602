"""Generate the golden fixtures that pin the CPU oracle (and the CUDA path) to the reference.

Run in the build container, where the reference source tree is available:

    python tests/golden/make_golden.py <path to the reference's app directory>

It imports PlaneSite's own modules (planesite.gsift / features / matching) and runs their CPU
code paths on small seeded inputs, plus OpenCV SIFT (the reference's CPU extractor), and writes
compressed .npz files next to this script. Nothing at test time reads the reference tree.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fieldstitch_b200 import synth  # noqa: E402

# (name, h, w, seed, contrast, edge, max_kp, nfeat for the sift_gpu sequence)
SIFT_CASES = [
    ("s240x320_c04", 240, 320, 11, 0.04, 10.0, 8000, 300),
    ("s200x264_c015", 200, 264, 23, 0.015, 12.0, 12000, 250),
    ("s97x131_c04", 97, 131, 5, 0.04, 10.0, 8000, 60),
]


def sift_fixtures(gsift, features):
    out = {}
    for name, h, w, seed, contrast, edge, max_kp, nfeat in SIFT_CASES:
        img = synth.synth_image(h, w, seed)
        kps, st = gsift.detect(img, gpu=False, max_kp=max_kp, contrast=contrast, edge=edge)
        sel = np.arange(len(kps["x"]), dtype=np.int64)
        desc = gsift.describe(st, kps, sel)
        out[name + "/img"] = img
        out[name + "/params"] = np.array([contrast, edge, max_kp, nfeat], np.float64)
        for k, v in kps.items():
            out[name + "/kp_" + k] = v
        out[name + "/desc"] = desc
        # the per-photo GPU worker sequence (detect with the pipeline defaults -> spread -> describe)
        xy, d2, resp, _ = features.sift_gpu(img, nfeat, gpu=False)
        out[name + "/sg_xy"] = xy
        out[name + "/sg_desc"] = d2 if d2 is not None else np.zeros((0, 128), np.float32)
        out[name + "/sg_resp"] = resp
        # RootSIFT bytes of the feature file, through the reference's own writer
        path = os.path.join("/tmp", "fsb_golden_%s.npz" % name)
        features._save(path, xy, d2, resp, w, h)
        with np.load(path) as z:
            out[name + "/sg_u8"] = z["desc"]
        os.remove(path)
    # a flat image has no keypoints
    flat = np.full((64, 80), 128, np.uint8)
    kps, _ = gsift.detect(flat, gpu=False)
    out["flat/img"] = flat
    out["flat/n"] = np.array(len(kps["x"]))
    return out


def cv2_fixtures():
    import cv2
    out = {}
    for name, h, w, seed, contrast, edge, max_kp, nfeat in SIFT_CASES[:2]:
        img = synth.synth_image(h, w, seed)
        sift = cv2.SIFT_create(nfeatures=max_kp, nOctaveLayers=3, contrastThreshold=contrast,
                               edgeThreshold=edge, sigma=1.6)
        kps, desc = sift.detectAndCompute(img, None)
        out[name + "/xy"] = np.array([k.pt for k in kps], np.float32).reshape(-1, 2)
        out[name + "/size"] = np.array([k.size for k in kps], np.float32)
        out[name + "/angle"] = np.array([k.angle for k in kps], np.float32)
        out[name + "/response"] = np.array([k.response for k in kps], np.float32)
        out[name + "/octave"] = np.array([k.octave for k in kps], np.int32)
        out[name + "/desc"] = desc
    return out


def match_fixtures(matching):
    out = {}
    rng = np.random.default_rng(101)
    # dense ratio matching on SIFT-like u8 descriptors
    for name, na, nb, seed, ratio in [("bf_400x380", 400, 380, 3, 0.8), ("bf_257x300", 257, 300, 9, 0.85),
                                      ("bf_2x2", 2, 2, 4, 0.8)]:
        a, b, _ = synth.synth_descriptors(na, nb, seed)
        q, t = matching._ratio_match_bf(a.astype(np.float32), b.astype(np.float32), ratio)
        out[name + "/a"], out[name + "/b"] = a, b
        out[name + "/ratio"] = np.array(ratio)
        out[name + "/q"], out[name + "/t"] = q, t
    # one-to-one filter with ties on the distance
    q = np.array([0, 1, 2, 3, 4, 5, 6, 7], np.int64)
    t = np.array([5, 3, 5, 3, 9, 5, 1, 9], np.int64)
    dd = np.array([4, 2, 4, 1, 7, 3, 0, 7], np.float32)
    uq, ut = matching._unique(q, t, dd)
    out["uniq/q"], out["uniq/t"], out["uniq/dd"] = q, t, dd
    out["uniq/uq"], out["uniq/ut"] = uq, ut
    # guided matching: B keypoints are A's moved by a homography plus jitter, with distractors
    for name, n, seed, kc, radius in [("g_600_k16", 600, 21, 16, 24.0), ("g_600_k2", 600, 22, 2, 24.0),
                                      ("g_600_k1", 600, 23, 1, 24.0), ("g_500_all", 500, 24, 100000, 40.0)]:
        a, b, truth = synth.synth_descriptors(n, n, seed, true_frac=0.5)
        W, H = 640, 480
        ua = np.c_[rng.uniform(0, W, n), rng.uniform(0, H, n)]
        Hm = synth.random_homography(rng, H, W, rot_deg=5.0, scale=(0.95, 1.05), shift=30.0)
        ub = np.c_[rng.uniform(0, W, n), rng.uniform(0, H, n)]
        hit = truth >= 0
        ub[hit] = synth.apply_homography(Hm, ua[truth[hit]]) + rng.normal(0, 3.0, (hit.sum(), 2))
        fa, fb = a.astype(np.float32), b.astype(np.float32)
        A = {"und": ua, "desc": fa, "norm": (fa * fa).sum(1), "tree": None, "wh": (W, H)}
        B = {"und": ub, "desc": fb, "norm": (fb * fb).sum(1), "tree": None, "wh": (W, H)}
        qg, tg = matching._guided(A, B, Hm, radius, kc, 0.85)
        out[name + "/a"], out[name + "/b"] = a, b
        out[name + "/ua"], out[name + "/ub"], out[name + "/Hm"] = ua, ub, Hm
        out[name + "/args"] = np.array([radius, kc, 0.85, W, H], np.float64)
        out[name + "/q"], out[name + "/t"] = qg, tg
    return out


def main(ref_app):
    sys.path.insert(0, ref_app)
    from planesite import features, gsift, matching
    np.savez_compressed(os.path.join(HERE, "sift_ref.npz"), **sift_fixtures(gsift, features))
    np.savez_compressed(os.path.join(HERE, "sift_cv2.npz"), **cv2_fixtures())
    np.savez_compressed(os.path.join(HERE, "match_ref.npz"), **match_fixtures(matching))
    for f in ("sift_ref.npz", "sift_cv2.npz", "match_ref.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path to the reference's app directory>")
    main(sys.argv[1])
