"""Generate the fixture that pins the SIFT path at the benchmark's own configuration: 2640x1978
images, contrast 0.015, edge 12, keypoint caps 2000 and 16000 (detect's max_kp = 2.2 nfeat, as
features.sift_gpu sets it).

Run in the build container, where the reference source tree is available; the path of the
reference's `app` directory is a required argument:

    python tests/golden/make_headline.py <path to the reference's app directory>

It imports PlaneSite's own modules and runs their CPU code paths (gsift.detect / describe with
gpu=False, features.sift_gpu with gpu=False, features._save) on two seeded benchmark images, and
OpenCV SIFT with the same parameters. The images themselves are not stored: the test regenerates
them from their seeds (synth.synth_image) and checks a digest. The reference's CPU path takes a
few minutes at this size.
"""
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fieldstitch_b200 import synth  # noqa: E402

H, W = 1978, 2640
CONTRAST, EDGE = 0.015, 12.0
# (name, seed of synth.synth_image, nfeat): the first image of the benchmark's first two pairs
# (bench.py seeds pairs from 1000), with the two ends of the benchmark's keypoint-cap range
CASES = [("h1000_n16000", 1000, 16000), ("h1001_n2000", 1001, 2000)]
DESC_ROWS = 4000   # RootSIFT rows of the worker output kept in the fixture (the strongest)


def digest(img):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(img).tobytes()).digest()[:8], np.uint64)[0]


def main(ref_app):
    sys.path.insert(0, ref_app)
    import cv2
    from planesite import features, gsift
    out = {}
    for name, seed, nfeat in CASES:
        t0 = time.time()
        img = synth.synth_image(H, W, seed)
        max_kp = int(nfeat * 2.2)
        kps, _ = gsift.detect(img, gpu=False, max_kp=max_kp, contrast=CONTRAST, edge=EDGE)
        out[name + "/params"] = np.array([seed, nfeat, max_kp, CONTRAST, EDGE], np.float64)
        out[name + "/digest"] = np.array(digest(img), np.uint64)
        for k, v in kps.items():
            out[name + "/kp_" + k] = v
        # the per-photo worker sequence: detect (max_kp = 2.2 nfeat) -> spread -> describe -> _save
        xy, d2, resp, _ = features.sift_gpu(img, nfeat, gpu=False)
        path = os.path.join("/tmp", "fsb_headline_%s.npz" % name)
        features._save(path, xy, d2, resp, W, H)
        with np.load(path) as z:
            u8 = z["desc"]
        os.remove(path)
        out[name + "/sg_xy"] = xy
        out[name + "/sg_resp"] = resp
        out[name + "/sg_u8"] = u8[:DESC_ROWS]
        # OpenCV SIFT (the reference's CPU extractor, features.sift_cpu) with the same parameters
        sift = cv2.SIFT_create(nfeatures=max_kp, nOctaveLayers=3, contrastThreshold=CONTRAST,
                               edgeThreshold=EDGE, sigma=1.6)
        ck, cd = sift.detectAndCompute(img, None)
        out[name + "/cv_xy"] = np.array([k.pt for k in ck], np.float32).reshape(-1, 2)
        out[name + "/cv_angle"] = np.array([k.angle for k in ck], np.float32)
        print(name, "keypoints", len(kps["x"]), "worker", len(xy), "opencv", len(ck),
              "%.1f s" % (time.time() - t0), flush=True)
    np.savez_compressed(os.path.join(HERE, "headline.npz"), **out)
    print("headline.npz", os.path.getsize(os.path.join(HERE, "headline.npz")))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_headline.py <path to the reference's app directory>")
    main(sys.argv[1])
