"""Golden CLAHE fixtures: OpenCV's cv2.createCLAHE(clipLimit, tileGridSize).apply (the call of
features.prepare, app/planesite/features.py:70-71) on seeded synthetic images, including sides
that are and are not multiples of the tile count. Writes clahe.npz next to this script.

    python tests/golden/make_clahe.py
"""
import os
import sys

import cv2
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fieldstitch_b200 import synth  # noqa: E402

# (h, w, seed, clip, tiles x, tiles y)
CASES = [(120, 160, 1, 2.0, 8, 8), (117, 159, 2, 2.0, 8, 8), (120, 157, 3, 2.0, 8, 8), (97, 131, 4, 2.0, 8, 8),
         (80, 100, 5, 4.0, 4, 6), (64, 64, 6, 0.0, 8, 8)]


def main():
    out = {}
    for h, w, seed, clip, tx, ty in CASES:
        img = synth.synth_image(h, w, seed)
        name = "c%dx%d_%d" % (h, w, seed)
        out[name + "/img"] = img
        out[name + "/params"] = np.array([clip, tx, ty], np.float64)
        out[name + "/out"] = cv2.createCLAHE(clipLimit=clip, tileGridSize=(tx, ty)).apply(img)
    np.savez_compressed(os.path.join(HERE, "clahe.npz"), **out)


if __name__ == "__main__":
    main()
