"""CPU oracle: per-photo feature steps of PlaneSite (app/planesite/features.py).

TEST INFRASTRUCTURE ONLY (imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg; never by the fieldstitch_b200 package).

* ``spread``      - grid-spread keypoint selection (features.py:38-57).
* ``rootsift_u8`` - RootSIFT uint8 encoding of the feature file (features.py:74-86).
* ``sift_gpu_ref``- the detect -> spread -> describe sequence of ``sift_gpu`` (features.py:115-129)
                    computed with the gsift oracle.
* ``sift_cpu``    - the reference's OpenCV CPU extractor (features.py:89-104), used as the timed CPU
                    baseline and as the OpenCV parity oracle.
"""
import time

import numpy as np

from . import gsift_ref


def spread(x, y, resp, W, H, n, gx=12, gy=9, stable=True):
    """Indices of n keypoints spread over a gx*gy grid: per cell the strongest first, at most
    ceil(n/(gx*gy)) per cell, then the strongest of the rest (features.py:38-57).

    The reference sorts "the rest" with NumPy's default (unstable) argsort, so its order among
    equal responses depends on the machine's SIMD sort; ``stable=True`` fixes that tie order to
    ascending index (the CUDA path's rule); ``stable=False`` reproduces the reference call."""
    N = len(x)
    if N <= n:
        return np.arange(N, dtype=np.int64)
    resp = np.asarray(resp, np.float32)
    xs = np.asarray(x, np.float32)
    ys = np.asarray(y, np.float32)
    cx = np.clip((xs / W * gx).astype(int), 0, gx - 1)
    cy = np.clip((ys / H * gy).astype(int), 0, gy - 1)
    cell = cy * gx + cx
    order = np.lexsort((-resp, cell))
    cs = cell[order]
    rank = np.arange(N) - np.searchsorted(cs, cs, side="left")
    cap = int(np.ceil(n / (gx * gy)))
    sel = order[rank < cap]
    if len(sel) < n:
        rest = np.setdiff1d(np.arange(N), sel)
        o = np.argsort(-resp[rest], kind="stable") if stable else np.argsort(-resp[rest])
        sel = np.concatenate([sel, rest[o][: n - len(sel)]])
    return sel[:n].astype(np.int64)


def rootsift_u8(desc):
    """L1-normalise (+1e-7), square-root, x512, clip to [0,255], truncate to uint8, all in float32
    (features.py:80-82)."""
    d = np.asarray(desc, np.float32)
    d = d / (np.abs(d).sum(1, keepdims=True) + 1e-7)
    d = np.sqrt(d)
    return np.clip(d * 512.0, 0, 255).astype(np.uint8)


def sift_gpu_ref(g2, nfeat, stable=True):
    """The sift_gpu sequence with the oracle: detect(max_kp=int(2.2 nfeat)) -> spread -> stable
    sort by response -> describe. Returns (xy f32 (n,2), desc f32 (n,128) or None, resp f32)."""
    h, w = g2.shape[:2]
    kps, st = gsift_ref.detect(g2, max_kp=int(nfeat * 2.2))
    n = len(kps["x"])
    if n < 10:
        return np.zeros((0, 2), np.float32), None, np.zeros(0, np.float32)
    # the reference rebuilds Python floats from the float32 arrays; values are unchanged
    sel = spread(kps["x"], kps["y"], kps["response"], w, h, nfeat, stable=stable)
    sel = sel[np.argsort(-kps["response"][sel], kind="stable")]
    desc = gsift_ref.describe(st, kps, sel)
    xy = np.c_[kps["x"][sel], kps["y"][sel]].astype(np.float32)
    return xy, desc, kps["response"][sel].astype(np.float32)


def sift_cpu(g2, nfeat, contrast=0.015, edge=12, n_kp=None):
    """OpenCV SIFT as the reference's CPU worker calls it (features.py:89-104). Returns
    (xy, desc, resp, seconds spent in compute)."""
    import cv2
    sift = cv2.SIFT_create(nfeatures=int(nfeat * 2.2) if n_kp is None else n_kp,
                           contrastThreshold=contrast, edgeThreshold=edge)
    kps = sift.detect(g2, None)
    h, w = g2.shape[:2]
    if len(kps) < 10:
        return np.zeros((0, 2), np.float32), None, np.zeros(0, np.float32), 0.0
    t = time.perf_counter()
    xs = np.array([k.pt[0] for k in kps], np.float32)
    ys = np.array([k.pt[1] for k in kps], np.float32)
    rs = np.array([k.response for k in kps], np.float32)
    sel = spread(xs, ys, rs, w, h, nfeat, stable=False)
    kps = sorted([kps[i] for i in sel], key=lambda k: -k.response)
    kps, desc = sift.compute(g2, kps)
    if desc is None:
        return np.zeros((0, 2), np.float32), None, np.zeros(0, np.float32), 0.0
    xy = np.array([k.pt for k in kps], np.float32)
    resp = np.array([k.response for k in kps], np.float32)
    return xy, desc, resp, time.perf_counter() - t
