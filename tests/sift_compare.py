"""Keypoint / descriptor comparison helpers shared by the parity tests."""
import numpy as np
from scipy.spatial import cKDTree


def angle_diff(a, b):
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)) % 360.0
    return np.minimum(d, 360.0 - d)


def pair_keypoints(ref_xy, ref_ang, got_xy, got_ang, pos_tol=0.01, ang_tol=0.1):
    """For each reference keypoint, the index of a got keypoint within pos_tol px and ang_tol
    degrees (closest angle among position candidates), or -1."""
    ref_xy = np.asarray(ref_xy, np.float64).reshape(-1, 2)
    got_xy = np.asarray(got_xy, np.float64).reshape(-1, 2)
    out = np.full(len(ref_xy), -1, np.int64)
    if len(ref_xy) == 0 or len(got_xy) == 0:
        return out
    tree = cKDTree(got_xy)
    cands = tree.query_ball_point(ref_xy, r=pos_tol + 1e-12)
    for i, c in enumerate(cands):
        if not c:
            continue
        c = np.asarray(c)
        da = angle_diff(ref_ang[i], np.asarray(got_ang)[c])
        j = int(np.argmin(da))
        if da[j] <= ang_tol:
            out[i] = c[j]
    return out


def paired_fraction(ref, got, pos_tol=0.01, ang_tol=0.1):
    """(fraction of ref keypoints paired, pairing array). ref/got: dicts with x, y, angle."""
    p = pair_keypoints(np.c_[ref["x"], ref["y"]], ref["angle"], np.c_[got["x"], got["y"]], got["angle"],
                       pos_tol, ang_tol)
    return (p >= 0).mean() if len(p) else 1.0, p
