"""Drop-in for PlaneSite's track building (app/planesite/recon.py:14-54) on the B200.

``build_tracks(pairs, nfeat, n_img)``: pairs is a list of (i, j, qi, tj) verified matches (the
pair workers' output), nfeat the number of features of every photo. Returns (tid, img, feat,
n_tracks) int64: one observation per tracked feature, listed by track then by global feature
index; a track is a connected component of at least two matched features with no two features of
the same photo, tracks numbered in the order of their smallest global feature index. The
connected components, the duplicate-photo test and the numbering run on the device.
"""
import ctypes

import numpy as np

from . import _lib


def build_tracks(pairs, nfeat, n_img, device=0):
    nfeat = np.asarray(nfeat, np.int64)
    offsets = np.ascontiguousarray(np.r_[0, np.cumsum(nfeat)].astype(np.int64))
    if len(offsets) != n_img + 1:
        raise ValueError("one feature count per photo")
    rows = [offsets[i] + np.asarray(qi, np.int64) for i, j, qi, tj in pairs]
    cols = [offsets[j] + np.asarray(tj, np.int64) for i, j, qi, tj in pairs]
    z = np.zeros(0, np.int64)
    if not rows:
        return z, z, z, 0
    u = np.ascontiguousarray(np.concatenate(rows))
    v = np.ascontiguousarray(np.concatenate(cols))
    if len(u) != len(v):
        raise ValueError("qi and tj differ in length")
    if len(u) == 0:
        return z, z, z, 0
    cap = 2 * len(u)
    tid, img, feat = np.empty(cap, np.int64), np.empty(cap, np.int64), np.empty(cap, np.int64)
    n_obs, n_tr = ctypes.c_int64(), ctypes.c_int64()
    ctx = _lib.context(device)
    _lib.check(ctx.lib.fsb_build_tracks(ctx.handle, _lib.ptr(u), _lib.ptr(v), len(u), _lib.ptr(offsets), int(n_img),
                                        _lib.ptr(tid), _lib.ptr(img), _lib.ptr(feat), ctypes.byref(n_obs),
                                        ctypes.byref(n_tr)), "fsb_build_tracks")
    n = n_obs.value
    return tid[:n].copy(), img[:n].copy(), feat[:n].copy(), int(n_tr.value)
