"""CPU oracle: descriptor matching of PlaneSite (app/planesite/matching.py).

TEST INFRASTRUCTURE ONLY (imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg; never by the fieldstitch_b200 package).

Descriptors are RootSIFT uint8 vectors held as float32 (matching.py:59), so every squared
distance na + nb - 2 a.b is an integer below 2^24 and float32 BLAS computes it exactly; the
results below are therefore determined by the values alone (ties on the best distance always fail
the ratio test because ratio < 1).
"""
import numpy as np


def unique(q, t, dd):
    """One-to-one on the target: for each t keep the entry with the smallest dd, ties to the
    earlier position; output ordered by t (matching.py:103-110)."""
    if len(q) == 0:
        return q, t
    order = np.lexsort((dd, t))
    ts = t[order]
    first = np.r_[True, ts[1:] != ts[:-1]]
    keep = order[first]
    return q[keep], t[keep]


def ratio_match_bf(da, db, ratio, na=None, nb=None):
    """Exhaustive nearest / second-nearest ratio test with one float32 GEMM
    (matching.py:86-100). Returns (q, t) int64."""
    if len(da) < 2 or len(db) < 2:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    da = np.asarray(da, np.float32)
    db = np.asarray(db, np.float32)
    na = (da * da).sum(1) if na is None else na
    nb = (db * db).sum(1) if nb is None else nb
    d2 = na[:, None] + nb[None, :] - 2.0 * (da @ db.T)
    two = np.argpartition(d2, 1, axis=1)[:, :2]
    r = np.arange(len(da))
    a0, a1 = d2[r, two[:, 0]], d2[r, two[:, 1]]
    first = np.where(a0 <= a1, two[:, 0], two[:, 1])
    b1 = np.maximum(np.minimum(a0, a1), 0)
    b2 = np.maximum(np.maximum(a0, a1), 0)
    ok = np.sqrt(b1) < ratio * np.sqrt(b2)
    return unique(r[ok].astype(np.int64), first[ok].astype(np.int64), b1[ok].astype(np.float32))


def perspective(xy, Hm):
    """Project (n,2) float64 points through a 3x3 homography (the cv2.perspectiveTransform call of
    matching.py:115)."""
    import cv2
    return cv2.perspectiveTransform(np.asarray(xy, np.float64).reshape(-1, 1, 2), np.asarray(Hm, np.float64)).reshape(-1, 2)


def guided_from_pred(pred, a_desc, b_und, b_desc, wh_b, radius, kc, ratio, a_norm=None, b_norm=None,
                     ties="tree"):
    """Guided matching given predicted positions of A's keypoints in B (matching.py:116-152):
    keep predictions inside B +- radius; candidates = the kc nearest B keypoints strictly within
    radius (cKDTree); float32 distances; top-2 ratio test; one-to-one filter.
    ``kc=None`` takes every B keypoint within radius. ``ties``: "tree" keeps cKDTree's own order
    among B keypoints at equal distance (the reference's call); "index" keeps the smaller index
    (SIFT lists several orientations of one position, so equal distances at the kc-th candidate
    are common on real keypoints; cKDTree's order among them is implementation-defined)."""
    from scipy.spatial import cKDTree
    a_desc = np.asarray(a_desc, np.float32)
    b_desc = np.asarray(b_desc, np.float32)
    a_norm = (a_desc * a_desc).sum(1) if a_norm is None else a_norm
    b_norm = (b_desc * b_desc).sum(1) if b_norm is None else b_norm
    nb = len(b_und)
    Wb, Hb = wh_b
    inside = np.nonzero((pred[:, 0] > -radius) & (pred[:, 0] < Wb + radius)
                        & (pred[:, 1] > -radius) & (pred[:, 1] < Hb + radius))[0]
    if len(inside) == 0 or nb == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    tree = cKDTree(b_und)
    k = nb if kc is None else min(kc, nb)
    if ties == "index" and kc is not None and k < nb:
        kq = min(nb, k + 32)
        dist, idx = tree.query(pred[inside], k=kq, distance_upper_bound=radius)
        if kq == 1:
            dist, idx = dist[:, None], idx[:, None]
        order = np.lexsort((np.where(idx < nb, idx, nb), dist))[:, :k]
        idx = np.take_along_axis(idx, order, axis=1)
    else:
        dist, idx = tree.query(pred[inside], k=k, distance_upper_bound=radius)
    if idx.ndim == 1:
        idx = idx[:, None]
    valid = idx < nb
    has = valid.any(1)
    inside, idx, valid = inside[has], idx[has], valid[has]
    if len(inside) == 0:
        # the reference reaches np.concatenate([]) here and raises ValueError (caught by
        # match_pair's handler); the drop-in returns no matches instead
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    idx = np.where(valid, idx, 0)
    qs, ts, ds = [], [], []
    # the reference uses 1024-query chunks; smaller chunks for large k only bound memory
    chunk = max(1, min(1024, (1 << 21) // max(k, 1)))
    for s0 in range(0, len(inside), chunk):
        sl = slice(s0, s0 + chunk)
        da = a_desc[inside[sl]]
        cand = b_desc[idx[sl]]
        d2 = a_norm[inside[sl], None] + b_norm[idx[sl]] - 2 * np.matmul(cand, da[:, :, None])[:, :, 0]
        d2 = np.where(valid[sl], np.maximum(d2, 0), np.inf)
        o = np.argpartition(d2, 1, axis=1)[:, :2] if d2.shape[1] > 2 else np.argsort(d2, axis=1)[:, :2]
        r = np.arange(d2.shape[0])
        a0 = d2[r, o[:, 0]]
        a1 = d2[r, o[:, 1]] if d2.shape[1] > 1 else np.full(len(r), np.inf)
        best = np.where(a0 <= a1, o[:, 0], o[:, 1]) if d2.shape[1] > 1 else o[:, 0]
        b1 = np.minimum(a0, a1)
        b2 = np.maximum(a0, a1)
        with np.errstate(invalid="ignore"):
            ok = np.isfinite(b1) & (np.sqrt(b1) < ratio * np.sqrt(b2))
        qs.append(inside[sl][ok])
        ts.append(idx[sl][r[ok], best[ok]])
        ds.append(b1[ok])
    return unique(np.concatenate(qs), np.concatenate(ts), np.concatenate(ds))


def guided(A, B, Hm, radius, kc, ratio):
    """``_guided(A, B, Hm, radius, kc, ratio)`` (matching.py:113-152) on feature dicts with keys
    und (n,2) float64, desc (n,128) float32, norm (n,), wh (W, H)."""
    pred = perspective(A["und"], Hm)
    return guided_from_pred(pred, A["desc"], B["und"], B["desc"], B["wh"], radius, kc, ratio,
                            A.get("norm"), B.get("norm"))


def predict(u, Ki, Ri, Ci, Kj, Rj, Cj, zg):
    """Ground-plane prior (matching.py:155-172): back-project undistorted pixels of image i to
    the plane z = zg and project them into image j. Returns (pred (n,2), ok)."""
    rays = np.c_[u, np.ones(len(u))] @ np.linalg.inv(Ki).T
    d = rays @ Ri
    dz = d[:, 2]
    dz = np.where(np.abs(dz) < 1e-6, -1e-6, dz)
    t = (zg - Ci[2]) / dz
    G = Ci[None] + t[:, None] * d
    q = (G - Cj[None]) @ Rj.T @ Kj.T
    z = q[:, 2]
    ok = (t > 0) & (z > 0)
    z = np.where(np.abs(z) < 1e-9, 1e-9, z)
    return q[:, :2] / z[:, None], ok
