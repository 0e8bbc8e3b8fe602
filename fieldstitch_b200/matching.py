"""Drop-in for PlaneSite's descriptor matching (app/planesite/matching.py:86-152) on the B200.

* ``_ratio_match_bf(da, db, ratio, na=None, nb=None, precision="fp32")`` - exhaustive ratio test
  (matching.py:86-100) + ``_unique``. ``precision`` picks the distance engine; every engine
  returns the same pairs.
* ``_guided(A, B, Hm, radius, kc, ratio)`` - prior-guided matching (matching.py:113-152).
  ``guided_from_pred`` takes predicted positions directly (the ground-plane prior of
  matching.py:155-172, or any other prior); ``kc=None`` takes every B keypoint within radius.
* ``_unique(q, t, dd)`` - one-to-one filter on the target (matching.py:103-110).
* ``match_pair((i, j))`` with ``init_worker`` / ``set_context`` / ``_get`` / ``load_features`` -
  the pair worker (matching.py:17-64, 155-253): coarse exhaustive match, ground-plane prior
  (``predict_ground``), RANSAC homography, guided match and fundamental verification; keypoint
  undistortion (``undistort_pixels``, camera.py:5-31) and the prior run on the device.

Descriptors are the feature file's uint8 RootSIFT vectors (uint8 arrays, or float arrays holding
uint8 values as the reference does). ``na``/``nb`` must be the squared norms when given (the
reference callers pass exactly those); the device recomputes them.
"""
import ctypes
import math
import os
import pickle
from collections import OrderedDict

import cv2
import numpy as np

from . import _lib


def _out(n):
    return np.empty(max(n, 1), np.int64), np.empty(max(n, 1), np.int64)


def _ratio_match_bf(da, db, ratio, na=None, nb=None, precision="fp32", device=0):
    if len(da) < 2 or len(db) < 2:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    a = _lib.as_u8_desc(da, "da")
    b = _lib.as_u8_desc(db, "db")
    ctx = _lib.context(device)
    q, t = _out(len(a))
    n = ctypes.c_int32()
    _lib.check(ctx.lib.fsb_match_bf(ctx.handle, _lib.ptr(a), len(a), _lib.ptr(b), len(b), float(ratio),
                                    _lib.PREC[precision], _lib.ptr(q), _lib.ptr(t), ctypes.byref(n)), "fsb_match_bf")
    return q[:n.value].copy(), t[:n.value].copy()


def ratio_match_bf_batch_d(a_list, b_list, ratio, precision="bf16", device=0, out=None):
    """Many independent ``_ratio_match_bf`` problems in one call on device-resident descriptors.

    ``a_list[p]``, ``b_list[p]`` are CUDA tensors (uint8, n x 128, contiguous) on ``device``.
    Returns a list of (q, t) int64 CUDA tensors, ordered by target like ``_ratio_match_bf``
    (views into ``out[p]`` when given: pairs of int64 CUDA tensors with at least len(a_list[p])
    elements each, reused across calls). With ``precision`` "bf16" or "fp8" every pair goes
    through one persistent tensor-core launch.
    """
    import torch
    if len(a_list) != len(b_list):
        raise ValueError("a_list and b_list differ in length")
    n = len(a_list)
    for x in list(a_list) + list(b_list):
        if x.dtype != torch.uint8 or x.dim() != 2 or x.shape[1] != 128 or not x.is_contiguous() or not x.is_cuda:
            raise ValueError("descriptors must be contiguous CUDA uint8 tensors of shape (n, 128)")
    ctx = _lib.context(device)
    if out is None:
        outs = [(torch.empty(max(len(a), 1), dtype=torch.int64, device=a.device),
                 torch.empty(max(len(a), 1), dtype=torch.int64, device=a.device)) for a in a_list]
    else:
        outs = list(out)
        if len(outs) != n or any(len(q) < len(a) or len(t) < len(a) or q.dtype != torch.int64 or t.dtype != torch.int64
                                 for (q, t), a in zip(outs, a_list)):
            raise ValueError("out must hold one (q, t) pair of int64 tensors of length >= na per pair")
    P = ctypes.c_void_p * max(n, 1)
    I = ctypes.c_int32 * max(n, 1)
    pa = P(*[a.data_ptr() for a in a_list])
    pb = P(*[b.data_ptr() for b in b_list])
    na = I(*[len(a) for a in a_list])
    nb = I(*[len(b) for b in b_list])
    pq = P(*[o[0].data_ptr() for o in outs])
    pt = P(*[o[1].data_ptr() for o in outs])
    cnt = I()
    torch.cuda.current_stream(device).synchronize()
    _lib.check(ctx.lib.fsb_match_bf_batch_d(ctx.handle, n, pa, na, pb, nb, float(ratio), _lib.PREC[precision],
                                            pq, pt, cnt), "fsb_match_bf_batch_d")
    return [(o[0][:cnt[i]], o[1][:cnt[i]]) for i, o in enumerate(outs)]


def guided_from_pred_batch_d(problems, radius, kc, ratio, device=0, out=None):
    """Many ``guided_from_pred`` problems in one call on device-resident data, as one CUDA graph.

    ``problems[p]`` = (pred float64 (na,2), a uint8 (na,128), b_xy float64 (nb,2), b uint8 (nb,128),
    (w_b, h_b)), CUDA tensors on ``device``. ``out[p]`` (optional, reused across calls): a pair of
    int64 CUDA tensors of length >= na. Returns [(q, t)] per pair, ordered by target.
    """
    import torch
    n = len(problems)
    for pred, a, bxy, b, _ in problems:
        for x, dt, w in ((pred, torch.float64, 2), (a, torch.uint8, 128), (bxy, torch.float64, 2),
                         (b, torch.uint8, 128)):
            if x.dtype != dt or x.dim() != 2 or x.shape[1] != w or not x.is_contiguous() or not x.is_cuda:
                raise ValueError("expected contiguous CUDA tensors: pred/b_xy float64 (n,2), a/b uint8 (n,128)")
        if len(pred) != len(a) or len(bxy) != len(b):
            raise ValueError("positions and descriptors differ in length")
    ctx = _lib.context(device)
    if out is None:
        out = [(torch.empty(max(len(pr), 1), dtype=torch.int64, device=pr.device),
                torch.empty(max(len(pr), 1), dtype=torch.int64, device=pr.device)) for pr, _, _, _, _ in problems]
    P = ctypes.c_void_p * max(n, 1)
    I = ctypes.c_int32 * max(n, 1)
    D = ctypes.c_double * max(n, 1)
    k = 0 if kc is None else int(kc)
    cnt = I()
    torch.cuda.current_stream(device).synchronize()
    _lib.check(ctx.lib.fsb_match_guided_batch_d(
        ctx.handle, n, P(*[x[0].data_ptr() for x in problems]), P(*[x[1].data_ptr() for x in problems]),
        I(*[len(x[1]) for x in problems]), P(*[x[2].data_ptr() for x in problems]),
        P(*[x[3].data_ptr() for x in problems]), I(*[len(x[3]) for x in problems]),
        D(*[float(x[4][0]) for x in problems]), D(*[float(x[4][1]) for x in problems]), float(radius), k,
        float(ratio), P(*[o[0].data_ptr() for o in out]), P(*[o[1].data_ptr() for o in out]), cnt),
        "fsb_match_guided_batch_d")
    return [(o[0][:cnt[i]], o[1][:cnt[i]]) for i, o in enumerate(out)]


_STAGE = {}


def match_guided_batch(problems, radius, kc=None, ratio=0.85, device=0):
    """Batched guided matching on host arrays: ``problems[p]`` = (pred (na,2), a_desc (na,128),
    b_xy (nb,2), b_desc (nb,128), (w_b, h_b)) as ``guided_from_pred`` takes them (descriptors uint8
    or their float32 values). The data go to the device in one copy per kind into buffers kept
    between calls with the same sizes (so a repeated batch replays its graph), every pair runs in
    one ``guided_from_pred_batch_d`` call and the results come back in one copy; returns [(q, t)]
    int64 numpy arrays per pair, each equal to ``guided_from_pred`` on that pair."""
    import torch
    if kc is not None and int(kc) < 1:
        raise ValueError("kc must be >= 1 or None")
    dev = torch.device("cuda", device)
    n = len(problems)
    if n == 0:
        return []
    preds, As, bxys, Bs, whs = [], [], [], [], []
    for pred, a_desc, b_xy, b_desc, wh in problems:
        As.append(np.ascontiguousarray(_lib.as_u8_desc(a_desc, "A desc")))
        Bs.append(np.ascontiguousarray(_lib.as_u8_desc(b_desc, "B desc")))
        preds.append(np.asarray(pred, np.float64).reshape(-1, 2))
        bxys.append(np.asarray(b_xy, np.float64).reshape(-1, 2))
        whs.append((float(wh[0]), float(wh[1])))
        if len(preds[-1]) != len(As[-1]) or len(bxys[-1]) != len(Bs[-1]):
            raise ValueError("positions and descriptors differ in length")
    na = [len(a) for a in As]
    nb = [len(b) for b in Bs]
    key = (device, tuple(na), tuple(nb))
    if key not in _STAGE:
        _STAGE.clear()
        A, Bn = max(sum(na), 1), max(sum(nb), 1)
        _STAGE[key] = {"pred": torch.empty((A, 2), dtype=torch.float64, device=dev),
                       "a": torch.empty((A, 128), dtype=torch.uint8, device=dev),
                       "bxy": torch.empty((Bn, 2), dtype=torch.float64, device=dev),
                       "b": torch.empty((Bn, 128), dtype=torch.uint8, device=dev),
                       "q": torch.empty(A + n, dtype=torch.int64, device=dev),
                       "t": torch.empty(A + n, dtype=torch.int64, device=dev)}
    st = _STAGE[key]
    oa = np.r_[0, np.cumsum(na)].astype(np.int64)
    ob = np.r_[0, np.cumsum(nb)].astype(np.int64)
    st["pred"][:oa[-1]].copy_(torch.from_numpy(np.concatenate(preds) if oa[-1] else np.zeros((0, 2))))
    st["a"][:oa[-1]].copy_(torch.from_numpy(np.concatenate(As) if oa[-1] else np.zeros((0, 128), np.uint8)))
    st["bxy"][:ob[-1]].copy_(torch.from_numpy(np.concatenate(bxys) if ob[-1] else np.zeros((0, 2))))
    st["b"][:ob[-1]].copy_(torch.from_numpy(np.concatenate(Bs) if ob[-1] else np.zeros((0, 128), np.uint8)))
    staged, out = [], []
    for p in range(n):
        staged.append((st["pred"][oa[p]:oa[p + 1]], st["a"][oa[p]:oa[p + 1]], st["bxy"][ob[p]:ob[p + 1]],
                       st["b"][ob[p]:ob[p + 1]], whs[p]))
        # output slots: na[p] + 1 entries per pair (at least one, so that every pointer is distinct)
        out.append((st["q"][oa[p] + p:oa[p + 1] + p + 1], st["t"][oa[p] + p:oa[p + 1] + p + 1]))
    res = guided_from_pred_batch_d(staged, radius, kc, ratio, device=device, out=out)
    lens = [len(q) for q, _ in res]
    if sum(lens) == 0:
        e = np.zeros(0, np.int64)
        return [(e, e) for _ in range(n)]
    qa = torch.cat([q for q, _ in res]).cpu().numpy()
    ta = torch.cat([t for _, t in res]).cpu().numpy()
    cut = np.cumsum(lens)[:-1]
    return list(zip(np.split(qa, cut), np.split(ta, cut)))


def tc_stats(device=0):
    """Statistics of the last tensor-core dense match on this thread's context for ``device``:
    rows, rows recomputed exactly (certificate not settled), largest / mean absolute error of the
    approximate best squared distance against the exact one."""
    ctx = _lib.context(device)
    r, f = ctypes.c_int64(), ctypes.c_int64()
    mx, mean = ctypes.c_double(), ctypes.c_double()
    _lib.check(ctx.lib.fsb_match_tc_stats(ctx.handle, ctypes.byref(r), ctypes.byref(f), ctypes.byref(mx),
                                          ctypes.byref(mean)), "fsb_match_tc_stats")
    return {"rows": r.value, "fallback_rows": f.value, "max_abs_err": mx.value, "mean_abs_err": mean.value}


def perspective(xy, Hm, device=0):
    """cv2.perspectiveTransform of (n,2) float64 points on the device (matching.py:115)."""
    xy = np.ascontiguousarray(np.asarray(xy, np.float64).reshape(-1, 2))
    h = np.ascontiguousarray(np.asarray(Hm, np.float64).reshape(9))
    out = np.empty_like(xy)
    if len(xy):
        ctx = _lib.context(device)
        _lib.check(ctx.lib.fsb_perspective(ctx.handle, _lib.ptr(xy), len(xy), _lib.ptr(h), _lib.ptr(out)),
                   "fsb_perspective")
    return out


def guided_from_pred(pred, a_desc, b_xy, b_desc, wh_b, radius, kc, ratio, device=0):
    """Guided matching given predicted positions of A's keypoints in B's frame."""
    a = _lib.as_u8_desc(a_desc, "A desc")
    b = _lib.as_u8_desc(b_desc, "B desc")
    pred = np.ascontiguousarray(np.asarray(pred, np.float64).reshape(-1, 2))
    bxy = np.ascontiguousarray(np.asarray(b_xy, np.float64).reshape(-1, 2))
    if len(pred) != len(a) or len(bxy) != len(b):
        raise ValueError("positions and descriptors differ in length")
    if len(a) == 0 or len(b) == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    ctx = _lib.context(device)
    q, t = _out(len(a))
    n = ctypes.c_int32()
    k = 0 if kc is None else int(min(kc, len(b)))
    if kc is not None and k < 1:
        raise ValueError("kc must be >= 1 or None")
    wb, hb = wh_b
    _lib.check(ctx.lib.fsb_match_guided(ctx.handle, _lib.ptr(pred), _lib.ptr(a), len(a), _lib.ptr(bxy), _lib.ptr(b),
                                        len(b), float(wb), float(hb), float(radius), k, float(ratio), _lib.ptr(q),
                                        _lib.ptr(t), ctypes.byref(n)), "fsb_match_guided")
    return q[:n.value].copy(), t[:n.value].copy()


def _guided(A, B, Hm, radius, kc, ratio, device=0):
    """matching._guided (app/planesite/matching.py:113-152) on feature dicts with keys und (n,2),
    desc (n,128) and wh (W, H)."""
    pred = perspective(A["und"], Hm, device)
    return guided_from_pred(pred, A["desc"], B["und"], B["desc"], B["wh"], radius, kc, ratio, device)


def _unique(q, t, dd, device=0):
    """matching._unique (app/planesite/matching.py:103-110): per target t keep the entry with the
    smallest dd (ties: earlier position); output ordered by t."""
    q = np.ascontiguousarray(np.asarray(q, np.int64))
    t = np.ascontiguousarray(np.asarray(t, np.int64))
    dd = np.ascontiguousarray(np.asarray(dd, np.float32))
    if len(q) == 0:
        return q, t
    if not (len(q) == len(t) == len(dd)):
        raise ValueError("q, t and dd differ in length")
    ctx = _lib.context(device)
    qo, to = _out(len(q))
    n = ctypes.c_int32()
    _lib.check(ctx.lib.fsb_unique(ctx.handle, _lib.ptr(q), _lib.ptr(t), _lib.ptr(dd), len(q), _lib.ptr(qo),
                                  _lib.ptr(to), ctypes.byref(n)), "fsb_unique")
    return qo[:n.value].copy(), to[:n.value].copy()


# ------------------------------------------------------------------ camera geometry (device)
def undistort_pixels(uv, k, device=0):
    """camera.undistort_pixels (app/planesite/camera.py:5-31) on the device: distorted pixels
    (n,2) -> ideal pinhole pixels with the same f, cx, cy; k = (f, cx, cy, k1, k2, p1, p2, k3).
    float64, 25 fixed-point iterations in the reference's operation order."""
    uv = np.ascontiguousarray(np.asarray(uv, np.float64).reshape(-1, 2))
    k8 = np.ascontiguousarray(np.asarray(k, np.float64).reshape(8))
    out = np.empty_like(uv)
    if len(uv):
        ctx = _lib.context(device)
        _lib.check(ctx.lib.fsb_undistort_pixels(ctx.handle, _lib.ptr(uv), len(uv), _lib.ptr(k8), _lib.ptr(out)),
                   "fsb_undistort_pixels")
    return out


def predict_ground(u, K_i, R_i, C_i, K_j, R_j, C_j, zg, device=0):
    """The ground-plane prior of matching._predict (app/planesite/matching.py:155-172) on the
    device: where undistorted pixels u (n,2) of image i land in image j when their rays meet the
    plane z = zg. Returns (pred (n,2) float64, ok (n,) bool)."""
    u = np.ascontiguousarray(np.asarray(u, np.float64).reshape(-1, 2))
    mats = [np.ascontiguousarray(np.asarray(m, np.float64).reshape(-1))
            for m in (np.linalg.inv(np.asarray(K_i, np.float64)), R_i, C_i, K_j, R_j, C_j)]
    pred = np.empty_like(u)
    ok = np.zeros(len(u), np.uint8)
    if len(u):
        ctx = _lib.context(device)
        _lib.check(ctx.lib.fsb_predict_ground(ctx.handle, _lib.ptr(u), len(u), *[_lib.ptr(m) for m in mats],
                                              float(zg), _lib.ptr(pred), _lib.ptr(ok)), "fsb_predict_ground")
    return pred, ok.astype(bool)


# ------------------------------------------------------------------ geometric verification
def find_homography_batch(problems, thr, iters=1024, seed=0, device=0):
    """RANSAC homographies of many pairs in one launch (cv2.findHomography(src, dst, cv2.RANSAC,
    thr) as matching.match_pair calls it, app/planesite/matching.py:226). problems: list of (src
    (n,2), dst (n,2)). Returns a list of (H (3,3) float64 or None, mask (n,1) uint8) per pair, in the
    shape OpenCV returns; None where a pair has fewer than 4 correspondences or no usable sample."""
    src = [np.asarray(s, np.float64).reshape(-1, 2) for s, _ in problems]
    dst = [np.asarray(d, np.float64).reshape(-1, 2) for _, d in problems]
    if any(len(a) != len(b) for a, b in zip(src, dst)):
        raise ValueError("src and dst differ in length")
    off = np.ascontiguousarray(np.r_[0, np.cumsum([len(a) for a in src])].astype(np.int64))
    S = np.ascontiguousarray(np.concatenate(src) if src else np.zeros((0, 2)))
    D = np.ascontiguousarray(np.concatenate(dst) if dst else np.zeros((0, 2)))
    P = len(problems)
    H = np.zeros((max(P, 1), 9))
    mask = np.zeros(max(len(S), 1), np.uint8)
    n_in = np.zeros(max(P, 1), np.int32)
    if P:
        ctx = _lib.context(device)
        _lib.check(ctx.lib.fsb_find_homography_batch(ctx.handle, P, _lib.ptr(off), _lib.ptr(S), _lib.ptr(D),
                                                     float(thr), int(iters), int(seed) & (2 ** 64 - 1), _lib.ptr(H),
                                                     _lib.ptr(mask), _lib.ptr(n_in)), "fsb_find_homography_batch")
    out = []
    for p in range(P):
        m = mask[off[p]:off[p + 1]].reshape(-1, 1).copy()
        out.append((None if not H[p].any() else H[p].reshape(3, 3).copy(), m))
    return out


def find_fundamental_batch(problems, thr, iters=2048, seed=0, device=0):
    """Fundamental matrices of many pairs in one launch (matching._verify's
    cv2.findFundamentalMat(pi, pj, USAC_MAGSAC, thr, 0.999, 10000), app/planesite/matching.py:175-191,
    batched): seven-point samples, inliers by Sampson distance <= thr (OpenCV's MAGSAC mask rule), eight-point
    least-squares refinement. problems: list of (pi (n,2), pj (n,2)). Returns a list of (F (3,3)
    float64 or None, mask (n,1) uint8) per pair, as OpenCV returns them; None where a pair has fewer
    than 8 correspondences or no candidate with 8 inliers."""
    src = [np.asarray(s, np.float64).reshape(-1, 2) for s, _ in problems]
    dst = [np.asarray(d, np.float64).reshape(-1, 2) for _, d in problems]
    if any(len(a) != len(b) for a, b in zip(src, dst)):
        raise ValueError("src and dst differ in length")
    off = np.ascontiguousarray(np.r_[0, np.cumsum([len(a) for a in src])].astype(np.int64))
    S = np.ascontiguousarray(np.concatenate(src) if src else np.zeros((0, 2)))
    D = np.ascontiguousarray(np.concatenate(dst) if dst else np.zeros((0, 2)))
    P = len(problems)
    F = np.zeros((max(P, 1), 9))
    mask = np.zeros(max(len(S), 1), np.uint8)
    n_in = np.zeros(max(P, 1), np.int32)
    if P:
        ctx = _lib.context(device)
        _lib.check(ctx.lib.fsb_find_fundamental_batch(ctx.handle, P, _lib.ptr(off), _lib.ptr(S), _lib.ptr(D),
                                                      float(thr), int(iters), int(seed) & (2 ** 64 - 1), _lib.ptr(F),
                                                      _lib.ptr(mask), _lib.ptr(n_in)), "fsb_find_fundamental_batch")
    out = []
    for p in range(P):
        m = mask[off[p]:off[p + 1]].reshape(-1, 1).copy()
        out.append((None if not F[p].any() else F[p].reshape(3, 3).copy(), m))
    return out


def find_fundamental(pi, pj, thr, iters=2048, seed=0, device=0):
    """One pair of find_fundamental_batch: (F or None, mask)."""
    return find_fundamental_batch([(pi, pj)], thr, iters, seed, device)[0]


def find_homography(src, dst, thr, iters=1024, seed=0, device=0):
    """One pair of find_homography_batch: (H or None, mask)."""
    return find_homography_batch([(src, dst)], thr, iters, seed, device)[0]


# ------------------------------------------------------------------ feature files
def load_features(feat_dir, i, W, H):
    """matching.load_features (app/planesite/matching.py:29-35): keypoints of feature file i in
    full-resolution pixels (float64) and its uint8 RootSIFT descriptors."""
    with np.load(os.path.join(feat_dir, "%d.npz" % i)) as d:
        xy = d["xy"].astype(np.float64)
        desc = d["desc"]
        if len(xy):
            rw, rh = d["red_wh"]
            xy = (xy + 0.5) * np.array([W / float(rw), H / float(rh)]) - 0.5
    return xy, desc


def load_xy(feat_dir, i, W, H):
    """matching.load_xy (app/planesite/matching.py:38-45): keypoint coordinates only."""
    return load_features(feat_dir, i, W, H)[0]


# ------------------------------------------------------------------ pair matching (worker side)
# The worker context is the reference's pickled dict (feat_dir, W, H, K, dist, R, C, zg,
# has_rot, prior_tol, guided_radius, min_inliers, ransac_thr and the optional n_coarse,
# guided, guided_k, ratio, use_prior); init_worker / set_context install it per process.
_CTX = None
_CACHE = OrderedDict()
_CACHE_MAX = 48


def init_worker(ctx_file):
    """matching.init_worker (app/planesite/matching.py:17-26): load the pickled worker context."""
    with open(ctx_file, "rb") as f:
        set_context(pickle.load(f))
    try:
        cv2.setNumThreads(1)
    except Exception:
        pass


def set_context(ctx):
    global _CTX
    _CTX = ctx
    _CACHE.clear()


def _get(i, device=0):
    """matching._get (app/planesite/matching.py:48-64): feature file i with undistorted keypoints
    (on the device), uint8 descriptors and their squared norms, cached (least recently used)."""
    if i in _CACHE:
        _CACHE.move_to_end(i)
        return _CACHE[i]
    c = _CTX
    xy, desc = load_features(c["feat_dir"], i, c["W"][i], c["H"][i])
    und = xy
    if len(xy):
        K, dd = c["K"][i], c["dist"][i]
        und = undistort_pixels(xy, (K[0, 0], K[0, 2], K[1, 2], dd[0], dd[1], dd[2], dd[3], dd[4]), device)
    d = np.ascontiguousarray(desc, np.uint8)
    df = d.astype(np.float32)
    item = {"xy": xy, "und": und, "desc": d, "norm": (df * df).sum(1), "wh": (c["W"][i], c["H"][i])}
    _CACHE[i] = item
    while len(_CACHE) > _CACHE_MAX:
        _CACHE.popitem(last=False)
    return item


def _predict(u, i, j, device=0):
    """matching._predict (app/planesite/matching.py:155-172) with the worker context's cameras."""
    c = _CTX
    return predict_ground(u, c["K"][i], c["R"][i], c["C"][i], c["K"][j], c["R"][j], c["C"][j], c["zg"][i], device)


def _prior_filter(q, t, ui, uj, i, j, tol, device=0):
    """Keeps the pairs whose prior prediction of ui[q] lands within tol of uj[t]."""
    pred, ok = _predict(ui[q], i, j, device)
    keep = ok & (np.linalg.norm(pred - uj[t], axis=1) < tol)
    return q[keep], t[keep]


def _verify(c, i, j, ui, uj, q, t, device=0):
    """matching._verify (app/planesite/matching.py:175-191): fundamental-matrix inliers (OpenCV
    USAC_MAGSAC, plain RANSAC where MAGSAC rejects a degenerate set); with the context's
    ransac="device", the device's batched fundamental RANSAC (statistically equal, not identical)."""
    pi, pj = ui[q].astype(np.float32), uj[t].astype(np.float32)
    F = mask = None
    if c.get("ransac", "opencv") == "device":
        F, mask = find_fundamental(pi.astype(np.float64), pj.astype(np.float64), c["ransac_thr"], device=device)
        if F is None or mask is None:
            return None, None, 0
        inl = mask.ravel().astype(bool)
        return q[inl], t[inl], int(inl.sum())
    for method in (getattr(cv2, "USAC_MAGSAC", cv2.FM_RANSAC), cv2.FM_RANSAC):
        try:
            F, mask = cv2.findFundamentalMat(pi, pj, method, c["ransac_thr"], 0.999, 10000)
            break
        except cv2.error:
            continue
    if F is None or mask is None:
        return None, None, 0
    inl = mask.ravel().astype(bool)
    return q[inl], t[inl], int(inl.sum())


def _similarity(c, i, ui, uj, q, t):
    """matching._similarity (app/planesite/matching.py:194-202): (rotation, scale, tx, ty) of the
    inliers' partial affine fit, or None."""
    try:
        M, _ = cv2.estimateAffinePartial2D(ui[q].astype(np.float32), uj[t].astype(np.float32), method=cv2.RANSAC,
                                           ransacReprojThreshold=0.02 * max(c["W"][i], c["H"][i]))
    except Exception:
        return None
    if M is None:
        return None
    return (math.atan2(M[1, 0], M[0, 0]), math.hypot(M[0, 0], M[1, 0]), float(M[0, 2]), float(M[1, 2]))


def _ratio_match(da, db, ratio, checks=None, device=0):
    """The reference's exhaustive fallback (matching.py:74-83, a FLANN kd-forest ratio test) as the
    exact device ratio test: the same ratio rule on the true nearest neighbours."""
    return _ratio_match_bf(da, db, ratio, device=device)


def _coarse_guided(c, i, j, A, B, use_prior, tol, device):
    """Stage 1 of matching.match_pair (app/planesite/matching.py:217-233): the strongest n_coarse
    features of each image, prior-filtered, give a RANSAC homography; guided matching around it
    and fundamental verification. Returns (q, t, n_in) or None."""
    ui, uj = A["und"], B["und"]
    n1 = c.get("n_coarse", 1500)
    if not (c.get("guided", True) and len(ui) > n1 // 2):
        return None
    q1, t1 = _ratio_match_bf(A["desc"][:n1], B["desc"][:n1], 0.85, device=device)
    if use_prior and len(q1):
        q1, t1 = _prior_filter(q1, t1, ui, uj, i, j, tol, device)
    if len(q1) < 12:
        return None
    thr = 0.012 * max(c["W"][i], c["H"][i])
    if c.get("ransac", "opencv") == "device":   # the device RANSAC (statistically equal, not identical)
        Hm, hm = find_homography(ui[q1], uj[t1], thr, device=device)
    else:
        Hm, hm = cv2.findHomography(ui[q1], uj[t1], cv2.RANSAC, thr)
    if Hm is None or hm is None or hm.sum() < 10:
        return None
    radius = c["guided_radius"] * max(c["W"][j], c["H"][j])
    q, t = _guided(A, B, Hm, radius, c.get("guided_k", 24), 0.85, device)
    if len(q) < c["min_inliers"]:
        return None
    q, t, n_in = _verify(c, i, j, ui, uj, q, t, device)
    if q is None or n_in < max(c["min_inliers"], 40):
        return None
    return q, t, n_in


def match_pair(task, device=0):
    """matching.match_pair (app/planesite/matching.py:205-253) for task (i, j): returns
    (i, j, q int32, t int32, similarity, n_inliers), or (i, j, None, None, None or an error tuple,
    n) as the reference does. Descriptor matching (coarse exhaustive, guided, fallback) and the
    camera geometry run on the device; RANSAC and the fundamental / similarity fits are OpenCV's,
    as in the reference, unless the context sets ransac="device" (the stage-1 homography and the
    fundamental verification then run on the device)."""
    i, j = task
    c = _CTX
    try:
        A, B = _get(i, device), _get(j, device)
        ui, uj = A["und"], B["und"]
        if len(ui) < 30 or len(uj) < 30:
            return i, j, None, None, None, 0
        use_prior = c["has_rot"][i] and c["has_rot"][j] and c.get("use_prior", True)
        tol = c["prior_tol"] * max(c["W"][j], c["H"][j])
        result = _coarse_guided(c, i, j, A, B, use_prior, tol, device)
        if result is None:
            # exhaustive fallback (matching.py:234-246)
            q, t = _ratio_match(A["desc"], B["desc"], c.get("ratio", 0.8), c.get("checks", 48), device)
            if use_prior and len(q):
                q, t = _prior_filter(q, t, ui, uj, i, j, tol, device)
            if len(q) < 20:
                return i, j, None, None, None, 0
            q, t, n_in = _verify(c, i, j, ui, uj, q, t, device)
            if q is None or n_in < c["min_inliers"]:
                return i, j, None, None, None, n_in
            result = (q, t, n_in)
        q, t, n_in = result
        return i, j, q.astype(np.int32), t.astype(np.int32), _similarity(c, i, ui, uj, q, t), n_in
    except Exception as e:  # the reference reports a worker error in the similarity slot
        import traceback
        tb = traceback.extract_tb(e.__traceback__)[-1]
        return i, j, None, None, ("error", "%s: %s (%s line %d)" % (type(e).__name__, e, os.path.basename(tb.filename),
                                                                    tb.lineno)), 0
