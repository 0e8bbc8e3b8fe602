"""Drop-in for PlaneSite's descriptor matching (app/planesite/matching.py:86-152) on the B200.

* ``_ratio_match_bf(da, db, ratio, na=None, nb=None, precision="fp32")`` - exhaustive ratio test
  (matching.py:86-100) + ``_unique``. ``precision`` picks the distance engine; every engine
  returns the same pairs.
* ``_guided(A, B, Hm, radius, kc, ratio)`` - prior-guided matching (matching.py:113-152).
  ``guided_from_pred`` takes predicted positions directly (the ground-plane prior of
  matching.py:155-172, or any other prior); ``kc=None`` takes every B keypoint within radius.
* ``_unique(q, t, dd)`` - one-to-one filter on the target (matching.py:103-110).

Descriptors are the feature file's uint8 RootSIFT vectors (uint8 arrays, or float arrays holding
uint8 values as the reference does). ``na``/``nb`` must be the squared norms when given (the
reference callers pass exactly those); the device recomputes them.
"""
import ctypes

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
