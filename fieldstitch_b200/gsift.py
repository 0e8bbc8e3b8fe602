"""Drop-in for PlaneSite's ``gsift.detect`` / ``gsift.describe`` (app/planesite/gsift.py:435-525)
running on the B200 through libfsb200.

Same signatures and outputs: ``detect`` returns (dict of host arrays x, y, size, angle, response
(float32), octave, layer (int32), state); ``describe(state, kps, sel)`` returns float32 (n, 128)
descriptors with L2 norm 512 (unrounded, OpenCV scaling). The state owns the device-resident
gradient atlas and is released when it is garbage-collected (or by ``state.close()``).

There is no CPU path: ``gpu=False`` raises. This is the one deliberate signature difference: the
reference's ``detect(gray, gpu=False, ...)`` defaults to its NumPy path, this module's ``gpu``
defaults to True, so a caller relying on the default gets the GPU (the reference's own GPU worker,
features.sift_gpu, passes gpu=True explicitly, features.py:119; only its start-up self-test calls
the CPU default, as the comparison side). ``exact=True`` selects float64 blur accumulation
(bit-identical pyramid to the reference's NumPy/SciPy path) and float64 descriptor sample math.
"""
import ctypes
import time

import numpy as np

from . import _lib

KEYS = ("x", "y", "size", "angle", "response", "octave", "layer")


class State:
    """Handle of a detect result (fsb_state): the device gradient atlas used by describe()."""

    def __init__(self, ctx, handle, shape, exact):
        self.ctx = ctx
        self.handle = handle
        self.shape = shape
        self.exact = exact

    def close(self):
        if self.handle:
            _lib.load().fsb_state_free(self.handle)
            self.handle = None

    def atlas(self):
        """(shapes [(R, C)], DoG list of (5,R,C), magnitude list of (3,R,C), angle list of (3,R,C))
        copied to host - the reference state's `_Atlas` content per octave."""
        lib = _lib.load()
        n = ctypes.c_int32()
        rows = np.zeros(16, np.int32)
        cols = np.zeros(16, np.int32)
        _lib.check(lib.fsb_state_geometry(self.handle, ctypes.byref(n), _lib.ptr(rows), _lib.ptr(cols)), "geometry")
        shapes = [(int(rows[o]), int(cols[o])) for o in range(n.value)]
        out = []
        for which, layers in ((0, 5), (1, 3), (2, 3)):
            tot = sum(layers * r * c for r, c in shapes)
            buf = np.empty(tot, np.float32)
            _lib.check(lib.fsb_state_atlas(self.handle, which, _lib.ptr(buf), tot), "fsb_state_atlas")
            per, at = [], 0
            for r, c in shapes:
                per.append(buf[at:at + layers * r * c].reshape(layers, r, c))
                at += layers * r * c
            out.append(per)
        return shapes, out[0], out[1], out[2]

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


def _params(contrast, edge, max_kp, exact):
    return _lib.SiftParams(float(contrast), float(edge), int(max_kp), _lib.SIFT_EXACT_BLUR if exact else 0)


def _gray(gray):
    g = np.asarray(gray)
    if g.ndim != 2:
        raise ValueError("gray must be a 2-D uint8 image, got shape %s" % (g.shape,))
    if g.dtype != np.uint8:
        raise ValueError("gray must be uint8, got %s" % g.dtype)
    if g.strides[1] != 1 or g.strides[0] < g.shape[1]:
        g = np.ascontiguousarray(g)
    return g


def detect(gray, gpu=True, max_kp=12000, contrast=0.015, edge=12.0, timings=None, exact=False, device=0):
    """Oriented SIFT keypoints, strongest first (gsift.detect, app/planesite/gsift.py:435)."""
    if not gpu:
        raise NotImplementedError("fieldstitch_b200 runs SIFT on the GPU only (no CPU fallback)")
    t0 = time.perf_counter()
    g = _gray(gray)
    ctx = _lib.context(device)
    lib = ctx.lib
    p = _params(contrast, edge, max_kp, exact)
    st = _lib.c_vp()
    n = ctypes.c_int32()
    _lib.check(lib.fsb_detect(ctx.handle, _lib.ptr(g), g.shape[0], g.shape[1], g.strides[0], ctypes.byref(p),
                              ctypes.byref(st), ctypes.byref(n)), "fsb_detect")
    state = State(ctx, st.value, g.shape, exact)
    n = n.value
    if n == 0:
        kps = {k: np.zeros(0, np.float32) for k in KEYS}
    else:
        kps = {k: np.empty(n, np.float32) for k in KEYS[:5]}
        kps["octave"] = np.empty(n, np.int32)
        kps["layer"] = np.empty(n, np.int32)
        _lib.check(lib.fsb_state_keypoints(state.handle, *[_lib.ptr(kps[k]) for k in KEYS]), "fsb_state_keypoints")
    if timings is not None:
        timings["detect"] = timings.get("detect", 0.0) + time.perf_counter() - t0
    return kps, state


def describe(state, kps, sel, budget=2.5e6, timings=None, rootsift=False):
    """128-d descriptors of kps[sel] (gsift.describe, app/planesite/gsift.py:480). ``budget`` is
    accepted for signature compatibility (the device kernel needs no chunking). With
    ``rootsift=True`` returns (desc float32, RootSIFT uint8) with the feature-file encoding."""
    t0 = time.perf_counter()
    sel = np.asarray(sel, np.int64)
    n = len(sel)
    desc = np.zeros((n, 128), np.float32)
    u8 = np.zeros((n, 128), np.uint8) if rootsift else None
    if n:
        if not isinstance(state, State) or not state.handle:
            raise ValueError("state must be the live state returned by detect()")
        cols = [np.ascontiguousarray(np.asarray(kps[k])[sel], np.float32) for k in ("x", "y", "size", "angle")]
        cols += [np.ascontiguousarray(np.asarray(kps[k])[sel], np.int32) for k in ("octave", "layer")]
        lib = state.ctx.lib
        _lib.check(lib.fsb_describe(state.ctx.handle, state.handle, n, *[_lib.ptr(c) for c in cols],
                                    _lib.ptr(desc), _lib.ptr(u8)), "fsb_describe")
    if timings is not None:
        timings["describe"] = timings.get("describe", 0.0) + time.perf_counter() - t0
    return (desc, u8) if rootsift else desc


def cv2_octave(kps):
    """OpenCV's packed keypoint octave for detect's keypoints: octave byte (o - 1) & 255 (o = 0 is
    the 2x upsampled octave), layer << 8, round((X2 + 0.5) * 255) << 16 with X2 the sub-layer offset
    of the refinement, recovered from size = 1.6 * 2^((layer + X2) / 3) * 2^o (gsift.py:462-470)."""
    o = np.asarray(kps["octave"], np.int64)
    layer = np.asarray(kps["layer"], np.int64)
    scl = np.asarray(kps["size"], np.float64) / np.exp2(o.astype(np.float64))
    x2 = 3.0 * np.log2(np.maximum(scl, 1e-30) / 1.6) - layer
    sub = np.clip(np.rint((x2 + 0.5) * 255.0), 0, 255).astype(np.int64)
    return (((o - 1) & 255) | (layer << 8) | (sub << 16)).astype(np.int64)


def to_cv2_keypoints(kps):
    """detect's keypoints as a list of cv2.KeyPoint (pt, size, angle, response, packed octave), the
    form cv2.SIFT.detect returns, for code that consumes OpenCV keypoints."""
    import cv2
    packed = cv2_octave(kps)
    return [cv2.KeyPoint(float(x), float(y), float(s), float(a), float(r), int(p))
            for x, y, s, a, r, p in zip(kps["x"], kps["y"], kps["size"], kps["angle"], kps["response"], packed)]


def detect_batch(grays, max_kp=12000, contrast=0.015, edge=12.0, exact=False, streams=4, device=0):
    """detect() of every image, spread over `streams` contexts (one CUDA stream each). Returns a
    list of (kps, state); each state belongs to the context that detected it and may be used by
    describe() once the batch has returned."""
    from .features import _batch
    return _batch(lambda g: detect(g, True, max_kp, contrast, edge, None, exact, device), list(grays), streams)
