"""ctypes binding of libfsb200.so (the C ABI declared in include/fsb200.h).

The library is loaded from this package directory only; if it is missing the import of any
entry point fails loudly (there is no CPU fallback).
"""
import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfsb200.so")

FSB_OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "out of device memory", 3: "CUDA error", 4: "timeout",
          5: "invalid state", 6: "unsupported", 7: "capacity overflow"}
PREC = {"fp32": 0, "bf16": 1, "fp8": 2}
SIFT_EXACT_BLUR = 1

c_i32, c_i64, c_f32, c_f64, c_vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_float, ctypes.c_double, ctypes.c_void_p


class SiftParams(ctypes.Structure):
    _fields_ = [("contrast", ctypes.c_double), ("edge", ctypes.c_double), ("max_kp", ctypes.c_int32),
                ("flags", ctypes.c_int32)]


# (name, restype, argtypes); pointers are passed as c_void_p
SIGNATURES = [
    ("fsb_version", c_i32, []),
    ("fsb_last_error", ctypes.c_char_p, []),
    ("fsb_create", c_i32, [c_i32, c_vp]),
    ("fsb_destroy", c_i32, [c_vp]),
    ("fsb_sync", c_i32, [c_vp, c_i32]),
    ("fsb_stream", c_vp, [c_vp]),
    ("fsb_device_bytes", c_i64, [c_vp]),
    ("fsb_detect", c_i32, [c_vp, c_vp, c_i32, c_i32, c_i32, c_vp, c_vp, c_vp]),
    ("fsb_state_keypoints", c_i32, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("fsb_describe", c_i32, [c_vp, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("fsb_state_free", c_i32, [c_vp]),
    ("fsb_state_geometry", c_i32, [c_vp, c_vp, c_vp, c_vp]),
    ("fsb_state_atlas", c_i32, [c_vp, c_i32, c_vp, c_i64]),
    ("fsb_sift_features", c_i32, [c_vp, c_vp, c_i32, c_i32, c_i32, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("fsb_match_bf", c_i32, [c_vp, c_vp, c_i32, c_vp, c_i32, c_f32, c_i32, c_vp, c_vp, c_vp]),
    ("fsb_match_guided", c_i32, [c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_i32, c_f64, c_f64, c_f64, c_i32, c_f32,
                                 c_vp, c_vp, c_vp]),
    ("fsb_unique", c_i32, [c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_vp]),
    ("fsb_perspective", c_i32, [c_vp, c_vp, c_i32, c_vp, c_vp]),
    ("fsb_undistort_pixels", c_i32, [c_vp, c_vp, c_i32, c_vp, c_vp]),
    ("fsb_build_tracks", c_i32, [c_vp, c_vp, c_vp, c_i64, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("fsb_find_homography_batch", c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, ctypes.c_double, c_i32, ctypes.c_uint64,
                                          c_vp, c_vp, c_vp]),
    ("fsb_sift_features_batch_d", c_i32, [c_vp, c_i32, c_vp, c_i32, c_i32, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp,
                                          c_vp, c_vp, c_i32]),
    ("fsb_sift_features_batch_hd", c_i32, [c_vp, c_i32, c_vp, c_vp, c_i32, c_i32, c_i32, c_vp, c_vp, c_vp, c_vp,
                                           c_vp, c_vp, c_vp, c_i32]),
    ("fsb_pyramid_batch_d", c_i32, [c_vp, c_i32, c_vp, c_i32, c_i32, c_i32, c_i32, c_i32]),
    ("fsb_find_fundamental_batch", c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, ctypes.c_double, c_i32, ctypes.c_uint64,
                                           c_vp, c_vp, c_vp]),
    ("fsb_spread", c_i32, [c_vp, c_vp, c_vp, c_vp, c_i32, c_i32, c_i32, c_i32, c_i32, c_vp, c_vp]),
    ("fsb_decode_gray_d", c_i32, [c_vp, c_vp, c_i64, c_i32, c_vp, c_i64, c_vp, c_vp]),
    ("fsb_prepare_gray", c_i32, [c_vp, c_vp, c_i64, c_i32, ctypes.c_double, c_vp, c_i64, c_vp, c_vp]),
    ("fsb_clahe", c_i32, [c_vp, c_vp, c_i32, c_i32, c_i32, ctypes.c_double, c_i32, c_i32, c_vp, c_i32]),
    ("fsb_clahe_d", c_i32, [c_vp, c_vp, c_i32, c_i32, c_i32, ctypes.c_double, c_i32, c_i32, c_vp, c_i32]),
    ("fsb_predict_ground", c_i32, [c_vp, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_double,
                                   c_vp, c_vp]),
    ("fsb_launch_count", c_i64, []),
    ("fsb_timing", c_i32, [c_vp, c_i32]),
    ("fsb_stage_times", c_i32, [c_vp, c_vp, c_vp, c_i32]),
    ("fsb_sift_features_d", c_i32, [c_vp, c_vp, c_i32, c_i32, c_i32, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("fsb_project_d", c_i32, [c_vp, c_vp, c_i32, c_vp, c_vp, c_vp]),
    ("fsb_project_batch_d", c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("fsb_match_guided_d", c_i32, [c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_i32, c_f64, c_f64, c_f64, c_i32, c_f32,
                                   c_vp, c_vp, c_vp]),
    ("fsb_match_bf_d", c_i32, [c_vp, c_vp, c_i32, c_vp, c_i32, c_f32, c_i32, c_vp, c_vp, c_vp]),
    ("fsb_match_bf_noalloc", c_i32, [c_vp, c_i32, c_vp, c_i32, c_f32, c_vp, c_vp, c_vp, c_vp]),
    ("fsb_match_bf_batch_d", c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_f32, c_i32, c_vp, c_vp, c_vp]),
    ("fsb_match_tc_stats", c_i32, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("fsb_sift_features_ex_d", c_i32, [c_vp, c_vp, c_i32, c_i32, c_i32, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp,
                                       c_vp, c_vp, c_vp]),
    ("fsb_match_guided_cand_d", c_i32, [c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_i32, c_f64, c_f64, c_f64, c_i32,
                                        c_vp, c_vp]),
    ("fsb_match_guided_batch_d", c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_f64, c_i32,
                                         c_f32, c_vp, c_vp, c_vp]),
    ("fsb_autotune_table", c_i32, [ctypes.c_char_p, c_i32]),
    ("fsb_mlp_param_count", c_i32, []),
    ("fsb_mlp_trainable_count", c_i32, []),
    ("fsb_mlp_features_d", c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                   c_f32, c_vp]),
    ("fsb_mlp_grad_d", c_i32, [c_vp, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp]),
    ("fsb_mlp_train_d", c_i32, [c_vp, c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_i32, c_i32, c_f32, ctypes.c_uint32,
                                c_vp]),
    ("fsb_mlp_infer_d", c_i32, [c_vp, c_vp, c_i32, c_vp, c_i32, c_vp]),
    ("fsb_mlp_filter_d", c_i32, [c_vp, c_i32, c_vp, c_vp, c_vp, c_f32, c_f32, c_i32, c_vp, c_vp, c_vp]),
]

STAGES = ("upload", "pyramid", "extrema", "refine", "orientation", "sort", "spread", "describe", "match", "tc_dense")

_lib = None
_lock = threading.Lock()


def load():
    """Loads libfsb200.so and declares every entry point (raises if the library is missing)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError("libfsb200.so is not built (run `python -m fieldstitch_b200.build`); "
                                   "fieldstitch_b200 has no CPU fallback")
            lib = ctypes.CDLL(LIB_PATH)
            for name, res, args in SIGNATURES:
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def check(status, what=""):
    if status != FSB_OK:
        msg = load().fsb_last_error().decode(errors="replace")
        raise RuntimeError("%s failed (%s): %s" % (what or "fsb call", STATUS.get(status, status), msg))


def ptr(a):
    """Raw data pointer of a numpy array (None for None)."""
    return None if a is None else a.ctypes.data


class Context:
    """One fsb_ctx (one CUDA stream on one device)."""

    def __init__(self, device=0):
        self.lib = load()
        h = c_vp()
        check(self.lib.fsb_create(device, ctypes.byref(h)), "fsb_create(device=%d)" % device)
        self.handle = h.value
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self.lib.fsb_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def sync(self, timeout_ms=60000):
        check(self.lib.fsb_sync(self.handle, timeout_ms), "fsb_sync")

    def device_bytes(self):
        return int(self.lib.fsb_device_bytes(self.handle))

    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        return int(self.lib.fsb_stream(self.handle) or 0)

    def timing(self, on=True):
        check(self.lib.fsb_timing(self.handle, 1 if on else 0), "fsb_timing")

    def stage_times(self):
        """{stage: (milliseconds, calls)} accumulated since the last call (then reset)."""
        ms = np.zeros(len(STAGES), np.float64)
        n = np.zeros(len(STAGES), np.int64)
        check(self.lib.fsb_stage_times(self.handle, ptr(ms), ptr(n), len(STAGES)), "fsb_stage_times")
        return {s: (float(ms[i]), int(n[i])) for i, s in enumerate(STAGES)}


def launch_count():
    """Kernel launches issued by libfsb200 in this process."""
    return int(load().fsb_launch_count())


_tls = threading.local()


def context(device=0):
    """The calling thread's context for `device` (contexts are single-threaded)."""
    ctxs = getattr(_tls, "ctxs", None)
    if ctxs is None:
        ctxs = _tls.ctxs = {}
    if device not in ctxs:
        ctxs[device] = Context(device)
    return ctxs[device]


def as_u8_desc(d, name="descriptors"):
    """uint8 (n,128) C-contiguous view of descriptors given as uint8 or as integral float arrays
    (the reference holds uint8 RootSIFT descriptors as float32, app/planesite/matching.py:59)."""
    d = np.asarray(d)
    if d.ndim != 2 or (d.shape[0] and d.shape[1] != 128):
        raise ValueError("%s must be (n, 128), got %s" % (name, d.shape))
    if d.dtype == np.uint8:
        return np.ascontiguousarray(d)
    u = d.astype(np.uint8)
    if not np.array_equal(u, d):
        raise ValueError("%s must hold uint8 values (0..255 integers)" % name)
    return np.ascontiguousarray(u)


def autotune_table():
    """{key: variant} of the launch-variant autotuner's choices in this process."""
    lib = load()
    n = int(lib.fsb_autotune_table(None, 0))
    buf = ctypes.create_string_buffer(max(n, 1))
    lib.fsb_autotune_table(buf, n)
    out = {}
    for line in buf.value.decode().splitlines():
        k, v = line.rsplit(" ", 1)
        out[k] = int(v)
    return out
