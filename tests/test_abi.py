"""CPU-side checks of the C ABI boundary: the library loads, exports every entry point that
include/fsb200.h declares, and rejects bad calls with a status (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from fieldstitch_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fsb200.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fsb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    for n in ("fsb_create", "fsb_detect", "fsb_describe", "fsb_sift_features", "fsb_match_bf",
              "fsb_match_guided", "fsb_unique", "fsb_perspective"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(declared()) <= bound, set(declared()) - bound


def test_null_context_is_rejected_with_a_status():
    lib = _lib.load()
    n = ctypes.c_int32(-1)
    st = lib.fsb_match_bf(None, None, 0, None, 0, 0.8, 0, None, None, ctypes.byref(n))
    assert st == 1
    assert b"invalid argument" in lib.fsb_last_error()
    assert lib.fsb_create(0, None) == 1


def test_unknown_precision_rejected():
    lib = _lib.load()
    n = ctypes.c_int32()
    a = np.zeros((4, 128), np.uint8)
    # a bogus (non-null) context pointer is never dereferenced before argument validation
    st = lib.fsb_match_bf(ctypes.c_void_p(1), _lib.ptr(a), 4, _lib.ptr(a), 4, 0.8, 17, _lib.ptr(a), _lib.ptr(a),
                          ctypes.byref(n))
    assert st == 1


def test_create_fails_cleanly_without_gpu():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = _lib.load()
    h = ctypes.c_void_p()
    st = lib.fsb_create(0, ctypes.byref(h))
    assert st != 0 and h.value is None
    assert len(lib.fsb_last_error()) > 0


def test_host_validation():
    from fieldstitch_b200 import gsift, matching
    with pytest.raises(NotImplementedError):
        gsift.detect(np.zeros((32, 32), np.uint8), gpu=False)
    with pytest.raises(ValueError):
        _lib.as_u8_desc(np.full((3, 128), 0.5, np.float32))
    with pytest.raises(ValueError):
        _lib.as_u8_desc(np.zeros((3, 64), np.uint8))
    assert _lib.as_u8_desc(np.full((2, 128), 7.0, np.float32)).dtype == np.uint8
    q, t = matching._ratio_match_bf(np.zeros((1, 128), np.float32), np.zeros((5, 128), np.float32), 0.8)
    assert len(q) == len(t) == 0


def test_spread_arguments_checked_before_the_device():
    """fsb_spread rejects unsorted responses, a bad order code and negative sizes with a status
    before touching the context (a bogus non-null context pointer is never dereferenced)."""
    lib = _lib.load()
    x = np.arange(5, dtype=np.float32)
    r_up = np.arange(5, dtype=np.float32)          # ascending: not detect's order
    r_dn = r_up[::-1].copy()
    sel = np.zeros(5, np.int32)
    n = ctypes.c_int32(-1)
    bogus = ctypes.c_void_p(1)
    P = _lib.ptr
    assert lib.fsb_spread(bogus, P(x), P(x), P(r_up), 5, 100, 100, 3, 0, P(sel), ctypes.byref(n)) == 1
    assert b"response-descending" in lib.fsb_last_error()
    assert lib.fsb_spread(bogus, P(x), P(x), P(r_dn), 5, 100, 100, 3, 7, P(sel), ctypes.byref(n)) == 1
    assert lib.fsb_spread(bogus, P(x), P(x), P(r_dn), -1, 100, 100, 3, 0, P(sel), ctypes.byref(n)) == 1
    assert lib.fsb_spread(bogus, P(x), P(x), P(r_dn), 5, 0, 100, 3, 0, P(sel), ctypes.byref(n)) == 1
    from fieldstitch_b200 import features
    with pytest.raises(ValueError):
        features._spread([], 100, 100, 10, gx=8)


def test_pyramid_batch_arguments_checked_before_the_device():
    """fsb_pyramid_batch_d rejects a null context, negative counts, bad sizes, a chain count outside
    1..32 and null image pointers with a status before touching the device (a bogus non-null
    context pointer is never dereferenced); an empty batch is a no-op."""
    lib = _lib.load()
    bogus = ctypes.c_void_p(1)
    P2 = ctypes.c_void_p * 2
    imgs = P2(16, 32)
    assert lib.fsb_pyramid_batch_d(None, 2, imgs, 100, 100, 100, 0, 2) == 1
    assert lib.fsb_pyramid_batch_d(bogus, -1, imgs, 100, 100, 100, 0, 2) == 1
    assert lib.fsb_pyramid_batch_d(bogus, 0, None, 0, 0, 0, 0, 2) == 0
    assert lib.fsb_pyramid_batch_d(bogus, 2, None, 100, 100, 100, 0, 2) == 1
    assert lib.fsb_pyramid_batch_d(bogus, 2, imgs, 100, 100, 50, 0, 2) == 1
    assert lib.fsb_pyramid_batch_d(bogus, 2, imgs, 40000, 100, 100, 0, 2) == 1
    assert lib.fsb_pyramid_batch_d(bogus, 2, imgs, 100, 100, 100, 0, 0) == 1
    assert b"chains" in lib.fsb_last_error()
    assert lib.fsb_pyramid_batch_d(bogus, 2, imgs, 100, 100, 100, 0, 33) == 1
    assert lib.fsb_pyramid_batch_d(bogus, 2, P2(16, None), 100, 100, 100, 0, 2) == 1
    assert b"null image" in lib.fsb_last_error()
