"""Device CLAHE (the contrast equalisation of features.prepare) through the C ABI: identical to
OpenCV's output on the golden fixtures and to the oracle at the bench's image size, on strided
input and on images smaller than the tile grid."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "clahe.npz")


def test_clahe_matches_opencv_fixtures():
    from fieldstitch_b200 import features
    with np.load(GOLDEN) as z:
        for n in [k[:-4] for k in z.files if k.endswith("/img")]:
            clip, tx, ty = z[n + "/params"]
            np.testing.assert_array_equal(features.clahe(z[n + "/img"], clip, (int(tx), int(ty))), z[n + "/out"],
                                          err_msg=n)


@pytest.mark.parametrize("hw", [(1978, 2640), (1001, 1333), (8, 24), (7, 7), (3, 40)])
def test_clahe_matches_oracle(hw):
    from fieldstitch_b200 import features, synth
    from oracle import clahe_ref
    img = synth.synth_image(*hw, 12)
    ref = clahe_ref.clahe(img)
    np.testing.assert_array_equal(features.clahe(img), ref)
    strided = np.zeros((hw[0], hw[1] + 13), np.uint8)
    strided[:, 5:5 + hw[1]] = img
    np.testing.assert_array_equal(features.clahe(strided[:, 5:5 + hw[1]]), ref)


def test_clahe_rejects_bad_tile_grids():
    from fieldstitch_b200 import features
    for tiles in ((0, 8), (17, 16)):
        with pytest.raises(RuntimeError):
            features.clahe(np.zeros((64, 64), np.uint8), 2.0, tiles)


def _jpeg(color, seed=7, hw=(989, 1320)):
    import cv2
    from fieldstitch_b200 import synth
    img = synth.synth_image(*hw, seed)
    src = cv2.merge([img, np.roll(img, 5, 1), np.roll(img, 9, 0)]) if color else img
    ok, enc = cv2.imencode(".jpg", src, [cv2.IMWRITE_JPEG_QUALITY, 92])
    assert ok
    return enc.ravel()


def _decode(buf, r):
    import ctypes

    import torch
    from fieldstitch_b200 import _lib
    ctx = _lib.context(0)
    dev = torch.empty(1 << 22, dtype=torch.uint8, device="cuda")
    h, w = ctypes.c_int32(), ctypes.c_int32()
    _lib.check(ctx.lib.fsb_decode_gray_d(ctx.handle, _lib.ptr(buf), len(buf), r, ctypes.c_void_p(dev.data_ptr()),
                                         dev.numel(), ctypes.byref(h), ctypes.byref(w)), "fsb_decode_gray_d")
    torch.cuda.synchronize()
    return dev[:h.value * w.value].cpu().numpy().reshape(h.value, w.value)


@pytest.mark.parametrize("color", [True, False])
def test_jpeg_decode_against_opencv(color):
    """Luma plane by nvJPEG against OpenCV's grayscale read (the reference's decode): full size
    within the inverse DCT's rounding (max 2 levels, mean < 0.05); reduced reads (block means where
    OpenCV scales inside the DCT) mean < 0.3, 99th percentile <= 2, max <= 8 levels; same sizes."""
    import cv2
    buf = _jpeg(color)
    for r, flag in ((1, cv2.IMREAD_GRAYSCALE), (2, cv2.IMREAD_REDUCED_GRAYSCALE_2),
                    (4, cv2.IMREAD_REDUCED_GRAYSCALE_4), (8, cv2.IMREAD_REDUCED_GRAYSCALE_8)):
        ref = cv2.imdecode(buf, flag | cv2.IMREAD_IGNORE_ORIENTATION)
        got = _decode(buf, r)
        assert got.shape == ref.shape, (r, got.shape, ref.shape)
        d = np.abs(got.astype(np.int32) - ref.astype(np.int32))
        if r == 1:
            assert d.max() <= 2 and d.mean() < 0.05, (r, d.max(), d.mean())
        else:
            assert d.mean() < 0.3 and np.percentile(d, 99) <= 2 and d.max() <= 8, (r, d.mean(), d.max())


def test_prepare_gpu_against_opencv_pipeline():
    """features.prepare_gpu (device decode + CLAHE) against OpenCV decode + OpenCV CLAHE (the
    reference's prepare): CLAHE amplifies the decode differences locally; mean < 0.8 levels,
    99th percentile <= 6."""
    import cv2
    from fieldstitch_b200 import features
    buf = _jpeg(True, 3)
    cl = cv2.createCLAHE(clipLimit=2.0, tileGridSize=(8, 8))
    for r, flag in ((1, cv2.IMREAD_GRAYSCALE), (2, cv2.IMREAD_REDUCED_GRAYSCALE_2)):
        ref = cl.apply(cv2.imdecode(buf, flag | cv2.IMREAD_IGNORE_ORIENTATION))
        got = features.prepare_gpu(buf, r)
        d = np.abs(got.astype(np.int32) - ref.astype(np.int32))
        assert got.shape == ref.shape and d.mean() < 0.8 and np.percentile(d, 99) <= 6, (r, d.mean())
    with pytest.raises(RuntimeError):
        features.prepare_gpu(np.zeros(100, np.uint8), 1)
