"""The sync-free batched extraction (fsb_sift_features_batch_d: every count on the device, the batch
captured as one CUDA graph with several images in flight) returns exactly what the host-driven
per-image path (fsb_sift_features_d, features.sift_gpu's sequence) returns: the same feature
counts, coordinates, responses and RootSIFT bytes, on the first call (capture) and on replays,
for uneven keypoint caps including caps above the keypoint count and a flat image."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _per_image(F, img, nfeat):
    xy, u8, resp = F.features.sift_gpu_u8(img, nfeat)
    return xy, u8, resp


@pytest.mark.parametrize("hw,chains", [((989, 1320), 3), ((495, 660), 8)])
def test_batch_extraction_equals_per_image(hw, chains):
    import torch

    import fieldstitch_b200 as F
    from fieldstitch_b200 import synth
    h, w = hw
    dev = torch.device("cuda", 0)
    imgs = [synth.synth_image(h, w, 300 + k) for k in range(7)]
    imgs[5] = np.full((h, w), 90, np.uint8)          # no keypoints
    nfeats = [3000, 500, 12000, 800, 20000, 1000, 64]
    d_imgs = [torch.from_numpy(im).to(dev) for im in imgs]
    nmax = max(nfeats)
    xy = [torch.zeros((nmax, 2), dtype=torch.float32, device=dev) for _ in imgs]
    u8 = [torch.zeros((nmax, 128), dtype=torch.uint8, device=dev) for _ in imgs]
    rs = [torch.zeros(nmax, dtype=torch.float32, device=dev) for _ in imgs]
    want = [_per_image(F, im, nf) for im, nf in zip(imgs, nfeats)]
    for rep in range(3):   # capture, then replays
        for t in xy + u8 + rs:
            t.zero_()
        counts = F.features.sift_gpu_batch_d(d_imgs, nfeats, xy, u8, rs, chains=chains)
        for k, (wxy, wu8, wrs) in enumerate(want):
            n = len(wxy)
            assert counts[k] == n, (rep, k, counts[k], n)
            np.testing.assert_array_equal(xy[k][:n].cpu().numpy(), wxy)
            np.testing.assert_array_equal(u8[k][:n].cpu().numpy(), wu8)
            np.testing.assert_array_equal(rs[k][:n].cpu().numpy(), wrs)
    assert counts[5] == 0 and counts[2] > 0


def test_batch_extraction_rejects_bad_arguments():
    import ctypes

    from fieldstitch_b200 import _lib
    ctx = _lib.context(0)
    prm = _lib.SiftParams(0.015, 12.0, 0, 0)
    P1, I1 = ctypes.c_void_p * 1, ctypes.c_int32 * 1
    st = ctx.lib.fsb_sift_features_batch_d(ctx.handle, 1, P1(16), 100, 100, 100, ctypes.byref(prm), I1(10), P1(16),
                                           None, P1(16), ctypes.c_void_p(16), None, 0)
    assert st == 1 and b"chains" in ctx.lib.fsb_last_error()
    assert ctx.lib.fsb_sift_features_batch_d(ctx.handle, 0, None, 0, 0, 0, ctypes.byref(prm), None, None, None,
                                             None, None, None, 4) == 0


def test_host_batch_api_equals_per_image():
    """features.sift_gpu_u8_batch (host arrays in and out: one upload, one graph, one download per
    kind) returns sift_gpu_u8's output image by image, on two calls in a row."""
    import fieldstitch_b200 as F
    from fieldstitch_b200 import synth
    imgs = [synth.synth_image(600, 800, 500 + k) for k in range(5)]
    nfeats = [2000, 300, 5000, 50, 1200]
    want = [_per_image(F, im, nf) for im, nf in zip(imgs, nfeats)]
    for _ in range(2):
        got = F.features.sift_gpu_u8_batch(imgs, nfeats, chains=2)
        for (gxy, gu8, grs), (wxy, wu8, wrs) in zip(got, want):
            np.testing.assert_array_equal(gxy, wxy)
            np.testing.assert_array_equal(gu8, wu8)
            np.testing.assert_array_equal(grs, wrs)


def test_extract_and_match_equals_per_pair_calls():
    """frontend.extract_and_match (features kept on the device between the two graphs) returns the
    matches of the per-image / per-pair host calls (sift_gpu_u8, guided_from_pred), on two calls."""
    import fieldstitch_b200 as F
    from fieldstitch_b200 import synth
    h, w = 700, 900
    pairs_src = [synth.synth_pair(h, w, 700 + k) for k in range(3)]
    imgs = [im for a, b, _ in pairs_src for im in (a, b)]
    nfeats = [3000, 2500, 800, 4000, 1500, 1500]
    pairs = [(0, 1), (2, 3), (4, 5), (1, 0)]
    priors = [pairs_src[0][2], pairs_src[1][2], pairs_src[2][2], np.linalg.inv(pairs_src[0][2])]
    offs = [synth.prior_noise(5000, 40 + p) for p in range(len(pairs))]
    feats = [F.features.sift_gpu_u8(im, nf) for im, nf in zip(imgs, nfeats)]
    want = []
    for (i, j), H, o in zip(pairs, priors, offs):
        xa = feats[i][0]
        pred = synth.apply_homography(H, xa) + o[:len(xa)].astype(np.float64)
        want.append(F.matching.guided_from_pred(pred, feats[i][1], feats[j][0].astype(np.float64), feats[j][1],
                                                (w, h), 40.0, 16, 0.85))
    for _ in range(2):
        got, fe = F.frontend.extract_and_match(imgs, nfeats, pairs, priors, 40.0, 16, 0.85, offsets=offs,
                                               chains=3, return_features=True)
        for (gq, gt), (wq, wt) in zip(got, want):
            assert len(wq) > 0
            np.testing.assert_array_equal(gq, wq)
            np.testing.assert_array_equal(gt, wt)
        for (gxy, gu8, grs), (wxy, wu8, wrs) in zip(fe, feats):
            np.testing.assert_array_equal(gxy, wxy)
            np.testing.assert_array_equal(gu8, wu8)


def _pinned(a):
    import torch
    t = torch.empty(a.shape, dtype=torch.uint8, pin_memory=True)
    t.numpy()[...] = a
    return t


def test_graph_uploads_from_page_locked_images():
    """fsb_sift_features_batch_hd (the uploads captured in the extraction graph, each image's chain
    waiting for its own upload): the per-image results, on the capture and on replays whose host
    buffers are other page-locked arrays (the uploads re-pointed, the graph kept), with the batch
    larger than the chains so later uploads overlap earlier extractions."""
    import fieldstitch_b200 as F
    from fieldstitch_b200 import synth
    imgs = [synth.synth_image(600, 800, 900 + k) for k in range(7)]
    nfeats = [2000, 300, 5000, 50, 1200, 800, 2500]
    want = [_per_image(F, im, nf) for im, nf in zip(imgs, nfeats)]
    assert F.features._all_pinned([_pinned(imgs[0]).numpy()])
    for rep in range(3):
        hold = [_pinned(im) for im in imgs]   # new page-locked buffers every call
        got = F.features.sift_gpu_u8_batch([t.numpy() for t in hold], nfeats, chains=3)
        for k, ((gxy, gu8, grs), (wxy, wu8, wrs)) in enumerate(zip(got, want)):
            np.testing.assert_array_equal(gxy, wxy, err_msg="call %d image %d" % (rep, k))
            np.testing.assert_array_equal(gu8, wu8)
            np.testing.assert_array_equal(grs, wrs)


def test_graph_uploads_reject_pageable_memory():
    import ctypes

    import torch

    from fieldstitch_b200 import _lib
    ctx = _lib.context(0)
    prm = _lib.SiftParams(0.015, 12.0, 0, 0)
    img = np.zeros((64, 64), np.uint8)   # pageable
    d = torch.zeros((64, 64), dtype=torch.uint8, device="cuda:0")
    xy = torch.zeros((10, 2), dtype=torch.float32, device="cuda:0")
    u8 = torch.zeros((10, 128), dtype=torch.uint8, device="cuda:0")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda:0")
    P1, I1 = ctypes.c_void_p * 1, ctypes.c_int32 * 1
    st = ctx.lib.fsb_sift_features_batch_hd(ctx.handle, 1, P1(img.ctypes.data), P1(d.data_ptr()), 64, 64, 64,
                                            ctypes.byref(prm), I1(10), P1(xy.data_ptr()), None, P1(u8.data_ptr()),
                                            ctypes.c_void_p(cnt.data_ptr()), None, 2)
    assert st == 1 and b"page-locked" in ctx.lib.fsb_last_error()


def test_extract_and_match_from_page_locked_images():
    """frontend.extract_and_match with page-locked images (the uploads inside the extraction graph)
    returns the matches of the pageable-input path."""
    import fieldstitch_b200 as F
    from fieldstitch_b200 import synth
    h, w = 700, 900
    src = [synth.synth_pair(h, w, 800 + k) for k in range(3)]
    imgs = [im for a, b, _ in src for im in (a, b)]
    nfeats = [3000, 2500, 800, 4000, 1500, 1500]
    pairs = [(0, 1), (2, 3), (4, 5)]
    priors = [s[2] for s in src]
    offs = [synth.prior_noise(5000, 60 + p) for p in range(len(pairs))]
    want = F.frontend.extract_and_match(imgs, nfeats, pairs, priors, 40.0, 16, 0.85, offsets=offs, chains=2)
    for _ in range(2):
        hold = [_pinned(im) for im in imgs]
        got = F.frontend.extract_and_match([t.numpy() for t in hold], nfeats, pairs, priors, 40.0, 16, 0.85,
                                           offsets=offs, chains=2)
        for (gq, gt), (wq, wt) in zip(got, want):
            assert len(wq) > 0
            np.testing.assert_array_equal(gq, wq)
            np.testing.assert_array_equal(gt, wt)


def test_pyramid_batch_runs_and_leaves_extraction_unchanged():
    """fsb_pyramid_batch_d (the pyramid stage of a batch alone, one graph, several chains) runs on
    its capture and replays, rejects bad arguments, and a batched extraction on the same context
    afterwards still equals the per-image path."""
    import ctypes

    import torch

    import fieldstitch_b200 as F
    from fieldstitch_b200 import _lib, synth
    h, w = 495, 660
    dev = torch.device("cuda", 0)
    imgs = [synth.synth_image(h, w, 700 + k) for k in range(5)]
    d_imgs = [torch.from_numpy(im).to(dev) for im in imgs]
    ctx = _lib.context(0)
    Pv = ctypes.c_void_p * len(imgs)
    arr = Pv(*[t.data_ptr() for t in d_imgs])
    for _ in range(3):
        _lib.check(ctx.lib.fsb_pyramid_batch_d(ctx.handle, len(imgs), arr, h, w, w, 0, 3), "pyramid batch")
    assert ctx.lib.fsb_pyramid_batch_d(ctx.handle, len(imgs), arr, h, w, w, 0, 0) == 1
    assert b"chains" in ctx.lib.fsb_last_error()
    assert ctx.lib.fsb_pyramid_batch_d(ctx.handle, 1, Pv(None), h, w, w, 0, 2) == 1
    assert ctx.lib.fsb_pyramid_batch_d(ctx.handle, 0, None, 0, 0, 0, 0, 2) == 0
    nfeats = [1500, 400, 3000, 800, 50]
    nmax = max(nfeats)
    xy = [torch.zeros((nmax, 2), dtype=torch.float32, device=dev) for _ in imgs]
    u8 = [torch.zeros((nmax, 128), dtype=torch.uint8, device=dev) for _ in imgs]
    rs = [torch.zeros(nmax, dtype=torch.float32, device=dev) for _ in imgs]
    counts = F.features.sift_gpu_batch_d(d_imgs, nfeats, xy, u8, rs, chains=3)
    for k, (im, nf) in enumerate(zip(imgs, nfeats)):
        wxy, wu8, wrs = _per_image(F, im, nf)
        n = len(wxy)
        assert counts[k] == n
        np.testing.assert_array_equal(xy[k][:n].cpu().numpy(), wxy)
        np.testing.assert_array_equal(u8[k][:n].cpu().numpy(), wu8)
