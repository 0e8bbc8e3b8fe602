"""Drop-in for PlaneSite's per-photo GPU feature step (app/planesite/features.py:74-129).

``sift_gpu(g2, nfeat)`` keeps the reference's signature and return value (xy float32 (n,2), desc
float32 (n,128) or None, resp float32 (n,), seconds spent describing) but runs detect -> grid
spread -> stable response sort -> describe -> RootSIFT in one device pass (fsb_sift_features).
``sift_gpu_u8`` also returns the RootSIFT uint8 bytes of the feature file, computed on the device,
and ``save_features`` writes the reference's .npz feature-file format.
"""
import ctypes
import time

import numpy as np

from . import _lib
from .gsift import _gray, _params


def _extract(g2, nfeat, contrast, edge, exact, want_desc, want_u8, device):
    g = _gray(g2)
    ctx = _lib.context(device)
    nf = int(nfeat)
    xy = np.empty((max(nf, 0), 2), np.float32)
    resp = np.empty(max(nf, 0), np.float32)
    desc = np.empty((max(nf, 0), 128), np.float32) if want_desc else None
    u8 = np.empty((max(nf, 0), 128), np.uint8) if want_u8 else None
    n = ctypes.c_int32()
    p = _params(contrast, edge, 0, exact)
    _lib.check(ctx.lib.fsb_sift_features(ctx.handle, _lib.ptr(g), g.shape[0], g.shape[1], g.strides[0],
                                         ctypes.byref(p), nf, _lib.ptr(xy), _lib.ptr(resp), _lib.ptr(desc),
                                         _lib.ptr(u8), ctypes.byref(n)), "fsb_sift_features")
    n = n.value
    return xy[:n], (desc[:n] if desc is not None else None), resp[:n], (u8[:n] if u8 is not None else None)


def spread_arrays(x, y, resp, W, H, n, response_order=False, device=0):
    """features._spread (app/planesite/features.py:38-57) on the device over keypoint arrays in
    response-descending order (detect's order): int64 indices of min(len, n) keypoints spread over
    a 12 x 9 grid, in _spread's order, or (response_order=True) after the stable response sort of
    features.py:126. Ties among equal responses go by index."""
    xs = np.ascontiguousarray(x, np.float32)
    ys = np.ascontiguousarray(y, np.float32)
    rs = np.ascontiguousarray(resp, np.float32)
    if not (len(xs) == len(ys) == len(rs)):
        raise ValueError("x, y and resp differ in length")
    ctx = _lib.context(device)
    out = np.empty(max(min(len(xs), int(n)), 1), np.int32)
    k = ctypes.c_int32()
    _lib.check(ctx.lib.fsb_spread(ctx.handle, _lib.ptr(xs), _lib.ptr(ys), _lib.ptr(rs), len(xs), int(W), int(H),
                                  int(n), 1 if response_order else 0, _lib.ptr(out), ctypes.byref(k)), "fsb_spread")
    return out[:k.value].astype(np.int64)


def _spread(kps, W, H, n, gx=12, gy=9):
    """features._spread with the reference's signature: kps are objects with .pt and .response
    (cv2.KeyPoint or the reference's _KP), in response-descending order; returns a list of ints."""
    if (gx, gy) != (12, 9):
        raise ValueError("the device selection uses the reference's 12 x 9 grid")
    if len(kps) <= n:
        return list(range(len(kps)))
    xy = np.array([k.pt for k in kps], np.float32).reshape(-1, 2)
    r = np.array([k.response for k in kps], np.float32)
    return spread_arrays(xy[:, 0], xy[:, 1], r, W, H, n).tolist()


def sift_gpu(g2, nfeat, gpu=True, contrast=0.015, edge=12.0, exact=False, device=0):
    """features.sift_gpu (app/planesite/features.py:115-129): (xy, desc, resp, t_desc); returns
    zeros and None when fewer than 10 keypoints are found."""
    if not gpu:
        raise NotImplementedError("fieldstitch_b200 runs SIFT on the GPU only (no CPU fallback)")
    t = time.perf_counter()
    xy, desc, resp, _ = _extract(g2, nfeat, contrast, edge, exact, True, False, device)
    if len(xy) == 0:
        return np.zeros((0, 2), np.float32), None, np.zeros(0, np.float32), 0.0
    return xy, desc, resp, time.perf_counter() - t


def sift_gpu_u8(g2, nfeat, contrast=0.015, edge=12.0, exact=False, device=0):
    """(xy, rootsift uint8 (n,128), resp): the feature-file content of features._save
    (app/planesite/features.py:74-86) with the RootSIFT encoding done on the device."""
    xy, _, resp, u8 = _extract(g2, nfeat, contrast, edge, exact, False, True, device)
    if len(xy) < 10:
        return np.zeros((0, 2), np.float32), np.zeros((0, 128), np.uint8), np.zeros(0, np.float32)
    return xy, u8, resp


def save_features(out_npz, xy, desc_u8, resp, w, h):
    """Writes the feature file in the reference's format (keys xy, desc, resp, red_wh;
    app/planesite/features.py:74-86). Returns the number of features written."""
    if desc_u8 is None or len(xy) < 10:
        np.savez(out_npz, xy=np.zeros((0, 2), np.float32), desc=np.zeros((0, 128), np.uint8),
                 resp=np.zeros(0, np.float32), red_wh=np.array([w, h], np.int32))
        return 0
    np.savez(out_npz, xy=np.asarray(xy, np.float32), desc=np.asarray(desc_u8, np.uint8),
             resp=np.asarray(resp, np.float32), red_wh=np.array([w, h], np.int32))
    return len(xy)


def _batch(fn, items, streams):
    """Runs fn over items on `streams` host threads, each driving its own context (CUDA stream and
    workspaces), so one image's host-side steps overlap the others' kernels; results in order."""
    from concurrent.futures import ThreadPoolExecutor
    streams = max(1, min(int(streams), len(items)))
    if streams == 1:
        return [fn(x) for x in items]
    with ThreadPoolExecutor(max_workers=streams) as ex:
        return list(ex.map(fn, items))


def sift_gpu_batch(images, nfeats, streams=4, contrast=0.015, edge=12.0, exact=False, device=0):
    """Batched feature extraction: sift_gpu_u8 of every image (nfeats: one cap per image or one
    for all), spread over `streams` contexts. Returns a list of (xy, rootsift uint8, resp)."""
    nf = list(nfeats) if np.ndim(nfeats) else [int(nfeats)] * len(images)
    if len(nf) != len(images):
        raise ValueError("one keypoint cap per image")
    jobs = list(zip(images, nf))
    return _batch(lambda j: sift_gpu_u8(j[0], j[1], contrast, edge, exact, device), jobs, streams)


def sift_gpu_batch_d(images, nfeats, out_xy, out_u8, out_resp=None, chains=16, contrast=0.015, edge=12.0,
                     exact=False, device=0, host_images=None):
    """Batched feature extraction on device data with no host wait inside the batch
    (fsb_sift_features_batch_d: one CUDA graph, `chains` images in flight). images: same-size
    uint8 CUDA tensors; nfeats: one cap per image; out_xy[i] (>= nfeat, 2) float32, out_u8[i]
    (>= nfeat, 128) uint8 and optionally out_resp[i] CUDA tensors. With host_images (page-locked
    host arrays or CPU tensors, one per image, rows as long as the device images'), the graph
    uploads host_images[i] into images[i] itself, overlapping the uploads with the extraction
    (fsb_sift_features_batch_hd). Returns the feature counts (host list); equal to sift_gpu_u8 /
    fsb_sift_features_d image by image."""
    import ctypes

    import torch
    n = len(images)
    if n == 0:
        return []
    nf = list(nfeats) if np.ndim(nfeats) else [int(nfeats)] * n
    h, w = images[0].shape
    if any(tuple(im.shape) != (h, w) for im in images):
        raise ValueError("the images of a batch share one size")
    stride = images[0].stride(0)
    ctx = _lib.context(device)
    Pv, Iv = ctypes.c_void_p * n, ctypes.c_int32 * n
    counts = torch.empty(n, dtype=torch.int32, device=images[0].device)
    h_counts = Iv()
    prm = _lib.SiftParams(float(contrast), float(edge), 0, _lib.SIFT_EXACT_BLUR if exact else 0)
    outs = (Iv(*[int(v) for v in nf]), Pv(*[t.data_ptr() for t in out_xy]),
            Pv(*[t.data_ptr() for t in out_resp]) if out_resp is not None else None,
            Pv(*[t.data_ptr() for t in out_u8]), ctypes.c_void_p(counts.data_ptr()), h_counts, int(chains))
    torch.cuda.current_stream(images[0].device).synchronize()
    if host_images is None:
        _lib.check(ctx.lib.fsb_sift_features_batch_d(ctx.handle, n, Pv(*[im.data_ptr() for im in images]), h, w,
                                                     stride, ctypes.byref(prm), *outs), "fsb_sift_features_batch_d")
    else:
        hp = []
        for im in host_images:
            if isinstance(im, torch.Tensor):
                ok = im.dtype == torch.uint8 and tuple(im.shape) == (h, w) and im.stride(0) == stride
                hp.append(im.data_ptr())
            else:
                ok = im.dtype == np.uint8 and im.shape == (h, w) and im.strides == (stride, 1)
                hp.append(im.ctypes.data)
            if not ok:
                raise ValueError("host images: uint8 (%d, %d) with %d-byte rows" % (h, w, stride))
        _lib.check(ctx.lib.fsb_sift_features_batch_hd(ctx.handle, n, Pv(*hp), Pv(*[im.data_ptr() for im in images]),
                                                      h, w, stride, ctypes.byref(prm), *outs),
                   "fsb_sift_features_batch_hd")
    return [h_counts[i] for i in range(n)]


def _all_pinned(images):
    """True when every image is a host array in page-locked memory (the graph can upload it)."""
    import torch
    for im in images:
        a = np.asarray(im)
        if a.dtype != np.uint8 or not a.flags["C_CONTIGUOUS"] or not torch.from_numpy(a).is_pinned():
            return False
    return True


_BATCH_BUFS = {}


def sift_gpu_u8_batch(images, nfeats, chains=16, contrast=0.015, edge=12.0, exact=False, device=0):
    """sift_gpu_u8 of many same-size host images as one sync-free batch: one CUDA graph extracts
    them all (fsb_sift_features_batch_d; images in page-locked memory are uploaded by the graph
    itself, overlapping the extraction: fsb_sift_features_batch_hd) and the results come back. Returns [(xy float32 (n,2), RootSIFT
    uint8 (n,128), resp float32 (n,))], equal to sift_gpu_u8 image by image. The device buffers are
    kept between calls of the same shape, so a repeated batch replays its graph."""
    import torch
    n = len(images)
    if n == 0:
        return []
    nf = list(nfeats) if np.ndim(nfeats) else [int(nfeats)] * n
    h, w = np.asarray(images[0]).shape
    dev = torch.device("cuda", device)
    nmax = max(1, max(int(v) for v in nf))
    key = (n, h, w, nmax, device)
    if key not in _BATCH_BUFS:
        _BATCH_BUFS.clear()
        _BATCH_BUFS[key] = {"img": torch.empty((n, h, w), dtype=torch.uint8, device=dev),
                            "xy": torch.empty((n, nmax, 2), dtype=torch.float32, device=dev),
                            "u8": torch.empty((n, nmax, 128), dtype=torch.uint8, device=dev),
                            "rs": torch.empty((n, nmax), dtype=torch.float32, device=dev)}
    b = _BATCH_BUFS[key]
    host = None
    if _all_pinned(images):   # the graph uploads them, overlapping the extraction
        host = [np.asarray(im) for im in images]
    else:
        for i, im in enumerate(images):
            b["img"][i].copy_(torch.from_numpy(np.ascontiguousarray(im, np.uint8)))
    counts = sift_gpu_batch_d([b["img"][i] for i in range(n)], nf, [b["xy"][i] for i in range(n)],
                              [b["u8"][i] for i in range(n)], [b["rs"][i] for i in range(n)], chains, contrast,
                              edge, exact, device, host_images=host)
    # the valid rows of every image gathered on the device, one copy per kind back to the host
    if sum(counts) == 0:
        return [(np.zeros((0, 2), np.float32), np.zeros((0, 128), np.uint8), np.zeros(0, np.float32)) for _ in counts]
    xy = torch.cat([b["xy"][i, :c] for i, c in enumerate(counts)]).cpu().numpy()
    u8 = torch.cat([b["u8"][i, :c] for i, c in enumerate(counts)]).cpu().numpy()
    rs = torch.cat([b["rs"][i, :c] for i, c in enumerate(counts)]).cpu().numpy()
    cut = np.cumsum(counts)[:-1]
    return list(zip(np.split(xy, cut), np.split(u8, cut), np.split(rs, cut)))


def clahe(gray, clip=2.0, tiles=(8, 8), device=0):
    """cv2.createCLAHE(clipLimit=clip, tileGridSize=tiles).apply(gray) on the device (the contrast
    equalisation of features.prepare, app/planesite/features.py:70-71): identical uint8 output."""
    g = _gray(gray)
    out = np.empty(g.shape, np.uint8)
    ctx = _lib.context(device)
    _lib.check(ctx.lib.fsb_clahe(ctx.handle, _lib.ptr(g), g.shape[0], g.shape[1], g.strides[0], float(clip),
                                 int(tiles[0]), int(tiles[1]), _lib.ptr(out), out.strides[0]), "fsb_clahe")
    return out


def prepare(buf, reduce, thumb_path, device=0):
    """features.prepare (app/planesite/features.py:60-71): decode once (OpenCV, reduced-size JPEG
    decoding as the reference does), write the colour thumbnail if missing, and return the grey
    image contrast-equalised by CLAHE (clip 2.0, 8 x 8 tiles) on the device."""
    import os

    import cv2
    flag_col = {1: cv2.IMREAD_COLOR, 2: cv2.IMREAD_REDUCED_COLOR_2, 4: cv2.IMREAD_REDUCED_COLOR_4,
                8: cv2.IMREAD_REDUCED_COLOR_8}
    flag_gray = {1: cv2.IMREAD_GRAYSCALE, 2: cv2.IMREAD_REDUCED_GRAYSCALE_2, 4: cv2.IMREAD_REDUCED_GRAYSCALE_4,
                 8: cv2.IMREAD_REDUCED_GRAYSCALE_8}
    if thumb_path and not os.path.exists(thumb_path):
        col = cv2.imdecode(buf, flag_col[reduce] | cv2.IMREAD_IGNORE_ORIENTATION)
        if col is None:
            raise IOError("cannot decode image")
        th = cv2.resize(col, ((col.shape[1] + 1) * reduce // 8, (col.shape[0] + 1) * reduce // 8),
                        interpolation=cv2.INTER_AREA) if reduce < 8 else col
        ok, enc = cv2.imencode(".jpg", th, [cv2.IMWRITE_JPEG_QUALITY, 88])
        if not ok:
            raise IOError("encode failed")
        enc.tofile(thumb_path)
        gray = cv2.cvtColor(col, cv2.COLOR_BGR2GRAY)
    else:
        gray = cv2.imdecode(buf, flag_gray[reduce] | cv2.IMREAD_IGNORE_ORIENTATION)
        if gray is None:
            raise IOError("cannot decode image")
    return clahe(gray, 2.0, (8, 8), device)


def prepare_gpu(buf, reduce=1, clip=2.0, device=0):
    """The grey half of features.prepare (app/planesite/features.py:60-71) entirely on the device:
    nvJPEG decode of the luma plane (reduced by block means for reduce 2, 4, 8), then CLAHE (clip,
    8 x 8 tiles). buf holds the JPEG file's bytes. Full-size decodes agree with OpenCV's grayscale
    read to the inverse DCT's rounding; reduced ones approximately (OpenCV scales inside the DCT)."""
    data = np.ascontiguousarray(np.frombuffer(buf, np.uint8) if not isinstance(buf, np.ndarray) else buf, np.uint8)
    ctx = _lib.context(device)
    h, w = ctypes.c_int32(), ctypes.c_int32()
    cap = 1 << 22
    while True:
        out = np.empty(cap, np.uint8)
        st = ctx.lib.fsb_prepare_gray(ctx.handle, _lib.ptr(data), len(data), int(reduce), float(clip), _lib.ptr(out),
                                      cap, ctypes.byref(h), ctypes.byref(w))
        if st == 0 or h.value * w.value <= cap:
            _lib.check(st, "fsb_prepare_gray")
            return out[:h.value * w.value].reshape(h.value, w.value)
        cap = h.value * w.value
