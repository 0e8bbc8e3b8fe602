"""The feature front end of a flight in one call: SIFT of every photo and prior-guided matching of
every pair, with the features kept in device memory between the two stages.

In the reference, the feature workers write one npz file per photo (features._save,
app/planesite/features.py:74-86) and the pair workers read them back (matching._get,
app/planesite/matching.py:48-64) before guided matching (matching._guided, matching.py:113-152).
``extract_and_match`` does the same work for a batch: one CUDA graph extracts every image
(features.sift_gpu_batch_d; images in page-locked memory are uploaded by that graph, each
image's extraction starting once its own upload is done), every pair's prior prediction is
projected on the device, one CUDA graph matches every pair (matching.guided_from_pred_batch_d),
and the match lists come back in one copy. The features come back too when asked for (one copy
per kind).
"""
import ctypes

import numpy as np

from . import _lib, features, matching

_BUFS = {}


def _buffers(n_img, h, w, nmax, n_pairs, device):
    import torch
    key = (n_img, h, w, nmax, n_pairs, device)
    if key not in _BUFS:
        _BUFS.clear()
        dev = torch.device("cuda", device)
        _BUFS[key] = {"img": torch.empty((n_img, h, w), dtype=torch.uint8, device=dev),
                      "xy": torch.empty((n_img, nmax, 2), dtype=torch.float32, device=dev),
                      "u8": torch.empty((n_img, nmax, 128), dtype=torch.uint8, device=dev),
                      "rs": torch.empty((n_img, nmax), dtype=torch.float32, device=dev),
                      "bxy": torch.empty((n_img, nmax, 2), dtype=torch.float64, device=dev),
                      "pred": torch.empty((n_pairs, nmax, 2), dtype=torch.float64, device=dev),
                      "off": torch.zeros((n_pairs, nmax, 2), dtype=torch.float32, device=dev),
                      "q": torch.empty((n_pairs, nmax), dtype=torch.int64, device=dev),
                      "t": torch.empty((n_pairs, nmax), dtype=torch.int64, device=dev)}
    return _BUFS[key]


def extract_and_match(images, nfeats, pairs, priors, radius, kc=16, ratio=0.85, offsets=None, chains=16,
                      return_features=False, contrast=0.015, edge=12.0, device=0):
    """Features of every image and guided matches of every pair.

    images: same-size uint8 host arrays (page-locked ones are uploaded inside the extraction
    graph, overlapping the extraction of the images before them); nfeats: one
    keypoint cap per image (features.sift_gpu's nfeat); pairs: list of (i, j) image indices;
    priors: one 3x3 homography per pair mapping image i pixels to image j pixels (the GNSS /
    gimbal prior of matching._predict in homography form); offsets: optional per-pair float32
    (>= n_i, 2) additions to the predictions (a prior's error). Matching is matching._guided's:
    candidates the kc nearest image-j keypoints within radius of the prediction, exact
    distances, ratio test, one match per target. Returns [(q, t)] int64 per pair and, with
    return_features, [(xy, rootsift uint8, resp)] per image (sift_gpu_u8's output)."""
    import torch
    n_img, P = len(images), len(pairs)
    if n_img == 0:
        return ([], []) if return_features else []
    h, w = np.asarray(images[0]).shape
    nf = list(nfeats) if np.ndim(nfeats) else [int(nfeats)] * n_img
    nmax = max(1, max(int(v) for v in nf))
    b = _buffers(n_img, h, w, nmax, max(P, 1), device)
    host = None
    if features._all_pinned(images):   # uploaded by the extraction graph, overlapping the extraction
        host = [np.asarray(im) for im in images]
    else:
        for i, im in enumerate(images):
            b["img"][i].copy_(torch.from_numpy(np.ascontiguousarray(im, np.uint8)))
    if offsets is not None:
        off = np.zeros((max(P, 1), nmax, 2), np.float32)
        for p, o in enumerate(offsets):
            o = np.asarray(o, np.float32).reshape(-1, 2)[:nmax]
            off[p, :len(o)] = o
        b["off"].copy_(torch.from_numpy(off))
    counts = features.sift_gpu_batch_d([b["img"][i] for i in range(n_img)], nf, [b["xy"][i] for i in range(n_img)],
                                       [b["u8"][i] for i in range(n_img)], [b["rs"][i] for i in range(n_img)], chains,
                                       contrast, edge, False, device, host_images=host)
    if P:
        # image j's keypoints as float64 positions, every pair's prediction, on the device
        ctx = _lib.context(device)
        nset = n_img + P
        Pv, Iv = ctypes.c_void_p * nset, ctypes.c_int32 * nset
        hm = np.concatenate([np.tile(np.eye(3).reshape(9), n_img)] +
                            [np.asarray(H, np.float64).reshape(9) for H in priors])
        hm = np.ascontiguousarray(hm)
        xs = Pv(*[b["xy"][i].data_ptr() for i in range(n_img)] + [b["xy"][i].data_ptr() for i, _ in pairs])
        ns = Iv(*(counts + [counts[i] for i, _ in pairs]))
        offs = Pv(*([None] * n_img + [b["off"][p].data_ptr() if offsets is not None else None for p in range(P)]))
        outs = Pv(*[b["bxy"][i].data_ptr() for i in range(n_img)] + [b["pred"][p].data_ptr() for p in range(P)])
        torch.cuda.current_stream(device).synchronize()
        _lib.check(ctx.lib.fsb_project_batch_d(ctx.handle, nset, xs, ns, _lib.ptr(hm), offs, outs), "projections")
        probs = [(b["pred"][p, :counts[i]], b["u8"][i, :counts[i]], b["bxy"][j, :counts[j]], b["u8"][j, :counts[j]],
                  (float(w), float(h))) for p, (i, j) in enumerate(pairs)]
        res = matching.guided_from_pred_batch_d(probs, radius, kc, ratio, device=device,
                                                out=[(b["q"][p], b["t"][p]) for p in range(P)])
        lens = [len(q) for q, _ in res]
        if sum(lens):
            qa = torch.cat([q for q, _ in res]).cpu().numpy()
            ta = torch.cat([t for _, t in res]).cpu().numpy()
            cut = np.cumsum(lens)[:-1]
            matches = list(zip(np.split(qa, cut), np.split(ta, cut)))
        else:
            e = np.zeros(0, np.int64)
            matches = [(e, e) for _ in range(P)]
    else:
        matches = []
    if not return_features:
        return matches
    if sum(counts) == 0:
        feats = [(np.zeros((0, 2), np.float32), np.zeros((0, 128), np.uint8), np.zeros(0, np.float32))
                 for _ in counts]
    else:
        xy = torch.cat([b["xy"][i, :c] for i, c in enumerate(counts)]).cpu().numpy()
        u8 = torch.cat([b["u8"][i, :c] for i, c in enumerate(counts)]).cpu().numpy()
        rs = torch.cat([b["rs"][i, :c] for i, c in enumerate(counts)]).cpu().numpy()
        cut = np.cumsum(counts)[:-1]
        feats = list(zip(np.split(xy, cut), np.split(u8, cut), np.split(rs, cut)))
    return matches, feats
