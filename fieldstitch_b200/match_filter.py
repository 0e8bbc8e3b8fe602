"""Learned match filter for prior-guided matching (no counterpart in the reference).

PlaneSite accepts a query's best guided candidate by the ratio test (matching._guided,
app/planesite/matching.py:142-146) and then verifies the accepted set with a RANSAC homography
(matching.py:205-233). Here an 8-64-64-1 MLP scores every query's best candidate from 8 features
(ratio, best distance, log2 scale ratio, angle difference, prior residual, both responses,
octave); it is trained on the GPU (libfsb200's own forward/backward/Adam kernels, one CUDA graph
per epoch) on labels that the plain pipeline produces by its own verification: a candidate is an
inlier when the RANSAC homography fitted to the plain pipeline's matches maps it within 2 px.
The plain ratio test stays the fallback (``MatchFilter.matches`` without a trained network) and
the yardstick of the filter's precision and recall (``score``).

Device data are torch CUDA tensors (torch is used only for device memory here).
"""
import ctypes

import numpy as np

from . import _lib

N_FEATURES = 8
LABEL_PX = 2.0


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def extract(img, nfeat, contrast=0.015, edge=12.0, device=0):
    """SIFT (the sift_gpu sequence) of a uint8 CUDA image: dict of CUDA tensors xy (n,2), resp,
    u8 (n,128) RootSIFT, size, angle, octave."""
    import torch
    ctx = _lib.context(device)
    h, w = img.shape
    dev = img.device
    nf = int(nfeat)
    out = {"xy": torch.empty((nf, 2), dtype=torch.float32, device=dev),
           "resp": torch.empty(nf, dtype=torch.float32, device=dev),
           "u8": torch.empty((nf, 128), dtype=torch.uint8, device=dev),
           "size": torch.empty(nf, dtype=torch.float32, device=dev),
           "angle": torch.empty(nf, dtype=torch.float32, device=dev),
           "octave": torch.empty(nf, dtype=torch.int32, device=dev)}
    n = ctypes.c_int32()
    prm = _lib.SiftParams(contrast, edge, 0, 0)
    torch.cuda.current_stream(dev).synchronize()
    _lib.check(ctx.lib.fsb_sift_features_ex_d(ctx.handle, _p(img), h, w, img.stride(0), ctypes.byref(prm), nf,
                                              _p(out["xy"]), _p(out["resp"]), None, _p(out["u8"]),
                                              _p(out["size"]), _p(out["angle"]), _p(out["octave"]),
                                              ctypes.byref(n)), "fsb_sift_features_ex_d")
    return {k: v[:n.value] for k, v in out.items()}


def candidates(pred, A, B, wh_b, radius, kc, device=0):
    """Best guided candidate of every query (before the ratio test): t1 int32 (-1: none),
    b12 float32 (n,2) = (b1, b2). pred: float64 CUDA (na,2) predicted positions in B."""
    import torch
    ctx = _lib.context(device)
    na, nb = len(A["xy"]), len(B["xy"])
    t1 = torch.empty(max(na, 1), dtype=torch.int32, device=pred.device)
    b12 = torch.empty((max(na, 1), 2), dtype=torch.float32, device=pred.device)
    bxy = B["xy"].double().contiguous()
    torch.cuda.current_stream(pred.device).synchronize()
    _lib.check(ctx.lib.fsb_match_guided_cand_d(ctx.handle, _p(pred), _p(A["u8"]), na, _p(bxy), _p(B["u8"]), nb,
                                               float(wh_b[0]), float(wh_b[1]), float(radius),
                                               0 if kc is None else int(kc), _p(t1), _p(b12)),
               "fsb_match_guided_cand_d")
    return t1[:na], b12[:na]


def features(t1, b12, pred, A, B, radius, device=0):
    """(na, 8) float32 CUDA features of the candidates (zeros where t1 < 0)."""
    import torch
    ctx = _lib.context(device)
    n = len(t1)
    feat = torch.empty((max(n, 1), N_FEATURES), dtype=torch.float32, device=t1.device)
    if n:
        _lib.check(ctx.lib.fsb_mlp_features_d(ctx.handle, n, _p(t1), _p(b12), _p(pred), _p(B["xy"]),
                                              _p(A["size"]), _p(A["angle"]), _p(A["resp"]), _p(A["octave"]),
                                              _p(B["size"]), _p(B["angle"]), _p(B["resp"]), float(radius),
                                              _p(feat)), "fsb_mlp_features_d")
    return feat[:n]


def accept(t1, b12, nb, prob=None, threshold=0.5, ratio=0.85, device=0):
    """One-to-one matches (q, t) int64 CUDA, ordered by target: candidates with prob > threshold,
    or (prob None) the ratio test of matching._guided."""
    import torch
    ctx = _lib.context(device)
    n = len(t1)
    q = torch.empty(max(n, 1), dtype=torch.int64, device=t1.device)
    t = torch.empty(max(n, 1), dtype=torch.int64, device=t1.device)
    cnt = ctypes.c_int32()
    _lib.check(ctx.lib.fsb_mlp_filter_d(ctx.handle, n, _p(t1), _p(b12), _p(prob), float(threshold), float(ratio),
                                        int(nb), _p(q), _p(t), ctypes.byref(cnt)), "fsb_mlp_filter_d")
    return q[:cnt.value], t[:cnt.value]


def ransac_labels(xy_a, xy_b, q, t, t1, px=LABEL_PX, reproj=3.0):
    """Labels of the plain pipeline's verification: fit a RANSAC homography (cv2) to the plain
    matches (q, t) and label every candidate (query i, target t1[i]) an inlier when it maps within
    `px` pixels. Host numpy in, (labels float32 (na,), homography or None) out."""
    import cv2
    na = len(t1)
    lab = np.zeros(na, np.float32)
    if len(q) < 8:
        return lab, None
    Hm, _ = cv2.findHomography(xy_a[q].astype(np.float64), xy_b[t].astype(np.float64), cv2.RANSAC, reproj)
    if Hm is None:
        return lab, None
    ok = t1 >= 0
    if ok.any():
        src = np.c_[xy_a[ok].astype(np.float64), np.ones(ok.sum())] @ Hm.T
        proj = src[:, :2] / src[:, 2:3]
        err = np.linalg.norm(proj - xy_b[t1[ok]].astype(np.float64), axis=1)
        lab[np.flatnonzero(ok)] = (err < px).astype(np.float32)
    return lab, Hm


def score(q, labels):
    """(precision, recall, true positives) of accepted queries q against per-query labels."""
    q = np.asarray(q)
    pos = float(labels.sum())
    tp = float(labels[q].sum()) if len(q) else 0.0
    prec = tp / len(q) if len(q) else 0.0
    rec = tp / pos if pos else 0.0
    return prec, rec, tp


class MatchFilter:
    """The 8-64-64-1 network: parameters in one float32 CUDA vector (layout of include/fsb200.h)."""

    def __init__(self, params=None, device=0):
        import torch
        self.device = device
        lib = _lib.load()
        self.n_param = int(lib.fsb_mlp_param_count())
        self.n_train = int(lib.fsb_mlp_trainable_count())
        self.params = None
        if params is not None:
            p = torch.as_tensor(np.asarray(params, np.float32)).to(torch.device("cuda", device))
            if p.numel() != self.n_param:
                raise ValueError("expected %d parameters" % self.n_param)
            self.params = p.contiguous()

    @property
    def trained(self):
        return self.params is not None

    def init(self, feat, seed=0):
        """He-initialised network whose input normalisation is the mean / std of `feat`."""
        import torch
        rng = np.random.default_rng(seed)
        f = feat.double()
        mu = f.mean(0).cpu().numpy()
        sig = f.std(0).cpu().numpy()
        sig = np.where(sig > 1e-6, sig, 1.0)
        h, nf = 64, N_FEATURES
        p = np.zeros(self.n_param, np.float64)
        o = 0
        p[o:o + h * nf] = rng.normal(0, np.sqrt(2.0 / nf), h * nf); o += h * nf + h
        p[o:o + h * h] = rng.normal(0, np.sqrt(2.0 / h), h * h); o += h * h + h
        p[o:o + h] = rng.normal(0, np.sqrt(1.0 / h), h); o += h + 1
        p[o:o + nf] = mu
        p[o + nf:o + 2 * nf] = sig
        self.params = torch.as_tensor(p.astype(np.float32)).to(torch.device("cuda", self.device)).contiguous()

    def fit(self, feat, label, epochs=20, batch=8192, lr=2e-3, seed=0):
        """Mini-batch Adam on the GPU; returns the mean loss of every epoch."""
        import torch
        if self.params is None:
            self.init(feat, seed)
        ctx = _lib.context(self.device)
        dev = self.params.device
        m = torch.zeros(self.n_train, dtype=torch.float32, device=dev)
        v = torch.zeros(self.n_train, dtype=torch.float32, device=dev)
        feat = feat.contiguous()
        label = label.float().contiguous()
        losses = np.zeros(max(epochs, 1), np.float64)
        torch.cuda.current_stream(dev).synchronize()
        _lib.check(ctx.lib.fsb_mlp_train_d(ctx.handle, _p(self.params), _p(m), _p(v), len(label), _p(feat),
                                           _p(label), int(epochs), int(batch), float(lr), int(seed) & 0xffffffff,
                                           _lib.ptr(losses)), "fsb_mlp_train_d")
        return losses[:epochs]

    def predict(self, feat, bf16=True):
        """Inlier probabilities (n,) float32 CUDA; BF16 inference by default."""
        import torch
        ctx = _lib.context(self.device)
        n = len(feat)
        prob = torch.empty(max(n, 1), dtype=torch.float32, device=feat.device)
        torch.cuda.current_stream(feat.device).synchronize()
        _lib.check(ctx.lib.fsb_mlp_infer_d(ctx.handle, _p(self.params), n, _p(feat.contiguous()), 1 if bf16 else 0,
                                           _p(prob)), "fsb_mlp_infer_d")
        return prob[:n]

    def grad(self, feat, label):
        """(mean BCE loss, gradient (trainable count,) float32 CUDA)."""
        import torch
        ctx = _lib.context(self.device)
        g = torch.empty(self.n_train, dtype=torch.float32, device=self.params.device)
        loss = ctypes.c_double()
        torch.cuda.current_stream(feat.device).synchronize()
        _lib.check(ctx.lib.fsb_mlp_grad_d(ctx.handle, _p(self.params), len(label), _p(feat.contiguous()),
                                          _p(label.float().contiguous()), _p(g), ctypes.byref(loss)),
                   "fsb_mlp_grad_d")
        return loss.value, g

    def matches(self, t1, b12, nb, feat=None, threshold=0.5, ratio=0.85, bf16=True):
        """Filtered one-to-one matches; without a trained network (or features) the plain ratio
        test decides (the fallback)."""
        prob = self.predict(feat, bf16) if (self.trained and feat is not None) else None
        return accept(t1, b12, nb, prob, threshold, ratio, self.device)

    def save(self, path):
        np.savez(path, params=self.params.cpu().numpy())

    @classmethod
    def load(cls, path, device=0):
        return cls(np.load(path)["params"], device)


def label_pair(img_a, img_b, H_true, nfeat_a, nfeat_b, noise, radius=40.0, kc=16, ratio=0.85, device=0):
    """One synthetic pair through the plain pipeline: SIFT of both images, prior = true homography
    + `noise` (host (>= na, 2) pixels), guided candidates, features, the plain ratio-test matches
    and their RANSAC labels. Returns a dict (CUDA tensors feat, label, t1, b12; host q_plain,
    label_true: candidates within LABEL_PX of the true homography; nb)."""
    import torch
    dev = torch.device("cuda", device)
    h, w = img_a.shape
    A = extract(torch.as_tensor(img_a).to(dev), nfeat_a, device=device)
    B = extract(torch.as_tensor(img_b).to(dev), nfeat_b, device=device)
    xa = A["xy"].cpu().numpy().astype(np.float64)
    xb = B["xy"].cpu().numpy().astype(np.float64)
    na, nb = len(xa), len(xb)
    src = np.c_[xa, np.ones(na)] @ np.asarray(H_true, np.float64).T
    proj = src[:, :2] / src[:, 2:3]
    pred = torch.as_tensor(proj + np.asarray(noise, np.float64)[:na]).to(dev).contiguous()
    t1, b12 = candidates(pred, A, B, (w, h), radius, kc, device)
    feat = features(t1, b12, pred, A, B, radius, device)
    q, t = accept(t1, b12, nb, None, ratio=ratio, device=device)
    t1h = t1.cpu().numpy()
    lab, Hm = ransac_labels(xa, xb, q.cpu().numpy(), t.cpu().numpy(), t1h)
    ok = t1h >= 0
    true = np.zeros(na, np.float32)
    if ok.any():
        true[ok] = (np.linalg.norm(proj[ok] - xb[t1h[ok]], axis=1) < LABEL_PX).astype(np.float32)
    return {"feat": feat, "label": torch.as_tensor(lab).to(dev), "t1": t1, "b12": b12, "nb": nb,
            "q_plain": q.cpu().numpy(), "label_host": lab, "label_true": true, "has_cand": ok, "H_ransac": Hm}
