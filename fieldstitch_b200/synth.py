"""Seeded synthetic inputs for the SIFT + guided-matching workloads.

Nothing here is measured: these functions only build inputs with the shapes, sizes and value
distributions of the benchmark workloads (no public dataset is involved).

* ``synth_image``: sum of random Gaussian blobs (sigma 2-30 px, signed amplitudes up to 255) plus
  1/f band-limited noise, rescaled to uint8 [0, 255].
* ``random_homography`` / ``warp_pair``: image B = A warped by a random homography (rotation
  +-10 deg, scale 0.9-1.1, translation +-200 px about the image centre) plus Gaussian noise
  (sigma 3), clipped to uint8.
* ``synth_descriptors``: SIFT-like 128-d uint8 descriptors (non-negative Gamma(0.6) draws,
  L2-normalised, clipped at 0.2, renormalised, x512, rounded and saturated) with a fraction of
  the B rows being copies of A rows with +-4 byte noise.
"""
import math

import numpy as np


def _blob_field(rng, h, w, n_blobs):
    img = np.zeros((h, w), np.float32)
    ys = rng.uniform(0, h, n_blobs)
    xs = rng.uniform(0, w, n_blobs)
    sig = rng.uniform(2.0, 30.0, n_blobs)
    amp = rng.uniform(-255.0, 255.0, n_blobs)
    for y, x, s, a in zip(ys, xs, sig, amp):
        r = int(math.ceil(3.5 * s))
        y0, y1 = max(0, int(y) - r), min(h, int(y) + r + 1)
        x0, x1 = max(0, int(x) - r), min(w, int(x) + r + 1)
        if y0 >= y1 or x0 >= x1:
            continue
        gy = np.exp(-((np.arange(y0, y1, dtype=np.float32) - y) ** 2) / (2 * s * s))
        gx = np.exp(-((np.arange(x0, x1, dtype=np.float32) - x) ** 2) / (2 * s * s))
        img[y0:y1, x0:x1] += np.float32(a) * gy[:, None] * gx[None, :]
    return img


def _pink_noise(rng, h, w, fmin=1.0 / 512, fmax=0.45):
    white = rng.standard_normal((h, w)).astype(np.float32)
    spec = np.fft.rfft2(white)
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.rfftfreq(w)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    band = (f >= fmin) & (f <= fmax)
    scale = np.where(band, 1.0 / np.maximum(f, fmin), 0.0)
    out = np.fft.irfft2(spec * scale, s=(h, w)).astype(np.float32)
    return out / max(float(out.std()), 1e-6)


def synth_image(h, w, seed, n_blobs=400, noise_weight=0.6):
    """uint8 (h, w) image: Gaussian blobs + 1/f band-limited noise, rescaled so that the 0.5 and
    99.5 percentiles map to 0 and 255 (clipped)."""
    rng = np.random.default_rng(seed)
    blobs = _blob_field(rng, h, w, n_blobs)
    bs = float(blobs.std()) or 1.0
    img = blobs / bs + np.float32(noise_weight) * _pink_noise(rng, h, w)
    lo, hi = (float(v) for v in np.percentile(img[::4, ::4], [0.5, 99.5]))
    img = (img - lo) * (255.0 / max(hi - lo, 1e-6))
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def random_homography(rng, h, w, rot_deg=10.0, scale=(0.9, 1.1), shift=200.0):
    """3x3 float64 homography: rotation and scale about the image centre, then a translation."""
    th = math.radians(rng.uniform(-rot_deg, rot_deg))
    s = rng.uniform(*scale)
    tx, ty = rng.uniform(-shift, shift, 2)
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    c, si = math.cos(th) * s, math.sin(th) * s
    to_c = np.array([[1, 0, -cx], [0, 1, -cy], [0, 0, 1]], np.float64)
    rs = np.array([[c, -si, 0], [si, c, 0], [0, 0, 1]], np.float64)
    back = np.array([[1, 0, cx + tx], [0, 1, cy + ty], [0, 0, 1]], np.float64)
    return back @ rs @ to_c


def warp_pair(img, rng, noise_sigma=3.0, **hkw):
    """Returns (B, H): B = img warped by a random homography H (A pixel -> B pixel) + noise."""
    import cv2
    h, w = img.shape
    H = random_homography(rng, h, w, **hkw)
    warped = cv2.warpPerspective(img, H, (w, h), flags=cv2.INTER_LINEAR, borderMode=cv2.BORDER_REFLECT_101)
    noisy = warped.astype(np.float32) + rng.normal(0.0, noise_sigma, warped.shape).astype(np.float32)
    return np.clip(np.rint(noisy), 0, 255).astype(np.uint8), H


def synth_pair(h, w, seed):
    """(A, B, H) image pair from one seed."""
    a = synth_image(h, w, seed)
    rng = np.random.default_rng(seed + 7919)
    b, H = warp_pair(a, rng)
    return a, b, H


def flight_pair(args):
    """One pair of the batched guided-matching workload: (A, B, H, nfeat_A, nfeat_B) for
    (h, w, seed). Keypoint caps are drawn uniformly from [2000, 16000]."""
    h, w, seed = args
    a, b, H = synth_pair(h, w, seed)
    rng = np.random.default_rng(seed + 104729)
    na, nb = (int(v) for v in rng.integers(2000, 16001, 2))
    return a, b, H, na, nb


def prior_noise(n, seed, sigma=15.0):
    """Gaussian prior error (n, 2) float32 in pixels (GNSS/gimbal prior sigma)."""
    return np.random.default_rng(seed + 1299709).normal(0.0, sigma, (n, 2)).astype(np.float32)


def apply_homography(H, xy):
    """Project (n, 2) points by a 3x3 homography (float64)."""
    xy = np.asarray(xy, np.float64)
    p = np.c_[xy, np.ones(len(xy))] @ np.asarray(H, np.float64).T
    return p[:, :2] / p[:, 2:3]


def _sift_like(rng, n, d=128):
    v = rng.gamma(0.6, 1.0, (n, d)).astype(np.float32)
    v /= np.maximum(np.linalg.norm(v, axis=1, keepdims=True), 1e-12)
    v = np.minimum(v, 0.2)
    v /= np.maximum(np.linalg.norm(v, axis=1, keepdims=True), 1e-12)
    return np.clip(np.rint(v * 512.0), 0, 255).astype(np.uint8)


def synth_descriptors(na, nb, seed, true_frac=0.3, noise=4):
    """(A u8 (na,128), B u8 (nb,128), truth) where truth[j] = A row copied into B row j, or -1."""
    rng = np.random.default_rng(seed)
    a = _sift_like(rng, na)
    b = _sift_like(rng, nb)
    n_true = int(round(true_frac * min(na, nb)))
    rows_b = rng.choice(nb, n_true, replace=False)
    rows_a = rng.choice(na, n_true, replace=False)
    jitter = rng.integers(-noise, noise + 1, (n_true, a.shape[1]))
    b[rows_b] = np.clip(a[rows_a].astype(np.int32) + jitter, 0, 255).astype(np.uint8)
    truth = np.full(nb, -1, np.int64)
    truth[rows_b] = rows_a
    return a, b, truth


def synth_descriptors_device(na, nb, seed, device=0, true_frac=0.3, noise=4):
    """``synth_descriptors`` drawn on the GPU with torch (same distribution: gamma(0.6) magnitudes,
    L2-normalised, clipped at 0.2, renormalised, x512 rounded to uint8; a ``true_frac`` share of B
    rows are copies of A rows with uniform +-noise byte jitter). Returns (A, B, truth) CUDA tensors;
    for benchmark batches too large to draw on the host."""
    import torch
    dev = torch.device("cuda", device)
    with torch.random.fork_rng(devices=[dev]):
        torch.manual_seed(seed)

        def sift_like(n):
            v = torch._standard_gamma(torch.full((n, 128), 0.6, device=dev))
            v = v / v.norm(dim=1, keepdim=True).clamp_min(1e-12)
            v = v.clamp_max(0.2)
            v = v / v.norm(dim=1, keepdim=True).clamp_min(1e-12)
            return torch.round(v * 512.0).clamp(0, 255).to(torch.uint8)

        a = sift_like(na)
        b = sift_like(nb)
        n_true = int(round(true_frac * min(na, nb)))
        rows_b = torch.randperm(nb, device=dev)[:n_true]
        rows_a = torch.randperm(na, device=dev)[:n_true]
        jitter = torch.randint(-noise, noise + 1, (n_true, 128), device=dev, dtype=torch.int32)
        b[rows_b] = (a[rows_a].to(torch.int32) + jitter).clamp(0, 255).to(torch.uint8)
        truth = torch.full((nb,), -1, dtype=torch.int64, device=dev)
        truth[rows_b] = rows_a
    return a.contiguous(), b.contiguous(), truth


# --------------------------------------------------------------------------- synthetic flight
# One seeded procedural terrain texture, nadir frames cropped from it along a lawnmower grid, the
# true frame-to-frame homographies and the GNSS neighbour pair list of the reference's pipeline.

def flight_terrain(seed, h=16000, w=20000, device=0):
    """uint8 (h, w) CUDA tensor: the terrain texture of the synthetic flight, drawn on the GPU with
    torch: Gaussian blobs at three scales (impulses convolved in the frequency domain, sigma 4, 14
    and 40 px) plus 1/f band-limited noise, rescaled so that the 0.5 and 99.5 percentiles map to 0
    and 255."""
    import torch
    dev = torch.device("cuda", device)
    g = torch.Generator(device=dev).manual_seed(int(seed))
    fy = torch.fft.fftfreq(h, device=dev)[:, None]
    fx = torch.fft.rfftfreq(w, device=dev)[None, :]
    f2 = fx * fx + fy * fy
    # 1/f noise in the band [1/1024, 0.45] cycles per pixel
    spec = torch.fft.rfft2(torch.randn((h, w), generator=g, device=dev))
    f = torch.sqrt(f2)
    spec *= torch.where((f >= 1.0 / 1024) & (f <= 0.45), 1.0 / torch.clamp(f, min=1.0 / 1024), torch.zeros_like(f))
    noise = torch.fft.irfft2(spec, s=(h, w))
    del spec
    noise /= noise.std().clamp_min(1e-6)
    # blobs: about one per 13 000 px at each scale, signed amplitudes
    blobs = torch.zeros((h, w), device=dev)
    for sigma in (4.0, 14.0, 40.0):
        n = int(h * w / 13000)
        imp = torch.zeros((h, w), device=dev)
        ys = torch.randint(0, h, (n,), generator=g, device=dev)
        xs = torch.randint(0, w, (n,), generator=g, device=dev)
        amp = torch.rand((n,), generator=g, device=dev) * 2.0 - 1.0
        imp.index_put_((ys, xs), amp, accumulate=True)
        sp = torch.fft.rfft2(imp)
        sp *= torch.exp(-2.0 * (torch.pi ** 2) * sigma * sigma * f2) * (2.0 * torch.pi * sigma * sigma)
        blobs += torch.fft.irfft2(sp, s=(h, w))
        del imp, sp
    img = blobs / blobs.std().clamp_min(1e-6) + 0.6 * noise
    del blobs, noise
    lo, hi = torch.quantile(img[::8, ::8].reshape(-1)[:16_000_000], torch.tensor([0.005, 0.995], device=dev))
    img = (img - lo) * (255.0 / float(max(hi - lo, 1e-6)))
    return torch.clamp(torch.round(img), 0, 255).to(torch.uint8)


def lawnmower(seed, lines=20, per_line=20, W=2640, H=1978, forward=0.8, side=0.7, margin=200.0,
              yaw_deg=3.0, scale_jitter=0.02):
    """Frame poses of a serpentine lawnmower flight over the terrain: (n, 4) float64 rows (cx, cy,
    yaw in radians, scale) in terrain pixels, flight lines along the terrain's y axis (the frames'
    short side along track) with the given forward / side overlap, the return lines flown with
    the heading turned by 180 deg, each frame with uniform +-yaw_deg yaw and +-scale_jitter scale."""
    rng = np.random.default_rng(seed)
    step_y, step_x = (1.0 - forward) * H, (1.0 - side) * W
    out = []
    for l in range(lines):
        ks = range(per_line) if l % 2 == 0 else range(per_line - 1, -1, -1)
        for k in ks:
            cx = margin + W / 2.0 + step_x * l
            cy = margin + H / 2.0 + step_y * k
            yaw = math.radians(rng.uniform(-yaw_deg, yaw_deg)) + (0.0 if l % 2 == 0 else math.pi)
            out.append((cx, cy, yaw, 1.0 + rng.uniform(-scale_jitter, scale_jitter)))
    return np.array(out, np.float64)


def frame_to_terrain(pose, W=2640, H=1978):
    """3x3 map of frame pixels to terrain pixels for pose (cx, cy, yaw, scale)."""
    cx, cy, yaw, s = pose
    c, si = math.cos(yaw) * s, math.sin(yaw) * s
    return np.array([[c, -si, cx - c * (W - 1) / 2.0 + si * (H - 1) / 2.0],
                     [si, c, cy - si * (W - 1) / 2.0 - c * (H - 1) / 2.0],
                     [0.0, 0.0, 1.0]])


def frame_homography(pose_i, pose_j, W=2640, H=1978):
    """The true homography of frame i pixels to frame j pixels."""
    return np.linalg.inv(frame_to_terrain(pose_j, W, H)) @ frame_to_terrain(pose_i, W, H)


def render_frames(terrain, poses, W=2640, H=1978, noise_sigma=2.0, seed=0):
    """(n, H, W) uint8 CUDA tensor: each frame the terrain resampled (bilinear) at its pose, plus
    Gaussian noise, rounded and clipped."""
    import torch
    dev = terrain.device
    th, tw = terrain.shape
    src = terrain.to(torch.float32)[None, None]
    g = torch.Generator(device=dev).manual_seed(int(seed) + 17)
    v, u = torch.meshgrid(torch.arange(H, device=dev, dtype=torch.float64),
                          torch.arange(W, device=dev, dtype=torch.float64), indexing="ij")
    out = torch.empty((len(poses), H, W), dtype=torch.uint8, device=dev)
    for k, pose in enumerate(poses):
        M = torch.tensor(frame_to_terrain(pose, W, H), device=dev)
        x = M[0, 0] * u + M[0, 1] * v + M[0, 2]
        y = M[1, 0] * u + M[1, 1] * v + M[1, 2]
        # align_corners=True: -1 and 1 are the centres of the first and last terrain pixels
        grid = torch.stack((x / (tw - 1) * 2 - 1, y / (th - 1) * 2 - 1), -1).to(torch.float32)[None]
        fr = torch.nn.functional.grid_sample(src, grid, mode="bilinear", padding_mode="border", align_corners=True)[0, 0]
        fr += noise_sigma * torch.randn(fr.shape, generator=g, device=dev)
        out[k] = torch.clamp(torch.round(fr), 0, 255).to(torch.uint8)
    return out


def gnss_pairs(centers, W=2640, H=1978, neighbors=16, sigma=0.0, seed=0):
    """Candidate pairs of the reference's pipeline (app/planesite/pipeline.py:452-476) from frame
    positions (GNSS, here the frame centres plus N(0, sigma) noise, in terrain pixels at unit
    scale): the `neighbors` nearest frames within 2 x 0.95 x half the long footprint side, plus the
    next two frames in flight order when within twice that half side. Sorted (i < j) list."""
    from scipy.spatial import cKDTree
    xy = np.asarray(centers, np.float64)[:, :2]
    if sigma > 0:
        xy = xy + np.random.default_rng(seed).normal(0.0, sigma, xy.shape)
    n = len(xy)
    tree = cKDTree(xy)
    k = min(n - 1, neighbors)
    dists, nbrs = tree.query(xy, k=k + 1)
    half_long = max(W, H) / 2.0
    pairs = set()
    for i in range(n):
        for d, j in zip(dists[i][1:], nbrs[i][1:]):
            if j < n and d < 2 * half_long * 0.95:
                pairs.add((min(i, int(j)), max(i, int(j))))
    for i in range(n - 1):
        for off in (1, 2):
            j = i + off
            if j < n and np.hypot(*(xy[i] - xy[j])) < 2 * half_long:
                pairs.add((i, j))
    return sorted(pairs)
