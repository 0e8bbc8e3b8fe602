"""CPU oracle: SIFT detector + descriptor of PlaneSite's ``gsift`` (its NumPy/SciPy path).

TEST INFRASTRUCTURE ONLY. This module is the checker for the CUDA path: it may be imported by
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / reference leg of ``bench.py``,
and never by the ``fieldstitch_b200`` package.

It restates the reference algorithm (app/planesite/gsift.py) with the same float32/float64
arithmetic in the same order, so that its outputs are bit-identical to the reference's CPU path on
the same machine (pinned by tests/test_oracle_golden.py against fixtures produced by running the
reference itself). The structure differs from the reference: octaves are processed one at a time
instead of being packed into one flat atlas, and the refinement loop works per octave.

Float semantics that matter (NumPy 2, NEP 50): Python float scalars combined with float32 arrays
stay float32; ``scipy.ndimage.correlate1d`` accumulates in float64 and rounds once to float32;
``np.bincount`` accumulates weights in float64 in input order.
"""
import math

import numpy as np
import scipy.ndimage as ndi

N_LAYERS = 3          # gsift.py:13
SIGMA = 1.6           # gsift.py:14
INIT_SIGMA = 0.5      # gsift.py:15
BORDER = 5            # gsift.py:16
MAX_INTERP = 5        # gsift.py:17
ORI_BINS = 36         # gsift.py:18
ORI_RADIUS = 4.5      # gsift.py:19
ORI_SIG = 1.5         # gsift.py:20
ORI_PEAK = 0.8        # gsift.py:21
D_WIDTH = 4           # gsift.py:22
D_BINS = 8            # gsift.py:23
D_SCL = 3.0           # gsift.py:24
D_MAG_THR = 0.2       # gsift.py:25
ORI_R_MAX = int(round(ORI_RADIUS * SIGMA * 2.0 ** ((N_LAYERS + 0.5) / N_LAYERS)))   # gsift.py:224 (16)


# ------------------------------------------------------------------------------------------ taps
def gauss_taps(sigma):
    """Normalised Gaussian taps, length round(8*sigma+1)|1, built in float64, stored float32
    (gsift.py:52-56)."""
    n = int(round(sigma * 8 + 1)) | 1
    t = np.arange(n, dtype=np.float64) - (n - 1) / 2.0
    g = np.exp(-t * t / (2 * sigma * sigma))
    return (g / g.sum()).astype(np.float32)


def blur_sigmas():
    """(base sigma, [sigma of layer 1..5 increments]) (gsift.py:59-72)."""
    k = 2.0 ** (1.0 / N_LAYERS)
    inc = []
    for i in range(1, N_LAYERS + 3):
        prev = k ** (i - 1) * SIGMA
        tot = prev * k
        inc.append(math.sqrt(tot * tot - prev * prev))
    base = math.sqrt(max(SIGMA * SIGMA - (2 * INIT_SIGMA) ** 2, 0.01))
    return base, inc


def all_taps():
    base, inc = blur_sigmas()
    return gauss_taps(base), [gauss_taps(s) for s in inc]


# --------------------------------------------------------------------------------------- pyramid
def blur(img, taps):
    """Separable correlation, rows axis first then columns, mirror (reflect-101) borders
    (gsift.py:85-87)."""
    t = ndi.correlate1d(img, taps, axis=0, mode="mirror")
    return ndi.correlate1d(t, taps, axis=1, mode="mirror")


def upsample2(a):
    """2x bilinear, pixel-centre aligned, clamped edges; weights 0.75/0.25 in float32, first along
    rows then along columns (gsift.py:90-102)."""
    def rows(x):
        up = np.concatenate([x[:1], x[:-1]], axis=0)
        dn = np.concatenate([x[1:], x[-1:]], axis=0)
        out = np.empty((2 * x.shape[0], x.shape[1]), np.float32)
        out[0::2] = 0.75 * x + 0.25 * up
        out[1::2] = 0.75 * x + 0.25 * dn
        return out
    return np.ascontiguousarray(rows(np.ascontiguousarray(rows(a).T)).T)


def n_octaves(shape):
    """Octave budget (gsift.py:167); the loop also stops when an octave is smaller than
    2*BORDER+4 (gsift.py:171)."""
    return max(1, int(round(math.log2(min(shape)) - 2)) + 1)


def build_pyramid(gray):
    """Returns a list of octaves; each is dict(gauss=[6 layers], dog=(5,R,C) float32)
    (gsift.py:158-179)."""
    base_taps, inc_taps = all_taps()
    img = np.asarray(gray, dtype=np.float32) * (1.0 / 255.0)
    cur = blur(upsample2(img), base_taps)
    octs = []
    for _ in range(n_octaves(gray.shape)):
        if min(cur.shape) < 2 * BORDER + 4:
            break
        g = [cur]
        for tp in inc_taps:
            g.append(blur(g[-1], tp))
        dog = np.stack([g[i + 1] - g[i] for i in range(N_LAYERS + 2)])
        octs.append({"gauss": g, "dog": dog})
        cur = g[N_LAYERS][::2, ::2]
    return octs


def gradients(oct_):
    """Magnitude and angle (degrees in [0,360)) of gauss layers 1..3, zero on the one-pixel
    border (gsift.py:256-267). Returns (3,R,C) float32 arrays."""
    G = np.stack(oct_["gauss"][1:N_LAYERS + 1])
    dx = np.zeros_like(G)
    dy = np.zeros_like(G)
    dx[:, 1:-1, 1:-1] = G[:, 1:-1, 2:] - G[:, 1:-1, :-2]
    dy[:, 1:-1, 1:-1] = G[:, :-2, 1:-1] - G[:, 2:, 1:-1]
    mag = np.sqrt(dx * dx + dy * dy)
    ang = np.degrees(np.arctan2(dy, dx))
    return mag, np.where(ang < 0, ang + 360.0, ang)


# ------------------------------------------------------------------------------ extrema + refine
def extrema(dog, contrast):
    """(l, r, c) int64 of 3x3x3 extrema of DoG layers 1..3 inside BORDER, ties included, beyond
    +-0.8*0.5*contrast/3 (gsift.py:293-319). Order: layer, row, column (flat index order)."""
    thr = 0.8 * 0.5 * contrast / N_LAYERS
    L, R, C = dog.shape
    core = dog[1:L - 1, BORDER:R - BORDER, BORDER:C - BORDER]
    hi = np.full(core.shape, -np.inf, np.float32)
    lo = np.full(core.shape, np.inf, np.float32)
    for dl in (-1, 0, 1):
        for dr in (-1, 0, 1):
            for dc in (-1, 0, 1):
                nb = dog[1 + dl:L - 1 + dl, BORDER + dr:R - BORDER + dr, BORDER + dc:C - BORDER + dc]
                hi = np.maximum(hi, nb)
                lo = np.minimum(lo, nb)
    keep = ((core >= hi) & (core > thr)) | ((core <= lo) & (core < -thr))
    l, r, c = np.nonzero(keep)
    return l + 1, r + BORDER, c + BORDER


def _local_fit(dog, l, r, c):
    """Value, gradient and Hessian of the DoG at integer voxels, float32, same operation order as
    gsift.py:274-290."""
    D = dog
    v = D[l, r, c]
    xp1, xm1 = D[l, r, c + 1], D[l, r, c - 1]
    yp1, ym1 = D[l, r + 1, c], D[l, r - 1, c]
    sp1, sm1 = D[l + 1, r, c], D[l - 1, r, c]
    grad = np.stack([(xp1 - xm1) * 0.5, (yp1 - ym1) * 0.5, (sp1 - sm1) * 0.5], 1)
    dxx = xp1 + xm1 - 2 * v
    dyy = yp1 + ym1 - 2 * v
    dss = sp1 + sm1 - 2 * v
    dxy = (D[l, r + 1, c + 1] - D[l, r + 1, c - 1] - D[l, r - 1, c + 1] + D[l, r - 1, c - 1]) * 0.25
    dxs = (D[l + 1, r, c + 1] - D[l + 1, r, c - 1] - D[l - 1, r, c + 1] + D[l - 1, r, c - 1]) * 0.25
    dys = (D[l + 1, r + 1, c] - D[l + 1, r - 1, c] - D[l - 1, r + 1, c] + D[l - 1, r - 1, c]) * 0.25
    return v, grad, (dxx, dyy, dss, dxy, dxs, dys)


def _solve3(h, g):
    """x = H^-1 g for the symmetric 3x3 H = [[xx xy xs][xy yy ys][xs ys ss]] by the adjugate, as
    gsift.py:182-198 (float32, sums left to right)."""
    dxx, dyy, dss, dxy, dxs, dys = h
    a, b, c = dxx, dxy, dxs
    d, e, f = dxy, dyy, dys
    gg, hh, i = dxs, dys, dss
    A = e * i - f * hh
    B = -(d * i - f * gg)
    C = d * hh - e * gg
    det = a * A + b * B + c * C
    ok = np.abs(det) > 1e-20
    det = np.where(ok, det, 1.0)
    rows = ((A, -(b * i - c * hh), b * f - c * e),
            (B, a * i - c * gg, -(a * f - c * d)),
            (C, -(a * hh - b * gg), a * e - b * d))
    g0, g1, g2 = g[:, 0], g[:, 1], g[:, 2]
    x = np.stack([(r0 / det) * g0 + (r1 / det) * g1 + (r2 / det) * g2 for r0, r1, r2 in rows], 1)
    return x, ok


def refine(dog, l, r, c, contrast, edge):
    """Sub-pixel refinement, contrast and edge tests (gsift.py:322-369). Returns a boolean keep
    mask and refined (l, r, c, X float32 (n,3), response float32) for the kept entries."""
    L, R, C = dog.shape
    n = l.size
    alive = np.ones(n, bool)
    done = np.zeros(n, bool)
    X = np.zeros((n, 3), np.float32)
    l, r, c = l.copy(), r.copy(), c.copy()
    for _ in range(MAX_INTERP):
        _, g, h = _local_fit(dog, l, r, c)
        x, ok = _solve3(h, g)
        x = -x
        alive &= ok
        conv = (np.abs(x) < 0.5).all(1)
        fresh = alive & ~done & conv
        X = np.where(fresh[:, None], x, X)
        done |= fresh
        moving = alive & ~done
        alive &= ~(moving & (np.abs(x) > 1e6).any(1))
        moving = alive & ~done
        with np.errstate(invalid="ignore"):
            step = np.rint(np.where(moving[:, None], x, 0)).astype(np.int64)
        c = c + step[:, 0]
        r = r + step[:, 1]
        l = l + step[:, 2]
        alive &= (l >= 1) & (l <= N_LAYERS) & (c >= BORDER) & (c < C - BORDER) & (r >= BORDER) & (r < R - BORDER)
        l = np.clip(l, 1, N_LAYERS)
        r = np.clip(r, BORDER, R - BORDER - 1)
        c = np.clip(c, BORDER, C - BORDER - 1)
    v, g, h = _local_fit(dog, l, r, c)
    dxx, dyy, _, dxy, _, _ = h
    contr = v + 0.5 * (g * X).sum(1)
    tr = dxx + dyy
    det = dxx * dyy - dxy * dxy
    keep = alive & done & (np.abs(contr) * N_LAYERS >= contrast) & (det > 0) & \
        (tr * tr * edge < (edge + 1) ** 2 * det)
    return keep, l[keep], r[keep], c[keep], X[keep], np.abs(contr[keep])


# --------------------------------------------------------------------------------- orientation
def orientation_hist(mag, ang, l, r, c, scl):
    """Raw 36-bin histograms (n,36) float32: Gaussian weight exp(-d2/(2*(1.5 scl)^2)) over the
    square window |i|,|j| <= min(rint(4.5 scl),16), interior pixels only, bin rint(ang*0.1) mod 36,
    summed in float64 in window row-major order (gsift.py:382-408)."""
    n = r.size
    R, C = mag.shape[1:]
    off = np.arange(-ORI_R_MAX, ORI_R_MAX + 1, dtype=np.int64)
    oi = np.repeat(off, off.size)[None]
    oj = np.tile(off, off.size)[None]
    d2 = (oi * oi + oj * oj).astype(np.float32)
    rad = np.rint(ORI_RADIUS * scl).astype(np.int64)[:, None]
    y = r[:, None] + oi
    x = c[:, None] + oj
    valid = (np.abs(oi) <= rad) & (np.abs(oj) <= rad) & (y > 0) & (y < R - 1) & (x > 0) & (x < C - 1)
    y = np.clip(y, 0, R - 1)
    x = np.clip(x, 0, C - 1)
    li = (l - 1)[:, None]
    sw = ORI_SIG * scl
    w = np.exp(-d2 / (2.0 * sw[:, None] ** 2))
    m = mag[li, y, x] * w * valid
    b = np.rint(ang[li, y, x] * (ORI_BINS / 360.0)).astype(np.int64) % ORI_BINS
    idx = (np.arange(n, dtype=np.int64)[:, None] * ORI_BINS + b).ravel()
    return np.bincount(idx, weights=m.ravel(), minlength=n * ORI_BINS).astype(np.float32).reshape(n, ORI_BINS)


def orientation_peaks(hist):
    """Smoothed-histogram peaks (gsift.py:415-432): returns (row index, angle float32). Smoothing
    [1,4,6,4,1]/16 circular in float32; peaks above both neighbours and >= 0.8 max; parabolic
    refinement (the bin offset is float32, the bin position and angle float64)."""
    sh = lambda k: np.roll(hist, k, 1)   # noqa: E731
    h = (sh(2) + sh(-2)) * (1.0 / 16) + (sh(1) + sh(-1)) * (4.0 / 16) + hist * (6.0 / 16)
    top = h.max(1, keepdims=True)
    left = np.roll(h, 1, 1)
    right = np.roll(h, -1, 1)
    pk = (h > left) & (h > right) & (h >= ORI_PEAK * top) & (top > 0)
    row, j = np.nonzero(pk)
    hl, hc, hr = left[row, j], h[row, j], right[row, j]
    den = hl - 2 * hc + hr
    den = np.where(np.abs(den) < 1e-12, -1e-12, den)
    pos = j + 0.5 * (hl - hr) / den
    pos = np.where(pos < 0, pos + ORI_BINS, pos)
    pos = np.where(pos >= ORI_BINS, pos - ORI_BINS, pos)
    angle = 360.0 - (360.0 / ORI_BINS) * pos
    angle = np.where(np.abs(angle - 360.0) < 1e-4, 0.0, angle)
    return row, angle.astype(np.float32)


# ---------------------------------------------------------------------------------------- detect
class State:
    """What describe() needs from detect(): per octave (R, C, mag, ang)."""

    def __init__(self, octs):
        self.shapes = [o["dog"].shape[1:] for o in octs]
        self.grads = [gradients(o) for o in octs]


def detect(gray, max_kp=12000, contrast=0.015, edge=12.0):
    """Oriented keypoints, strongest first (gsift.py:435-477). Returns (dict of arrays x, y, size,
    angle, response (float32), octave, layer (int32); State)."""
    octs = build_pyramid(gray)
    st = State(octs)
    per = []
    for o, oc in enumerate(octs):
        dog = oc["dog"]
        l, r, c = extrema(dog, contrast)
        if l.size == 0:
            continue
        keep, l, r, c, X, resp = refine(dog, l, r, c, contrast, edge)
        if l.size == 0:
            continue
        scl = SIGMA * 2.0 ** ((l.astype(np.float32) + X[:, 2]) / N_LAYERS)
        mag, ang = st.grads[o]
        kp, angle = orientation_peaks(orientation_hist(mag, ang, l, r, c, scl))
        f = np.float32(2.0 ** np.float32(o)) * 0.5
        per.append({
            "x": (c[kp].astype(np.float32) + X[kp, 0]) * f,
            "y": (r[kp].astype(np.float32) + X[kp, 1]) * f,
            "size": scl[kp] * 2 * f,
            "angle": angle,
            "response": resp[kp],
            "octave": np.full(kp.size, o, np.int32),
            "layer": l[kp].astype(np.int32),
        })
    keys = ("x", "y", "size", "angle", "response", "octave", "layer")
    if not per:
        return {k: np.zeros(0, np.float32) for k in keys}, st
    cat = {k: np.concatenate([p[k] for p in per]) for k in keys}
    order = np.argsort(-cat["response"], kind="stable")[:max_kp]
    return {k: v[order] for k, v in cat.items()}, st


# -------------------------------------------------------------------------------------- describe
def describe(st, kps, sel):
    """128-d descriptors (float32, L2 norm 512, OpenCV scaling, not rounded) for kps[sel]
    (gsift.py:480-525, 800-871): keypoint geometry in float64, rotated 4x4 spatial x 8 angle
    trilinear histogram over a 6x6x10 padded grid summed in float64, angle wrap fold, L2 clip at
    0.2 and renormalisation in float32."""
    sel = np.asarray(sel, np.int64)
    n = len(sel)
    out = np.zeros((n, D_WIDTH * D_WIDTH * D_BINS), np.float32)
    if n == 0:
        return out
    o = kps["octave"][sel].astype(np.int64)
    li = kps["layer"][sel].astype(np.int64)
    f = 1.0 / (2.0 ** o * 0.5)
    px = kps["x"][sel] * f
    py = kps["y"][sel] * f
    scl = kps["size"][sel] * f * 0.5
    ori = 360.0 - kps["angle"][sel]
    ori = np.where(np.abs(ori - 360.0) < 1e-4, 0.0, ori)
    shp = np.array(st.shapes, np.int64)
    rows, cols = shp[o, 0], shp[o, 1]
    rad = np.rint(D_SCL * scl * 1.4142135623730951 * (D_WIDTH + 1) * 0.5).astype(np.int64)
    rad = np.minimum(rad, np.sqrt(rows * rows + cols * cols).astype(np.int64))
    for k in range(n):
        out[k] = _descr_one(st.grads[o[k]], li[k], px[k], py[k], scl[k], ori[k], rad[k], rows[k], cols[k])
    return out


def _descr_one(grad, li, px, py, scl, ori, rad, rows, cols):
    d, nb = D_WIDTH, D_BINS
    mag, ang = grad[0][li - 1], grad[1][li - 1]
    off = np.arange(-rad, rad + 1, dtype=np.float32)
    oi = np.repeat(off, off.size)
    oj = np.tile(off, off.size)
    hw = D_SCL * scl
    t = np.radians(ori)
    cos_t = np.cos(t) / hw
    sin_t = np.sin(t) / hw
    c_rot = oj * cos_t - oi * sin_t
    r_rot = oj * sin_t + oi * cos_t
    rbin = r_rot + d / 2.0 - 0.5
    cbin = c_rot + d / 2.0 - 0.5
    y = np.int64(np.rint(py)) + oi.astype(np.int64)
    x = np.int64(np.rint(px)) + oj.astype(np.int64)
    ok = (rbin > -1) & (rbin < d) & (cbin > -1) & (cbin < d) & (y > 0) & (y < rows - 1) & (x > 0) & (x < cols - 1)
    y = np.clip(y, 0, rows - 1)
    x = np.clip(x, 0, cols - 1)
    w = np.exp((c_rot * c_rot + r_rot * r_rot) * (-1.0 / (d * d * 0.5)))
    m = mag[y, x] * w * ok
    obin = (ang[y, x] - ori) * (nb / 360.0)
    r0, c0, o0 = np.floor(rbin), np.floor(cbin), np.floor(obin)
    rb, cb, ob = rbin - r0, cbin - c0, obin - o0
    o0 = o0.astype(np.int64)
    o0 = np.where(o0 < 0, o0 + nb, o0)
    o0 = np.where(o0 >= nb, o0 - nb, o0)
    r0 = r0.astype(np.int64)
    c0 = c0.astype(np.int64)
    # trilinear split of m into the 8 neighbouring cells (same subtraction order as the reference)
    v_r1 = m * rb
    v_r0 = m - v_r1
    v_rc11 = v_r1 * cb
    v_rc10 = v_r1 - v_rc11
    v_rc01 = v_r0 * cb
    v_rc00 = v_r0 - v_rc01
    parts = []
    for v in (v_rc00, v_rc01, v_rc10, v_rc11):
        hi = v * ob
        parts.append((v - hi, hi))
    s1, s2 = nb + 2, (d + 2) * (nb + 2)
    base = ((r0 + 1) * (d + 2) + c0 + 1) * (nb + 2) + o0
    base = np.where(ok, base, 0)
    # contribution order of the reference: (000, 001, 010, 011, 100, 101, 110, 111) blocks
    idx = np.concatenate([base, base + 1, base + s1, base + s1 + 1,
                          base + s2, base + s2 + 1, base + s2 + s1, base + s2 + s1 + 1])
    val = np.concatenate([parts[0][0], parts[0][1], parts[1][0], parts[1][1],
                          parts[2][0], parts[2][1], parts[3][0], parts[3][1]])
    hist = np.bincount(idx, weights=val, minlength=s2 * (d + 2)).astype(np.float32).reshape(d + 2, d + 2, nb + 2)
    hist[..., 0] += hist[..., nb]
    hist[..., 1] += hist[..., nb + 1]
    dst = hist[1:d + 1, 1:d + 1, :nb].reshape(1, d * d * nb)
    nrm = np.sqrt((dst * dst).sum(1, keepdims=True))
    dst = np.minimum(dst, nrm * D_MAG_THR)
    nrm = np.sqrt((dst * dst).sum(1, keepdims=True))
    return (dst * (512.0 / np.maximum(nrm, 1e-7)))[0]
