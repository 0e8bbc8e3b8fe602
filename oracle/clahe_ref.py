"""CPU oracle: the CLAHE contrast equalisation of features.prepare (app/planesite/features.py:70-71,
cv2.createCLAHE(clipLimit=2.0, tileGridSize=(8, 8)).apply).

TEST INFRASTRUCTURE ONLY (imported by tests/; never by the fieldstitch_b200 package).

OpenCV's CLAHE is a published algorithm (contrast-limited adaptive histogram equalisation) with
OpenCV-specific choices, restated here from its documented behaviour and pinned against OpenCV's
own output (tests/golden/make_clahe.py):
  * tiles: when either side is not a multiple of its tile count, both sides are extended at the far
    edge by reflect-101 (a side that is a multiple by a whole tile);
  * clip at max(int(clip * area / 256), 1) counts; the excess is spread evenly over the 256 bins and
    the remainder one count every max(256 / remainder, 1) bins from bin 0;
  * LUT = round-half-even(float32(cumulative count) * float32(255 / area));
  * output = round-half-even of the float32 blend (a xa1 + b xa) ya1 + (c xa1 + d xa) ya of the
    four nearest tiles' LUT values, xa from x / tile_w - 0.5 (float32, no fused multiply-add).
"""
import numpy as np


def clahe(img, clip=2.0, tiles=(8, 8)):
    img = np.asarray(img, np.uint8)
    H, W = img.shape
    tx, ty = tiles
    src = img
    if W % tx or H % ty:
        src = np.pad(img, ((0, ty - H % ty), (0, tx - W % tx)), mode="reflect")
    tw, th = src.shape[1] // tx, src.shape[0] // ty
    area = tw * th
    lut_scale = np.float32(255.0) / np.float32(area)
    climit = max(int(clip * area / 256), 1) if clip > 0 else 1 << 30
    luts = np.zeros((ty, tx, 256), np.uint8)
    for j in range(ty):
        for i in range(tx):
            h = np.bincount(src[j * th:(j + 1) * th, i * tw:(i + 1) * tw].ravel(), minlength=256).astype(np.int64)
            excess = int(np.maximum(h - climit, 0).sum())
            h = np.minimum(h, climit)
            batch, resid = divmod(excess, 256)
            h += batch
            if resid:
                step = max(256 // resid, 1)
                h[np.arange(0, 256, step)[:resid]] += 1
            v = np.cumsum(h).astype(np.float32) * lut_scale
            luts[j, i] = np.clip(np.rint(v), 0, 255).astype(np.uint8)
    f32 = np.float32
    inv_tw, inv_th = f32(1.0) / f32(tw), f32(1.0) / f32(th)
    txf = np.arange(W, dtype=f32) * inv_tw - f32(0.5)
    tyf = np.arange(H, dtype=f32) * inv_th - f32(0.5)
    tx1, ty1 = np.floor(txf).astype(np.int64), np.floor(tyf).astype(np.int64)
    xa, ya = txf - tx1.astype(f32), tyf - ty1.astype(f32)
    xa1, ya1 = f32(1) - xa, f32(1) - ya
    tx2, tx1 = np.minimum(tx1 + 1, tx - 1), np.maximum(tx1, 0)
    ty2, ty1 = np.minimum(ty1 + 1, ty - 1), np.maximum(ty1, 0)
    out = np.empty_like(img)
    for y in range(H):
        l1, l2, v = luts[ty1[y]], luts[ty2[y]], img[y]
        r1 = l1[tx1, v].astype(f32) * xa1 + l1[tx2, v].astype(f32) * xa
        r2 = l2[tx1, v].astype(f32) * xa1 + l2[tx2, v].astype(f32) * xa
        res = r1 * ya1[y] + r2 * ya[y]
        out[y] = np.clip(np.rint(res), 0, 255).astype(np.uint8)
    return out
