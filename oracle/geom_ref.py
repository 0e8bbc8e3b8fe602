"""CPU oracle: camera geometry of PlaneSite's matching stage.

TEST INFRASTRUCTURE ONLY (imported by tests/; never by the fieldstitch_b200 package).

Restates in NumPy float64, with the reference's operation order:
  undistort_pixels  Brown-Conrady undistortion by 25 fixed-point iterations
                    (app/planesite/camera.py:5-31)
  predict_ground    the ground-plane prior of matching._predict (app/planesite/matching.py:155-172)
"""
import numpy as np


def undistort_normalized(uv, k, iters=25):
    """Pixels (n,2) -> undistorted normalised coordinates; k = f, cx, cy, k1, k2, p1, p2, k3
    (camera.py:5-24). The radial factor is clamped to 0.2 where its magnitude falls below."""
    f, cx, cy, k1, k2, p1, p2, k3 = [float(v) for v in k]
    uv = np.asarray(uv, np.float64).reshape(-1, 2)
    xd = (uv[:, 0] - cx) / f
    yd = (uv[:, 1] - cy) / f
    x, y = xd.copy(), yd.copy()
    if not (k1 == 0 and k2 == 0 and k3 == 0 and p1 == 0 and p2 == 0):
        for _ in range(iters):
            r2 = x * x + y * y
            rad = 1 + k1 * r2 + k2 * r2 * r2 + k3 * r2 * r2 * r2
            rad = np.where(np.abs(rad) < 0.2, 0.2, rad)
            tx = 2 * p1 * x * y + p2 * (r2 + 2 * x * x)
            ty = p1 * (r2 + 2 * y * y) + 2 * p2 * x * y
            x, y = (xd - tx) / rad, (yd - ty) / rad
    return np.c_[x, y]


def undistort_pixels(uv, k):
    """camera.py:27-31: undistorted normalised coordinates back to pixels with the same f, cx, cy."""
    n = undistort_normalized(uv, k)
    return np.c_[n[:, 0] * k[0] + k[1], n[:, 1] * k[0] + k[2]]


def predict_ground(u, K_i, R_i, C_i, K_j, R_j, C_j, zg):
    """matching.py:155-172: ray of each undistorted pixel of image i (world direction R_i^T K_i^-1
    [u 1]), intersected with z = zg, projected by K_j R_j (G - C_j). ok: the plane is hit in front
    of camera i and the point is in front of camera j. Returns (pred (n,2), ok (n,))."""
    u = np.asarray(u, np.float64).reshape(-1, 2)
    rays = np.c_[u, np.ones(len(u))] @ np.linalg.inv(np.asarray(K_i, np.float64)).T
    d = rays @ np.asarray(R_i, np.float64)
    dz = np.where(np.abs(d[:, 2]) < 1e-6, -1e-6, d[:, 2])
    t = (zg - C_i[2]) / dz
    G = np.asarray(C_i, np.float64)[None] + t[:, None] * d
    q = (G - np.asarray(C_j, np.float64)[None]) @ np.asarray(R_j, np.float64).T @ np.asarray(K_j, np.float64).T
    z = q[:, 2]
    ok = (t > 0) & (z > 0)
    z = np.where(np.abs(z) < 1e-9, 1e-9, z)
    return q[:, :2] / z[:, None], ok
