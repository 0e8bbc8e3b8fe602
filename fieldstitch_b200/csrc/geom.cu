// Camera geometry of the matching stage, float64 on the device:
//   k_undistort  Brown-Conrady undistortion of keypoint pixels (app/planesite/camera.py:5-31):
//                25 fixed-point iterations, the reference's expression order; compiled with
//                --fmad=false so every operation rounds once, as NumPy's float64 does.
//   k_predict    the ground-plane prior of app/planesite/matching.py:155-172: the ray of an
//                undistorted pixel of image i, intersected with the plane z = zg, projected into
//                image j. The 3x3 products are summed left to right (NumPy's BLAS may group
//                them differently, so the prediction agrees to rounding, not bit for bit).
#include "fsb_internal.cuh"

namespace fsb {
namespace {

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

struct Cam8 {
    double f, cx, cy, k1, k2, p1, p2, k3;
};

__global__ void k_undistort(const double* __restrict__ uv, int n, Cam8 k, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double xd = (uv[2 * i] - k.cx) / k.f;
    const double yd = (uv[2 * i + 1] - k.cy) / k.f;
    double x = xd, y = yd;
    if (!(k.k1 == 0.0 && k.k2 == 0.0 && k.k3 == 0.0 && k.p1 == 0.0 && k.p2 == 0.0)) {
        for (int it = 0; it < 25; ++it) {
            const double r2 = x * x + y * y;
            double rad = 1.0 + k.k1 * r2 + k.k2 * r2 * r2 + k.k3 * r2 * r2 * r2;
            if (fabs(rad) < 0.2) rad = 0.2;
            const double dx = 2.0 * k.p1 * x * y + k.p2 * (r2 + 2.0 * x * x);
            const double dy = k.p1 * (r2 + 2.0 * y * y) + 2.0 * k.p2 * x * y;
            x = (xd - dx) / rad;
            y = (yd - dy) / rad;
        }
    }
    out[2 * i] = x * k.f + k.cx;
    out[2 * i + 1] = y * k.f + k.cy;
}

struct PredictArgs {
    double kinv_i[9], r_i[9], c_i[3], k_j[9], r_j[9], c_j[3], zg;
};

__global__ void k_predict(const double* __restrict__ u, int n, PredictArgs a, double* __restrict__ pred,
                          uint8_t* __restrict__ ok) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double p[3] = {u[2 * i], u[2 * i + 1], 1.0};
    double ray[3], d[3], e[3], q[3];
    for (int r = 0; r < 3; ++r) ray[r] = p[0] * a.kinv_i[3 * r] + p[1] * a.kinv_i[3 * r + 1] + p[2] * a.kinv_i[3 * r + 2];
    for (int c = 0; c < 3; ++c) d[c] = ray[0] * a.r_i[c] + ray[1] * a.r_i[3 + c] + ray[2] * a.r_i[6 + c];   // rays @ Ri
    double dz = d[2];
    if (fabs(dz) < 1e-6) dz = -1e-6;
    const double t = (a.zg - a.c_i[2]) / dz;
    const double g[3] = {a.c_i[0] + t * d[0] - a.c_j[0], a.c_i[1] + t * d[1] - a.c_j[1], a.c_i[2] + t * d[2] - a.c_j[2]};
    for (int r = 0; r < 3; ++r) e[r] = g[0] * a.r_j[3 * r] + g[1] * a.r_j[3 * r + 1] + g[2] * a.r_j[3 * r + 2];   // @ Rj^T
    for (int r = 0; r < 3; ++r) q[r] = e[0] * a.k_j[3 * r] + e[1] * a.k_j[3 * r + 1] + e[2] * a.k_j[3 * r + 2];   // @ Kj^T
    double z = q[2];
    ok[i] = (t > 0.0 && z > 0.0) ? 1 : 0;
    if (fabs(z) < 1e-9) z = 1e-9;
    pred[2 * i] = q[0] / z;
    pred[2 * i + 1] = q[1] / z;
}

}  // namespace

int32_t run_undistort(const double* d_uv, int n, const double* k8, double* d_out, cudaStream_t s) {
    if (n <= 0) return FSB_OK;
    const Cam8 k{k8[0], k8[1], k8[2], k8[3], k8[4], k8[5], k8[6], k8[7]};
    k_undistort<<<blocks(n, 256), 256, 0, s>>>(d_uv, n, k, d_out);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

int32_t run_predict(const double* d_u, int n, const double* kinv_i, const double* r_i, const double* c_i,
                    const double* k_j, const double* r_j, const double* c_j, double zg, double* d_pred, uint8_t* d_ok,
                    cudaStream_t s) {
    if (n <= 0) return FSB_OK;
    PredictArgs a{};
    for (int m = 0; m < 9; ++m) {
        a.kinv_i[m] = kinv_i[m];
        a.r_i[m] = r_i[m];
        a.k_j[m] = k_j[m];
        a.r_j[m] = r_j[m];
    }
    for (int m = 0; m < 3; ++m) {
        a.c_i[m] = c_i[m];
        a.c_j[m] = c_j[m];
    }
    a.zg = zg;
    k_predict<<<blocks(n, 256), 256, 0, s>>>(d_u, n, a, d_pred, d_ok);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

}  // namespace fsb
