// Geometric verification of the pair worker on the device: RANSAC homography fits of many pairs in
// one launch (the cv2.findHomography(src, dst, cv2.RANSAC, thr) of matching.match_pair,
// app/planesite/matching.py:226, batched). One CTA per pair:
//   * coordinates are normalised per pair (centroid, mean distance sqrt(2)) for the solves;
//   * each thread draws hypotheses from a counter-based generator (seed, pair, hypothesis): four
//     distinct correspondences, rejected when three of them are collinear or when the orientation
//     of a triple differs between the two images; the homography with h33 = 1 from the 8 x 8 DLT
//     system by Gaussian elimination with partial pivoting, float64;
//   * a correspondence is an inlier when its squared reprojection error is at most thr^2 (as
//     OpenCV's RANSAC compares it); the hypothesis with the most inliers wins (ties: the lower
//     hypothesis index, so the result does not depend on the schedule);
//   * the mask is the winner's inliers (as OpenCV returns its RANSAC mask); the homography is then
//     refined by linear least squares over those inliers (OpenCV refines by Levenberg-Marquardt),
//     normalised to h33 = 1.
// Random sampling differs from OpenCV's, so results agree statistically, not bit for bit.
#include "fsb_internal.cuh"

namespace fsb {
namespace {

constexpr int RT = 256;   // threads per pair

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// solves the n x n system M x = r (M row-major, n <= 8) in place; false when singular
__device__ bool solve(double* M, double* r, int n) {
    for (int c = 0; c < n; ++c) {
        int piv = c;
        double best = fabs(M[c * n + c]);
        for (int k = c + 1; k < n; ++k)
            if (fabs(M[k * n + c]) > best) {
                best = fabs(M[k * n + c]);
                piv = k;
            }
        if (!(best > 1e-12)) return false;
        if (piv != c) {
            for (int k = 0; k < n; ++k) {
                const double t = M[c * n + k];
                M[c * n + k] = M[piv * n + k];
                M[piv * n + k] = t;
            }
            const double t = r[c];
            r[c] = r[piv];
            r[piv] = t;
        }
        for (int k = c + 1; k < n; ++k) {
            const double f = M[k * n + c] / M[c * n + c];
            for (int j = c; j < n; ++j) M[k * n + j] -= f * M[c * n + j];
            r[k] -= f * r[c];
        }
    }
    for (int c = n - 1; c >= 0; --c) {
        double v = r[c];
        for (int j = c + 1; j < n; ++j) v -= M[c * n + j] * r[j];
        r[c] = v / M[c * n + c];
    }
    return true;
}

__device__ __forceinline__ double area2(double ax, double ay, double bx, double by, double cx, double cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

struct Norm {
    double cx, cy, s;   // x' = (x - cx) * s
};

// squared reprojection error in pixels of correspondence k under the normalised homography h (h33 = 1)
__device__ __forceinline__ double err2(const double* h, const double2* src, const double2* dst, int k, const Norm& ns,
                                       const Norm& nd) {
    const double x = (src[k].x - ns.cx) * ns.s, y = (src[k].y - ns.cy) * ns.s;
    const double w = h[6] * x + h[7] * y + 1.0;
    if (fabs(w) < 1e-12) return 1e300;
    const double u = (h[0] * x + h[1] * y + h[2]) / w, v = (h[3] * x + h[4] * y + h[5]) / w;
    const double du = (u / nd.s + nd.cx) - dst[k].x, dv = (v / nd.s + nd.cy) - dst[k].y;
    return du * du + dv * dv;
}

__global__ void __launch_bounds__(RT) k_ransac_h(const long long* __restrict__ off, const double2* __restrict__ src,
                                                 const double2* __restrict__ dst, double thr2, int iters,
                                                 unsigned long long seed, double* __restrict__ H,
                                                 uint8_t* __restrict__ mask, int* __restrict__ n_inl) {
    const int p = blockIdx.x, tid = threadIdx.x;
    const long long o = off[p];
    const int n = (int)(off[p + 1] - o);
    src += o;
    dst += o;
    __shared__ double s_red[RT / 32][3];
    __shared__ int s_best[2];
    __shared__ double s_h[9];
    __shared__ double s_ne[RT / 32][72];   // per-warp partial normal equations (summed in warp order)
    // normalisation of both point sets (centroid, mean distance sqrt(2))
    double sx = 0, sy = 0, dx = 0, dy = 0;
    for (int k = tid; k < n; k += RT) {
        sx += src[k].x; sy += src[k].y; dx += dst[k].x; dy += dst[k].y;
    }
    auto block_sum = [&](double a, double b, double c, double* out3) {
        for (int sh = 16; sh; sh >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, sh);
            b += __shfl_xor_sync(0xffffffffu, b, sh);
            c += __shfl_xor_sync(0xffffffffu, c, sh);
        }
        __syncthreads();
        if ((tid & 31) == 0) { s_red[tid >> 5][0] = a; s_red[tid >> 5][1] = b; s_red[tid >> 5][2] = c; }
        __syncthreads();
        out3[0] = out3[1] = out3[2] = 0;
        for (int w = 0; w < RT / 32; ++w) { out3[0] += s_red[w][0]; out3[1] += s_red[w][1]; out3[2] += s_red[w][2]; }
    };
    if (n < 4) {
        if (tid < 9) H[9 * p + tid] = 0.0;
        for (int k = tid; k < n; k += RT) mask[o + k] = 0;
        if (tid == 0) n_inl[p] = 0;
        return;
    }
    double t3[3], u3[3];
    block_sum(sx, sy, 0.0, t3);
    block_sum(dx, dy, 0.0, u3);
    Norm ns{t3[0] / n, t3[1] / n, 0}, nd{u3[0] / n, u3[1] / n, 0};
    double ds = 0, dd = 0;
    for (int k = tid; k < n; k += RT) {
        ds += hypot(src[k].x - ns.cx, src[k].y - ns.cy);
        dd += hypot(dst[k].x - nd.cx, dst[k].y - nd.cy);
    }
    block_sum(ds, dd, 0.0, t3);
    ns.s = t3[0] > 0 ? 1.4142135623730951 * n / t3[0] : 1.0;
    nd.s = t3[1] > 0 ? 1.4142135623730951 * n / t3[1] : 1.0;
    // hypotheses
    int best_cnt = -1, best_hyp = 0x7fffffff;
    double best_h[8] = {};
    for (int hyp = tid; hyp < iters; hyp += RT) {
        int id[4];
        unsigned long long st = mix64(seed ^ ((unsigned long long)p << 32) ^ (unsigned long long)hyp * 0x2545F4914F6CDD1Dull);
        for (int k = 0; k < 4; ++k) {
            for (int tries = 0; tries < 64; ++tries) {
                st = mix64(st);
                const int c = (int)(st % (unsigned long long)n);
                bool dup = false;
                for (int j = 0; j < k; ++j) dup |= id[j] == c;
                id[k] = c;
                if (!dup) break;
            }
        }
        bool ok = id[0] != id[1] && id[0] != id[2] && id[0] != id[3] && id[1] != id[2] && id[1] != id[3] && id[2] != id[3];
        double X[4], Y[4], U[4], V[4];
        for (int k = 0; k < 4 && ok; ++k) {
            X[k] = (src[id[k]].x - ns.cx) * ns.s;
            Y[k] = (src[id[k]].y - ns.cy) * ns.s;
            U[k] = (dst[id[k]].x - nd.cx) * nd.s;
            V[k] = (dst[id[k]].y - nd.cy) * nd.s;
        }
        // no three collinear, same orientation of every triple in both images
        const int tri[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
        for (int t = 0; t < 4 && ok; ++t) {
            const double a = area2(X[tri[t][0]], Y[tri[t][0]], X[tri[t][1]], Y[tri[t][1]], X[tri[t][2]], Y[tri[t][2]]);
            const double b = area2(U[tri[t][0]], V[tri[t][0]], U[tri[t][1]], V[tri[t][1]], U[tri[t][2]], V[tri[t][2]]);
            if (fabs(a) < 1e-6 || fabs(b) < 1e-6 || (a > 0) != (b > 0)) ok = false;
        }
        double h[9];
        if (ok) {
            double M[64], r[8];
            for (int k = 0; k < 4; ++k) {
                double* m0 = M + 16 * k;
                double* m1 = m0 + 8;
                m0[0] = X[k]; m0[1] = Y[k]; m0[2] = 1; m0[3] = 0; m0[4] = 0; m0[5] = 0;
                m0[6] = -U[k] * X[k]; m0[7] = -U[k] * Y[k];
                m1[0] = 0; m1[1] = 0; m1[2] = 0; m1[3] = X[k]; m1[4] = Y[k]; m1[5] = 1;
                m1[6] = -V[k] * X[k]; m1[7] = -V[k] * Y[k];
                r[2 * k] = U[k];
                r[2 * k + 1] = V[k];
            }
            ok = solve(M, r, 8);
            for (int k = 0; k < 8; ++k) h[k] = r[k];
            h[8] = 1.0;
        }
        if (!ok) continue;
        int cnt = 0;
        for (int k = 0; k < n; ++k) cnt += err2(h, src, dst, k, ns, nd) <= thr2;
        if (cnt > best_cnt || (cnt == best_cnt && hyp < best_hyp)) {
            best_cnt = cnt;
            best_hyp = hyp;
            for (int k = 0; k < 8; ++k) best_h[k] = h[k];
        }
    }
    // block argmax: most inliers, then lowest hypothesis index
    if (tid == 0) { s_best[0] = -1; s_best[1] = 0x7fffffff; }
    __syncthreads();
    atomicMax(&s_best[0], best_cnt);
    __syncthreads();
    if (best_cnt == s_best[0] && best_cnt >= 0) atomicMin(&s_best[1], best_hyp);
    __syncthreads();
    if (s_best[0] < 0) {   // no usable sample
        if (tid < 9) H[9 * p + tid] = 0.0;
        for (int k = tid; k < n; k += RT) mask[o + k] = 0;
        if (tid == 0) n_inl[p] = 0;
        return;
    }
    if (best_cnt == s_best[0] && best_hyp == s_best[1]) {
        for (int k = 0; k < 8; ++k) s_h[k] = best_h[k];
        s_h[8] = 1.0;
    }
    __syncthreads();
    // mask of the winner; normal equations of the least-squares DLT over its inliers
    double ne[72];
    for (int k = 0; k < 72; ++k) ne[k] = 0.0;
    for (int k = tid; k < n; k += RT) {
        const bool in = err2(s_h, src, dst, k, ns, nd) <= thr2;
        mask[o + k] = in ? 1 : 0;
        if (!in) continue;
        const double x = (src[k].x - ns.cx) * ns.s, y = (src[k].y - ns.cy) * ns.s;
        const double u = (dst[k].x - nd.cx) * nd.s, v = (dst[k].y - nd.cy) * nd.s;
        const double a0[8] = {x, y, 1, 0, 0, 0, -u * x, -u * y}, a1[8] = {0, 0, 0, x, y, 1, -v * x, -v * y};
        for (int i = 0; i < 8; ++i) {
            for (int j = 0; j < 8; ++j) ne[8 * i + j] += a0[i] * a0[j] + a1[i] * a1[j];
            ne[64 + i] += a0[i] * u + a1[i] * v;
        }
    }
    for (int k = 0; k < 72; ++k) {
        double v = ne[k];
        for (int sh = 16; sh; sh >>= 1) v += __shfl_xor_sync(0xffffffffu, v, sh);
        if ((tid & 31) == 0) s_ne[tid >> 5][k] = v;
    }
    __syncthreads();
    if (tid == 0) {
        double M[64], r[8], hn[9];
        for (int k = 0; k < 72; ++k) {
            double v = 0.0;
            for (int w = 0; w < RT / 32; ++w) v += s_ne[w][k];
            if (k < 64)
                M[k] = v;
            else
                r[k - 64] = v;
        }
        if (solve(M, r, 8)) {
            for (int k = 0; k < 8; ++k) hn[k] = r[k];
        } else {
            for (int k = 0; k < 8; ++k) hn[k] = s_h[k];
        }
        hn[8] = 1.0;
        // back to pixels: H = Td^-1 Hn Ts, Ts = [[s,0,-s cx],[0,s,-s cy],[0,0,1]]
        const double Ts[9] = {ns.s, 0, -ns.s * ns.cx, 0, ns.s, -ns.s * ns.cy, 0, 0, 1};
        const double Ti[9] = {1 / nd.s, 0, nd.cx, 0, 1 / nd.s, nd.cy, 0, 0, 1};
        double A[9], B[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) A[3 * i + j] = hn[3 * i] * Ts[j] + hn[3 * i + 1] * Ts[3 + j] + hn[3 * i + 2] * Ts[6 + j];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) B[3 * i + j] = Ti[3 * i] * A[j] + Ti[3 * i + 1] * A[3 + j] + Ti[3 * i + 2] * A[6 + j];
        const double z = B[8];
        for (int k = 0; k < 9; ++k) H[9 * p + k] = fabs(z) > 0 ? B[k] / z : B[k];
        n_inl[p] = s_best[0];
    }
}

}  // namespace

int32_t run_ransac_h(const long long* d_off, int n_pairs, const double2* d_src, const double2* d_dst, double thr,
                     int iters, unsigned long long seed, double* d_H, uint8_t* d_mask, int* d_ninl, cudaStream_t s) {
    if (n_pairs <= 0) return FSB_OK;
    k_ransac_h<<<n_pairs, RT, 0, s>>>(d_off, d_src, d_dst, thr * thr, iters, seed, d_H, d_mask, d_ninl);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

}  // namespace fsb
