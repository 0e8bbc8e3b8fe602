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

// -------------------------------------------------------------------------------------------------
// Fundamental-matrix verification of the pair worker on the device: matching._verify's
// cv2.findFundamentalMat(pi, pj, USAC_MAGSAC, thr, 0.999, 10000) (app/planesite/matching.py:175-191)
// for many pairs in one launch. One CTA per pair:
//   * both point sets normalised (centroid, mean distance sqrt(2)), float64 throughout;
//   * hypotheses from seven distinct correspondences (counter-based draws): the 7 x 9 epipolar
//     system reduced by Gaussian elimination with partial pivoting to its two-dimensional null
//     space F1, F2 (samples of lower rank are rejected), det(a F1 + (1 - a) F2) = 0 solved as a
//     cubic: one to three candidates per sample;
//   * a correspondence is an inlier when its Sampson distance (the first-order geometric error of
//     x2^T F x1 = 0, in pixels) is at most thr, the rule OpenCV's USAC_MAGSAC applies to the mask
//     it returns; the candidate with the most inliers wins (ties: lower hypothesis, then lower root
//     index: schedule-independent);
//   * local optimisation: the normalised eight-point least squares over the winner's inliers (the
//     smallest eigenvector of A^T A by cyclic Jacobi), rank 2 enforced by removing the smallest
//     singular direction, kept while it does not lose inliers (two rounds);
//   * F in pixels scaled to F33 = 1 (unit norm when F33 is near zero), the mask of its inliers.
// MAGSAC++ scores hypotheses by marginalising over the noise scale; the score here is the plain
// inlier count, and random samples differ, so the masks agree statistically, not bit for bit.
namespace fsb {
namespace {

__device__ __forceinline__ double det3(const double* m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// real roots of c3 a^3 + c2 a^2 + c1 a + c0 (at most 3); returns the count
__device__ int cubic_roots(double c3, double c2, double c1, double c0, double* r) {
    const double scale = fmax(fmax(fabs(c3), fabs(c2)), fmax(fabs(c1), fabs(c0)));
    if (!(scale > 0)) return 0;
    if (fabs(c3) <= 1e-12 * scale) {   // quadratic (or linear)
        if (fabs(c2) <= 1e-12 * scale) {
            if (fabs(c1) <= 1e-12 * scale) return 0;
            r[0] = -c0 / c1;
            return 1;
        }
        const double d = c1 * c1 - 4 * c2 * c0;
        if (d < 0) return 0;
        const double q = -0.5 * (c1 + copysign(sqrt(d), c1));
        int n = 0;
        if (q != 0) r[n++] = c0 / q;
        r[n++] = q / c2;
        return n;
    }
    const double a = c2 / c3, b = c1 / c3, c = c0 / c3;
    const double Q = (a * a - 3 * b) / 9, R = (2 * a * a * a - 9 * a * b + 27 * c) / 54;
    const double Q3 = Q * Q * Q;
    if (R * R < Q3) {
        const double th = acos(fmin(1.0, fmax(-1.0, R / sqrt(Q3))));
        const double s = -2 * sqrt(Q);
        r[0] = s * cos(th / 3) - a / 3;
        r[1] = s * cos((th + 2 * M_PI) / 3) - a / 3;
        r[2] = s * cos((th - 2 * M_PI) / 3) - a / 3;
        return 3;
    }
    const double A = -copysign(cbrt(fabs(R) + sqrt(R * R - Q3)), R);
    const double B = A != 0 ? Q / A : 0;
    r[0] = (A + B) - a / 3;
    return 1;
}

// two-dimensional null space of the 7 x 9 system M (row-major, destroyed): false below rank 7
__device__ bool null2(double* M, double* f1, double* f2) {
    int pivc[7];
    int row = 0;
    int freec[2], nf = 0;
    for (int c = 0; c < 9; ++c) {
        int piv = -1;
        double best = 1e-10;
        for (int k = row; k < 7; ++k)
            if (fabs(M[k * 9 + c]) > best) {
                best = fabs(M[k * 9 + c]);
                piv = k;
            }
        if (piv < 0 || row == 7) {
            if (nf == 2) return false;
            freec[nf++] = c;
            continue;
        }
        if (piv != row)
            for (int j = 0; j < 9; ++j) {
                const double t = M[row * 9 + j];
                M[row * 9 + j] = M[piv * 9 + j];
                M[piv * 9 + j] = t;
            }
        const double inv = 1.0 / M[row * 9 + c];
        for (int j = c; j < 9; ++j) M[row * 9 + j] *= inv;
        for (int k = 0; k < 7; ++k) {
            if (k == row) continue;
            const double f = M[k * 9 + c];
            if (f != 0)
                for (int j = c; j < 9; ++j) M[k * 9 + j] -= f * M[row * 9 + j];
        }
        pivc[row++] = c;
    }
    if (row != 7 || nf != 2) return false;
    // reduced row echelon form: x_pivot = - sum over free columns of M[row][free] x_free
    for (int v = 0; v < 2; ++v) {
        double* f = v ? f2 : f1;
        for (int j = 0; j < 9; ++j) f[j] = 0;
        f[freec[v]] = 1;
        for (int k = 0; k < 7; ++k) f[pivc[k]] = -M[k * 9 + freec[v]];
    }
    return true;
}

// symmetric n x n eigen-decomposition by cyclic Jacobi (A destroyed, V columns = eigenvectors)
template <int n>
__device__ void jacobi_eig(double* A, double* V, double* ev) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) V[i * n + j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 30; ++sweep) {
        double off = 0, tot = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                tot += A[i * n + j] * A[i * n + j];
                if (i != j) off += A[i * n + j] * A[i * n + j];
            }
        if (off <= 1e-30 * tot) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[p * n + q];
                if (fabs(apq) < 1e-300) continue;
                const double th = (A[q * n + q] - A[p * n + p]) / (2 * apq);
                const double t = copysign(1.0, th) / (fabs(th) + sqrt(th * th + 1));
                const double c = 1 / sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < n; ++k) {   // A = J^T A J
                    const double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * vkq;
                    V[k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < n; ++i) ev[i] = A[i * n + i];
}

// F (normalised coordinates) to pixels: F_pix = T2^T F T1, T = [[s,0,-s cx],[0,s,-s cy],[0,0,1]]
__device__ void denorm_f(const double* f, const Norm& n1, const Norm& n2, double* out) {
    const double T1[9] = {n1.s, 0, -n1.s * n1.cx, 0, n1.s, -n1.s * n1.cy, 0, 0, 1};
    const double T2t[9] = {n2.s, 0, 0, 0, n2.s, 0, -n2.s * n2.cx, -n2.s * n2.cy, 1};
    double A[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[3 * i + j] = f[3 * i] * T1[j] + f[3 * i + 1] * T1[3 + j] + f[3 * i + 2] * T1[6 + j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[3 * i + j] = T2t[3 * i] * A[j] + T2t[3 * i + 1] * A[3 + j] + T2t[3 * i + 2] * A[6 + j];
}

// squared Sampson distance (pixels) of correspondence (x1, x2) at most thr2:
// (x2^T F x1)^2 <= thr2 ((F x1)_1^2 + (F x1)_2^2 + (F^T x2)_1^2 + (F^T x2)_2^2)
__device__ __forceinline__ bool f_inlier(const double* F, double2 a, double2 b, double thr2) {
    const double l0 = F[0] * a.x + F[1] * a.y + F[2], l1 = F[3] * a.x + F[4] * a.y + F[5];
    const double l2 = F[6] * a.x + F[7] * a.y + F[8];
    const double m0 = F[0] * b.x + F[3] * b.y + F[6], m1 = F[1] * b.x + F[4] * b.y + F[7];
    const double e = b.x * l0 + b.y * l1 + l2;
    const double den = l0 * l0 + l1 * l1 + m0 * m0 + m1 * m1;
    return den > 0 && e * e <= thr2 * den;
}

constexpr int FT = 256;

__global__ void __launch_bounds__(FT) k_ransac_f(const long long* __restrict__ off, const double2* __restrict__ src,
                                                 const double2* __restrict__ dst, double thr2, int iters,
                                                 unsigned long long seed, double* __restrict__ Fout,
                                                 uint8_t* __restrict__ mask, int* __restrict__ n_inl) {
    const int p = blockIdx.x, tid = threadIdx.x;
    const long long o = off[p];
    const int n = (int)(off[p + 1] - o);
    src += o;
    dst += o;
    __shared__ double s_red[FT / 32][3];
    __shared__ int s_best[3];
    __shared__ double s_f[9], s_fn[9];
    __shared__ double s_ne[FT / 32][45];
    __shared__ int s_cnt[FT / 32];
    auto block_sum = [&](double a, double b, double* out2) {
        for (int sh = 16; sh; sh >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, sh);
            b += __shfl_xor_sync(0xffffffffu, b, sh);
        }
        __syncthreads();
        if ((tid & 31) == 0) { s_red[tid >> 5][0] = a; s_red[tid >> 5][1] = b; }
        __syncthreads();
        out2[0] = out2[1] = 0;
        for (int w = 0; w < FT / 32; ++w) { out2[0] += s_red[w][0]; out2[1] += s_red[w][1]; }
    };
    auto fail = [&]() {
        if (tid < 9) Fout[9 * p + tid] = 0.0;
        for (int k = tid; k < n; k += FT) mask[o + k] = 0;
        if (tid == 0) n_inl[p] = 0;
    };
    if (n < 8) {
        fail();
        return;
    }
    double t2[2], u2[2];
    double sx = 0, sy = 0, dx = 0, dy = 0;
    for (int k = tid; k < n; k += FT) { sx += src[k].x; sy += src[k].y; dx += dst[k].x; dy += dst[k].y; }
    block_sum(sx, sy, t2);
    block_sum(dx, dy, u2);
    Norm n1{t2[0] / n, t2[1] / n, 0}, n2{u2[0] / n, u2[1] / n, 0};
    double ds = 0, dd = 0;
    for (int k = tid; k < n; k += FT) {
        ds += hypot(src[k].x - n1.cx, src[k].y - n1.cy);
        dd += hypot(dst[k].x - n2.cx, dst[k].y - n2.cy);
    }
    block_sum(ds, dd, t2);
    n1.s = t2[0] > 0 ? 1.4142135623730951 * n / t2[0] : 1.0;
    n2.s = t2[1] > 0 ? 1.4142135623730951 * n / t2[1] : 1.0;
    int best_cnt = -1, best_key = 0x7fffffff;
    double best_f[9] = {};
    for (int hyp = tid; hyp < iters; hyp += FT) {
        int id[7];
        unsigned long long st = mix64(seed ^ ((unsigned long long)p << 32) ^ (unsigned long long)hyp * 0x2545F4914F6CDD1Dull);
        bool ok = true;
        for (int k = 0; k < 7; ++k) {
            bool dup = true;
            for (int tries = 0; tries < 64 && dup; ++tries) {
                st = mix64(st);
                id[k] = (int)(st % (unsigned long long)n);
                dup = false;
                for (int j = 0; j < k; ++j) dup |= id[j] == id[k];
            }
            ok = ok && !dup;
        }
        if (!ok) continue;
        double M[63];
        for (int k = 0; k < 7; ++k) {
            const double x = (src[id[k]].x - n1.cx) * n1.s, y = (src[id[k]].y - n1.cy) * n1.s;
            const double u = (dst[id[k]].x - n2.cx) * n2.s, v = (dst[id[k]].y - n2.cy) * n2.s;
            double* m = M + 9 * k;
            m[0] = u * x; m[1] = u * y; m[2] = u; m[3] = v * x; m[4] = v * y; m[5] = v; m[6] = x; m[7] = y; m[8] = 1;
        }
        double f1[9], f2[9];
        if (!null2(M, f1, f2)) continue;
        // det(F2 + a D), D = F1 - F2, at a = 0, 1, -1, 2 -> cubic coefficients
        double D[9], T[9];
        for (int k = 0; k < 9; ++k) D[k] = f1[k] - f2[k];
        const double d0 = det3(f2), d1 = det3(f1);
        for (int k = 0; k < 9; ++k) T[k] = f2[k] - D[k];
        const double dm = det3(T);
        for (int k = 0; k < 9; ++k) T[k] = f2[k] + 2 * D[k];
        const double dp = det3(T);
        const double c0 = d0, c3 = (dp - 3 * d1 + 3 * d0 - dm) / 6, c2 = (d1 + dm) / 2 - d0, c1 = d1 - d0 - c2 - c3;
        double roots[3];
        const int nr = cubic_roots(c3, c2, c1, c0, roots);
        for (int ri = 0; ri < nr; ++ri) {
            double fn[9], fp[9];
            for (int k = 0; k < 9; ++k) fn[k] = f2[k] + roots[ri] * D[k];
            denorm_f(fn, n1, n2, fp);
            int cnt = 0;
            for (int k = 0; k < n; ++k) cnt += f_inlier(fp, src[k], dst[k], thr2);
            const int key = hyp * 4 + ri;
            if (cnt > best_cnt || (cnt == best_cnt && key < best_key)) {
                best_cnt = cnt;
                best_key = key;
                for (int k = 0; k < 9; ++k) best_f[k] = fp[k];
            }
        }
    }
    if (tid == 0) { s_best[0] = -1; s_best[1] = 0x7fffffff; }
    __syncthreads();
    atomicMax(&s_best[0], best_cnt);
    __syncthreads();
    if (best_cnt == s_best[0] && best_cnt >= 0) atomicMin(&s_best[1], best_key);
    __syncthreads();
    if (s_best[0] < 8) {
        fail();
        return;
    }
    if (best_cnt == s_best[0] && best_key == s_best[1])
        for (int k = 0; k < 9; ++k) s_f[k] = best_f[k];
    __syncthreads();
    int cur = s_best[0];
    // local optimisation: eight-point least squares over the current inliers (normalised coordinates)
    for (int round = 0; round < 2; ++round) {
        double ne[45];
        for (int k = 0; k < 45; ++k) ne[k] = 0;
        for (int k = tid; k < n; k += FT) {
            if (!f_inlier(s_f, src[k], dst[k], thr2)) continue;
            const double x = (src[k].x - n1.cx) * n1.s, y = (src[k].y - n1.cy) * n1.s;
            const double u = (dst[k].x - n2.cx) * n2.s, v = (dst[k].y - n2.cy) * n2.s;
            const double a[9] = {u * x, u * y, u, v * x, v * y, v, x, y, 1};
            int idx = 0;
            for (int i = 0; i < 9; ++i)
                for (int j = i; j < 9; ++j) ne[idx++] += a[i] * a[j];
        }
        for (int k = 0; k < 45; ++k) {
            double v = ne[k];
            for (int sh = 16; sh; sh >>= 1) v += __shfl_xor_sync(0xffffffffu, v, sh);
            if ((tid & 31) == 0) s_ne[tid >> 5][k] = v;
        }
        __syncthreads();
        if (tid == 0) {
            double A[81], V[81], ev[9];
            int idx = 0;
            for (int i = 0; i < 9; ++i)
                for (int j = i; j < 9; ++j) {
                    double v = 0;
                    for (int w = 0; w < FT / 32; ++w) v += s_ne[w][idx];
                    A[i * 9 + j] = A[j * 9 + i] = v;
                    ++idx;
                }
            jacobi_eig<9>(A, V, ev);
            int m = 0;
            for (int i = 1; i < 9; ++i)
                if (ev[i] < ev[m]) m = i;
            double f[9];
            for (int i = 0; i < 9; ++i) f[i] = V[i * 9 + m];
            // rank 2: remove the direction of F's smallest singular value (F <- F (I - w w^T))
            double G[9], W[9], gv[3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) G[3 * i + j] = f[i] * f[j] + f[3 + i] * f[3 + j] + f[6 + i] * f[6 + j];
            jacobi_eig<3>(G, W, gv);
            int s = 0;
            for (int i = 1; i < 3; ++i)
                if (gv[i] < gv[s]) s = i;
            const double w3[3] = {W[s], W[3 + s], W[6 + s]};
            double fr[9];
            for (int i = 0; i < 3; ++i) {
                const double fw = f[3 * i] * w3[0] + f[3 * i + 1] * w3[1] + f[3 * i + 2] * w3[2];
                for (int j = 0; j < 3; ++j) fr[3 * i + j] = f[3 * i + j] - fw * w3[j];
            }
            denorm_f(fr, n1, n2, s_fn);
        }
        __syncthreads();
        int c = 0;
        for (int k = tid; k < n; k += FT) c += f_inlier(s_fn, src[k], dst[k], thr2);
        for (int sh = 16; sh; sh >>= 1) c += __shfl_xor_sync(0xffffffffu, c, sh);
        if ((tid & 31) == 0) s_cnt[tid >> 5] = c;
        __syncthreads();
        int tot = 0;
        for (int w = 0; w < FT / 32; ++w) tot += s_cnt[w];
        __syncthreads();
        if (tot < cur) break;   // uniform: every thread sees the same total
        cur = tot;
        if (tid < 9) s_f[tid] = s_fn[tid];
        __syncthreads();
    }
    for (int k = tid; k < n; k += FT) mask[o + k] = f_inlier(s_f, src[k], dst[k], thr2) ? 1 : 0;
    if (tid == 0) {
        const double z = s_f[8];
        double nrm = 0;
        for (int k = 0; k < 9; ++k) nrm += s_f[k] * s_f[k];
        nrm = sqrt(nrm);
        const double sc = fabs(z) > 1e-12 * nrm ? z : nrm;
        for (int k = 0; k < 9; ++k) Fout[9 * p + k] = sc != 0 ? s_f[k] / sc : s_f[k];
        n_inl[p] = cur;
    }
}

}  // namespace

int32_t run_ransac_f(const long long* d_off, int n_pairs, const double2* d_src, const double2* d_dst, double thr,
                     int iters, unsigned long long seed, double* d_F, uint8_t* d_mask, int* d_ninl, cudaStream_t s) {
    if (n_pairs <= 0) return FSB_OK;
    k_ransac_f<<<n_pairs, FT, 0, s>>>(d_off, d_src, d_dst, thr * thr, iters, seed, d_F, d_mask, d_ninl);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

}  // namespace fsb
