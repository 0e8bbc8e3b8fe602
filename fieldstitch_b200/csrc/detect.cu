// Keypoint detection and description on the DoG / gradient atlases.
//
// Compiled with --fmad=false: every float32 expression below is evaluated with the reference's
// rounding (one rounding per operation, in the written order), so integer positions, sub-pixel
// offsets and responses follow app/planesite/gsift.py bit for bit given the same DoG values.
//
//   k_extrema   3x3x3 extrema of DoG layers 1..3 (gsift.py:293-319), warp-aggregated append
//   k_refine    sub-pixel fit, contrast and edge tests (gsift.py:322-369), thread per candidate
//   k_orient    36-bin orientation histogram + smoothing + peaks (gsift.py:372-432), warp per
//               keypoint, exact fixed-point accumulation (order-independent, deterministic)
//   sort        stable radix sorts: (extremum index, bin) then response descending (gsift.py:471)
//   k_gather    keypoint fields in input-image pixels (gsift.py:462-474)
//   k_describe  rotated 4x4x8 trilinear histogram, L2 clip/renormalise (gsift.py:480-525,
//               800-871) and RootSIFT bytes (features.py:80-82), warp per keypoint
//   spread      grid-spread selection of features.py:38-57
#include <cub/cub.cuh>

#include <cmath>

#include "fsb_internal.cuh"

namespace fsb {
namespace {

struct DetectConsts {
    Geometry g;
    float pthr, contrast, edge, e1sq;
    long long vox_off[MAXO + 1];
};

constexpr double kHistScale = 1125899906842624.0;        // 2^50, orientation histogram fixed point
constexpr double kHistInv = 1.0 / 1125899906842624.0;
constexpr double kDescScale = 281474976710656.0;         // 2^48, descriptor histogram fixed point
constexpr double kDescInv = 1.0 / 281474976710656.0;

__device__ __forceinline__ int find_octave(const Geometry& g, long long f) {
    int o = 0;
    while (o + 1 < g.n_oct && f >= g.dog_off[o + 1]) ++o;
    return o;
}

// warp-aggregated append of `flag` entries into out[], counter shared by the grid
template <class T>
__device__ __forceinline__ void warp_append(bool flag, const T& v, T* out, uint32_t* counter, uint32_t cap) {
    const unsigned m = __ballot_sync(0xffffffffu, flag);
    if (!m) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (flag) {
        const uint32_t pos = base + __popc(m & ((1u << lane) - 1u));
        if (pos < cap) out[pos] = v;
    }
}

__global__ void __launch_bounds__(256) k_extrema(const float* __restrict__ DF, DetectConsts k,
                                                 uint32_t* __restrict__ cand, uint32_t* counter,
                                                 uint32_t cap) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool ext = false;
    uint32_t fidx = 0;
    if (t < k.vox_off[k.g.n_oct]) {
        int o = 0;
        while (t >= k.vox_off[o + 1]) ++o;
        const int R = k.g.R[o], C = k.g.C[o];
        const int iw = C - 2 * BORDER, ih = R - 2 * BORDER;
        const long long loc = t - k.vox_off[o], per = (long long)iw * ih;
        const int l = (int)(loc / per) + 1;
        const long long rem = loc - (long long)(l - 1) * per;
        const int r = (int)(rem / iw) + BORDER;
        const int c = (int)(rem - (long long)(r - BORDER) * iw) + BORDER;
        const long long RC = (long long)R * C;
        const long long kk = k.g.dog_off[o] + l * RC + (long long)r * C + c;
        const float v = DF[kk];
        bool mx = v > k.pthr, mn = v < -k.pthr;
        if (mx || mn) {
#pragma unroll
            for (int dl = -1; dl <= 1; ++dl)
#pragma unroll
                for (int dr = -1; dr <= 1; ++dr)
#pragma unroll
                    for (int dc = -1; dc <= 1; ++dc) {
                        const float u = DF[kk + dl * RC + dr * C + dc];
                        mx = mx && !(u > v);
                        mn = mn && !(u < v);
                    }
        }
        ext = mx || mn;
        fidx = (uint32_t)kk;
    }
    warp_append(ext, fidx, cand, counter, cap);
}

struct Fit {
    float v, dx, dy, ds, dxx, dyy, dss, dxy, dxs, dys;
};

// finite-difference gradient and Hessian at an integer voxel (gsift.py:274-290)
__device__ __forceinline__ Fit local_fit(const float* __restrict__ D, long long k, long long C, long long RC) {
    Fit f;
    f.v = D[k];
    const float xp1 = D[k + 1], xm1 = D[k - 1], yp1 = D[k + C], ym1 = D[k - C];
    const float sp1 = D[k + RC], sm1 = D[k - RC];
    f.dx = (xp1 - xm1) * 0.5f;
    f.dy = (yp1 - ym1) * 0.5f;
    f.ds = (sp1 - sm1) * 0.5f;
    f.dxx = (xp1 + xm1) - 2.f * f.v;
    f.dyy = (yp1 + ym1) - 2.f * f.v;
    f.dss = (sp1 + sm1) - 2.f * f.v;
    f.dxy = (((D[k + C + 1] - D[k + C - 1]) - D[k - C + 1]) + D[k - C - 1]) * 0.25f;
    f.dxs = (((D[k + RC + 1] - D[k + RC - 1]) - D[k - RC + 1]) + D[k - RC - 1]) * 0.25f;
    f.dys = (((D[k + RC + C] - D[k + RC - C]) - D[k - RC + C]) + D[k - RC - C]) * 0.25f;
    return f;
}

__global__ void __launch_bounds__(128) k_refine(const float* __restrict__ DF, DetectConsts k,
                                                const uint32_t* __restrict__ cand, const uint32_t* n_cand,
                                                uint32_t cap_cand, Refined* __restrict__ out,
                                                uint32_t* counter, uint32_t cap) {
    const uint32_t n = min(*n_cand, cap_cand);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t i = base + threadIdx.x;
        bool good = false;
        Refined e{};
        if (i < n) {
            const uint32_t f = cand[i];
            const int o = find_octave(k.g, f);
            const int R = k.g.R[o], C = k.g.C[o];
            const long long RC = (long long)R * C, ob = k.g.dog_off[o];
            const long long loc = (long long)f - ob;
            int l = (int)(loc / RC);
            const long long rem = loc - (long long)l * RC;
            int r = (int)(rem / C);
            int c = (int)(rem - (long long)r * C);
            float X0 = 0.f, X1 = 0.f, X2 = 0.f;
            bool done = false;
            for (int it = 0; it < MAX_INTERP; ++it) {
                const Fit F = local_fit(DF, ob + l * RC + (long long)r * C + c, C, RC);
                // adjugate solve of H x = g (gsift.py:182-198); x = -H^-1 g
                const float a = F.dxx, b = F.dxy, cc = F.dxs, d = F.dxy, ee = F.dyy, ff = F.dys;
                const float gg = F.dxs, hh = F.dys, ii = F.dss;
                const float A = ee * ii - ff * hh, B = -(d * ii - ff * gg), Cc = d * hh - ee * gg;
                const float det = (a * A + b * B) + cc * Cc;
                if (!(fabsf(det) > 1e-20f)) break;
                const float i00 = A / det, i01 = -(b * ii - cc * hh) / det, i02 = (b * ff - cc * ee) / det;
                const float i10 = B / det, i11 = (a * ii - cc * gg) / det, i12 = -(a * ff - cc * d) / det;
                const float i20 = Cc / det, i21 = -(a * hh - b * gg) / det, i22 = (a * ee - b * d) / det;
                const float x0 = -((i00 * F.dx + i01 * F.dy) + i02 * F.ds);
                const float x1 = -((i10 * F.dx + i11 * F.dy) + i12 * F.ds);
                const float x2 = -((i20 * F.dx + i21 * F.dy) + i22 * F.ds);
                if (fabsf(x0) < 0.5f && fabsf(x1) < 0.5f && fabsf(x2) < 0.5f) {
                    X0 = x0; X1 = x1; X2 = x2;
                    done = true;
                    break;
                }
                if (!(fabsf(x0) <= 1e6f && fabsf(x1) <= 1e6f && fabsf(x2) <= 1e6f)) break;   // also NaN
                c += (int)rintf(x0);
                r += (int)rintf(x1);
                l += (int)rintf(x2);
                if (l < 1 || l > N_LAYERS || c < BORDER || c >= C - BORDER || r < BORDER || r >= R - BORDER) break;
            }
            if (done) {
                const Fit F = local_fit(DF, ob + l * RC + (long long)r * C + c, C, RC);
                const float contr = F.v + 0.5f * ((F.dx * X0 + F.dy * X1) + F.ds * X2);
                const float tr = F.dxx + F.dyy;
                const float dt = F.dxx * F.dyy - F.dxy * F.dxy;
                if (fabsf(contr) * (float)N_LAYERS >= k.contrast && dt > 0.f && (tr * tr) * k.edge < k.e1sq * dt) {
                    good = true;
                    e.f = f; e.o = (int16_t)o; e.l = (int16_t)l; e.r = r; e.c = c;
                    e.x0 = X0; e.x1 = X1; e.x2 = X2;
                    e.resp = fabsf(contr);
                }
            }
        }
        warp_append(good, e, out, counter, cap);
    }
}

// keypoint scale in octave pixels: 1.6 * 2^((l + x2) / 3) (gsift.py:462)
__device__ __forceinline__ float kp_scale(int l, float x2) {
    const float t = ((float)l + x2) / 3.f;
    return 1.6f * exp2f(t);
}

constexpr int ORI_WARPS = 8;

__global__ void __launch_bounds__(ORI_WARPS * 32) k_orient(const float* __restrict__ MAG, const float* __restrict__ ANG,
                                                           DetectConsts k, const Refined* __restrict__ ref,
                                                           const uint32_t* n_ref, uint32_t cap_ref,
                                                           Oriented* __restrict__ out, uint32_t* counter,
                                                           uint32_t cap) {
    __shared__ unsigned long long s_hist[ORI_WARPS][ORI_BINS];
    __shared__ float s_raw[ORI_WARPS][ORI_BINS];
    __shared__ float s_sm[ORI_WARPS][ORI_BINS];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n = min(*n_ref, cap_ref);
    const uint32_t nw = gridDim.x * ORI_WARPS;
    for (uint32_t i = blockIdx.x * ORI_WARPS + wid; i < n; i += nw) {
        const Refined e = ref[i];
        const int o = e.o, R = k.g.R[o], C = k.g.C[o];
        const float scl = kp_scale(e.l, e.x2);
        const int rad = min((int)rintf(4.5f * scl), ORI_R_MAX);
        const float sw = 1.5f * scl;
        const float den = 2.f * (sw * sw);
        const int W = 2 * rad + 1;
        const long long gb = k.g.grad_off[o] + (long long)(e.l - 1) * R * C;
        for (int b = lane; b < ORI_BINS; b += 32) s_hist[wid][b] = 0ull;
        __syncwarp();
        for (int s = lane; s < W * W; s += 32) {
            const int ii = s / W - rad, jj = s - (s / W) * W - rad;
            const int y = e.r + ii, x = e.c + jj;
            if (y > 0 && y < R - 1 && x > 0 && x < C - 1) {
                const long long gi = gb + (long long)y * C + x;
                const float d2 = (float)(ii * ii + jj * jj);
                const float w = expf(-d2 / den);
                const float m = MAG[gi] * w;
                int b = (int)rintf(ANG[gi] * 0.1f);
                b = ((b % ORI_BINS) + ORI_BINS) % ORI_BINS;
                atomicAdd(&s_hist[wid][b], (unsigned long long)llrint((double)m * kHistScale));
            }
        }
        __syncwarp();
        for (int b = lane; b < ORI_BINS; b += 32) s_raw[wid][b] = (float)((double)s_hist[wid][b] * kHistInv);
        __syncwarp();
        float hmax = 0.f;
        for (int b = lane; b < ORI_BINS; b += 32) {
            const float* h = s_raw[wid];
            const float v = ((h[(b + 34) % 36] + h[(b + 2) % 36]) * 0.0625f + (h[(b + 35) % 36] + h[(b + 1) % 36]) * 0.25f) +
                            h[b] * 0.375f;
            s_sm[wid][b] = v;
            hmax = fmaxf(hmax, v);
        }
#pragma unroll
        for (int sh = 16; sh; sh >>= 1) hmax = fmaxf(hmax, __shfl_xor_sync(0xffffffffu, hmax, sh));
        __syncwarp();
        const float thr = 0.8f * hmax;
        for (int b0 = 0; b0 < 64; b0 += 32) {
            const int b = b0 + lane;
            bool pk = false;
            Oriented ent{};
            if (b < ORI_BINS) {
                const float* h = s_sm[wid];
                const float hl = h[(b + 35) % 36], hc = h[b], hr = h[(b + 1) % 36];
                pk = hc > hl && hc > hr && hc >= thr && hmax > 0.f;
                if (pk) {
                    float dn = (hl - 2.f * hc) + hr;
                    if (fabsf(dn) < 1e-12f) dn = -1e-12f;
                    const float off = (0.5f * (hl - hr)) / dn;
                    double pos = (double)b + (double)off;
                    if (pos < 0.0) pos += 36.0;
                    if (pos >= 36.0) pos -= 36.0;
                    double ang = 360.0 - 10.0 * pos;
                    if (fabs(ang - 360.0) < 1e-4) ang = 0.0;
                    ent.ri = i; ent.j = b; ent.angle = (float)ang;
                }
            }
            warp_append(pk, ent, out, counter, cap);
        }
        __syncwarp();
    }
}

__global__ void k_sort_keys_a(const Oriented* __restrict__ ori, const Refined* __restrict__ ref, uint32_t n,
                              unsigned long long* __restrict__ key, uint32_t* __restrict__ val) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Oriented e = ori[i];
    key[i] = ((unsigned long long)ref[e.ri].f << 6) | (unsigned long long)e.j;
    val[i] = i;
}

__global__ void k_sort_keys_b(const Oriented* __restrict__ ori, const Refined* __restrict__ ref,
                              const uint32_t* __restrict__ order, uint32_t n, uint32_t* __restrict__ key) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    key[i] = ~__float_as_uint(ref[ori[order[i]].ri].resp);
}

__global__ void k_gather(const Oriented* __restrict__ ori, const Refined* __restrict__ ref,
                         const uint32_t* __restrict__ order, uint32_t n, float* kx, float* ky, float* ksize,
                         float* kang, float* kresp, int32_t* koct, int32_t* klayer) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Oriented e = ori[order[i]];
    const Refined r = ref[e.ri];
    const float f = (float)(1 << r.o) * 0.5f;
    const float scl = kp_scale(r.l, r.x2);
    kx[i] = ((float)r.c + r.x0) * f;
    ky[i] = ((float)r.r + r.x1) * f;
    ksize[i] = (scl * 2.f) * f;
    kang[i] = e.angle;
    kresp[i] = r.resp;
    koct[i] = r.o;
    klayer[i] = r.l;
}

// ------------------------------------------------------------------------------ descriptor
constexpr int DESC_WARPS = 4;
constexpr int DH = (D_WIDTH + 2) * (D_WIDTH + 2) * (D_BINS + 2);   // 360

// NumPy's float32 sum of 128 contiguous values: eight strided partial sums, then a fixed tree.
__device__ __forceinline__ float np_sum128(const float* v, int lane) {
    float r = 0.f;
    if (lane < 8) {
        r = v[lane];
        for (int i = 8 + lane; i < 128; i += 8) r = r + v[i];
    }
    const float r1 = __shfl_down_sync(0xffffffffu, r, 1);
    const float p = r + r1;                                // lanes 0,2,4,6: (r0+r1),(r2+r3),...
    const float p2 = __shfl_down_sync(0xffffffffu, p, 2);
    const float q = p + p2;                                // lanes 0,4: ((r0+r1)+(r2+r3)), ((r4+r5)+(r6+r7))
    const float q4 = __shfl_down_sync(0xffffffffu, q, 4);
    return __shfl_sync(0xffffffffu, q + q4, 0);
}

template <bool EXACT>
__global__ void __launch_bounds__(DESC_WARPS * 32) k_describe(const float* __restrict__ MAG, const float* __restrict__ ANG,
                                                              Geometry g, int n, const float* __restrict__ kx,
                                                              const float* __restrict__ ky, const float* __restrict__ ks,
                                                              const float* __restrict__ ka, const int32_t* __restrict__ ko,
                                                              const int32_t* __restrict__ kl, float* __restrict__ desc,
                                                              uint8_t* __restrict__ u8) {
    __shared__ unsigned long long s_hist[DESC_WARPS][DH];
    __shared__ float s_d[DESC_WARPS][128];
    __shared__ float s_t[DESC_WARPS][128];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = gridDim.x * DESC_WARPS;
    for (int k = blockIdx.x * DESC_WARPS + wid; k < n; k += nw) {
        // keypoint geometry in float64 as the reference's host code computes it (gsift.py:490-501)
        const int o = ko[k], li = kl[k];
        const double f = 1.0 / (exp2((double)o) * 0.5);
        const double px = (double)kx[k] * f, py = (double)ky[k] * f;
        const double scl = (double)ks[k] * f * 0.5;
        double ori = 360.0 - (double)ka[k];
        if (fabs(ori - 360.0) < 1e-4) ori = 0.0;
        const int rows = g.R[o], cols = g.C[o];
        long long rad = llrint(3.0 * scl * 1.4142135623730951 * 5.0 * 0.5);
        const long long rmax = (long long)sqrt((double)rows * rows + (double)cols * cols);
        if (rad > rmax) rad = rmax;
        const int R = (int)rad, W = 2 * R + 1;
        const long long gb = g.grad_off[o] + (long long)(li - 1) * rows * cols;
        const int pr = (int)rint(py), pc = (int)rint(px);
        const double hw = 3.0 * scl;
        const double t = ori * 0.017453292519943295;   // np.radians
        const double cos_d = cos(t) / hw, sin_d = sin(t) / hw;
        const float cos_f = (float)cos_d, sin_f = (float)sin_d, ori_f = (float)ori;
        for (int b = lane; b < DH; b += 32) s_hist[wid][b] = 0ull;
        __syncwarp();
        for (int s = lane; s < W * W; s += 32) {
            const int ii = s / W - R, jj = s - (s / W) * W - R;
            const int y = pr + ii, x = pc + jj;
            if (!(y > 0 && y < rows - 1 && x > 0 && x < cols - 1)) continue;
            int r0, c0, o0;
            double vv[8];
            if (EXACT) {
                const double c_rot = (double)jj * cos_d - (double)ii * sin_d;
                const double r_rot = (double)jj * sin_d + (double)ii * cos_d;
                const double rbin = (r_rot + 2.0) - 0.5, cbin = (c_rot + 2.0) - 0.5;
                if (!(rbin > -1.0 && rbin < 4.0 && cbin > -1.0 && cbin < 4.0)) continue;
                const long long gi = gb + (long long)y * cols + x;
                const double w = exp((c_rot * c_rot + r_rot * r_rot) * (-1.0 / 8.0));
                const double m = (double)MAG[gi] * w;
                const double obin = ((double)ANG[gi] - ori) * (8.0 / 360.0);
                const double fr = floor(rbin), fc = floor(cbin), fo = floor(obin);
                const double rb = rbin - fr, cb = cbin - fc, ob = obin - fo;
                r0 = (int)fr; c0 = (int)fc; o0 = (int)fo;
                const double v_r1 = m * rb, v_r0 = m - v_r1;
                const double v_rc11 = v_r1 * cb, v_rc10 = v_r1 - v_rc11;
                const double v_rc01 = v_r0 * cb, v_rc00 = v_r0 - v_rc01;
                vv[1] = v_rc00 * ob; vv[0] = v_rc00 - vv[1];
                vv[3] = v_rc01 * ob; vv[2] = v_rc01 - vv[3];
                vv[5] = v_rc10 * ob; vv[4] = v_rc10 - vv[5];
                vv[7] = v_rc11 * ob; vv[6] = v_rc11 - vv[7];
            } else {
                const float c_rot = (float)jj * cos_f - (float)ii * sin_f;
                const float r_rot = (float)jj * sin_f + (float)ii * cos_f;
                const float rbin = r_rot + 1.5f, cbin = c_rot + 1.5f;
                if (!(rbin > -1.f && rbin < 4.f && cbin > -1.f && cbin < 4.f)) continue;
                const long long gi = gb + (long long)y * cols + x;
                const float w = expf((c_rot * c_rot + r_rot * r_rot) * (-1.f / 8.f));
                const float m = MAG[gi] * w;
                const float obin = (ANG[gi] - ori_f) * (8.f / 360.f);
                const float fr = floorf(rbin), fc = floorf(cbin), fo = floorf(obin);
                const float rb = rbin - fr, cb = cbin - fc, ob = obin - fo;
                r0 = (int)fr; c0 = (int)fc; o0 = (int)fo;
                const float v_r1 = m * rb, v_r0 = m - v_r1;
                const float v_rc11 = v_r1 * cb, v_rc10 = v_r1 - v_rc11;
                const float v_rc01 = v_r0 * cb, v_rc00 = v_r0 - v_rc01;
                float t1;
                t1 = v_rc00 * ob; vv[1] = t1; vv[0] = v_rc00 - t1;
                t1 = v_rc01 * ob; vv[3] = t1; vv[2] = v_rc01 - t1;
                t1 = v_rc10 * ob; vv[5] = t1; vv[4] = v_rc10 - t1;
                t1 = v_rc11 * ob; vv[7] = t1; vv[6] = v_rc11 - t1;
            }
            if (o0 < 0) o0 += D_BINS;
            if (o0 >= D_BINS) o0 -= D_BINS;
            const int idx = ((r0 + 1) * (D_WIDTH + 2) + c0 + 1) * (D_BINS + 2) + o0;
            unsigned long long* h = s_hist[wid];
            // (r, c, o) corners: 000 001 010 011 100 101 110 111
            atomicAdd(h + idx, (unsigned long long)llrint(vv[0] * kDescScale));
            atomicAdd(h + idx + 1, (unsigned long long)llrint(vv[1] * kDescScale));
            atomicAdd(h + idx + 10, (unsigned long long)llrint(vv[2] * kDescScale));
            atomicAdd(h + idx + 11, (unsigned long long)llrint(vv[3] * kDescScale));
            atomicAdd(h + idx + 60, (unsigned long long)llrint(vv[4] * kDescScale));
            atomicAdd(h + idx + 61, (unsigned long long)llrint(vv[5] * kDescScale));
            atomicAdd(h + idx + 70, (unsigned long long)llrint(vv[6] * kDescScale));
            atomicAdd(h + idx + 71, (unsigned long long)llrint(vv[7] * kDescScale));
        }
        __syncwarp();
        // float32 histogram, fold the angle wrap bins, keep the 4x4x8 interior (gsift.py:789-793)
        float* d = s_d[wid];
        for (int q = lane; q < 128; q += 32) {
            const int rc = q >> 3, ob = q & 7;
            const int r = (rc >> 2) + 1, c = (rc & 3) + 1;
            const unsigned long long* h = s_hist[wid] + (r * (D_WIDTH + 2) + c) * (D_BINS + 2);
            float v = (float)((double)h[ob] * kDescInv);
            if (ob < 2) v = v + (float)((double)h[ob + D_BINS] * kDescInv);
            d[q] = v;
        }
        __syncwarp();
        float sq[4];
        for (int u = 0; u < 4; ++u) sq[u] = d[lane + 32 * u];
        float* tmp = s_t[wid];
        for (int u = 0; u < 4; ++u) tmp[lane + 32 * u] = sq[u] * sq[u];
        __syncwarp();
        const float n1 = sqrtf(np_sum128(tmp, lane));
        const float clip = n1 * 0.2f;
        for (int u = 0; u < 4; ++u) sq[u] = fminf(sq[u], clip);
        __syncwarp();
        for (int u = 0; u < 4; ++u) tmp[lane + 32 * u] = sq[u] * sq[u];
        __syncwarp();
        const float n2 = sqrtf(np_sum128(tmp, lane));
        const float sc = 512.f / fmaxf(n2, 1e-7f);
        for (int u = 0; u < 4; ++u) sq[u] = sq[u] * sc;
        if (desc)
            for (int u = 0; u < 4; ++u) desc[(size_t)k * 128 + lane + 32 * u] = sq[u];
        if (u8) {
            __syncwarp();
            for (int u = 0; u < 4; ++u) tmp[lane + 32 * u] = fabsf(sq[u]);
            __syncwarp();
            const float l1 = np_sum128(tmp, lane) + 1e-7f;
            for (int u = 0; u < 4; ++u) {
                float v = sqrtf(sq[u] / l1) * 512.f;
                v = fminf(fmaxf(v, 0.f), 255.f);
                u8[(size_t)k * 128 + lane + 32 * u] = (uint8_t)v;
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------------ spread
__global__ void k_cells(const float* __restrict__ x, const float* __restrict__ y, int n, float W, float H,
                        uint32_t* __restrict__ cell, uint32_t* __restrict__ iota) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int cx = (int)(x[i] / W * 12.f), cy = (int)(y[i] / H * 9.f);
    cx = min(max(cx, 0), 11);
    cy = min(max(cy, 0), 8);
    cell[i] = (uint32_t)(cy * 12 + cx);
    iota[i] = (uint32_t)i;
}

// positions sorted by cell (ties by index): flag the first `cap` of each cell
__global__ void k_cell_rank(const uint32_t* __restrict__ cell_sorted, int n, int cap, uint8_t* __restrict__ flag) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    // rank = p - first position with the same cell (binary search, cells are sorted)
    const uint32_t c = cell_sorted[p];
    int lo = 0, hi = p;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (cell_sorted[mid] < c) lo = mid + 1; else hi = mid;
    }
    flag[p] = (p - lo) < cap ? 1 : 0;
}

__global__ void k_mark(const uint32_t* __restrict__ sel, int n_sel, uint8_t* __restrict__ chosen) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_sel) chosen[sel[i]] = 1;
}

__global__ void k_not(const uint8_t* __restrict__ a, uint8_t* __restrict__ b, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i] ? 0 : 1;
}

__global__ void k_resp_keys(const uint32_t* __restrict__ sel, int n, const float* __restrict__ resp,
                            uint32_t* __restrict__ key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) key[i] = ~__float_as_uint(resp[sel[i]]);
}

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

DetectConsts make_consts(const Geometry& g, double contrast, double edge) {
    DetectConsts k{};
    k.g = g;
    k.pthr = (float)(0.8 * 0.5 * contrast / N_LAYERS);
    k.contrast = (float)contrast;
    k.edge = (float)edge;
    k.e1sq = (float)((edge + 1.0) * (edge + 1.0));
    long long acc = 0;
    for (int o = 0; o < g.n_oct; ++o) {
        k.vox_off[o] = acc;
        acc += (long long)N_LAYERS * (g.R[o] - 2 * BORDER) * (g.C[o] - 2 * BORDER);
    }
    k.vox_off[g.n_oct] = acc;
    return k;
}

}  // namespace

// Full detection pipeline; contrast/edge in double as the reference's Python floats.
int32_t run_detect(fsb_ctx* ctx, Workspace& ws, double contrast, double edge, int max_kp) {
    cudaStream_t s = ctx->stream;
    const Geometry& g = ws.g;
    const DetectConsts k = make_consts(g, contrast, edge);
    uint32_t* cnt = ws.counters.as<uint32_t>();
    const float* DF = ws.dog.as<float>();
    uint32_t h_cnt[3];
    ctx->stage_begin(ST_EXTREMA);
    for (int attempt = 0; attempt < 3; ++attempt) {
        FSB_CUDA(cudaMemsetAsync(cnt, 0, 3 * sizeof(uint32_t), s));
        const long long nvox = k.vox_off[g.n_oct];
        if (nvox > 0) {
            k_extrema<<<blocks(nvox, 256), 256, 0, s>>>(DF, k, ws.cand.as<uint32_t>(), cnt, (uint32_t)ws.cap_cand);
            note_launch();
        }
        FSB_CUDA(cudaGetLastError());
        FSB_CUDA(cudaMemcpyAsync(h_cnt, cnt, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaStreamSynchronize(s));
        if (h_cnt[0] <= ws.cap_cand) break;
        ws.cap_cand = (size_t)h_cnt[0] + (h_cnt[0] >> 3) + 1024;
        FSB_TRY(ws.cand.ensure(ws.cap_cand * sizeof(uint32_t)));
    }
    ctx->stage_end(ST_EXTREMA);
    const uint32_t n_cand = h_cnt[0];
    if (n_cand == 0) { ws.n_kp = 0; return FSB_OK; }
    if (ws.cap_ref < n_cand) {
        ws.cap_ref = n_cand;
        FSB_TRY(ws.refined.ensure(ws.cap_ref * sizeof(Refined)));
    }
    ctx->stage_begin(ST_REFINE);
    k_refine<<<blocks(n_cand, 128), 128, 0, s>>>(DF, k, ws.cand.as<uint32_t>(), cnt, (uint32_t)ws.cap_cand,
                                                 ws.refined.as<Refined>(), cnt + 1, (uint32_t)ws.cap_ref);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    FSB_CUDA(cudaMemcpyAsync(h_cnt + 1, cnt + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    ctx->stage_end(ST_REFINE);
    const uint32_t n_ref = h_cnt[1];
    if (n_ref == 0) { ws.n_kp = 0; return FSB_OK; }
    uint32_t n_ori = 0;
    ctx->stage_begin(ST_ORIENT);
    for (int attempt = 0; attempt < 3; ++attempt) {
        if (ws.cap_ori < (size_t)n_ref * 2 + 1024) ws.cap_ori = (size_t)n_ref * 2 + 1024;
        FSB_TRY(ws.oriented.ensure(ws.cap_ori * sizeof(Oriented)));
        FSB_CUDA(cudaMemsetAsync(cnt + 2, 0, sizeof(uint32_t), s));
        const unsigned ob = blocks(n_ref, ORI_WARPS);
        k_orient<<<ob < 148 * 16 ? ob : 148 * 16, ORI_WARPS * 32, 0, s>>>(
            ws.mag.as<float>(), ws.ang.as<float>(), k, ws.refined.as<Refined>(), cnt + 1, (uint32_t)ws.cap_ref,
            ws.oriented.as<Oriented>(), cnt + 2, (uint32_t)ws.cap_ori);
        note_launch();
        FSB_CUDA(cudaGetLastError());
        FSB_CUDA(cudaMemcpyAsync(h_cnt + 2, cnt + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaStreamSynchronize(s));
        n_ori = h_cnt[2];
        if (n_ori <= ws.cap_ori) break;
        ws.cap_ori = (size_t)n_ori + 1024;
    }
    ctx->stage_end(ST_ORIENT);
    if (n_ori > ws.cap_ori) { set_error("orientation list overflow"); return FSB_ERR_OVERFLOW; }
    if (n_ori == 0) { ws.n_kp = 0; return FSB_OK; }
    ctx->stage_begin(ST_SORT);
    // stable two-key sort: (extremum index, bin) ascending, then response descending
    FSB_TRY(ws.keys_a.ensure((size_t)n_ori * 8 * 2));
    FSB_TRY(ws.vals_a.ensure((size_t)n_ori * 4 * 2));
    FSB_TRY(ws.keys_b.ensure((size_t)n_ori * 4 * 2));
    FSB_TRY(ws.vals_b.ensure((size_t)n_ori * 4 * 2));
    unsigned long long* ka = ws.keys_a.as<unsigned long long>();
    uint32_t* va = ws.vals_a.as<uint32_t>();
    uint32_t* kb = ws.keys_b.as<uint32_t>();
    uint32_t* vb = ws.vals_b.as<uint32_t>();
    int fbits = 1;
    while ((1ull << fbits) < (unsigned long long)g.dog_off[g.n_oct]) ++fbits;
    const int end_a = fbits + 6;
    size_t t1 = 0, t2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, ka, ka + n_ori, va, va + n_ori, (int)n_ori, 0, end_a, s);
    cub::DeviceRadixSort::SortPairs(nullptr, t2, kb, kb + n_ori, vb, vb + n_ori, (int)n_ori, 0, 32, s);
    FSB_TRY(ws.sort_tmp.ensure(t1 > t2 ? t1 : t2));
    size_t tb = ws.sort_tmp.bytes;
    k_sort_keys_a<<<blocks(n_ori, 256), 256, 0, s>>>(ws.oriented.as<Oriented>(), ws.refined.as<Refined>(), n_ori, ka, va);
    FSB_CUDA(cub::DeviceRadixSort::SortPairs(ws.sort_tmp.p, tb, ka, ka + n_ori, va, va + n_ori, (int)n_ori, 0, end_a, s));
    k_sort_keys_b<<<blocks(n_ori, 256), 256, 0, s>>>(ws.oriented.as<Oriented>(), ws.refined.as<Refined>(), va + n_ori,
                                                     n_ori, kb);
    tb = ws.sort_tmp.bytes;
    FSB_CUDA(cub::DeviceRadixSort::SortPairs(ws.sort_tmp.p, tb, kb, kb + n_ori, va + n_ori, vb, (int)n_ori, 0, 32, s));
    const uint32_t n_keep = n_ori < (uint32_t)max_kp ? n_ori : (uint32_t)max_kp;
    const size_t nb4 = (size_t)(n_keep ? n_keep : 1) * 4;
    FSB_TRY(ws.kx.ensure(nb4));
    FSB_TRY(ws.ky.ensure(nb4));
    FSB_TRY(ws.ksize.ensure(nb4));
    FSB_TRY(ws.kangle.ensure(nb4));
    FSB_TRY(ws.kresp.ensure(nb4));
    FSB_TRY(ws.koct.ensure(nb4));
    FSB_TRY(ws.klayer.ensure(nb4));
    if (n_keep)
        k_gather<<<blocks(n_keep, 256), 256, 0, s>>>(ws.oriented.as<Oriented>(), ws.refined.as<Refined>(), vb, n_keep,
                                                     ws.kx.as<float>(), ws.ky.as<float>(), ws.ksize.as<float>(),
                                                     ws.kangle.as<float>(), ws.kresp.as<float>(), ws.koct.as<int32_t>(),
                                                     ws.klayer.as<int32_t>());
    note_launch(n_keep ? 3 : 2);
    FSB_CUDA(cudaGetLastError());
    ctx->stage_end(ST_SORT);
    ws.n_kp = (int)n_keep;
    return FSB_OK;
}

int32_t run_describe_mode(const Workspace& ws, int n, const float* d_x, const float* d_y, const float* d_size,
                          const float* d_angle, const int32_t* d_oct, const int32_t* d_layer, float* d_desc,
                          uint8_t* d_u8, bool exact, cudaStream_t s) {
    if (n <= 0) return FSB_OK;
    const unsigned nb = blocks(n, DESC_WARPS);
    const unsigned grid = nb < 148u * 32u ? nb : 148u * 32u;
    if (exact)
        k_describe<true><<<grid, DESC_WARPS * 32, 0, s>>>(ws.mag.as<float>(), ws.ang.as<float>(), ws.g, n, d_x, d_y,
                                                          d_size, d_angle, d_oct, d_layer, d_desc, d_u8);
    else
        k_describe<false><<<grid, DESC_WARPS * 32, 0, s>>>(ws.mag.as<float>(), ws.ang.as<float>(), ws.g, n, d_x, d_y,
                                                           d_size, d_angle, d_oct, d_layer, d_desc, d_u8);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

int32_t run_describe(const Workspace& ws, int n, const float* d_x, const float* d_y, const float* d_size,
                     const float* d_angle, const int32_t* d_oct, const int32_t* d_layer, float* d_desc,
                     uint8_t* d_u8, cudaStream_t s) {
    return run_describe_mode(ws, n, d_x, d_y, d_size, d_angle, d_oct, d_layer, d_desc, d_u8, false, s);
}

// grid-spread selection of nfeat keypoints out of the detected (response-sorted) ones,
// features.py:38-57 followed by the stable response sort of features.py:126. Writes the selected
// keypoint indices to d_sel and their count to *n_sel.
int32_t run_spread(const Workspace& ws, int nfeat, int32_t* d_sel_out, int* n_sel, fsb_ctx* ctx, cudaStream_t s) {
    const int n = ws.n_kp;
    uint32_t* sel = reinterpret_cast<uint32_t*>(d_sel_out);
    if (n <= nfeat) {
        // every keypoint, already in stable response order
        std::vector<uint32_t> idx(n);
        for (int i = 0; i < n; ++i) idx[i] = (uint32_t)i;
        if (n) FSB_CUDA(cudaMemcpyAsync(sel, idx.data(), n * 4, cudaMemcpyHostToDevice, s));
        FSB_CUDA(cudaStreamSynchronize(s));
        *n_sel = n;
        return FSB_OK;
    }
    const size_t N = (size_t)n;
    FSB_TRY(ctx->s_misc.ensure(N * 4 * 7 + N * 2 + 64));
    uint32_t* cell = ctx->s_misc.as<uint32_t>();
    uint32_t* iota = cell + N;
    uint32_t* cell_s = iota + N;
    uint32_t* idx_s = cell_s + N;
    uint32_t* rest = idx_s + N;
    uint32_t* keyb = rest + N;
    uint8_t* flag = reinterpret_cast<uint8_t*>(keyb + 2 * N);
    uint8_t* chosen = flag + N;
    FSB_TRY(ctx->s_i32.ensure(64));
    int* d_cnt = ctx->s_i32.as<int>();
    k_cells<<<blocks(n, 256), 256, 0, s>>>(ws.kx.as<float>(), ws.ky.as<float>(), n, (float)ws.g.w, (float)ws.g.h, cell, iota);
    size_t t1 = 0, t2 = 0, t3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, cell, cell_s, iota, idx_s, n, 0, 7, s);
    cub::DeviceSelect::Flagged(nullptr, t2, idx_s, flag, sel, d_cnt, n, s);
    cub::DeviceRadixSort::SortPairs(nullptr, t3, keyb, keyb, sel, sel, nfeat, 0, 32, s);
    size_t tmax = t1 > t2 ? t1 : t2;
    tmax = tmax > t3 ? tmax : t3;
    FSB_TRY(ctx->s_misc2.ensure(tmax + N * 8 + 256));
    void* tmp = ctx->s_misc2.p;
    uint32_t* sel2 = reinterpret_cast<uint32_t*>(static_cast<char*>(tmp) + ((tmax + 255) / 256) * 256);
    size_t tb = tmax;
    FSB_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, cell, cell_s, iota, idx_s, n, 0, 7, s));
    const int cap = (nfeat + 107) / 108;
    k_cell_rank<<<blocks(n, 256), 256, 0, s>>>(cell_s, n, cap, flag);
    tb = tmax;
    FSB_CUDA(cub::DeviceSelect::Flagged(tmp, tb, idx_s, flag, sel2, d_cnt, n, s));
    int n1 = 0;
    FSB_CUDA(cudaMemcpyAsync(&n1, d_cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    if (n1 > nfeat) n1 = nfeat;
    if (n1 < nfeat) {
        FSB_CUDA(cudaMemsetAsync(chosen, 0, N, s));
        if (n1 > 0) k_mark<<<blocks(n1, 256), 256, 0, s>>>(sel2, n1, chosen);
        k_not<<<blocks(n, 256), 256, 0, s>>>(chosen, flag, n);
        tb = tmax;
        FSB_CUDA(cub::DeviceSelect::Flagged(tmp, tb, iota, flag, rest, d_cnt + 2, n, s));
        // rest is in index order == response order (ties by index)
        FSB_CUDA(cudaMemcpyAsync(sel2 + n1, rest, (size_t)(nfeat - n1) * 4, cudaMemcpyDeviceToDevice, s));
    }
    // stable sort of the selection by response, descending (features.py:126)
    k_resp_keys<<<blocks(nfeat, 256), 256, 0, s>>>(sel2, nfeat, ws.kresp.as<float>(), keyb);
    note_launch(n1 < nfeat ? 5 : 3);
    tb = tmax;
    FSB_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keyb, keyb + N, sel2, sel, nfeat, 0, 32, s));
    FSB_CUDA(cudaGetLastError());
    *n_sel = nfeat;
    return FSB_OK;
}

}  // namespace fsb
