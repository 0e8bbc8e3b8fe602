// Orientation histograms and 128-d descriptors (gather kernels over the gradient atlases).
//
// Compiled with --fmad=false (float32 expressions round once per operation, as the reference's).
// Both histograms are accumulated without atomics, in float64, in a fixed order, so results are
// deterministic and the float32 bins equal the reference's float64 bincount sums except in the
// last bit of rare cases:
//   k_orient    warp per refined extremum, visited in rank order (response descending); each
//               lane owns a private 36-bin float64 column in shared memory; bins are then summed
//               over lanes in lane order (gsift.py:372-432); the extremum's peaks go to its rank's
//               slots in bin order.
//   k_describe  warp per keypoint; lane u < 25 owns one unit square of the rotated bin grid and
//               visits each of its samples once (row by row, the column interval solved in closed
//               form), adding the sample's trilinear split with the reference's operation order
//               (gsift.py:528-591 for float32 sample math, gsift.py:800-871 for float64 in exact
//               mode) into private accumulators of the four cells it touches; then fixed-order
//               cell sums, fold, L2 clip at 0.2, renormalise to 512 and the RootSIFT bytes of the
//               feature file (features.py:80-82), with NumPy's float32 summation order.
#include <cmath>
#include <type_traits>

#include "fsb_internal.cuh"

namespace fsb {
namespace {

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// keypoint scale in octave pixels: 1.6 * 2^((l + x2) / 3) (gsift.py:462)
__device__ __forceinline__ float kp_scale(int l, float x2) {
    const float t = ((float)l + x2) / 3.f;
    return 1.6f * exp2f(t);
}

// --------------------------------------------------------------------------------- orientation
constexpr int OW = 4;   // warps per block

// Acc = double reproduces the reference's float64 bincount in every case that matters (exact
// mode); Acc = float (per-lane sums of at most 35 samples, then a float64 lane reduction) halves
// the shared memory for occupancy in the default mode.
template <class Acc>
__global__ void __launch_bounds__(OW * 32) k_orient(const float* __restrict__ MAG, const float* __restrict__ ANG,
                                                    Geometry g, const Refined* __restrict__ ref,
                                                    const uint32_t* __restrict__ order, uint32_t k0, uint32_t k1,
                                                    const uint32_t* __restrict__ d_range,
                                                    Oriented* __restrict__ slots, uint32_t* __restrict__ cnt,
                                                    uint32_t* total) {
    if (d_range) {   // the rank range on the device ([k0, k1) of this pass)
        k0 = d_range[0];
        k1 = d_range[1];
    }
    __shared__ Acc s_acc[OW][ORI_BINS][33];
    __shared__ float s_raw[OW][ORI_BINS];
    __shared__ float s_sm[OW][ORI_BINS];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t nw = gridDim.x * OW;
    Acc (*acc)[33] = s_acc[wid];
    for (uint32_t t = k0 + blockIdx.x * OW + wid; t < k1; t += nw) {
        const uint32_t i = order[t];
        const Refined e = ref[i];
        const int o = e.o, R = g.R[o], C = g.C[o];
        const float scl = kp_scale(e.l, e.x2);
        const int rad = min((int)rintf(4.5f * scl), ORI_R_MAX);
        const float sw = 1.5f * scl;
        const float den = 2.f * (sw * sw);
        const int W = 2 * rad + 1;
        const long long gb = g.grad_off[o] + (long long)(e.l - 1) * R * C;
        for (int b = 0; b < ORI_BINS; ++b) acc[b][lane] = (Acc)0;
        // lane takes samples s = lane, lane + 32, ... of the W x W window (row-major); the window
        // position advances by (32 / W, 32 % W) per step, one division per keypoint
        const int dq = 32 / W, dr = 32 - dq * W;
        int ii = lane / W - rad, jj = lane - (lane / W) * W - rad;
        // two samples per step: both gathers are issued before either is accumulated (the
        // accumulation order of the lane is unchanged)
        for (int s = lane; s < W * W; s += 64) {
            int ii2 = ii + dq, jj2 = jj + dr;
            if (jj2 > rad) {
                jj2 -= W;
                ++ii2;
            }
            const int y1 = e.r + ii, x1 = e.c + jj, y2 = e.r + ii2, x2 = e.c + jj2;
            const bool in1 = y1 > 0 && y1 < R - 1 && x1 > 0 && x1 < C - 1;
            const bool in2 = s + 32 < W * W && y2 > 0 && y2 < R - 1 && x2 > 0 && x2 < C - 1;
            const long long g1 = gb + (long long)y1 * C + x1, g2 = gb + (long long)y2 * C + x2;
            const float m1 = in1 ? __ldg(MAG + g1) : 0.f, a1 = in1 ? __ldg(ANG + g1) : 0.f;
            const float m2 = in2 ? __ldg(MAG + g2) : 0.f, a2 = in2 ? __ldg(ANG + g2) : 0.f;
            if (in1) {
                const float w = expf(-(float)(ii * ii + jj * jj) / den);
                int b = (int)rintf(a1 * 0.1f);   // angles lie in [0, 360]: b in [0, 36]
                if (b >= ORI_BINS) b -= ORI_BINS;
                if (b < 0) b += ORI_BINS;
                acc[b][lane] += (Acc)(m1 * w);
            }
            if (in2) {
                const float w = expf(-(float)(ii2 * ii2 + jj2 * jj2) / den);
                int b = (int)rintf(a2 * 0.1f);
                if (b >= ORI_BINS) b -= ORI_BINS;
                if (b < 0) b += ORI_BINS;
                acc[b][lane] += (Acc)(m2 * w);
            }
            ii = ii2 + dq;
            jj = jj2 + dr;
            if (jj > rad) {
                jj -= W;
                ++ii;
            }
        }
        __syncwarp();
        for (int b = lane; b < ORI_BINS; b += 32) {
            double t = 0.0;
            for (int l = 0; l < 32; ++l) t += (double)acc[b][l];
            s_raw[wid][b] = (float)t;
        }
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
        uint32_t npk = 0;   // peaks of this extremum so far, in bin order
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
            const unsigned m = __ballot_sync(0xffffffffu, pk);
            if (pk) slots[(size_t)t * ORI_SLOTS + npk + __popc(m & ((1u << lane) - 1u))] = ent;
            npk += __popc(m);
        }
        if (lane == 0) {
            cnt[t] = npk;
            atomicAdd(total, npk);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------- descriptor
constexpr int DW = 4;            // warps per block (one keypoint per warp)
constexpr int NB = D_BINS + 1;   // orientation bins a cell can receive (o0 in 0..7, o0 + 1 in 1..8)
constexpr int NSQ = 25;          // unit squares of the padded 5 x 5 bin grid (floor(rbin), floor(cbin) in -1..3)

// NumPy's float32 sum of 128 contiguous values: eight strided partial sums, then a fixed tree.
__device__ __forceinline__ float np_sum128(const float* v, int lane) {
    float r = 0.f;
    if (lane < 8) {
        r = v[lane];
        for (int i = 8 + lane; i < 128; i += 8) r = r + v[i];
    }
    const float r1 = __shfl_down_sync(0xffffffffu, r, 1);
    const float p = r + r1;
    const float p2 = __shfl_down_sync(0xffffffffu, p, 2);
    const float q = p + p2;
    const float q4 = __shfl_down_sync(0xffffffffu, q, 4);
    return __shfl_sync(0xffffffffu, q + q4, 0);
}

// integer interval of j where lo <= a*j + b < hi (one extra on each side), clamped to [-R, R]
__device__ __forceinline__ void j_range(float a, float b, float lo, float hi, int R, int& j0, int& j1) {
    if (fabsf(a) < 1e-12f) {
        if (b >= lo - 1e-4f && b < hi + 1e-4f) { j0 = -R; j1 = R; } else { j0 = 1; j1 = 0; }
        return;
    }
    float u = (lo - b) / a, v = (hi - b) / a;
    if (u > v) { const float t = u; u = v; v = t; }
    j0 = max(-R, (int)floorf(u) - 1);
    j1 = min(R, (int)ceilf(v) + 1);
}

// One warp per keypoint. Lane u < 25 owns the unit square (R', C') = (u / 5 - 1, u % 5 - 1) of
// bin space: the samples with floor(rbin) = R' and floor(cbin) = C'. It walks the pixels of that
// rotated square row by row (column interval in closed form), and adds each sample's trilinear
// split (the reference's operation order) into its private accumulators for the four cells
// (R' + dr, C' + dc) it touches. Cell (R, C) then sums its four contributors in a fixed order.
template <bool EXACT>
__global__ void __launch_bounds__(DW * 32) k_describe(const float* __restrict__ MAG, const float* __restrict__ ANG,
                                                      Geometry g, int n, const int* __restrict__ d_n,
                                                      const float* __restrict__ kx,
                                                      const float* __restrict__ ky, const float* __restrict__ ks,
                                                      const float* __restrict__ ka, const int32_t* __restrict__ ko,
                                                      const int32_t* __restrict__ kl, float* __restrict__ desc,
                                                      uint8_t* __restrict__ u8) {
    typedef typename std::conditional<EXACT, double, float>::type Acc;
    __shared__ Acc s_acc[DW][4 * NB][32];
    __shared__ float s_d[DW][128];
    __shared__ float s_t[DW][128];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Acc (*acc)[32] = s_acc[wid];
    const int Rq = lane / 5 - 1, Cq = lane % 5 - 1;
    if (d_n) n = min(*d_n, n);   // the count on the device, n a capacity
    for (int k = blockIdx.x * DW + wid; k < n; k += gridDim.x * DW) {
        for (int b = 0; b < 4 * NB; ++b) acc[b][lane] = (Acc)0;
        // keypoint geometry in float64 as the reference's host code computes it (gsift.py:490-501)
        const int o = ko[k], li = kl[k];
        const double f = 1.0 / (exp2((double)o) * 0.5);
        const double px = (double)kx[k] * f, py = (double)ky[k] * f;
        const double scl = (double)ks[k] * f * 0.5;
        double ori = 360.0 - (double)ka[k];
        if (fabs(ori - 360.0) < 1e-4) ori = 0.0;
        const int rows = g.R[o], cols = g.C[o];
        long long radl = llrint(3.0 * scl * 1.4142135623730951 * 5.0 * 0.5);
        const long long rmax = (long long)sqrt((double)rows * rows + (double)cols * cols);
        if (radl > rmax) radl = rmax;
        const int rad = (int)radl;
        const long long gb = g.grad_off[o] + (long long)(li - 1) * rows * cols;
        const int pr = (int)rint(py), pc = (int)rint(px);
        const double hw = 3.0 * scl;
        const double t = ori * 0.017453292519943295;
        const double cos_d = cos(t) / hw, sin_d = sin(t) / hw;
        const float cos_f = (float)cos_d, sin_f = (float)sin_d, ori_f = (float)ori;
        if (lane < NSQ) {
            // pixel rows of this unit square: i = hw^2 (r_rot cos - c_rot sin) at its corners
            const float k2 = (float)(hw * hw);
            float imin = 1e30f, imax = -1e30f;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float rr = (float)(Rq + (q >> 1)) - 1.5f, cc = (float)(Cq + (q & 1)) - 1.5f;
                const float iv = k2 * (rr * cos_f - cc * sin_f);
                imin = fminf(imin, iv);
                imax = fmaxf(imax, iv);
            }
            const int i0 = max(-rad, (int)floorf(imin) - 1), i1 = min(rad, (int)ceilf(imax) + 1);
            for (int ii = i0; ii <= i1; ++ii) {
                const int y = pr + ii;
                if (!(y > 0 && y < rows - 1)) continue;
                int ja, jb, jc, jd;
                j_range(sin_f, (float)ii * cos_f + 1.5f, (float)Rq, (float)(Rq + 1), rad, ja, jb);
                j_range(cos_f, -(float)ii * sin_f + 1.5f, (float)Cq, (float)(Cq + 1), rad, jc, jd);
                const int j0 = max(ja, jc), j1 = min(jb, jd);
                const float* mrow = MAG + gb + (long long)y * cols;
                const float* arow = ANG + gb + (long long)y * cols;
                // four pixels per step: their gradient loads are issued before any is used, the
                // accumulation order stays pixel by pixel
                for (int jb = j0; jb <= j1; jb += 4) {
                float mv4[4], av4[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int x = pc + jb + u;
                    const bool in = jb + u <= j1 && x > 0 && x < cols - 1;
                    mv4[u] = in ? __ldg(mrow + x) : 0.f;
                    av4[u] = in ? __ldg(arow + x) : 0.f;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int jj = jb + u;
                    const int x = pc + jj;
                    if (!(jj <= j1 && x > 0 && x < cols - 1)) continue;
                    const float mval = mv4[u], aval = av4[u];
                    Acc v[8];
                    int o0;
                    if (EXACT) {
                        const double c_rot = (double)jj * cos_d - (double)ii * sin_d;
                        const double r_rot = (double)jj * sin_d + (double)ii * cos_d;
                        const double rbin = (r_rot + 2.0) - 0.5, cbin = (c_rot + 2.0) - 0.5;
                        if (!(rbin > -1.0 && rbin < 4.0 && cbin > -1.0 && cbin < 4.0)) continue;
                        const double fr = floor(rbin), fc = floor(cbin);
                        if ((int)fr != Rq || (int)fc != Cq) continue;
                        const double w = exp((c_rot * c_rot + r_rot * r_rot) * (-1.0 / 8.0));
                        const double m = (double)mval * w;
                        const double obin = ((double)aval - ori) * (8.0 / 360.0);
                        const double fo = floor(obin);
                        const double rb = rbin - fr, cb = cbin - fc, ob = obin - fo;
                        o0 = (int)fo;
                        const double v_r1 = m * rb, v_r0 = m - v_r1;
                        const double v_rc11 = v_r1 * cb, v_rc10 = v_r1 - v_rc11;
                        const double v_rc01 = v_r0 * cb, v_rc00 = v_r0 - v_rc01;
                        v[1] = v_rc00 * ob; v[0] = v_rc00 - v[1];
                        v[3] = v_rc01 * ob; v[2] = v_rc01 - v[3];
                        v[5] = v_rc10 * ob; v[4] = v_rc10 - v[5];
                        v[7] = v_rc11 * ob; v[6] = v_rc11 - v[7];
                    } else {
                        const float c_rot = (float)jj * cos_f - (float)ii * sin_f;
                        const float r_rot = (float)jj * sin_f + (float)ii * cos_f;
                        const float rbin = r_rot + 1.5f, cbin = c_rot + 1.5f;
                        if (!(rbin > -1.f && rbin < 4.f && cbin > -1.f && cbin < 4.f)) continue;
                        const float fr = floorf(rbin), fc = floorf(cbin);
                        if ((int)fr != Rq || (int)fc != Cq) continue;
                        const float w = expf((c_rot * c_rot + r_rot * r_rot) * (-1.f / 8.f));
                        const float m = mval * w;
                        const float obin = (aval - ori_f) * (8.f / 360.f);
                        const float fo = floorf(obin);
                        const float rb = rbin - fr, cb = cbin - fc, ob = obin - fo;
                        o0 = (int)fo;
                        const float v_r1 = m * rb, v_r0 = m - v_r1;
                        const float v_rc11 = v_r1 * cb, v_rc10 = v_r1 - v_rc11;
                        const float v_rc01 = v_r0 * cb, v_rc00 = v_r0 - v_rc01;
                        float h;
                        h = v_rc00 * ob; v[1] = h; v[0] = v_rc00 - h;
                        h = v_rc01 * ob; v[3] = h; v[2] = v_rc01 - h;
                        h = v_rc10 * ob; v[5] = h; v[4] = v_rc10 - h;
                        h = v_rc11 * ob; v[7] = h; v[6] = v_rc11 - h;
                    }
                    if (o0 < 0) o0 += D_BINS;
                    if (o0 >= D_BINS) o0 -= D_BINS;
                    // corners (dr, dc) = 00, 01, 10, 11 -> private cell slots 0..3
#pragma unroll
                    for (int c4 = 0; c4 < 4; ++c4) {
                        acc[c4 * NB + o0][lane] += v[2 * c4];
                        acc[c4 * NB + o0 + 1][lane] += v[2 * c4 + 1];
                    }
                }
                }
            }
        }
        __syncwarp();
        // cell (R, C) in 0..3 x 0..3 sums the squares (R - dr, C - dc) in a fixed order; fold the
        // angle wrap bin (gsift.py:789-793)
        for (int q = lane; q < 128; q += 32) {
            const int cell = q >> 3, ob = q & 7;
            const int R = cell >> 2, C = cell & 3;
            double sum0 = 0.0, sum8 = 0.0;
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4) {
                const int dr = c4 >> 1, dc = c4 & 1;
                const int sq = (R - dr + 1) * 5 + (C - dc + 1);
                sum0 += (double)acc[c4 * NB + ob][sq];
                if (ob == 0) sum8 += (double)acc[c4 * NB + D_BINS][sq];
            }
            float v = (float)sum0;
            if (ob == 0) v = v + (float)sum8;
            s_d[wid][q] = v;
        }
        __syncwarp();
        const float* d = s_d[wid];
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

}  // namespace

int32_t run_orient(const Workspace& ws, const Refined* ref, const uint32_t* order, uint32_t k0, uint32_t k1,
                   Oriented* slots, uint32_t* cnt, uint32_t* d_total, bool exact, cudaStream_t s) {
    if (k1 <= k0) return FSB_OK;
    const unsigned ob = blocks(k1 - k0, OW);
    const unsigned grid = ob < 148 * 32 ? ob : 148 * 32;
    if (exact)
        k_orient<double><<<grid, OW * 32, 0, s>>>(ws.mag.as<float>(), ws.ang.as<float>(), ws.g, ref, order, k0, k1,
                                                  nullptr, slots, cnt, d_total);
    else
        k_orient<float><<<grid, OW * 32, 0, s>>>(ws.mag.as<float>(), ws.ang.as<float>(), ws.g, ref, order, k0, k1,
                                                 nullptr, slots, cnt, d_total);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

int32_t run_describe_mode(const Workspace& ws, int n, const float* d_x, const float* d_y, const float* d_size,
                          const float* d_angle, const int32_t* d_oct, const int32_t* d_layer, float* d_desc,
                          uint8_t* d_u8, bool exact, cudaStream_t s) {
    if (n <= 0) return FSB_OK;
    const unsigned nb = blocks(n, DW);
    const unsigned grid = nb < 148u * 32u ? nb : 148u * 32u;
    if (exact)
        k_describe<true><<<grid, DW * 32, 0, s>>>(ws.mag.as<float>(), ws.ang.as<float>(), ws.g, n, nullptr, d_x, d_y,
                                                  d_size,
                                                  d_angle, d_oct, d_layer, d_desc, d_u8);
    else
        k_describe<false><<<grid, DW * 32, 0, s>>>(ws.mag.as<float>(), ws.ang.as<float>(), ws.g, n, nullptr, d_x, d_y,
                                                   d_size,
                                                   d_angle, d_oct, d_layer, d_desc, d_u8);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

// Orientation of ranks [d_range[0], d_range[1]) read on the device; grid sized for max_ranks ranks.
int32_t run_orient_dev(const Workspace& ws, const Refined* ref, const uint32_t* order, uint32_t max_ranks,
                       const uint32_t* d_range, Oriented* slots, uint32_t* cnt, uint32_t* d_total, bool exact,
                       cudaStream_t s) {
    if (max_ranks == 0) return FSB_OK;
    const unsigned ob = blocks(max_ranks, OW);
    const unsigned grid = ob < 148 * 32 ? ob : 148 * 32;
    if (exact)
        k_orient<double><<<grid, OW * 32, 0, s>>>(ws.mag.as<float>(), ws.ang.as<float>(), ws.g, ref, order, 0, 0,
                                                  d_range, slots, cnt, d_total);
    else
        k_orient<float><<<grid, OW * 32, 0, s>>>(ws.mag.as<float>(), ws.ang.as<float>(), ws.g, ref, order, 0, 0,
                                                 d_range, slots, cnt, d_total);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

// Descriptors of *d_n keypoints (read on the device; at most cap), grid sized for cap.
int32_t run_describe_dev(const Workspace& ws, int cap, const int* d_n, const float* d_x, const float* d_y,
                         const float* d_size, const float* d_angle, const int32_t* d_oct, const int32_t* d_layer,
                         float* d_desc, uint8_t* d_u8, bool exact, cudaStream_t s) {
    if (cap <= 0) return FSB_OK;
    const unsigned nb = blocks(cap, DW);
    const unsigned grid = nb < 148u * 32u ? nb : 148u * 32u;
    if (exact)
        k_describe<true><<<grid, DW * 32, 0, s>>>(ws.mag.as<float>(), ws.ang.as<float>(), ws.g, cap, d_n, d_x, d_y,
                                                  d_size, d_angle, d_oct, d_layer, d_desc, d_u8);
    else
        k_describe<false><<<grid, DW * 32, 0, s>>>(ws.mag.as<float>(), ws.ang.as<float>(), ws.g, cap, d_n, d_x, d_y,
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

}  // namespace fsb
