// Fused octave kernel: the five layer blurs of one octave in one pass over HBM.
//
// Reference: app/planesite/gsift.py:85-87 (separable mirror blur), 158-179 (layers, DoG,
// downsample), 244-267 (gradient magnitude / angle of gauss layers 1..3).
//
// A CTA owns a 168-column strip and a range of output rows and streams down the rows, S = 4 rows
// per step. Stage i (1..5) keeps the rows of L_{i-1} it still needs in a shared-memory ring
// (2 r_i + S rows; L0's ring has S more rows so the next step's rows load with cp.async while
// this step computes) and produces S new rows of L_i per step:
//   vertical pass   thread = (column pair, row pair): float2 loads of 2 r + 2 ring rows, two
//                   output rows, stored row-pair-interleaved;
//   horizontal pass thread = (row pair, column pair): r + 1 16-byte loads, two output columns
//                   of two rows, stored into the next ring.
// Arithmetic is packed FP32x2 (__ffma2_rn / __fadd2_rn) with symmetric tap pairing
// w_0 x_0 + sum_j w_j (x_-j + x_j): a mirrored input gives a bit-identical mirrored output, so
// mirroring L0 once when it is loaded reproduces the reference's per-layer reflect-101 borders.
// After each stage the epilogue writes, for the strip's output rows, the DoG L_i - L_{i-1}, the
// gradient of L_{i-1} (layers 1..3) and L_3[::2, ::2] (the next octave's base), with 16-byte
// stores where the row pitch allows. HBM traffic per octave pixel: L0 read once (plus the column
// halo) and 44 B written; no intermediate layer ever leaves the SM.
#include <cuda.h>

#include <cstring>

#include "fsb_internal.cuh"

namespace fsb {

__constant__ float2 c_tap2[6][14];   // (w_j, w_j) at distance j = 0..r of layer i's taps

int32_t upload_octave_taps(const float* taps, int stride, const int* counts) {
    float2 t[6][14] = {};
    for (int i = 0; i < 6; ++i) {
        const int r = counts[i] / 2;
        for (int j = 0; j <= r; ++j) t[i][j] = make_float2(taps[i * stride + r + j], taps[i * stride + r + j]);
    }
    FSB_CUDA(cudaMemcpyToSymbol(c_tap2, t, sizeof(t)));
    return FSB_OK;
}

namespace {

constexpr int NT = 256;      // threads per CTA
constexpr int SW = 168;      // output columns per strip
constexpr int S = 4;         // rows per step
constexpr int X0 = 44;       // L0 columns held left of the strip (keeps the load origin 16-byte aligned)
constexpr int HALO = 42;     // rows above / below a chunk that feed its outputs (5+6+8+10+13)

// radius of layer i's blur; first held column of layer i relative to the strip (x0 - H(i));
// held width of layer i (padded to 4); ring pitch and rows
__host__ __device__ constexpr int RAD(int i) { return i == 1 ? 5 : i == 2 ? 6 : i == 3 ? 8 : i == 4 ? 10 : i == 5 ? 13 : 0; }
__host__ __device__ constexpr int H(int i) { return i == 0 ? 44 : i == 1 ? 39 : i == 2 ? 33 : i == 3 ? 25 : i == 4 ? 15 : 2; }
__host__ __device__ constexpr int WIN(int i) { return i == 0 ? 256 : i == 1 ? 248 : i == 2 ? 236 : i == 3 ? 220 : i == 4 ? 200 : 172; }
__host__ __device__ constexpr int PITCH(int i) { return i == 0 ? 260 : WIN(i); }
__host__ __device__ constexpr int ROWS(int i) { return i == 0 ? 2 * 5 + 2 * S : i == 5 ? S : 2 * RAD(i + 1) + S; }
__host__ __device__ constexpr int LAG(int i) { return i == 1 ? 5 : i == 2 ? 11 : i == 3 ? 19 : i == 4 ? 29 : i == 5 ? 42 : 0; }
__host__ __device__ constexpr int off_of(int i) { return i == 0 ? 0 : off_of(i - 1) + ROWS(i - 1) * PITCH(i - 1); }
constexpr int T2_OFF = off_of(6);     // row-pair interleaved vertical outputs (float2 per column)
constexpr int T2_PITCH = 260;         // float2 per row pair
constexpr int SMEM_BYTES = (T2_OFF + 2 * T2_PITCH * 2) * 4;

struct Args {
    const float* L0;              // octave base, pitch C
    int R, C, rows_per_cta;
    float* dog[5];                // DoG planes R x C
    float* mag[3];                // gradient magnitude of layers 1..3
    float* ang[3];                // gradient angle of layers 1..3
    float* down;                  // next octave base or null
    int down_cols;
};

// 16-byte alignment of a plane address: the atlases pack octaves back to back, so an octave's
// planes can start off a 16-byte boundary even when its width is a multiple of 4
__device__ __forceinline__ bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

__device__ __forceinline__ int mir(int p, int n) {
    if (n == 1) return 0;
    while (p < 0 || p >= n) p = p < 0 ? -p : 2 * n - 2 - p;
    return p;
}

// slot of `row` in a ring of N rows, with row - base >= 0
template <int N>
__device__ __forceinline__ int slot_of(int row, int base) { return (row - base) % N; }

template <int N>
__device__ __forceinline__ int wrap(int s) { return s >= N ? s - N : s; }

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// rows [g, g + S) of L0 (mirrored) into ring 0: one 16-byte group per thread
__device__ __forceinline__ void load_rows(float* ring0, const Args& a, int x0, int g, int ybase, bool aligned) {
    const int s = threadIdx.x >> 6, q = threadIdx.x & 63;
    const int y = g + s;
    float* dst = ring0 + slot_of<ROWS(0)>(y, ybase) * PITCH(0) + 4 * q;
    const float* row = a.L0 + (size_t)mir(y, a.R) * a.C;
    const int x = x0 - X0 + 4 * q;
    if (aligned) {
        cp_async16(dst, row + x);
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) cp_async4(dst + k, row + mir(x + k, a.C));
    }
}

// sum_j w_j x[r + j] over j = -r..r for two lanes at once, with symmetric pairing
// w_0 x_0 + sum_j w_j (x_-j + x_j); two accumulation chains (odd / even j) for latency hiding.
// The pair sums commute, so a mirrored window gives a bit-identical result.
template <int TS, int r>
__device__ __forceinline__ float2 blur_pairs_t(const float2* x) {
    float2 a = __fmul2_rn(x[r], c_tap2[TS][0]);
    float2 b = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = r; j >= 1; --j) {
        const float2 p = __fadd2_rn(x[r - j], x[r + j]);
        if (j & 1)
            b = __ffma2_rn(p, c_tap2[TS][j], b);
        else
            a = __ffma2_rn(p, c_tap2[TS][j], a);
    }
    return __fadd2_rn(a, b);
}
template <int I>
__device__ __forceinline__ float2 blur_pairs(const float2* x) { return blur_pairs_t<I, RAD(I)>(x); }

// tap set TS held in registers for a whole pass (the empty asm keeps the compiler from re-reading
// the constant bank at every packed FMA, which takes no constant operand)
template <int TS, int r>
__device__ __forceinline__ void load_taps(float2 (&w)[r + 1]) {
#pragma unroll
    for (int j = 0; j <= r; ++j) {
        float2 t = c_tap2[TS][j];
        asm volatile("" : "+f"(t.x), "+f"(t.y));
        w[j] = t;
    }
}
// blur_pairs_t with the taps in registers: the same operations in the same order
template <int r>
__device__ __forceinline__ float2 blur_pairs_w(const float2* x, const float2 (&w)[r + 1]) {
    float2 a = __fmul2_rn(x[r], w[0]);
    float2 b = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = r; j >= 1; --j) {
        const float2 p = __fadd2_rn(x[r - j], x[r + j]);
        if (j & 1)
            b = __ffma2_rn(p, w[j], b);
        else
            a = __ffma2_rn(p, w[j], a);
    }
    return __fadd2_rn(a, b);
}

// rows yb, yb+1 (row pair rp) .. of L_I from L_{I-1} rows in `ring`; thread = (column pair, row pair)
template <int I>
__device__ __forceinline__ void vpass(const float* ring, float2* t2, int yb, int ybase) {
    constexpr int r = RAD(I), NR = ROWS(I - 1), P = PITCH(I - 1);
    constexpr int NP = WIN(I - 1) / 2 + 1;   // column pairs the horizontal pass reads
    const int cp = threadIdx.x & 127, rp = threadIdx.x >> 7;
    if (cp >= NP) return;
    const int s0 = slot_of<NR>(yb + 2 * rp - r, ybase);
    float2 x[2 * r + 2];
#pragma unroll
    for (int k = 0; k < 2 * r + 2; ++k)
        x[k] = *reinterpret_cast<const float2*>(ring + wrap<NR>(s0 + k) * P + 2 * cp);
    float2 o[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) o[s] = blur_pairs<I>(x + s);
    *reinterpret_cast<float4*>(t2 + rp * T2_PITCH + 2 * cp) = make_float4(o[0].x, o[1].x, o[0].y, o[1].y);
}

// L_I rows yb .. yb+3 from the interleaved vertical outputs; thread = (row pair, column pair)
template <int I>
__device__ __forceinline__ void hpass(const float2* t2, float* out, int yb, int ybase) {
    constexpr int r = RAD(I), NO = ROWS(I), P = PITCH(I);
    constexpr int NG = WIN(I) / 2;
    const int p = threadIdx.x >> 7, g = threadIdx.x & 127;
    if (g >= NG) return;
    const float4* src = reinterpret_cast<const float4*>(t2 + p * T2_PITCH + 2 * g);
    float2 y[2 * r + 2];
#pragma unroll
    for (int k = 0; k < r + 1; ++k) {
        const float4 v = src[k];
        y[2 * k] = make_float2(v.x, v.y);
        y[2 * k + 1] = make_float2(v.z, v.w);
    }
    float2 o[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) o[c] = blur_pairs<I>(y + c);
    const int s0 = slot_of<NO>(yb + 2 * p, ybase), s1 = wrap<NO>(s0 + 1);
    *reinterpret_cast<float2*>(out + s0 * P + 2 * g) = make_float2(o[0].x, o[1].x);
    *reinterpret_cast<float2*>(out + s1 * P + 2 * g) = make_float2(o[0].y, o[1].y);
}

// Gradient magnitude and direction (degrees in [0, 360)) of four pixels for the default (float32)
// pyramid: magnitude by the approximate square root (within a few ulps of sqrt), direction by
// octant reduction to t = min/max in [0, 1] (approximate reciprocal) and an odd polynomial for
// atan(t) in degrees. The
// coefficients were fitted here by iteratively reweighted least squares on Chebyshev nodes (max
// error 2.2e-6 deg; 7.4e-6 deg with float32 evaluation), so the angle stays well inside the
// reference's 0.1 deg keypoint tolerance. atan2(0, 0) = 0 as in the reference (border pixels).
// Pixels go through in pairs with packed FP32x2 arithmetic; every multiply and add is explicitly
// rounded (nothing is contracted into a fused multiply-add), so each engine that calls this
// function computes the same bits.
// the hardware's approximate square root and reciprocal (a few ulps; sqrt of 0 is 0)
__device__ __forceinline__ float sqrt_approx(float x) {
    float y;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void fast_grad4(const float (&dx)[4], const float (&dy)[4], float (&mag)[4],
                                           float (&ang)[4]) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const float2 X = make_float2(dx[2 * h], dx[2 * h + 1]), Y = make_float2(dy[2 * h], dy[2 * h + 1]);
        const float2 d2 = __fadd2_rn(__fmul2_rn(X, X), __fmul2_rn(Y, Y));
        const float2 m = make_float2(sqrt_approx(d2.x), sqrt_approx(d2.y));
        const float ax0 = fabsf(X.x), ay0 = fabsf(Y.x), ax1 = fabsf(X.y), ay1 = fabsf(Y.y);
        const float mx0 = fmaxf(ax0, ay0), mn0 = fminf(ax0, ay0), mx1 = fmaxf(ax1, ay1), mn1 = fminf(ax1, ay1);
        // min / max with the maximum kept above zero: 0 / tiny = 0 where both components vanish
        const float2 t = __fmul2_rn(make_float2(mn0, mn1),
                                    make_float2(rcp_approx(fmaxf(mx0, 1e-30f)), rcp_approx(fmaxf(mx1, 1e-30f))));
        const float2 z = __fmul2_rn(t, t);
        float2 p = make_float2(-2.323089093e-01f, -2.323089093e-01f);
        p = __ffma2_rn(p, z, make_float2(1.252652928e+00f, 1.252652928e+00f));
        p = __ffma2_rn(p, z, make_float2(-3.203537344e+00f, -3.203537344e+00f));
        p = __ffma2_rn(p, z, make_float2(5.524570187e+00f, 5.524570187e+00f));
        p = __ffma2_rn(p, z, make_float2(-7.969057098e+00f, -7.969057098e+00f));
        p = __ffma2_rn(p, z, make_float2(1.142854019e+01f, 1.142854019e+01f));
        p = __ffma2_rn(p, z, make_float2(-1.909660354e+01f, -1.909660354e+01f));
        p = __ffma2_rn(p, z, make_float2(5.729574144e+01f, 5.729574144e+01f));
        float2 a = __fmul2_rn(p, t);   // atan(min/max) in degrees, [0, 45]
        float2 f = __fadd2_rn(make_float2(90.f, 90.f), make_float2(-a.x, -a.y));
        a = make_float2(ay0 > ax0 ? f.x : a.x, ay1 > ax1 ? f.y : a.y);
        f = __fadd2_rn(make_float2(180.f, 180.f), make_float2(-a.x, -a.y));
        a = make_float2(X.x < 0.f ? f.x : a.x, X.y < 0.f ? f.y : a.y);
        f = __fadd2_rn(make_float2(360.f, 360.f), make_float2(-a.x, -a.y));   // atan2 < 0 maps to a + 360
        a = make_float2(Y.x < 0.f ? f.x : a.x, Y.y < 0.f ? f.y : a.y);
        mag[2 * h] = m.x;
        mag[2 * h + 1] = m.y;
        ang[2 * h] = a.x;
        ang[2 * h + 1] = a.y;
    }
}

// Gradient magnitude and angle at image row yy, columns x .. x+3, from a shared plane of pitch P
// (ctr points at (yy, x); the column left of x and right of x + 3 and the rows above and below are
// held): dx = right - left, dy = above - below, both zero on the image border as in the reference.
// One border test per group of four columns; the per-column test only where the group touches it.
template <int P>
__device__ __forceinline__ void grad4(const float* ctr, int yy, int x, int R, int C, float (&mg)[4], float (&an)[4]) {
    const float4 cc = *reinterpret_cast<const float4*>(ctr);
    const float4 up = *reinterpret_cast<const float4*>(ctr - P);
    const float4 dn = *reinterpret_cast<const float4*>(ctr + P);
    const float lf = ctr[-1], rt = ctr[4];
    float dx[4] = {__fsub_rn(cc.y, lf), __fsub_rn(cc.z, cc.x), __fsub_rn(cc.w, cc.y), __fsub_rn(rt, cc.z)};
    float dy[4] = {__fsub_rn(up.x, dn.x), __fsub_rn(up.y, dn.y), __fsub_rn(up.z, dn.z), __fsub_rn(up.w, dn.w)};
    if (!(yy > 0 && yy < R - 1 && x > 0 && x + 4 < C)) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (!(yy > 0 && yy < R - 1 && x + k > 0 && x + k < C - 1)) dx[k] = dy[k] = 0.f;
    }
    fast_grad4(dx, dy, mg, an);
}

// DoG of stage I (L_I - L_{I-1}), gradient of L_{I-1} (I = 2..4), L_3[::2, ::2] (I = 4)
template <int I>
__device__ __forceinline__ void epilogue(const float* prev, const float* cur, const Args& a, int x0, int yb, int ybase,
                                         int ya, int yz) {
    constexpr int PP = PITCH(I - 1), PR = ROWS(I - 1), CP = PITCH(I), CR = ROWS(I);
    constexpr int hp = H(I - 1), hc = H(I);
    const int e = threadIdx.x;
    if (e >= S * (SW / 4)) return;
    const int s = e / (SW / 4), q = e - s * (SW / 4);
    const int y = yb + s;
    const int xg = x0 + 4 * q;
    if (y < ya || y >= yz || xg >= a.C) return;
    const int ps = slot_of<PR>(y, ybase);
    const float* pr = prev + ps * PP + 4 * q + hp;
    const float* cr = cur + slot_of<CR>(y, ybase) * CP + 4 * q + hc;
    float d[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) d[k] = cr[k] - pr[k];
    const int at = y * a.C + xg;
    const bool vec = (a.C & 3) == 0 && xg + 4 <= a.C;
    float* dg = a.dog[I - 1] + at;
    if (vec && al16(dg)) {
        *reinterpret_cast<float4*>(dg) = make_float4(d[0], d[1], d[2], d[3]);
    } else {
        for (int k = 0; k < 4 && xg + k < a.C; ++k) dg[k] = d[k];
    }
    if (I >= 2 && I <= 4) {
        const float* up = prev + wrap<PR>(ps + PR - 1) * PP + 4 * q + hp;
        const float* dn = prev + wrap<PR>(ps + 1) * PP + 4 * q + hp;
        float mg[4], an[4], dx[4], dy[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int x = xg + k;
            dx[k] = dy[k] = 0.f;
            if (y > 0 && y < a.R - 1 && x > 0 && x < a.C - 1) {
                dx[k] = __fsub_rn(pr[k + 1], pr[k - 1]);
                dy[k] = __fsub_rn(up[k], dn[k]);
            }
        }
        fast_grad4(dx, dy, mg, an);
        float* m = a.mag[I - 2] + at;
        float* n = a.ang[I - 2] + at;
        if (vec && al16(m) && al16(n)) {
            *reinterpret_cast<float4*>(m) = make_float4(mg[0], mg[1], mg[2], mg[3]);
            *reinterpret_cast<float4*>(n) = make_float4(an[0], an[1], an[2], an[3]);
        } else {
            for (int k = 0; k < 4 && xg + k < a.C; ++k) {
                m[k] = mg[k];
                n[k] = an[k];
            }
        }
    }
    if (I == 4 && a.down && !(y & 1)) {
        float* o = a.down + (y >> 1) * a.down_cols + (xg >> 1);
        o[0] = pr[0];
        if (xg + 2 < a.C) o[1] = pr[2];
    }
}

__global__ void __launch_bounds__(NT, 2) k_octave(Args a) {
    extern __shared__ __align__(16) float sm[];
    float* ring0 = sm + off_of(0);
    float* ring1 = sm + off_of(1);
    float* ring2 = sm + off_of(2);
    float* ring3 = sm + off_of(3);
    float* ring4 = sm + off_of(4);
    float* ring5 = sm + off_of(5);
    float2* t2 = reinterpret_cast<float2*>(sm + T2_OFF);
    const int x0 = blockIdx.x * SW;
    const int ya = blockIdx.y * a.rows_per_cta;
    const int yz = min(a.R, ya + a.rows_per_cta);
    const int ybase = ya - 128;                             // keeps every (row - ybase) positive
    const int g0 = ya - HALO;
    const int steps = (yz - ya + 2 * HALO + S - 1) / S;
    const bool aligned = (a.C & 3) == 0 && al16(a.L0) && x0 - X0 >= 0 && x0 - X0 + WIN(0) <= a.C;
    load_rows(ring0, a, x0, g0, ybase, aligned);
    cp_commit();
    for (int t = 0; t < steps; ++t) {
        cp_wait_all();
        __syncthreads();
        const int g = g0 + t * S;                            // L0 rows g .. g+3 are in ring 0
        if (t + 1 < steps) load_rows(ring0, a, x0, g + S, ybase, aligned);
        cp_commit();
        // stage i produces rows g - LAG(i) .. g - LAG(i) + 3
        vpass<1>(ring0, t2, g - LAG(1), ybase);
        __syncthreads();
        hpass<1>(t2, ring1, g - LAG(1), ybase);
        __syncthreads();
        epilogue<1>(ring0, ring1, a, x0, g - LAG(1), ybase, ya, yz);
        vpass<2>(ring1, t2, g - LAG(2), ybase);
        __syncthreads();
        hpass<2>(t2, ring2, g - LAG(2), ybase);
        __syncthreads();
        epilogue<2>(ring1, ring2, a, x0, g - LAG(2), ybase, ya, yz);
        vpass<3>(ring2, t2, g - LAG(3), ybase);
        __syncthreads();
        hpass<3>(t2, ring3, g - LAG(3), ybase);
        __syncthreads();
        epilogue<3>(ring2, ring3, a, x0, g - LAG(3), ybase, ya, yz);
        vpass<4>(ring3, t2, g - LAG(4), ybase);
        __syncthreads();
        hpass<4>(t2, ring4, g - LAG(4), ybase);
        __syncthreads();
        epilogue<4>(ring3, ring4, a, x0, g - LAG(4), ybase, ya, yz);
        vpass<5>(ring4, t2, g - LAG(5), ybase);
        __syncthreads();
        hpass<5>(t2, ring5, g - LAG(5), ybase);
        __syncthreads();
        epilogue<5>(ring4, ring5, a, x0, g - LAG(5), ybase, ya, yz);
    }
    cp_wait_all();
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}


// bounded waits on a shared-memory mbarrier (TMA completion)
constexpr long long TSTRIP_TIMEOUT = 2000000000ll;   // cycles (about a second) for one TMA copy

__device__ __forceinline__ uint32_t s_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool s_mbar_test(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(s_addr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits (bounded) for one row block; every thread waits, then the CTA agrees on the outcome.
__device__ __forceinline__ bool s_mbar_wait(uint64_t* b, uint32_t parity) {
    bool ok = s_mbar_test(b, parity);
    if (!ok) {
        const long long t0 = clock64();
        while (!(ok = s_mbar_test(b, parity)) && clock64() - t0 < TSTRIP_TIMEOUT) {
        }
    }
    return ok;
}

// ------------------------------------------------------------------------------------------------
// Per-layer tiled kernels (float32 path), 128 x 32 outputs per CTA:
//   k_layer<I, RAD(I), false>  L_I of one octave from L_{I-1}: the same pair blurs and gradient as
//                              the fused kernel (bit-identical results), DoG, gradient of L_{I-1},
//                              L_{I-1}[::2, ::2]
//   k_layer<0, 5, true>        the octave-0 base: the 2x bilinear upsample of the uint8 image
//                              (the reference's float32 rounding, gsift.py:90-102) computed while the
//                              tile loads, from per-row / per-column source tables, blurred with tap
//                              set 0
// The input tile (16 columns and r rows of reflect-101 halo) arrives by 16-byte cp.async, the
// vertical pass keeps an 8-row sliding window of column pairs in registers, the horizontal pass
// reads the row-pair interleaved vertical outputs. No ring buffers: 3-4 CTAs per SM.
constexpr int LX = 128, LNT = 256;   // tile width, threads; the tile height LY is a template parameter
constexpr int LIN_C = LX + 32;   // input tile columns (16 of halo on each side)
constexpr int LIN_W = LX + 40;   // input tile pitch (floats): rows 2 apart differ by 64 bytes mod 128
constexpr int LT2_W = LX + 34;   // row-pair tile pitch (float2): 16 bytes past a multiple of 128, so
                                 // row pairs p and p + 1 start in opposite 16-byte bank groups

struct LayerArgs {
    const float* src;   // L_{I-1}, R x C
    const uint8_t* img; // base: uint8 image ih x iw, row pitch img_stride
    int img_stride, ih, iw;
    int R, C;
    float* dst;         // L_I or null
    float* dog;         // L_I - L_{I-1}
    float* mag;         // gradient of L_{I-1} or null
    float* ang;
    float* down;        // L_{I-1}[::2, ::2] or null
    int down_cols;
    int* err;           // set to 1 when the tile's TMA copy does not complete in time
};

// shared memory: the input tile (LIN_W floats per row), the row-pair tile, the TMA mbarrier
template <int r, int LY>
constexpr int layer_bar_off() {
    return (LY + 2 * r) * LIN_W * 4 + (LY / 2) * LT2_W * 8;
}
template <int r, int LY>
constexpr int layer_smem() {
    return layer_bar_off<r, LY>() + 16;
}

// The input tile (rows y0 - r .., columns x0 - 16 .., reflect-101 outside the plane) by
// per-thread cp.async (the caller commits and waits)
template <int r, int LY>
__device__ __forceinline__ void layer_load_cp(const LayerArgs& a, float* __restrict__ s_in, int x0, int y0) {
    constexpr int IH = LY + 2 * r;
    const int tid = threadIdx.x;
    if ((a.C & 3) == 0 && al16(a.src) && x0 >= 16 && x0 + LX + 16 <= a.C) {
        // eight lanes per row (the mirrored row address once per row), five 16-byte copies a lane
        static_assert(LIN_C / 4 == 40, "five copies of eight lanes per row");
        for (int row = tid >> 3; row < IH; row += LNT / 8) {
            const float* g = a.src + (size_t)mir(y0 - r + row, a.R) * a.C + (x0 - 16);
            float* d = s_in + row * LIN_W;
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                const int q = 4 * ((tid & 7) + 8 * k);
                cp_async16(d + q, g + q);
            }
        }
    } else {
        for (int i = tid; i < IH * LIN_C; i += LNT) {
            const int row = i / LIN_C, col = i - row * LIN_C;
            const float* g = a.src + (size_t)mir(y0 - r + row, a.R) * a.C + mir(x0 - 16 + col, a.C);
            cp_async4(s_in + row * LIN_W + col, g);
        }
    }
}

// Whether a tile's input lies inside the plane (no reflected row or column): such tiles arrive by
// one 2-D tensor copy of LIN_W x (LY + 2r) floats (the copy's last 8 columns are not read and may
// lie outside the plane, where the copy fills zeros)
template <int r, int LY>
__device__ __forceinline__ bool layer_tile_inside(const LayerArgs& a, int x0, int y0) {
    return y0 >= r && y0 + LY + r <= a.R && x0 >= 16 && x0 + LX + 16 <= a.C;
}
// thread 0: the tile's tensor copy into s_in, completion (bytes) on bar
template <int r, int LY>
__device__ __forceinline__ void layer_tma_issue(const CUtensorMap* tm, float* s_in, uint64_t* bar, int x0, int y0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s_addr(bar)),
                 "r"((LY + 2 * r) * LIN_W * 4)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(s_addr(s_in)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x0 - 16), "r"(y0 - r), "r"(s_addr(bar))
        : "memory");
}

// The passes of one tile once its input (s_in) is in shared memory: vertical pass into the
// row-pair tile t2, then the horizontal pass and the epilogue (L_I, DoG, gradient, downsample).
template <int TS, int r, bool BASE, int LY>
__device__ __forceinline__ void layer_compute(const LayerArgs& a, const float* __restrict__ s_in,
                                              float2* __restrict__ t2, int x0, int y0) {
    constexpr int d = r & 1;
    constexpr int NPAIR = (LX + 2 * r + 2 * d) / 2;
    const int tid = threadIdx.x;
    // vertical pass: column pair cp (V columns 2cp, 2cp+1 = image columns x0 - r - d + 2cp ..),
    // output rows 8g .. 8g + 7; stored row-pair interleaved at t2 index (V column + d)
    float2 w[r + 1];
    load_taps<TS, r>(w);
    for (int it = tid; it < NPAIR * (LY / 8); it += LNT) {
        const int cp = it % NPAIR, g = it / NPAIR;
        const float* base = s_in + (8 * g) * LIN_W + (16 - r - d + 2 * cp);
        float2 x[8 + 2 * r];
#pragma unroll
        for (int k = 0; k < 8 + 2 * r; ++k) x[k] = *reinterpret_cast<const float2*>(base + k * LIN_W);
#pragma unroll
        for (int sp = 0; sp < 4; ++sp) {
            const float2 o0 = blur_pairs_w<r>(x + 2 * sp, w), o1 = blur_pairs_w<r>(x + 2 * sp + 1, w);
            float2* dst = t2 + (4 * g + sp) * LT2_W + 2 * cp + d;
            dst[0] = make_float2(o0.x, o1.x);
            dst[1] = make_float2(o0.y, o1.y);
        }
    }
    __syncthreads();
    // horizontal pass: row pair p, output columns c .. c+3 (t2 indices c + 2d .. c + 2d + 3 + 2r).
    // A warp covers row pairs p, p + 1 x 64 columns. 16-byte loads are served 8 lanes at a time:
    // in each group of 8 lanes, four read row pair p and four row pair p + 1 (columns 4 apart, a
    // 32-byte stride: one bank parity per row pair, opposite parities by the pitch), so the 8
    // lanes cover all 32 banks once
    static_assert(LX == 128 && (LY / 2) % 2 == 0 && LNT % 32 == 0, "horizontal pass mapping");
    // Fast path for tiles whose outputs and gradient neighbourhoods lie inside the plane, with
    // 16-byte aligned planes and rows (uniform per CTA): no per-row bounds, border or alignment
    // tests and 32-bit offsets. Same arithmetic as the general path below, so the same bits.
    bool fast = (a.C & 3) == 0 && (long long)a.R * a.C < (1ll << 31) && x0 + LX <= a.C && y0 + LY <= a.R &&
                (!a.dst || al16(a.dst));
    if (!BASE)
        fast = fast && al16(a.dog) && (!a.mag || (al16(a.mag) && al16(a.ang))) && y0 >= 1 && y0 + LY <= a.R - 1 &&
               x0 >= 1 && x0 + LX < a.C;
    if (fast) {
        for (int it = tid; it < (LY / 2) * (LX / 4); it += LNT) {
            const int wi = it >> 5, l = it & 31;
            const int p = 2 * (wi >> 1) + ((l >> 2) & 1), c = 64 * (wi & 1) + 4 * ((l & 3) + 4 * (l >> 3));
            const int y = y0 + 2 * p, x = x0 + c;
            const float4* src = reinterpret_cast<const float4*>(t2 + p * LT2_W + c + 2 * d);
            float2 yv[4 + 2 * r];
#pragma unroll
            for (int k = 0; k < 2 + r; ++k) {
                const float4 v = src[k];
                yv[2 * k] = make_float2(v.x, v.y);
                yv[2 * k + 1] = make_float2(v.z, v.w);
            }
            float2 o[4];
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) o[cc] = blur_pairs_w<r>(yv + cc, w);
            const int at0 = y * a.C + x;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int at = at0 + h * a.C;
                const float4 lv = h ? make_float4(o[0].y, o[1].y, o[2].y, o[3].y)
                                    : make_float4(o[0].x, o[1].x, o[2].x, o[3].x);
                if (BASE) {
                    *reinterpret_cast<float4*>(a.dst + at) = lv;
                    continue;
                }
                const float* ctr = s_in + (2 * p + h + r) * LIN_W + 16 + c;   // L_{I-1} at (y + h, x)
                const float4 pv = *reinterpret_cast<const float4*>(ctr);
                *reinterpret_cast<float4*>(a.dog + at) = make_float4(lv.x - pv.x, lv.y - pv.y, lv.z - pv.z, lv.w - pv.w);
                if (a.dst) *reinterpret_cast<float4*>(a.dst + at) = lv;
                if (a.mag) {
                    const float4 up = *reinterpret_cast<const float4*>(ctr - LIN_W);
                    const float4 dn = *reinterpret_cast<const float4*>(ctr + LIN_W);
                    const float lf = ctr[-1], rt = ctr[4];
                    const float dx[4] = {__fsub_rn(pv.y, lf), __fsub_rn(pv.z, pv.x), __fsub_rn(pv.w, pv.y),
                                         __fsub_rn(rt, pv.z)};
                    const float dy[4] = {__fsub_rn(up.x, dn.x), __fsub_rn(up.y, dn.y), __fsub_rn(up.z, dn.z),
                                         __fsub_rn(up.w, dn.w)};
                    float mg[4], an[4];
                    fast_grad4(dx, dy, mg, an);
                    *reinterpret_cast<float4*>(a.mag + at) = make_float4(mg[0], mg[1], mg[2], mg[3]);
                    *reinterpret_cast<float4*>(a.ang + at) = make_float4(an[0], an[1], an[2], an[3]);
                }
                if (a.down && h == 0) {   // y is even: y0 and 2p are
                    float* o2 = a.down + (y >> 1) * a.down_cols + (x >> 1);
                    o2[0] = pv.x;
                    o2[1] = pv.z;
                }
            }
        }
        return;
    }
    for (int it = tid; it < (LY / 2) * (LX / 4); it += LNT) {
        const int wi = it >> 5, l = it & 31;
        const int p = 2 * (wi >> 1) + ((l >> 2) & 1), c = 64 * (wi & 1) + 4 * ((l & 3) + 4 * (l >> 3));
        const int y = y0 + 2 * p, x = x0 + c;
        if (y >= a.R || x >= a.C) continue;
        const float4* src = reinterpret_cast<const float4*>(t2 + p * LT2_W + c + 2 * d);
        float2 yv[4 + 2 * r];
#pragma unroll
        for (int k = 0; k < 2 + r; ++k) {
            const float4 v = src[k];
            yv[2 * k] = make_float2(v.x, v.y);
            yv[2 * k + 1] = make_float2(v.z, v.w);
        }
        float2 o[4];
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) o[cc] = blur_pairs_w<r>(yv + cc, w);   // (row y, row y+1) at column x+cc
        const bool vec = (a.C & 3) == 0 && x + 4 <= a.C;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int yy = y + h;
            if (yy >= a.R) break;
            const float lv[4] = {h ? o[0].y : o[0].x, h ? o[1].y : o[1].x, h ? o[2].y : o[2].x, h ? o[3].y : o[3].x};
            if (BASE) {
                const size_t at = (size_t)yy * a.C + x;
                if (vec && al16(a.dst)) {
                    *reinterpret_cast<float4*>(a.dst + at) = make_float4(lv[0], lv[1], lv[2], lv[3]);
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (x + k < a.C) a.dst[at + k] = lv[k];
                }
                continue;
            }
            const float* ctr = s_in + (2 * p + h + r) * LIN_W + 16 + c;   // L_{I-1} at (yy, x)
            const float4 pv = *reinterpret_cast<const float4*>(ctr);
            const float pr[4] = {pv.x, pv.y, pv.z, pv.w};
            float dg[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) dg[k] = lv[k] - pr[k];
            const size_t at = (size_t)yy * a.C + x;
            if (vec && al16(a.dog) && (!a.dst || al16(a.dst))) {
                *reinterpret_cast<float4*>(a.dog + at) = make_float4(dg[0], dg[1], dg[2], dg[3]);
                if (a.dst) *reinterpret_cast<float4*>(a.dst + at) = make_float4(lv[0], lv[1], lv[2], lv[3]);
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (x + k >= a.C) break;
                    a.dog[at + k] = dg[k];
                    if (a.dst) a.dst[at + k] = lv[k];
                }
            }
            if (a.mag) {
                float mg[4], an[4];
                grad4<LIN_W>(ctr, yy, x, a.R, a.C, mg, an);
                if (vec && al16(a.mag) && al16(a.ang)) {
                    *reinterpret_cast<float4*>(a.mag + at) = make_float4(mg[0], mg[1], mg[2], mg[3]);
                    *reinterpret_cast<float4*>(a.ang + at) = make_float4(an[0], an[1], an[2], an[3]);
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        if (x + k >= a.C) break;
                        a.mag[at + k] = mg[k];
                        a.ang[at + k] = an[k];
                    }
                }
            }
            if (a.down && !(yy & 1)) {
                float* o2 = a.down + (size_t)(yy >> 1) * a.down_cols + (x >> 1);
                o2[0] = pr[0];
                if (x + 2 < a.C) o2[1] = pr[2];
            }
        }
    }
}


template <int TS, int r, bool BASE, int LY>
__global__ void __launch_bounds__(LNT, r <= 10 ? 4 : 3) k_layer(const __grid_constant__ CUtensorMap tm, LayerArgs a,
                                                                int use_tma) {
    constexpr int d = r & 1;
    constexpr int IH = LY + 2 * r;
    constexpr int NPAIR = (LX + 2 * r + 2 * d) / 2;
    static_assert(layer_bar_off<r, LY>() % 16 == 0, "mbarrier alignment");
    extern __shared__ __align__(128) float sm[];
    float* s_in = sm;
    float2* t2 = reinterpret_cast<float2*>(sm + IH * LIN_W);
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * LX, y0 = blockIdx.y * LY;
    // input rows y0 - r .. y0 + LY + r - 1, columns x0 - 16 .. x0 + LX + 15 (reflect-101 outside)
    if (BASE) {
        // Source row / column pairs (iy, ny), (ix, nx) of every tile row / column (reflect-101 on
        // the upsampled grid). The source block they reach is staged once as scaled floats p, the
        // row-interpolated values vc = 0.75 p[iy] + 0.25 p[ny] are formed for every tile row over the
        // block's columns, and each upsampled sample is 0.75 vc[ix] + 0.25 vc[nx], four columns per
        // thread (gsift.py:90-102 rounding). Tables and vc live in the row-pair area and p in the
        // input tile until the vertical pass needs them. A block larger than the staging window
        // (mirror images of a tiny image) takes the per-sample global path.
        constexpr int VCW = 96, SRW = IH / 2 + 4;
        static_assert(!BASE || (2 * IH + 2 * LIN_C) * 4 + IH * VCW * 4 + 16 <= (LY / 2) * LT2_W * 8,
                      "base tables must fit the row-pair area");
        static_assert(!BASE || (SRW * VCW <= IH * LIN_W && IH % 2 == 0), "staged source block");
        int* ry = reinterpret_cast<int*>(t2);   // iy of tile row i, then ny
        int* rn = ry + IH;
        int* cxs = rn + IH;                      // ix of tile column c, then nx (16-byte aligned)
        int* cns = cxs + LIN_C;
        float* vcs = reinterpret_cast<float*>(cns + LIN_C);
        int* box = reinterpret_cast<int*>(vcs + IH * VCW);   // source row min / max, column min / max
        float* ps = s_in;
        if (tid < 4) box[tid] = (tid & 1) ? -1 : 0x7fffffff;
        __syncthreads();
        for (int i0 = 0; i0 < IH + LIN_C; i0 += LNT) {
            const int i = i0 + tid;
            int lo = 0x7fffffff, hi = -1, clo = 0x7fffffff, chi = -1;
            if (i < IH) {
                const int Y = mir(y0 - r + i, a.R), iy = Y >> 1;
                const int ny = (Y & 1) ? min(iy + 1, a.ih - 1) : max(iy - 1, 0);
                ry[i] = iy;
                rn[i] = ny;
                lo = min(iy, ny);
                hi = max(iy, ny);
            } else if (i < IH + LIN_C) {
                const int c = i - IH, X = mir(x0 - 16 + c, a.C), ix = X >> 1;
                const int nx = (X & 1) ? min(ix + 1, a.iw - 1) : max(ix - 1, 0);
                cxs[c] = ix;
                cns[c] = nx;
                clo = min(ix, nx);
                chi = max(ix, nx);
            }
            lo = __reduce_min_sync(0xffffffffu, lo);
            hi = __reduce_max_sync(0xffffffffu, hi);
            clo = __reduce_min_sync(0xffffffffu, clo);
            chi = __reduce_max_sync(0xffffffffu, chi);
            if ((tid & 31) == 0) {
                if (hi >= 0) {
                    atomicMin(&box[0], lo);
                    atomicMax(&box[1], hi);
                }
                if (chi >= 0) {
                    atomicMin(&box[2], clo);
                    atomicMax(&box[3], chi);
                }
            }
        }
        __syncthreads();
        const int sy0 = box[0], nsr = box[1] - box[0] + 1, sx0 = box[2], nsx = box[3] - box[2] + 1;
        const float sc = (float)(1.0 / 255.0);
        if (nsr <= SRW && nsx <= VCW) {
            for (int row = tid >> 5; row < nsr; row += LNT / 32) {
                const uint8_t* src = a.img + (size_t)(sy0 + row) * a.img_stride + sx0;
                for (int k = tid & 31; k < nsx; k += 32) ps[row * VCW + k] = __fmul_rn((float)__ldg(src + k), sc);
            }
            __syncthreads();
            for (int i = tid; i < IH * (VCW / 4); i += LNT) {
                const int row = i / (VCW / 4), q = 4 * (i - row * (VCW / 4));
                if (q >= nsx) continue;
                const float4 p0 = *reinterpret_cast<const float4*>(ps + (ry[row] - sy0) * VCW + q);
                const float4 p1 = *reinterpret_cast<const float4*>(ps + (rn[row] - sy0) * VCW + q);
                float4 v;
                v.x = __fadd_rn(__fmul_rn(0.75f, p0.x), __fmul_rn(0.25f, p1.x));
                v.y = __fadd_rn(__fmul_rn(0.75f, p0.y), __fmul_rn(0.25f, p1.y));
                v.z = __fadd_rn(__fmul_rn(0.75f, p0.z), __fmul_rn(0.25f, p1.z));
                v.w = __fadd_rn(__fmul_rn(0.75f, p0.w), __fmul_rn(0.25f, p1.w));
                *reinterpret_cast<float4*>(vcs + row * VCW + q) = v;
            }
            __syncthreads();
            // Tiles whose columns reflect at no image or source edge: column X = x0 - 16 + q + k
            // samples source columns X / 2 and X / 2 -+ 1 in a fixed pattern, so four outputs take
            // four consecutive row-interpolated values (the same products and sums as the tables)
            if (x0 >= 18 && x0 + LX + 15 <= a.C - 3 && sx0 == (x0 - 16) / 2 - 1) {
                for (int i = tid; i < IH * (LIN_C / 4); i += LNT) {
                    const int row = i / (LIN_C / 4), m = i - row * (LIN_C / 4);
                    const float* vr = vcs + row * VCW + 2 * m;   // source columns X / 2 - 1 .. + 2
                    const float2 lo = *reinterpret_cast<const float2*>(vr);
                    const float2 hi = *reinterpret_cast<const float2*>(vr + 2);
                    const float a1 = __fmul_rn(0.75f, lo.y), a2 = __fmul_rn(0.75f, hi.x);
                    float4 u;
                    u.x = __fadd_rn(a1, __fmul_rn(0.25f, lo.x));
                    u.y = __fadd_rn(a1, __fmul_rn(0.25f, hi.x));
                    u.z = __fadd_rn(a2, __fmul_rn(0.25f, lo.y));
                    u.w = __fadd_rn(a2, __fmul_rn(0.25f, hi.y));
                    *reinterpret_cast<float4*>(s_in + row * LIN_W + 4 * m) = u;
                }
            } else {
            for (int i = tid; i < IH * (LIN_C / 4); i += LNT) {
                const int row = i / (LIN_C / 4), q = 4 * (i - row * (LIN_C / 4));
                const int4 ix = *reinterpret_cast<const int4*>(cxs + q);
                const int4 nx = *reinterpret_cast<const int4*>(cns + q);
                const float* v = vcs + row * VCW - sx0;
                float4 u;
                u.x = __fadd_rn(__fmul_rn(0.75f, v[ix.x]), __fmul_rn(0.25f, v[nx.x]));
                u.y = __fadd_rn(__fmul_rn(0.75f, v[ix.y]), __fmul_rn(0.25f, v[nx.y]));
                u.z = __fadd_rn(__fmul_rn(0.75f, v[ix.z]), __fmul_rn(0.25f, v[nx.z]));
                u.w = __fadd_rn(__fmul_rn(0.75f, v[ix.w]), __fmul_rn(0.25f, v[nx.w]));
                *reinterpret_cast<float4*>(s_in + row * LIN_W + q) = u;
            }
            }
        } else {
            for (int i = tid; i < IH * LIN_C; i += LNT) {
                const int row = i / LIN_C, col = i - row * LIN_C;
                const uint8_t* r0 = a.img + (size_t)ry[row] * a.img_stride;
                const uint8_t* r1 = a.img + (size_t)rn[row] * a.img_stride;
                const int ix = cxs[col], nx = cns[col];
                const float vc = __fadd_rn(__fmul_rn(0.75f, __fmul_rn((float)__ldg(r0 + ix), sc)),
                                           __fmul_rn(0.25f, __fmul_rn((float)__ldg(r1 + ix), sc)));
                const float vn = __fadd_rn(__fmul_rn(0.75f, __fmul_rn((float)__ldg(r0 + nx), sc)),
                                           __fmul_rn(0.25f, __fmul_rn((float)__ldg(r1 + nx), sc)));
                s_in[row * LIN_W + col] = __fadd_rn(__fmul_rn(0.75f, vc), __fmul_rn(0.25f, vn));
            }
        }
    } else if (use_tma && (s_addr(s_in) & 127) == 0 && layer_tile_inside<r, LY>(a, x0, y0)) {
        // an interior tile: one tensor copy, completion on an mbarrier
        uint64_t* bar = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(sm) + layer_bar_off<r, LY>());
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s_addr(bar)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (tid == 0) layer_tma_issue<r, LY>(&tm, s_in, bar, x0, y0);
        if (__syncthreads_or(!s_mbar_wait(bar, 0))) {
            // the copy did not land in time: flag it, give it one more bounded wait (so that no copy
            // into this CTA's shared memory is left in flight when possible) and leave the tile
            if (tid == 0) atomicExch(a.err, 1);
            s_mbar_wait(bar, 0);
            return;
        }
    } else {
        layer_load_cp<r, LY>(a, s_in, x0, y0);
    }
    cp_commit();
    cp_wait_all();
    __syncthreads();
    layer_compute<TS, r, BASE, LY>(a, s_in, t2, x0, y0);
}

// Tensor map of a layer's source plane for the tile copies (box LIN_W x rows): needs 16-byte
// aligned rows and base and the box inside the plane's extent; 0 when not possible (the tiles then
// load by cp.async)
int layer_tensor_map(CUtensorMap* tm, const float* src, int R, int C, int rows) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc || (C & 3) != 0 || C < LIN_W || R < rows || (reinterpret_cast<uintptr_t>(src) & 15) != 0) return 0;
    const cuuint64_t dims[2] = {(cuuint64_t)C, (cuuint64_t)R};
    const cuuint64_t strides[1] = {(cuuint64_t)C * 4};
    const cuuint32_t box[2] = {(cuuint32_t)LIN_W, (cuuint32_t)rows};
    const cuuint32_t es[2] = {1, 1};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(src), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int TS, int r, bool BASE, int LY>
int32_t launch_layer_ly(const LayerArgs& a, cudaStream_t s) {
    static std::atomic<int> attr[64];
    FSB_TRY(smem_attr((const void*)k_layer<TS, r, BASE, LY>, layer_smem<r, LY>(), attr));
    static_assert(LY + 2 * r <= 256, "tensor copy box height");
    CUtensorMap tm;
    std::memset(&tm, 0, sizeof(tm));
    const int use_tma = !BASE && a.err ? layer_tensor_map(&tm, a.src, a.R, a.C, LY + 2 * r) : 0;
    dim3 grid((a.C + LX - 1) / LX, (a.R + LY - 1) / LY);
    k_layer<TS, r, BASE, LY><<<grid, LNT, layer_smem<r, LY>(), s>>>(tm, a, use_tma);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

// tile heights the autotuner chooses from (index 0 is the default)
constexpr int kTileHeights[3] = {32, 16, 64};

template <int TS, int r, bool BASE>
int32_t launch_layer_t(const LayerArgs& a, int variant, cudaStream_t s) {
    if constexpr (BASE) {   // the base tile's source tables need a tile height of at least 32
        return variant == 2 ? launch_layer_ly<TS, r, BASE, 64>(a, s) : launch_layer_ly<TS, r, BASE, 32>(a, s);
    } else {
        switch (variant) {
            case 1: return launch_layer_ly<TS, r, BASE, 16>(a, s);
            case 2: return launch_layer_ly<TS, r, BASE, 64>(a, s);
            default: return launch_layer_ly<TS, r, BASE, 32>(a, s);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Fused layer groups (float32 path): one persistent kernel computes consecutive layers of an
// octave for 128 x 32 output tiles,
//   group 0: L1, L2, L3 from L0 -> DoG 0..2, gradients of L1..L3, L3 and L3[::2, ::2]
//   group 1: L4, L5 from L3     -> DoG 3, 4
// Every level is held in shared memory on the tile plus the halo the levels above it need (row
// halo GH, column halo GXH; recomputed per tile), so the intermediate layers never reach HBM:
// per octave pixel the two launches read L0 and L3 and write the five DoG planes, six gradient
// planes, L3 and the downsample (14.25 octave planes of traffic where five per-layer launches move
// 20.25). Halo values outside the image equal the reflect-101 mirror of the values inside: the
// blur of a mirror-symmetric signal is mirror-symmetric and the pair sums of blur_pairs_t commute,
// so each level reproduces the per-layer kernels' values bit for bit. The passes are the per-layer
// kernel's (8-row register window of column pairs; row-pair-interleaved horizontal pass), with
// the DoG / gradient epilogue of a level run by the horizontal pass of the level above it. One
// CTA per SM walks the tiles; the next tile's input arrives by cp.async while this one computes.
constexpr int GX = 128, GY = 32, GNT = 512;

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

// One level of a group: the output level (row halo Ho, column halo Xo) blurred with radius r from
// the level below (Hi, Xi). The vertical pass covers input columns VS .. VS + VW - 1 (VS even);
// column j of its output sits at float2 index j + E of a row pair, so the horizontal pass's
// 16-byte loads start on an even index.
template <int Hi, int Xi, int Ho, int Xo, int r>
struct GLevel {
    static constexpr int HIN = Hi, XIN = Xi, HOUT = Ho, XOUT = Xo, RAD = r;
    static constexpr int NIN = GY + 2 * Hi, MIN = GX + 2 * Xi;     // input rows, columns (= pitch)
    static constexpr int NOUT = GY + 2 * Ho, MOUT = GX + 2 * Xo;   // output rows, columns (= pitch)
    static constexpr int ROFF = Hi - Ho - r;                       // input row of output row 0's first tap
    static constexpr int OFF = Xi - Xo - r;                        // input column of output column 0's first tap
    static constexpr int E = OFF & 1;
    static constexpr int VS = OFF - E;
    static constexpr int VW = (MOUT + 2 * r + E + 1) & ~1;
    static constexpr int VP = (VW + E + 1) & ~1;                   // float2 per row pair
    static constexpr int V_FLOATS = (NOUT / 2) * VP * 2;
    static constexpr int IN_FLOATS = NIN * MIN, OUT_FLOATS = NOUT * MOUT;
    static_assert(ROFF >= 0 && OFF >= 0 && Xi % 4 == 0 && Xo % 4 == 0, "level geometry");
    static_assert(VS + VW <= MIN, "vertical pass inside the input level");
};

template <int G>
struct GSpec;
template <>
struct GSpec<0> {
    using A = GLevel<20, 28, 15, 20, 5>;   // L0 -> L1
    using B = GLevel<15, 20, 9, 12, 6>;    // L1 -> L2
    using C = GLevel<9, 12, 1, 4, 8>;      // L2 -> L3 (halo 1: gradient of L3)
    static constexpr int BUF0 = (cmax(A::IN_FLOATS, cmax(B::V_FLOATS, C::V_FLOATS)) + 3) & ~3;   // L0 / V2 / V3
    static constexpr int BUF1 = (cmax(A::V_FLOATS, B::OUT_FLOATS) + 3) & ~3;                     // V1 / L2
    static constexpr int BUF2 = (cmax(A::OUT_FLOATS, C::OUT_FLOATS) + 3) & ~3;                   // L1 / L3
};
template <>
struct GSpec<1> {
    using A = GLevel<23, 28, 13, 16, 10>;   // L3 -> L4
    using B = GLevel<13, 16, 0, 0, 13>;     // L4 -> L5 (tile only)
    static constexpr int BUF0 = (cmax(A::IN_FLOATS, B::V_FLOATS) + 3) & ~3;   // L3 / V5
    static constexpr int BUF1 = (A::V_FLOATS + 3) & ~3;                       // V4
    static constexpr int BUF2 = (A::OUT_FLOATS + 3) & ~3;                     // L4
};
// two input buffers (this tile's, the next tile's) and the two others
template <int G>
constexpr int group_smem() {
    return (2 * GSpec<G>::BUF0 + GSpec<G>::BUF1 + GSpec<G>::BUF2) * 4;
}
static_assert(group_smem<0>() <= 227 * 1024 && group_smem<1>() <= 227 * 1024, "group shared memory");

struct GroupArgs {
    const float* src;   // the group's input level, R x C
    int R, C;
    int tiles_x, n_tiles;
    float* dog[3];      // DoG planes of the group's layers
    float* mag[3];      // group 0: gradients of L1, L2, L3
    float* ang[3];
    float* dst;         // group 0: L3
    float* down;        // group 0: L3[::2, ::2] or null
    int down_cols;
};

// input level of tile t (rows y0 - HIN .., columns x0 - XIN .., reflect-101 outside) by cp.async
template <class L>
__device__ __forceinline__ void g_load(const GroupArgs& a, int t, float* dst) {
    const int y0 = (t / a.tiles_x) * GY, cx = (t % a.tiles_x) * GX - L::XIN;
    if ((a.C & 3) == 0 && al16(a.src) && cx >= 0 && cx + L::MIN <= a.C) {
        // eight lanes per row (the mirrored row address once per row)
        for (int row = threadIdx.x >> 3; row < L::NIN; row += GNT / 8) {
            const float* g = a.src + (size_t)mir(y0 - L::HIN + row, a.R) * a.C + cx;
#pragma unroll
            for (int k = 0; k < (L::MIN / 4 + 7) / 8; ++k) {
                const int q = (threadIdx.x & 7) + 8 * k;
                if (q < L::MIN / 4) cp_async16(dst + row * L::MIN + 4 * q, g + 4 * q);
            }
        }
    } else {
        for (int i = threadIdx.x; i < L::NIN * L::MIN; i += GNT) {
            const int row = i / L::MIN, col = i - row * L::MIN;
            cp_async4(dst + row * L::MIN + col, a.src + (size_t)mir(y0 - L::HIN + row, a.R) * a.C + mir(cx + col, a.C));
        }
    }
}

// vertical pass of level L: thread item = (column pair, 8 output rows); the last group of a level
// whose height is not a multiple of 8 starts at row NOUT - 8 (rows it shares with the group before
// are written twice with the same values), so every load stays inside the input level. Only the
// level's rows below kmax and the columns its horizontal pass reads for output columns below jmax
// are computed (a tile that reaches past the image needs its level only to the halo beyond it).
template <int TS, class L>
__device__ __forceinline__ void g_vpass(const float* __restrict__ pin, float2* __restrict__ v, int kmax, int jmax) {
    constexpr int r = L::RAD, NQ = L::VW / 2, NG = (L::NOUT + 7) / 8;
    static_assert(L::NOUT >= 8 && L::NIN == L::NOUT + 2 * r + 2 * L::ROFF, "vertical pass rows");
    float2 w[r + 1];
    load_taps<TS, r>(w);
    const int qmax = jmax + 2 * r + L::E + 4;   // 2q below it: every column the needed items read
    for (int it = threadIdx.x; it < NQ * NG; it += GNT) {
        const int q = it % NQ, g = it / NQ;
        const int y8 = min(8 * g, L::NOUT - 8);
        if (y8 >= kmax || 2 * q >= qmax) continue;
        const float* base = pin + (y8 + L::ROFF) * L::MIN + L::VS + 2 * q;
        float2 x[8 + 2 * r];
#pragma unroll
        for (int k = 0; k < 8 + 2 * r; ++k) x[k] = *reinterpret_cast<const float2*>(base + k * L::MIN);
        float2* d = v + (y8 / 2) * L::VP + 2 * q + L::E;
#pragma unroll
        for (int sp = 0; sp < 4; ++sp) {
            const float2 o0 = blur_pairs_w<r>(x + 2 * sp, w), o1 = blur_pairs_w<r>(x + 2 * sp + 1, w);
            d[sp * L::VP] = make_float2(o0.x, o1.x);
            d[sp * L::VP + 1] = make_float2(o0.y, o1.y);
        }
    }
}

// horizontal pass of level L: thread item = (row pair, 4 columns); the level's rows go to `pout`
// (when not null) and epi(tile row of the upper row, tile column, upper row, lower row) runs for
// every item (it checks the tile bounds itself); items at rows from kmax or columns from jmax on
// are not needed and skipped
template <int TS, class L, class Epi>
__device__ __forceinline__ void g_hpass(const float2* __restrict__ v, float* __restrict__ pout, Epi epi, int kmax,
                                        int jmax) {
    constexpr int r = L::RAD, NC = L::MOUT / 4, NP = L::NOUT / 2;
    float2 w[r + 1];
    load_taps<TS, r>(w);
    for (int it = threadIdx.x; it < NP * NC; it += GNT) {
        const int p = it / NC, c = 4 * (it - p * NC);
        if (2 * p >= kmax || c >= jmax) continue;
        const float4* src = reinterpret_cast<const float4*>(v + p * L::VP + c + 2 * L::E);
        float2 yv[4 + 2 * r];
#pragma unroll
        for (int k = 0; k < 2 + r; ++k) {
            const float4 t = src[k];
            yv[2 * k] = make_float2(t.x, t.y);
            yv[2 * k + 1] = make_float2(t.z, t.w);
        }
        float2 o[4];
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) o[cc] = blur_pairs_w<r>(yv + cc, w);
        const float4 top = make_float4(o[0].x, o[1].x, o[2].x, o[3].x);
        const float4 bot = make_float4(o[0].y, o[1].y, o[2].y, o[3].y);
        if (pout) {
            *reinterpret_cast<float4*>(pout + (2 * p) * L::MOUT + c) = top;
            *reinterpret_cast<float4*>(pout + (2 * p + 1) * L::MOUT + c) = bot;
        }
        epi(2 * p - L::HOUT, c - L::XOUT, top, bot);
    }
}

__device__ __forceinline__ void g_store4(float* p, float4 v, bool vec, int left) {
    if (vec && al16(p)) {
        *reinterpret_cast<float4*>(p) = v;
    } else {
        const float w[4] = {v.x, v.y, v.z, v.w};
        for (int k = 0; k < 4 && k < left; ++k) p[k] = w[k];
    }
}

// at image row yy, columns xx .. xx + 3: the DoG cur - prev and, with mag set, the gradient of
// prev (prev points at prev(yy, xx) in a shared level of pitch P; the same arithmetic as k_layer)
template <int P>
__device__ __forceinline__ void g_dog_grad(const GroupArgs& a, int yy, int xx, const float* prev, float4 cur,
                                           float* dog, float* mag, float* ang) {
    const float4 pv = *reinterpret_cast<const float4*>(prev);
    const size_t at = (size_t)yy * a.C + xx;
    const bool vec = (a.C & 3) == 0;   // xx is a multiple of 4 below C
    g_store4(dog + at, make_float4(cur.x - pv.x, cur.y - pv.y, cur.z - pv.z, cur.w - pv.w), vec, a.C - xx);
    if (mag) {
        float mg[4], an[4];
        grad4<P>(prev, yy, xx, a.R, a.C, mg, an);
        g_store4(mag + at, make_float4(mg[0], mg[1], mg[2], mg[3]), vec, a.C - xx);
        g_store4(ang + at, make_float4(an[0], an[1], an[2], an[3]), vec, a.C - xx);
    }
}

// epilogue of a level: for the tile pixels of an item, DoG (this level - prev) and the gradient of
// prev, prev being the shared level (halo PH, PX, pitch P) below
template <int PH, int PX, int P>
struct GEpi {
    const GroupArgs& a;
    int y0, x0;
    const float* prev;
    float *dog, *mag, *ang;
    __device__ __forceinline__ void operator()(int ty, int tx, float4 top, float4 bot) const {
        if (tx < 0 || tx >= GX || x0 + tx >= a.C) return;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int t = ty + h;
            if (t < 0 || t >= GY || y0 + t >= a.R) continue;
            g_dog_grad<P>(a, y0 + t, x0 + tx, prev + (PH + t) * P + PX + tx, h ? bot : top, dog, mag, ang);
        }
    }
};

template <int G>
__global__ void __launch_bounds__(GNT, 1) k_group(GroupArgs a) {
    using Sp = GSpec<G>;
    using LA = typename Sp::A;
    extern __shared__ __align__(16) float sm[];
    float* b1 = sm + 2 * Sp::BUF0;
    float* b2 = b1 + Sp::BUF1;
    int t = blockIdx.x;
    if (t >= a.n_tiles) return;
    g_load<LA>(a, t, sm);
    cp_commit();
    for (int cur = 0; t < a.n_tiles; t += gridDim.x, cur ^= 1) {
        cp_wait_all();
        __syncthreads();   // this tile's input is in; every thread is done with the previous tile
        const int nt = t + gridDim.x;
        if (nt < a.n_tiles) g_load<LA>(a, nt, sm + (cur ^ 1) * Sp::BUF0);
        cp_commit();
        const int y0 = (t / a.tiles_x) * GY, x0 = (t % a.tiles_x) * GX;
        const int vy = min(GY, a.R - y0), vx = min(GX, a.C - x0);   // the tile's pixels inside the image
        float* b0 = sm + cur * Sp::BUF0;
        if constexpr (G == 0) {
            using LB = typename Sp::B;
            using LC = typename Sp::C;
            g_vpass<1, LA>(b0, reinterpret_cast<float2*>(b1), vy + 2 * LA::HOUT, vx + 2 * LA::XOUT);  // L0 -> V1
            __syncthreads();
            g_hpass<1, LA>(reinterpret_cast<const float2*>(b1), b2,                               // V1 -> L1
                           GEpi<LA::HIN, LA::XIN, LA::MIN>{a, y0, x0, b0, a.dog[0], nullptr, nullptr},
                           vy + 2 * LA::HOUT, vx + 2 * LA::XOUT);
            __syncthreads();
            g_vpass<2, LB>(b2, reinterpret_cast<float2*>(b0), vy + 2 * LB::HOUT, vx + 2 * LB::XOUT);  // L1 -> V2
            __syncthreads();
            g_hpass<2, LB>(reinterpret_cast<const float2*>(b0), b1,                               // V2 -> L2
                           GEpi<LB::HIN, LB::XIN, LB::MIN>{a, y0, x0, b2, a.dog[1], a.mag[0], a.ang[0]},
                           vy + 2 * LB::HOUT, vx + 2 * LB::XOUT);
            __syncthreads();
            g_vpass<3, LC>(b1, reinterpret_cast<float2*>(b0), vy + 2 * LC::HOUT, vx + 2 * LC::XOUT);  // L2 -> V3
            __syncthreads();
            g_hpass<3, LC>(reinterpret_cast<const float2*>(b0), b2,                               // V3 -> L3
                           GEpi<LC::HIN, LC::XIN, LC::MIN>{a, y0, x0, b1, a.dog[2], a.mag[1], a.ang[1]},
                           vy + 2 * LC::HOUT, vx + 2 * LC::XOUT);
            __syncthreads();
            // gradient of L3, L3 and L3[::2, ::2] on the tile
            for (int it = threadIdx.x; it < GY * (GX / 4); it += GNT) {
                const int ty = it / (GX / 4), tx = 4 * (it - ty * (GX / 4));
                const int yy = y0 + ty, xx = x0 + tx;
                if (yy >= a.R || xx >= a.C) continue;
                const float* l3 = b2 + (LC::HOUT + ty) * LC::MOUT + LC::XOUT + tx;
                const float4 v = *reinterpret_cast<const float4*>(l3);
                float mg[4], an[4];
                grad4<LC::MOUT>(l3, yy, xx, a.R, a.C, mg, an);
                const size_t at = (size_t)yy * a.C + xx;
                const bool vec = (a.C & 3) == 0;
                g_store4(a.mag[2] + at, make_float4(mg[0], mg[1], mg[2], mg[3]), vec, a.C - xx);
                g_store4(a.ang[2] + at, make_float4(an[0], an[1], an[2], an[3]), vec, a.C - xx);
                g_store4(a.dst + at, v, vec, a.C - xx);
                if (a.down && !(yy & 1)) {
                    float* o2 = a.down + (size_t)(yy >> 1) * a.down_cols + (xx >> 1);
                    o2[0] = v.x;
                    if (xx + 2 < a.C) o2[1] = v.z;
                }
            }
        } else {
            using LB = typename Sp::B;
            g_vpass<4, LA>(b0, reinterpret_cast<float2*>(b1), vy + 2 * LA::HOUT, vx + 2 * LA::XOUT);  // L3 -> V4
            __syncthreads();
            g_hpass<4, LA>(reinterpret_cast<const float2*>(b1), b2,                               // V4 -> L4
                           GEpi<LA::HIN, LA::XIN, LA::MIN>{a, y0, x0, b0, a.dog[0], nullptr, nullptr},
                           vy + 2 * LA::HOUT, vx + 2 * LA::XOUT);
            __syncthreads();
            g_vpass<5, LB>(b2, reinterpret_cast<float2*>(b0), vy + 2 * LB::HOUT, vx + 2 * LB::XOUT);  // L4 -> V5
            __syncthreads();
            g_hpass<5, LB>(reinterpret_cast<const float2*>(b0), nullptr,                          // V5 -> L5
                           GEpi<LB::HIN, LB::XIN, LB::MIN>{a, y0, x0, b2, a.dog[1], nullptr, nullptr},
                           vy + 2 * LB::HOUT, vx + 2 * LB::XOUT);
        }
    }
    cp_wait_all();
}

int sm_count() {
    static int n[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64) return 148;
    if (!n[dev] && cudaDeviceGetAttribute(&n[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) n[dev] = 148;
    return n[dev];
}

template <int G>
int32_t launch_group_t(GroupArgs a, cudaStream_t s) {
    static std::atomic<int> attr[64];
    FSB_TRY(smem_attr((const void*)k_group<G>, group_smem<G>(), attr));
    a.tiles_x = (a.C + GX - 1) / GX;
    a.n_tiles = a.tiles_x * ((a.R + GY - 1) / GY);
    const int grid = a.n_tiles < sm_count() ? a.n_tiles : sm_count();
    k_group<G><<<grid, GNT, group_smem<G>(), s>>>(a);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

// ------------------------------------------------------------------------------------------------
// Strip engine (float32 path): one launch per octave. A CTA owns a 128-column strip and a range of
// output rows and streams down it eight rows per step; all five layers of the octave are held in
// shared-memory row rings, so per octave pixel HBM sees one read of L0 (plus the strip's column
// halo) and the 44 bytes of DoG and gradient output, nothing else.
//
//   level i (L0 .. L4) ring: TN(i) rows of TWID(i) columns starting TH(i) columns left of the
//       strip; slot of image row y = (y - RB) mod TN(i). Ring 0 holds the 2 r_1 + 8 rows stage 1
//       reads plus the next eight rows arriving by TMA (one 2-D tensor copy per row, the row index
//       reflected at the image's top and bottom; columns outside the image are filled in from
//       global memory with the reflected column after the copy lands).
//   stage i (1 .. 5), at step t, produces rows Y_i = Y_1 - TLAG(i) .. + 7 of L_i, Y_1 = V0 + 8t + 3:
//       phase A  vertical pass of L_{i-1} into the row-pair interleaved buffer (thread = column
//                pair, all eight rows: 2 r + 8 loads); with it the gradient of L_{i-1} at rows
//                Y_i .. (i = 2..4, plus L3[::2, ::2] for i = 4) and the DoG L_{i-1} - L_{i-2} at
//                rows Y_{i-1} .. (i = 2..5), both on the strip's own columns;
//       phase B  horizontal pass (thread = row pair x four columns) into ring i; stage 5 writes the
//                DoG L5 - L4 from registers instead.
// The passes are the per-layer kernels' (the same packed pair blurs in the same order), so the
// outputs are bit-identical to theirs: L0 is mirrored once and every level computed on the
// extended domain is the mirror image of its interior (pair sums commute). A stage runs only while
// its rows are needed by the output range (the range widened by the later layers' radii).
constexpr int TW = 128, TSTEP = 8, TNT = 256;
__host__ __device__ constexpr int TH(int i) { return i == 0 ? 44 : i == 1 ? 38 : i == 2 ? 32 : i == 3 ? 24 : i == 4 ? 14 : 0; }
__host__ __device__ constexpr int TWID(int i) { return i == 0 ? 216 : i == 1 ? 204 : i == 2 ? 192 : i == 3 ? 176 : i == 4 ? 156 : 128; }
__host__ __device__ constexpr int TPITCH(int i) { return i == 0 ? 224 : TWID(i); }
__host__ __device__ constexpr int TN(int i) { return i == 0 ? 2 * 5 + 2 * TSTEP : 2 * RAD(i + 1) + TSTEP; }
// rows (and columns) of L_i needed beyond the output range
__host__ __device__ constexpr int TE(int i) { return i == 0 ? 42 : i == 1 ? 37 : i == 2 ? 31 : i == 3 ? 23 : i == 4 ? 13 : 0; }
__host__ __device__ constexpr int TLAG(int i) { return i == 1 ? 0 : i == 2 ? 6 : i == 3 ? 14 : i == 4 ? 24 : 37; }
// vertical pass of stage i: columns x0 - TH(i-1) .. (ring i-1 column j = V column j), TVW(i) of them,
// stored at float2 index j + TSD(i) % 2 so that the horizontal pass reads from an even index
__host__ __device__ constexpr int TVW(int i) { return TWID(i - 1); }
__host__ __device__ constexpr int TSD(int i) { return TH(i - 1) - TH(i) - RAD(i); }
constexpr int TVP = 218;   // float2 per row pair of the vertical-pass buffer
__host__ __device__ constexpr int toff(int i) { return i == 0 ? 0 : toff(i - 1) + TN(i - 1) * TPITCH(i - 1); }
constexpr int TVB_OFF = toff(5);
constexpr int TBAR_OFF = TVB_OFF + 4 * TVP * 2;
constexpr int TSMEM = TBAR_OFF * 4 + 32;
constexpr int TROW_BYTES = TWID(0) * 4;   // one TMA row copy
static_assert(TSD(1) >= 0 && TSD(2) >= 0 && TSD(3) >= 0 && TSD(4) >= 0 && TSD(5) >= 0, "strip halos");
static_assert(TVW(1) + TSD(1) % 2 <= TVP && TVW(5) + TSD(5) % 2 <= TVP, "vertical buffer width");
static_assert((toff(1) * 4) % 128 == 0 && (TPITCH(0) * 4) % 128 == 0, "TMA destinations 128-byte aligned");
static_assert(TSMEM <= 113 * 1024, "two CTAs per SM");

struct StripArgs {
    const float* L0;   // octave base, R x C, row pitch C
    int R, C, rows;    // rows: output rows per CTA
    float* dog[5];
    float* mag[3];
    float* ang[3];
    float* down;       // L3[::2, ::2] (pitch down_cols) or null
    int down_cols;
    int* err;          // set to 1 when a TMA wait gives up
};

// rows y .. y + 7 of L0 into ring 0: TMA (one thread issues eight row copies on `bar`) or, when
// tma is false, cp.async with reflected rows and columns
__device__ __forceinline__ void s_load_block(const CUtensorMap* tm, const StripArgs& a, float* ring0, uint64_t* bar,
                                             int x0, int y, int RB, bool tma) {
    if (tma) {
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s_addr(bar)),
                         "r"(TSTEP * TROW_BYTES)
                         : "memory");
#pragma unroll 1
            for (int k = 0; k < TSTEP; ++k) {
                const int row = y + k;
                float* dst = ring0 + ((row - RB) % TN(0)) * TPITCH(0);
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
                        s_addr(dst)),
                    "l"(reinterpret_cast<uint64_t>(tm)), "r"(x0 - TH(0)), "r"(mir(row, a.R)), "r"(s_addr(bar))
                    : "memory");
            }
        }
    } else {
        const int c = threadIdx.x;
        if (c < TWID(0)) {
            int xs = x0 - TH(0) + c;
            if (xs < 0 || xs >= a.C) xs = mir(xs, a.C);
#pragma unroll 1
            for (int k = 0; k < TSTEP; ++k) {
                const int row = y + k;
                cp_async4(ring0 + ((row - RB) % TN(0)) * TPITCH(0) + c, a.L0 + (size_t)mir(row, a.R) * a.C + xs);
            }
        }
        cp_commit();
    }
}

// After a TMA block landed: the columns outside the image (zero-filled) get their reflected values
__device__ __forceinline__ void s_fix_edges(const StripArgs& a, float* ring0, int x0, int y, int RB) {
    const int lo = TH(0) - x0;                 // ring columns [0, lo) are left of the image
    const int hi = a.C - (x0 - TH(0));         // ring columns [hi, TWID(0)) are right of it
    if (lo <= 0 && hi >= TWID(0)) return;
    for (int i = threadIdx.x; i < TSTEP * TWID(0); i += TNT) {
        const int k = i / TWID(0), c = i - k * TWID(0);
        if (c >= lo && c < hi) continue;
        const int row = y + k;
        ring0[((row - RB) % TN(0)) * TPITCH(0) + c] = __ldg(a.L0 + (size_t)mir(row, a.R) * a.C + mir(x0 - TH(0) + c, a.C));
    }
}

__device__ __forceinline__ void s_store4(float* p, float4 v, bool vec, int left) {
    if (vec) {
        *reinterpret_cast<float4*>(p) = v;
    } else {
        const float w[4] = {v.x, v.y, v.z, v.w};
        for (int k = 0; k < 4 && k < left; ++k) p[k] = w[k];
    }
}

template <int I>
__device__ __forceinline__ int s_slot(int row, int RB) { return (row - RB) % TN(I); }

struct StripCta {
    int x0, ya, yz, RB;
    bool vec;   // 16-byte stores of the output planes (C multiple of 4, planes aligned)
};

// vertical pass of stage I, column pair q: all eight rows Y .. Y + 7
template <int I>
__device__ __forceinline__ void s_vitem(const float* __restrict__ ring, float2* __restrict__ vb, int q, int s0,
                                        const float2 (&w)[RAD(I) + 1]) {
    constexpr int r = RAD(I), N = TN(I - 1), P = TPITCH(I - 1), dd = TSD(I) & 1;
    const float* base = ring + 2 * q;
    float2 x[2 * r + TSTEP];
    int s = s0;
#pragma unroll
    for (int k = 0; k < 2 * r + TSTEP; ++k) {
        x[k] = *reinterpret_cast<const float2*>(base + s * P);
        s = s + 1 == N ? 0 : s + 1;
    }
    float2* d = vb + 2 * q + dd;
#pragma unroll
    for (int sp = 0; sp < TSTEP / 2; ++sp) {
        const float2 o0 = blur_pairs_w<r>(x + 2 * sp, w), o1 = blur_pairs_w<r>(x + 2 * sp + 1, w);
        d[sp * TVP] = make_float2(o0.x, o1.x);
        d[sp * TVP + 1] = make_float2(o0.y, o1.y);
    }
}

// gradient of L_I (I = 1..3) at image row y, strip columns 4g .. 4g + 3, from ring I; for I = 3
// also L3[::2, ::2]
template <int I>
__device__ __forceinline__ void s_grad_item(const float* __restrict__ ring, const StripArgs& a, const StripCta& k,
                                            int y, int g) {
    constexpr int P = TPITCH(I);
    const int x = k.x0 + 4 * g;
    if (x >= a.C) return;
    const float* ct = ring + s_slot<I>(y, k.RB) * P + TH(I) + 4 * g;
    const float* up = ring + s_slot<I>(y - 1, k.RB) * P + TH(I) + 4 * g;
    const float* dn = ring + s_slot<I>(y + 1, k.RB) * P + TH(I) + 4 * g;
    const float2 c0 = *reinterpret_cast<const float2*>(ct), c1 = *reinterpret_cast<const float2*>(ct + 2);
    const float2 u0 = *reinterpret_cast<const float2*>(up), u1 = *reinterpret_cast<const float2*>(up + 2);
    const float2 d0 = *reinterpret_cast<const float2*>(dn), d1 = *reinterpret_cast<const float2*>(dn + 2);
    const float lf = ct[-1], rt = ct[4];
    float2 dxa = make_float2(__fsub_rn(c0.y, lf), __fsub_rn(c1.x, c0.x));
    float2 dxb = make_float2(__fsub_rn(c1.y, c0.y), __fsub_rn(rt, c1.x));
    float2 dya = make_float2(__fsub_rn(u0.x, d0.x), __fsub_rn(u0.y, d0.y));
    float2 dyb = make_float2(__fsub_rn(u1.x, d1.x), __fsub_rn(u1.y, d1.y));
    if (!(y > 0 && y < a.R - 1 && x > 0 && x + 4 < a.C)) {
        float dxv[4] = {dxa.x, dxa.y, dxb.x, dxb.y}, dyv[4] = {dya.x, dya.y, dyb.x, dyb.y};
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (!(y > 0 && y < a.R - 1 && x + j > 0 && x + j < a.C - 1)) dxv[j] = dyv[j] = 0.f;
        dxa = make_float2(dxv[0], dxv[1]);
        dxb = make_float2(dxv[2], dxv[3]);
        dya = make_float2(dyv[0], dyv[1]);
        dyb = make_float2(dyv[2], dyv[3]);
    }
    // the gradient of the other engines (same function, same roundings)
    const float dxv[4] = {dxa.x, dxa.y, dxb.x, dxb.y}, dyv[4] = {dya.x, dya.y, dyb.x, dyb.y};
    float mg[4], an[4];
    fast_grad4(dxv, dyv, mg, an);
    const size_t at = (size_t)y * a.C + x;
    s_store4(a.mag[I - 1] + at, make_float4(mg[0], mg[1], mg[2], mg[3]), k.vec, a.C - x);
    s_store4(a.ang[I - 1] + at, make_float4(an[0], an[1], an[2], an[3]), k.vec, a.C - x);
    if (I == 3 && a.down && !(y & 1)) {
        float* o = a.down + (size_t)(y >> 1) * a.down_cols + (x >> 1);
        o[0] = c0.x;
        if (x + 2 < a.C) o[1] = c1.x;
    }
}

// DoG L_I - L_{I-1} (I = 1..4) at image row y, strip columns 4g .. 4g + 3
template <int I>
__device__ __forceinline__ void s_dog_item(const float* __restrict__ ri, const float* __restrict__ rp, const StripArgs& a,
                                           const StripCta& k, int y, int g) {
    const int x = k.x0 + 4 * g;
    if (x >= a.C) return;
    const float* c = ri + s_slot<I>(y, k.RB) * TPITCH(I) + TH(I) + 4 * g;
    const float* p = rp + s_slot<I - 1>(y, k.RB) * TPITCH(I - 1) + TH(I - 1) + 4 * g;
    const float2 c0 = *reinterpret_cast<const float2*>(c), c1 = *reinterpret_cast<const float2*>(c + 2);
    const float2 p0 = *reinterpret_cast<const float2*>(p), p1 = *reinterpret_cast<const float2*>(p + 2);
    const float2 d0 = __fadd2_rn(c0, make_float2(-p0.x, -p0.y)), d1 = __fadd2_rn(c1, make_float2(-p1.x, -p1.y));
    s_store4(a.dog[I - 1] + (size_t)y * a.C + x, make_float4(d0.x, d0.y, d1.x, d1.y), k.vec, a.C - x);
}

// Phase A of stage I: vertical pass (rows Y .. Y + 7 of V_I), gradient of L_{I-1} at rows Y .., DoG
// L_{I-1} - L_{I-2} at rows Y + RAD(I) .. (the rows stage I-1 produced in this step)
template <int I>
__device__ __forceinline__ void s_phase_a(float* const* ring, float2* vb, const StripArgs& a, const StripCta& k, int Y,
                                          bool act) {
    constexpr int r = RAD(I);
    constexpr int NV = TVW(I) / 2, NVP = (NV + 31) & ~31;
    const int ylo = max(k.ya, 0), yhi = min(k.yz, a.R);
    const bool g_on = I >= 2 && I <= 4 && Y + TSTEP > ylo && Y < yhi;
    const int Yd = Y + r;   // rows of the DoG L_{I-1} - L_{I-2}
    const bool d_on = I >= 2 && Yd + TSTEP > ylo && Yd < yhi;
    const int nv = act ? NVP : 0;
    const int ng = g_on ? TSTEP * (TW / 4) : 0;
    const int nd = d_on ? TSTEP * (TW / 4) : 0;
    float2 w[r + 1];
    load_taps<I, r>(w);
    const int s0 = s_slot<I - 1>(Y - r, k.RB);
    for (int it = threadIdx.x; it < nv + ng + nd; it += TNT) {
        if (it < nv) {
            if (it < NV) s_vitem<I>(ring[I - 1], vb, it, s0, w);
        } else if (it < nv + ng) {
            if constexpr (I >= 2 && I <= 4) {
                const int j = it - nv, y = Y + j / (TW / 4);
                if (y >= ylo && y < yhi) s_grad_item<I - 1>(ring[I - 1], a, k, y, j % (TW / 4));
            }
        } else {
            if constexpr (I >= 2) {
                const int j = it - nv - ng, y = Yd + j / (TW / 4);
                if (y >= ylo && y < yhi) s_dog_item<I - 1>(ring[I - 1], ring[I - 2], a, k, y, j % (TW / 4));
            }
        }
    }
}

// Phase B of stage I: horizontal pass, thread = (row pair p, columns 4c .. 4c + 3 of ring I); stage 5
// writes the DoG L5 - L4 of the strip's columns instead of a ring
template <int I>
__device__ __forceinline__ void s_phase_b(float* const* ring, const float2* vb, const StripArgs& a, const StripCta& k,
                                          int Y) {
    constexpr int r = RAD(I), NC = TWID(I) / 4, off = TSD(I) + (TSD(I) & 1);
    float2 w[r + 1];
    load_taps<I, r>(w);
    const int it = threadIdx.x;
    if (it >= 4 * NC) return;
    const int p = it / NC, c = 4 * (it - p * NC);
    const float4* src = reinterpret_cast<const float4*>(vb + p * TVP + c + off);
    float2 yv[4 + 2 * r];
#pragma unroll
    for (int j = 0; j < 2 + r; ++j) {
        const float4 v = src[j];
        yv[2 * j] = make_float2(v.x, v.y);
        yv[2 * j + 1] = make_float2(v.z, v.w);
    }
    float2 o[4];
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) o[cc] = blur_pairs_w<r>(yv + cc, w);
    const float4 top = make_float4(o[0].x, o[1].x, o[2].x, o[3].x);
    const float4 bot = make_float4(o[0].y, o[1].y, o[2].y, o[3].y);
    const int y = Y + 2 * p;
    if constexpr (I < 5) {
        float* ri = ring[I];
        *reinterpret_cast<float4*>(ri + s_slot<I>(y, k.RB) * TPITCH(I) + c) = top;
        *reinterpret_cast<float4*>(ri + s_slot<I>(y + 1, k.RB) * TPITCH(I) + c) = bot;
    } else {
        const int x = k.x0 + c;
        if (x >= a.C) return;
        const int ylo = max(k.ya, 0), yhi = min(k.yz, a.R);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int yy = y + h;
            if (yy < ylo || yy >= yhi) continue;
            const float* pr = ring[4] + s_slot<4>(yy, k.RB) * TPITCH(4) + TH(4) + c;
            const float2 p0 = *reinterpret_cast<const float2*>(pr), p1 = *reinterpret_cast<const float2*>(pr + 2);
            const float4 l = h ? bot : top;
            const float2 d0 = __fadd2_rn(make_float2(l.x, l.y), make_float2(-p0.x, -p0.y));
            const float2 d1 = __fadd2_rn(make_float2(l.z, l.w), make_float2(-p1.x, -p1.y));
            s_store4(a.dog[4] + (size_t)yy * a.C + x, make_float4(d0.x, d0.y, d1.x, d1.y), k.vec, a.C - x);
        }
    }
}

template <int I>
__device__ __forceinline__ void s_stage(float* const* ring, float2* vb, const StripArgs& a, const StripCta& k, int Y1) {
    const int Y = Y1 - TLAG(I);
    const bool act = Y + TSTEP > k.ya - TE(I) && Y < k.yz + TE(I);
    s_phase_a<I>(ring, vb, a, k, Y, act);
    __syncthreads();
    if (act) s_phase_b<I>(ring, vb, a, k, Y);
    __syncthreads();
}

__global__ void __launch_bounds__(TNT, 2) k_strip(const __grid_constant__ CUtensorMap tmap, StripArgs a, int use_tma) {
    extern __shared__ __align__(1024) float sm_strip[];
    float* sm = sm_strip;
    float* ring[5] = {sm + toff(0), sm + toff(1), sm + toff(2), sm + toff(3), sm + toff(4)};
    float2* vb = reinterpret_cast<float2*>(sm + TVB_OFF);
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + TBAR_OFF);
    if (use_tma && (s_addr(sm) & 127) != 0) {   // TMA destinations must be 128-byte aligned
        if (threadIdx.x == 0) atomicExch(a.err, 2);
        return;
    }
    StripCta k;
    k.x0 = blockIdx.x * TW;
    k.ya = blockIdx.y * a.rows;
    k.yz = min(a.R, k.ya + a.rows);
    const int V0 = k.ya - TE(0);   // first L0 row held
    k.RB = V0 - 64;                // every row read is above RB
    k.vec = (a.C & 3) == 0;
    for (int i = 0; i < 5; ++i) k.vec = k.vec && al16(a.dog[i]);
    for (int i = 0; i < 3; ++i) k.vec = k.vec && al16(a.mag[i]) && al16(a.ang[i]);
    const bool tma = use_tma != 0;
    const int T = (k.yz - k.ya + TE(0) + TLAG(5) - 3 + TSTEP - 1) / TSTEP;   // steps
    if (tma && threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s_addr(bar)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(s_addr(bar + 1)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    s_load_block(&tmap, a, ring[0], bar, k.x0, V0, k.RB, tma);
    s_load_block(&tmap, a, ring[0], bar + 1, k.x0, V0 + TSTEP, k.RB, tma);
    for (int t = 0; t < T; ++t) {
        // blocks t and t + 1 (rows V0 + 8t .. V0 + 8t + 15) must be in ring 0
        if (tma) {
            bool ok = true;
            for (int b = (t == 0 ? 0 : t + 1); b <= t + 1; ++b) {
                ok = ok && s_mbar_wait(bar + (b & 1), (b >> 1) & 1);
                if (ok) s_fix_edges(a, ring[0], k.x0, V0 + TSTEP * b, k.RB);
            }
            if (__syncthreads_or(!ok)) {
                // flag it and give the copies still in flight (blocks t, t + 1) one more bounded wait
                // each before leaving
                if (threadIdx.x == 0) atomicExch(a.err, 1);
                for (int b = t; b <= t + 1; ++b) s_mbar_wait(bar + (b & 1), (b >> 1) & 1);
                return;
            }
        } else {
            cp_wait_all();
            __syncthreads();
        }
        // the rows of block t + 2 take the slots of rows no stage reads in this step
        if (t + 2 <= T) {
            if (tma && threadIdx.x == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            s_load_block(&tmap, a, ring[0], bar + (t & 1), k.x0, V0 + TSTEP * (t + 2), k.RB, tma);
        }
        const int Y1 = V0 + TSTEP * t + 3;
        s_stage<1>(ring, vb, a, k, Y1);
        s_stage<2>(ring, vb, a, k, Y1);
        s_stage<3>(ring, vb, a, k, Y1);
        s_stage<4>(ring, vb, a, k, Y1);
        s_stage<5>(ring, vb, a, k, Y1);
    }
    // every issued TMA block (0 .. T) was waited for inside the loop
    if (!tma) cp_wait_all();
}

}  // namespace

// One float32 octave by the strip engine (one launch): from the base L0 (R x C, pitch C), the five
// DoG planes at dog + k RC, gradients of L1..L3 at mag / ang + k RC, L3[::2, ::2] to down (pitch
// down_cols; null for the last octave). err (device) is set when a TMA wait gives up.
int32_t launch_octave_strip(const float* L0, int R, int C, float* dog, float* mag, float* ang, float* down,
                            int down_cols, int* err, cudaStream_t s) {
    static std::atomic<int> attr[64];
    FSB_TRY(smem_attr((const void*)k_strip, TSMEM, attr));
    StripArgs a{};
    a.L0 = L0;
    a.R = R;
    a.C = C;
    const long long RC = (long long)R * C;
    for (int i = 0; i < 5; ++i) a.dog[i] = dog + i * RC;
    for (int i = 0; i < 3; ++i) {
        a.mag[i] = mag + i * RC;
        a.ang[i] = ang + i * RC;
    }
    a.down = down;
    a.down_cols = down_cols;
    a.err = err;
    // TMA row copies need a 16-byte row pitch and base; the box is the 216-column L0 window
    CUtensorMap tm;
    std::memset(&tm, 0, sizeof(tm));
    int use_tma = 0;
    EncodeTiledFn enc = encode_tiled();
    if (enc && (C & 3) == 0 && C >= TWID(0) && (reinterpret_cast<uintptr_t>(L0) & 15) == 0) {
        const cuuint64_t dims[2] = {(cuuint64_t)C, (cuuint64_t)R};
        const cuuint64_t strides[1] = {(cuuint64_t)C * 4};
        const cuuint32_t box[2] = {(cuuint32_t)TWID(0), 1};
        const cuuint32_t es[2] = {1, 1};
        use_tma = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(L0), dims, strides, box, es,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    // about two CTAs per SM: strips x row chunks, chunk heights a multiple of the step
    const int strips = (C + TW - 1) / TW;
    int chunks = (2 * sm_count() + strips / 2) / strips;
    if (chunks < 1) chunks = 1;
    int rows = (R + chunks - 1) / chunks;
    rows = (rows + TSTEP - 1) / TSTEP * TSTEP;
    a.rows = rows;
    dim3 grid(strips, (R + rows - 1) / rows);
    k_strip<<<grid, TNT, TSMEM, s>>>(tm, a, use_tma);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

int32_t launch_octave_fused(const float* L0, int R, int C, float* dog, float* mag, float* ang, float* down,
                            int down_cols, cudaStream_t s) {
    static std::atomic<int> attr[64];
    FSB_TRY(smem_attr((const void*)k_octave, SMEM_BYTES, attr, 100));
    Args a;
    a.L0 = L0;
    a.R = R;
    a.C = C;
    const long long RC = (long long)R * C;
    for (int i = 0; i < 5; ++i) a.dog[i] = dog + i * RC;
    for (int i = 0; i < 3; ++i) {
        a.mag[i] = mag + i * RC;
        a.ang[i] = ang + i * RC;
    }
    a.down = down;
    a.down_cols = down_cols;
    // about two CTAs per SM over the whole octave
    const int strips = (C + SW - 1) / SW;
    int chunks = (2 * 148 + strips / 2) / strips;
    if (chunks < 1) chunks = 1;
    int rows = (R + chunks - 1) / chunks;
    if (rows < 32) rows = 32;
    a.rows_per_cta = rows;
    dim3 grid(strips, (R + rows - 1) / rows);
    k_octave<<<grid, NT, SMEM_BYTES, s>>>(a);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

}  // namespace fsb

namespace fsb {

int layer_tile_variants() { return 3; }
int layer_tile_height(int variant) { return kTileHeights[variant < 0 || variant > 2 ? 0 : variant]; }

// One layer of the float32 pyramid by the tiled per-layer kernel: L_layer from src (R x C), tile
// height layer_tile_height(variant).
int32_t launch_layer_fast(int layer, const float* src, int R, int C, float* dst, float* dog, float* mag, float* ang,
                          float* down, int down_cols, int variant, int* err, cudaStream_t s) {
    LayerArgs a{};
    a.err = err;
    a.src = src;
    a.R = R;
    a.C = C;
    a.dst = dst;
    a.dog = dog;
    a.mag = mag;
    a.ang = ang;
    a.down = down;
    a.down_cols = down_cols;
    switch (layer) {
        case 1: return launch_layer_t<1, 5, false>(a, variant, s);
        case 2: return launch_layer_t<2, 6, false>(a, variant, s);
        case 3: return launch_layer_t<3, 8, false>(a, variant, s);
        case 4: return launch_layer_t<4, 10, false>(a, variant, s);
        case 5: return launch_layer_t<5, 13, false>(a, variant, s);
        default: set_error("layer %d out of range", layer); return FSB_ERR_ARG;
    }
}


// Layers 1..3 of a float32 octave by the fused group kernel: from L0 (src, R x C), DoG planes
// 0..2 at dog, dog + RC, dog + 2RC, gradients of L1..L3 at mag / ang (+ RC, + 2RC), L3 to l3 and
// L3[::2, ::2] to down (null: last octave). down must not alias src (other tiles still read it).
int32_t launch_group_lower(const float* src, int R, int C, float* dog, float* mag, float* ang, float* l3, float* down,
                           int down_cols, cudaStream_t s) {
    const long long RC = (long long)R * C;
    GroupArgs a{};
    a.src = src;
    a.R = R;
    a.C = C;
    for (int k = 0; k < 3; ++k) {
        a.dog[k] = dog + k * RC;
        a.mag[k] = mag + k * RC;
        a.ang[k] = ang + k * RC;
    }
    a.dst = l3;
    a.down = down;
    a.down_cols = down_cols;
    return launch_group_t<0>(a, s);
}

// Layers 4, 5 of a float32 octave by the fused group kernel: from L3 (src), DoG planes 3, 4 at
// dog3, dog3 + RC.
int32_t launch_group_upper(const float* src, int R, int C, float* dog3, cudaStream_t s) {
    GroupArgs a{};
    a.src = src;
    a.R = R;
    a.C = C;
    a.dog[0] = dog3;
    a.dog[1] = dog3 + (long long)R * C;
    return launch_group_t<1>(a, s);
}

// The float32 octave-0 base: blur (tap set 0, radius 5) of the 2x upsampled uint8 image.
int32_t launch_base_fast(const uint8_t* img, int stride, int ih, int iw, float* dst, int variant, cudaStream_t s) {
    LayerArgs a{};
    a.img = img;
    a.img_stride = stride;
    a.ih = ih;
    a.iw = iw;
    a.R = 2 * ih;
    a.C = 2 * iw;
    a.dst = dst;
    return launch_layer_t<0, 5, true>(a, variant, s);
}

}  // namespace fsb
