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

// Gradient magnitude and direction (degrees in [0, 360)) for the default (float32) pyramid:
// magnitude through the reciprocal square root (within a few ulps of sqrt), direction by octant
// reduction to t = min/max in [0, 1] and an odd polynomial for atan(t) in degrees. The
// coefficients were fitted here by iteratively reweighted least squares on Chebyshev nodes
// (max error 2.2e-6 deg; 7.4e-6 deg with float32 evaluation), so the angle stays well inside the
// reference's 0.1 deg keypoint tolerance. atan2(0, 0) = 0 as in the reference (border pixels).
__device__ __forceinline__ void fast_grad(float dx, float dy, float& mag, float& ang) {
    const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
    mag = d2 > 0.f ? d2 * rsqrtf(d2) : 0.f;
    const float ax = fabsf(dx), ay = fabsf(dy);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    const float t = mx > 0.f ? __fdividef(mn, mx) : 0.f;
    const float z = t * t;
    float p = -2.323089093e-01f;
    p = fmaf(p, z, 1.252652928e+00f);
    p = fmaf(p, z, -3.203537344e+00f);
    p = fmaf(p, z, 5.524570187e+00f);
    p = fmaf(p, z, -7.969057098e+00f);
    p = fmaf(p, z, 1.142854019e+01f);
    p = fmaf(p, z, -1.909660354e+01f);
    p = fmaf(p, z, 5.729574144e+01f);
    float a = p * t;                       // atan(min/max) in degrees, [0, 45]
    if (ay > ax) a = 90.f - a;
    if (dx < 0.f) a = 180.f - a;
    if (dy < 0.f) a = 360.f - a;           // atan2 < 0 maps to a + 360 (may round to 360, as there)
    ang = a;
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
    if (vec) {
        *reinterpret_cast<float4*>(dg) = make_float4(d[0], d[1], d[2], d[3]);
    } else {
        for (int k = 0; k < 4 && xg + k < a.C; ++k) dg[k] = d[k];
    }
    if (I >= 2 && I <= 4) {
        const float* up = prev + wrap<PR>(ps + PR - 1) * PP + 4 * q + hp;
        const float* dn = prev + wrap<PR>(ps + 1) * PP + 4 * q + hp;
        float mg[4], an[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int x = xg + k;
            float dx = 0.f, dy = 0.f;
            if (y > 0 && y < a.R - 1 && x > 0 && x < a.C - 1) {
                dx = __fsub_rn(pr[k + 1], pr[k - 1]);
                dy = __fsub_rn(up[k], dn[k]);
            }
            fast_grad(dx, dy, mg[k], an[k]);
        }
        float* m = a.mag[I - 2] + at;
        float* n = a.ang[I - 2] + at;
        if (vec) {
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
    const bool aligned = (a.C & 3) == 0 && x0 - X0 >= 0 && x0 - X0 + WIN(0) <= a.C;
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
constexpr int LIN_W = LX + 32;   // input tile pitch (floats)
constexpr int LT2_W = LX + 32;   // row-pair tile pitch (float2)

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
};

template <int r, int LY>
constexpr int layer_smem() {
    return (LY + 2 * r) * LIN_W * 4 + (LY / 2) * LT2_W * 8;
}

template <int TS, int r, bool BASE, int LY>
__global__ void __launch_bounds__(LNT) k_layer(LayerArgs a) {
    constexpr int d = r & 1;
    constexpr int IH = LY + 2 * r;
    constexpr int NPAIR = (LX + 2 * r + 2 * d) / 2;
    extern __shared__ __align__(16) float sm[];
    float* s_in = sm;
    float2* t2 = reinterpret_cast<float2*>(sm + IH * LIN_W);
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * LX, y0 = blockIdx.y * LY;
    // input rows y0 - r .. y0 + LY + r - 1, columns x0 - 16 .. x0 + LX + 15 (reflect-101 outside)
    if (BASE) {
        // Source rows / columns of every tile row / column (reflect-101 on the upsampled grid),
        // then the row-interpolated values 0.75 a[iy] + 0.25 a[ny] of a window of source columns;
        // each upsampled sample is 0.75 vc[ix] + 0.25 vc[nx] (gsift.py:90-102 rounding). Tables and
        // window live in the row-pair area until the vertical pass needs it; a column outside the
        // window (mirrored columns of an edge tile) is computed from global memory.
        constexpr int VCW = 96;
        static_assert(!BASE || (2 * IH + 2 * LIN_W) * 4 + IH * VCW * 4 <= (LY / 2) * LT2_W * 8,
                      "base tables must fit the row-pair area");
        int* rtab = reinterpret_cast<int*>(t2);
        int* ctab = rtab + 2 * IH;
        float* vcs = reinterpret_cast<float*>(ctab + 2 * LIN_W);
        const int right = min(x0 + LX + 15, a.C - 1);
        int lo = x0 - 16;
        if (x0 + LX + 15 >= a.C) lo = min(lo, 2 * a.C - 2 - (x0 + LX + 15));
        const int sx0 = max(0, (lo >> 1) - 1);
        const int nsx = min(min(a.iw - 1, (right >> 1) + 1) - sx0 + 1, VCW);
        for (int i = tid; i < IH + LIN_W; i += LNT) {
            if (i < IH) {
                const int Y = mir(y0 - r + i, a.R), iy = Y >> 1;
                const int ny = (Y & 1) ? min(iy + 1, a.ih - 1) : max(iy - 1, 0);
                rtab[2 * i] = iy * a.img_stride;
                rtab[2 * i + 1] = ny * a.img_stride;
            } else {
                const int c = i - IH, X = mir(x0 - 16 + c, a.C), ix = X >> 1;
                const int nx = (X & 1) ? min(ix + 1, a.iw - 1) : max(ix - 1, 0);
                ctab[2 * c] = ix;
                ctab[2 * c + 1] = nx;
            }
        }
        __syncthreads();
        const float sc = (float)(1.0 / 255.0);
        for (int i = tid; i < IH * VCW; i += LNT) {
            const int row = i / VCW, k = i - row * VCW;
            if (k >= nsx) continue;
            const float p0 = __fmul_rn((float)__ldg(a.img + rtab[2 * row] + sx0 + k), sc);
            const float p1 = __fmul_rn((float)__ldg(a.img + rtab[2 * row + 1] + sx0 + k), sc);
            vcs[row * VCW + k] = __fadd_rn(__fmul_rn(0.75f, p0), __fmul_rn(0.25f, p1));
        }
        __syncthreads();
#pragma unroll 4
        for (int i = tid; i < IH * LIN_W; i += LNT) {
            const int row = i / LIN_W, col = i - row * LIN_W;
            const int ix = ctab[2 * col], nx = ctab[2 * col + 1];
            const int kx = ix - sx0, kn = nx - sx0;
            float vc, vn;
            if (kx >= 0 && kx < nsx && kn >= 0 && kn < nsx) {
                vc = vcs[row * VCW + kx];
                vn = vcs[row * VCW + kn];
            } else {
                const uint8_t* r0 = a.img + rtab[2 * row];
                const uint8_t* r1 = a.img + rtab[2 * row + 1];
                vc = __fadd_rn(__fmul_rn(0.75f, __fmul_rn((float)__ldg(r0 + ix), sc)),
                               __fmul_rn(0.25f, __fmul_rn((float)__ldg(r1 + ix), sc)));
                vn = __fadd_rn(__fmul_rn(0.75f, __fmul_rn((float)__ldg(r0 + nx), sc)),
                               __fmul_rn(0.25f, __fmul_rn((float)__ldg(r1 + nx), sc)));
            }
            s_in[row * LIN_W + col] = __fadd_rn(__fmul_rn(0.75f, vc), __fmul_rn(0.25f, vn));
        }
    } else if ((a.C & 3) == 0 && x0 >= 16 && x0 + LX + 16 <= a.C) {
        for (int i = tid; i < IH * (LIN_W / 4); i += LNT) {
            const int row = i / (LIN_W / 4), q = i - row * (LIN_W / 4);
            const float* g = a.src + (size_t)mir(y0 - r + row, a.R) * a.C + (x0 - 16 + 4 * q);
            cp_async16(s_in + row * LIN_W + 4 * q, g);
        }
    } else {
        for (int i = tid; i < IH * LIN_W; i += LNT) {
            const int row = i / LIN_W, col = i - row * LIN_W;
            const float* g = a.src + (size_t)mir(y0 - r + row, a.R) * a.C + mir(x0 - 16 + col, a.C);
            cp_async4(s_in + row * LIN_W + col, g);
        }
    }
    cp_commit();
    cp_wait_all();
    __syncthreads();
    // vertical pass: column pair cp (V columns 2cp, 2cp+1 = image columns x0 - r - d + 2cp ..),
    // output rows 8g .. 8g + 7; stored row-pair interleaved at t2 index (V column + d)
    for (int it = tid; it < NPAIR * (LY / 8); it += LNT) {
        const int cp = it % NPAIR, g = it / NPAIR;
        const float* base = s_in + (8 * g) * LIN_W + (16 - r - d + 2 * cp);
        float2 x[8 + 2 * r];
#pragma unroll
        for (int k = 0; k < 8 + 2 * r; ++k) x[k] = *reinterpret_cast<const float2*>(base + k * LIN_W);
#pragma unroll
        for (int sp = 0; sp < 4; ++sp) {
            const float2 o0 = blur_pairs_t<TS, r>(x + 2 * sp), o1 = blur_pairs_t<TS, r>(x + 2 * sp + 1);
            float2* dst = t2 + (4 * g + sp) * LT2_W + 2 * cp + d;
            dst[0] = make_float2(o0.x, o1.x);
            dst[1] = make_float2(o0.y, o1.y);
        }
    }
    __syncthreads();
    // horizontal pass: row pair p, output columns c .. c+3 (t2 indices c + 2d .. c + 2d + 3 + 2r)
    for (int it = tid; it < (LY / 2) * (LX / 4); it += LNT) {
        const int p = it / (LX / 4), c = 4 * (it - p * (LX / 4));
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
        for (int cc = 0; cc < 4; ++cc) o[cc] = blur_pairs_t<TS, r>(yv + cc);   // (row y, row y+1) at column x+cc
        const bool vec = (a.C & 3) == 0 && x + 4 <= a.C;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int yy = y + h;
            if (yy >= a.R) break;
            const float lv[4] = {h ? o[0].y : o[0].x, h ? o[1].y : o[1].x, h ? o[2].y : o[2].x, h ? o[3].y : o[3].x};
            if (BASE) {
                const size_t at = (size_t)yy * a.C + x;
                if (vec) {
                    *reinterpret_cast<float4*>(a.dst + at) = make_float4(lv[0], lv[1], lv[2], lv[3]);
                } else {
                    for (int k = 0; k < 4 && x + k < a.C; ++k) a.dst[at + k] = lv[k];
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
            if (vec) {
                *reinterpret_cast<float4*>(a.dog + at) = make_float4(dg[0], dg[1], dg[2], dg[3]);
                if (a.dst) *reinterpret_cast<float4*>(a.dst + at) = make_float4(lv[0], lv[1], lv[2], lv[3]);
            } else {
                for (int k = 0; k < 4 && x + k < a.C; ++k) {
                    a.dog[at + k] = dg[k];
                    if (a.dst) a.dst[at + k] = lv[k];
                }
            }
            if (a.mag) {
                float mg[4], an[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    float dx = 0.f, dy = 0.f;
                    if (yy > 0 && yy < a.R - 1 && x + k > 0 && x + k < a.C - 1) {
                        dx = __fsub_rn(ctr[k + 1], ctr[k - 1]);
                        dy = __fsub_rn(ctr[k - LIN_W], ctr[k + LIN_W]);
                    }
                    fast_grad(dx, dy, mg[k], an[k]);
                }
                if (vec) {
                    *reinterpret_cast<float4*>(a.mag + at) = make_float4(mg[0], mg[1], mg[2], mg[3]);
                    *reinterpret_cast<float4*>(a.ang + at) = make_float4(an[0], an[1], an[2], an[3]);
                } else {
                    for (int k = 0; k < 4 && x + k < a.C; ++k) {
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
int32_t launch_layer_ly(const LayerArgs& a, cudaStream_t s) {
    static bool attr[64] = {};
    int dev = 0;
    FSB_CUDA(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        FSB_CUDA(cudaFuncSetAttribute(k_layer<TS, r, BASE, LY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      layer_smem<r, LY>()));
        attr[dev] = true;
    }
    dim3 grid((a.C + LX - 1) / LX, (a.R + LY - 1) / LY);
    k_layer<TS, r, BASE, LY><<<grid, LNT, layer_smem<r, LY>(), s>>>(a);
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

}  // namespace

int32_t launch_octave_fused(const float* L0, int R, int C, float* dog, float* mag, float* ang, float* down,
                            int down_cols, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        FSB_CUDA(cudaFuncSetAttribute(k_octave, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
        FSB_CUDA(cudaFuncSetAttribute(k_octave, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        attr = true;
    }
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
                          float* down, int down_cols, int variant, cudaStream_t s) {
    LayerArgs a{};
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
