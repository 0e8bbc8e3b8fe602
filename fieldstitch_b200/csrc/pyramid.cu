// Gaussian / DoG pyramid with fused DoG, gradient and downsample epilogues.
//
// Reference: app/planesite/gsift.py:52-72 (taps), 85-102 (blur, 2x upsample), 158-179 (pyramid),
// 227-267 (DoG atlas, gradient magnitude / angle of gauss layers 1..3).
//
// Layout in HBM (per image):
//   DoG atlas   float32 [octave][layer 0..4][R][C], octave o at Geometry::dog_off[o]
//   MAG / ANG   float32 [octave][layer 1..3][R][C], octave o at Geometry::grad_off[o]
//   planes      three octave-0-sized float32 scratch planes for gauss layers in flight
//
// One launch per (octave, layer): a 64x32 output tile is staged through shared memory with its
// mirrored halo, blurred vertically then horizontally (the reference's axis order, with the
// intermediate rounded to float32), and the epilogue writes L_i, the DoG L_i - L_{i-1}, the
// gradient of L_{i-1} (layers 1..3) and the [::2, ::2] downsample of L_3 (next octave's base)
// from the tile already in shared memory, so none of those needs a separate pass over HBM.
#include <cmath>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "fsb_internal.cuh"

namespace fsb {

// Normalised Gaussian taps of gsift._gauss_kernel for the base sigma sqrt(1.6^2 - 1) and the five
// layer increments (float32 values, written as hex literals so they are exact).
// Tap set 0: base (11 taps); 1..5: layers 1..5 (11, 13, 17, 21, 27 taps).
static const int kTapCount[6] = {11, 11, 13, 17, 21, 27};
static const float kTaps[6][27] = {
    {0x1.bbb27cp-14f, 0x1.f04b54p-10f, 0x1.2469f0p-6f, 0x1.6b036ep-4f, 0x1.dac530p-3f, 0x1.4713cep-2f,
     0x1.dac530p-3f, 0x1.6b036ep-4f, 0x1.2469f0p-6f, 0x1.f04b54p-10f, 0x1.bbb27cp-14f},
    {0x1.4edfacp-14f, 0x1.a1407ap-10f, 0x1.0b5ddep-6f, 0x1.606d0ep-4f, 0x1.ddcdfcp-3f, 0x1.4d2364p-2f,
     0x1.ddcdfcp-3f, 0x1.606d0ep-4f, 0x1.0b5ddep-6f, 0x1.a1407ap-10f, 0x1.4edfacp-14f},
    {0x1.1f90cap-13f, 0x1.680080p-10f, 0x1.287054p-7f, 0x1.411cd4p-5f, 0x1.c995cap-4f, 0x1.ace486p-3f,
     0x1.086a76p-2f, 0x1.ace486p-3f, 0x1.c995cap-4f, 0x1.411cd4p-5f, 0x1.287054p-7f, 0x1.680080p-10f,
     0x1.1f90cap-13f},
    {0x1.719152p-15f, 0x1.4e5a92p-12f, 0x1.d0a8dcp-10f, 0x1.eff6b8p-8f, 0x1.9695c0p-6f, 0x1.ffffbap-5f,
     0x1.ef3104p-4f, 0x1.6fd80cp-3f, 0x1.a3bafcp-3f, 0x1.6fd80cp-3f, 0x1.ef3104p-4f, 0x1.ffffbap-5f,
     0x1.9695c0p-6f, 0x1.eff6b8p-8f, 0x1.d0a8dcp-10f, 0x1.4e5a92p-12f, 0x1.719152p-15f},
    {0x1.4ee0b6p-15f, 0x1.9634a6p-13f, 0x1.a141c6p-11f, 0x1.6af5d4p-9f, 0x1.0b5eb2p-7f, 0x1.4d9348p-6f,
     0x1.606e26p-5f, 0x1.3b51b8p-4f, 0x1.ddcf78p-4f, 0x1.3291c0p-3f, 0x1.4d246cp-3f, 0x1.3291c0p-3f,
     0x1.ddcf78p-4f, 0x1.3b51b8p-4f, 0x1.606e26p-5f, 0x1.4d9348p-6f, 0x1.0b5eb2p-7f, 0x1.6af5d4p-9f,
     0x1.a141c6p-11f, 0x1.9634a6p-13f, 0x1.4ee0b6p-15f},
    {0x1.36a04cp-16f, 0x1.1f903ep-14f, 0x1.df7c20p-13f, 0x1.67ffd2p-11f, 0x1.e6d384p-10f, 0x1.286fc4p-8f,
     0x1.451d18p-7f, 0x1.411c3ap-6f, 0x1.1d9ebap-5f, 0x1.c994eep-5f, 0x1.4a176ap-4f, 0x1.ace3b6p-4f,
     0x1.f5d90ep-4f, 0x1.0869f6p-3f, 0x1.f5d90ep-4f, 0x1.ace3b6p-4f, 0x1.4a176ap-4f, 0x1.c994eep-5f,
     0x1.1d9ebap-5f, 0x1.411c3ap-6f, 0x1.451d18p-7f, 0x1.286fc4p-8f, 0x1.e6d384p-10f, 0x1.67ffd2p-11f,
     0x1.df7c20p-13f, 0x1.1f903ep-14f, 0x1.36a04cp-16f},
};

__constant__ float c_taps[6][28];
__constant__ double c_taps_d[6][28];

int32_t upload_taps() {
    float f[6][28] = {};
    double d[6][28] = {};
    for (int s = 0; s < 6; ++s)
        for (int j = 0; j < kTapCount[s]; ++j) {
            f[s][j] = kTaps[s][j];
            d[s][j] = (double)kTaps[s][j];
        }
    FSB_CUDA(cudaMemcpyToSymbol(c_taps, f, sizeof(f)));
    FSB_CUDA(cudaMemcpyToSymbol(c_taps_d, d, sizeof(d)));
    return upload_octave_taps(&kTaps[0][0], 27, kTapCount);
}

Geometry make_geometry(int h, int w) {
    Geometry g{};
    g.h = h;
    g.w = w;
    int mn = h < w ? h : w;
    int budget = (int)std::nearbyint(std::log2((double)mn) - 2.0) + 1;   // gsift.py:167
    if (budget < 1) budget = 1;
    int R = 2 * h, C = 2 * w;
    long long dog = 0, grad = 0;
    g.n_oct = 0;
    for (int o = 0; o < budget && o < MAXO; ++o) {
        if ((R < C ? R : C) < 2 * BORDER + 4) break;                         // gsift.py:171
        g.R[o] = R;
        g.C[o] = C;
        g.dog_off[o] = dog;
        g.grad_off[o] = grad;
        dog += 5LL * R * C;
        grad += 3LL * R * C;
        g.n_oct = o + 1;
        R = (R + 1) / 2;   // layers[3][::2, ::2]
        C = (C + 1) / 2;
    }
    g.dog_off[g.n_oct] = dog;
    g.grad_off[g.n_oct] = grad;
    return g;
}

namespace {

constexpr int TX = 64, TY = 32, NT = 256;
// degrees per radian as NumPy's float32 rad2deg computes it: float(180) / float(pi)
constexpr float kRad2Deg = 0x1.ca5dc0p+5f;

__device__ __forceinline__ int mirror(int p, int n) {
    if (n == 1) return 0;
    while (p < 0 || p >= n) p = p < 0 ? -p : 2 * n - 2 - p;
    return p;
}

struct BlurArgs {
    const float* src;          // previous gauss layer (layer launches)
    const uint8_t* img;        // uint8 input (base launch)
    int img_stride, ih, iw;
    int rows, cols;
    float* dst;                // this layer, or null
    float* dog;                // DoG plane (this - previous), or null
    float* mag;                // gradient magnitude of the previous layer, or null
    float* ang;                // gradient angle of the previous layer (degrees), or null
    float* down;               // previous layer [::2, ::2], or null
    int down_cols;
};

// Bilinear 2x upsample sample of the uint8 image at (Y, X) of the 2h x 2w grid, float32 with the
// reference's rounding: a = u8 * float(1/255); t = 0.75 a[iy] + 0.25 a[ny] (rows first), then the
// same along columns (gsift.py:90-102, 160).
__device__ __forceinline__ float up2_sample(const BlurArgs& a, int Y, int X) {
    const float s = (float)(1.0 / 255.0);
    const int iy = Y >> 1, ix = X >> 1;
    const int ny = (Y & 1) ? min(iy + 1, a.ih - 1) : max(iy - 1, 0);
    const int nx = (X & 1) ? min(ix + 1, a.iw - 1) : max(ix - 1, 0);
    const uint8_t* r0 = a.img + (size_t)iy * a.img_stride;
    const uint8_t* r1 = a.img + (size_t)ny * a.img_stride;
    const float p00 = __fmul_rn((float)r0[ix], s), p10 = __fmul_rn((float)r1[ix], s);
    const float p01 = __fmul_rn((float)r0[nx], s), p11 = __fmul_rn((float)r1[nx], s);
    const float vc = __fadd_rn(__fmul_rn(0.75f, p00), __fmul_rn(0.25f, p10));
    const float vn = __fadd_rn(__fmul_rn(0.75f, p01), __fmul_rn(0.25f, p11));
    return __fadd_rn(__fmul_rn(0.75f, vc), __fmul_rn(0.25f, vn));
}

// Correlation of 2*RAD+1 samples p[0], p[stride], ... with tap set TS.
// EXACT: float64, centre term first, then symmetric pairs from the outside in, each product and
// sum rounded separately, one final rounding to float32 (scipy.ndimage.correlate1d's order).
template <int TS, int RAD, bool EXACT>
__device__ __forceinline__ float conv(const float* p, int stride) {
    if (EXACT) {
        double s = __dmul_rn((double)p[RAD * stride], c_taps_d[TS][RAD]);
#pragma unroll
        for (int j = RAD; j >= 1; --j)
            s = __dadd_rn(s, __dmul_rn(__dadd_rn((double)p[(RAD - j) * stride], (double)p[(RAD + j) * stride]),
                                       c_taps_d[TS][RAD - j]));
        return (float)s;
    } else {
        float s = 0.f;
#pragma unroll
        for (int j = 0; j <= 2 * RAD; ++j) s = fmaf(c_taps[TS][j], p[j * stride], s);
        return s;
    }
}

template <int TS, int RAD, bool EXACT, bool BASE>
__global__ void __launch_bounds__(NT) k_blur(BlurArgs a) {
    constexpr int IW = TX + 2 * RAD, IH = TY + 2 * RAD, SW = IW + 1;
    __shared__ float s_in[IH * SW];
    __shared__ float s_mid[TY * SW];
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    for (int i = threadIdx.x; i < IH * IW; i += NT) {
        const int yy = i / IW, xx = i - yy * IW;
        const int gy = mirror(y0 + yy - RAD, a.rows), gx = mirror(x0 + xx - RAD, a.cols);
        s_in[yy * SW + xx] = BASE ? up2_sample(a, gy, gx) : __ldg(a.src + (size_t)gy * a.cols + gx);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < TY * IW; i += NT) {
        const int yy = i / IW, xx = i - yy * IW;
        s_mid[yy * SW + xx] = conv<TS, RAD, EXACT>(&s_in[yy * SW + xx], SW);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < TY * TX; i += NT) {
        const int yy = i / TX, xx = i - yy * TX;
        const int gy = y0 + yy, gx = x0 + xx;
        if (gy >= a.rows || gx >= a.cols) continue;
        const float v = conv<TS, RAD, EXACT>(&s_mid[yy * SW + xx], 1);
        const size_t at = (size_t)gy * a.cols + gx;
        if (a.dst) a.dst[at] = v;
        const float* c = &s_in[(yy + RAD) * SW + xx + RAD];   // previous layer at (gy, gx)
        if (a.dog) a.dog[at] = __fsub_rn(v, c[0]);
        if (a.mag) {
            float dx = 0.f, dy = 0.f;
            if (gy > 0 && gy < a.rows - 1 && gx > 0 && gx < a.cols - 1) {
                dx = __fsub_rn(c[1], c[-1]);
                dy = __fsub_rn(c[-SW], c[SW]);
            }
            a.mag[at] = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
            float an = __fmul_rn(atan2f(dy, dx), kRad2Deg);
            a.ang[at] = an < 0.f ? __fadd_rn(an, 360.f) : an;
        }
        if (a.down && !(gy & 1) && !(gx & 1)) a.down[(size_t)(gy >> 1) * a.down_cols + (gx >> 1)] = c[0];
    }
}

template <int TS, int RAD, bool BASE>
void launch(bool exact, const BlurArgs& a, cudaStream_t s) {
    dim3 grid((a.cols + TX - 1) / TX, (a.rows + TY - 1) / TY);
    if (exact)
        k_blur<TS, RAD, true, BASE><<<grid, NT, 0, s>>>(a);
    else
        k_blur<TS, RAD, false, BASE><<<grid, NT, 0, s>>>(a);
    note_launch();
}

}  // namespace

// Float32 octave engines: the fused layer groups (k_group, octave.cu) by default; the tiled
// per-layer kernels (k_layer) with FSB_PYRAMID=layer; the fused streaming kernel (k_octave) for
// octaves at least kFusedMinCols wide with FSB_PYRAMID=fused.
static const int kFusedMinCols = 2000;

namespace {
struct LayerCall {
    int layer;
    const float* src;
    int R, C;
    float *dst, *dog, *mag, *ang, *down;
    int dc;
    int* err;   // error word of the tile copies' bounded waits
    cudaStream_t s;
};
int32_t run_layer_call(void* p, int v) {
    const LayerCall* c = static_cast<const LayerCall*>(p);
    return launch_layer_fast(c->layer, c->src, c->R, c->C, c->dst, c->dog, c->mag, c->ang, c->down, c->dc, v, c->err,
                             c->s);
}
struct BaseCall {
    const uint8_t* img;
    int stride, h, w;
    float* dst;
    cudaStream_t s;
};
int32_t run_base_call(void* p, int v) {
    const BaseCall* c = static_cast<const BaseCall*>(p);
    return launch_base_fast(c->img, c->stride, c->h, c->w, c->dst, v == 1 ? 2 : 0, c->s);   // heights 32, 64
}
// one tuned per-layer launch: the tile height is chosen per (layer, octave size);
// FSB_LAYER_VARIANT=k (read on every call) runs variant k everywhere instead, so each variant can
// be checked against the others
int32_t tuned_layer(int layer, const float* src, int R, int C, float* dst, float* dog, float* mag, float* ang,
                    float* down, int dc, int* err, cudaStream_t s) {
    LayerCall c{layer, src, R, C, dst, dog, mag, ang, down, dc, err, s};
    if (const char* fv = std::getenv("FSB_LAYER_VARIANT")) {
        const int v = std::atoi(fv);
        if (v >= 0 && v < layer_tile_variants()) return run_layer_call(&c, v);
    }
    char key[64];
    std::snprintf(key, sizeof(key), "k_layer%d_%dx%d", layer, R, C);
    int v = 0;
    return autotune(key, layer_tile_variants(), run_layer_call, &c, s, &v);
}
}  // namespace

// FSB_PYRAMID selects the float32 octave engine (all are bit-identical): unset, the autotuner picks
// per octave size between the per-layer kernels (variant 0, also with FSB_AUTOTUNE=0) and the
// fused layer groups (variant 1); "layer" / "group" force one; "fused" takes the streaming
// kernel for octaves at least kFusedMinCols wide. Read on every call.
enum class Engine { Auto, Group, Layer, Fused, Strip };
static Engine pyramid_engine() {
    const char* e = std::getenv("FSB_PYRAMID");
    if (e && std::strcmp(e, "layer") == 0) return Engine::Layer;
    if (e && std::strcmp(e, "group") == 0) return Engine::Group;
    if (e && std::strcmp(e, "strip") == 0) return Engine::Strip;
    if (e && std::strcmp(e, "fused") == 0) return Engine::Fused;
    return Engine::Auto;
}

namespace {
// One float32 octave from its base `src` (not written): DoG, gradient atlases, L3[::2, ::2] to
// `down`; x, y are scratch planes. Both variants leave the same outputs, so the tuner may run
// either any number of times.
struct OctaveCall {
    const float* src;
    int R, C;
    float *x, *y, *dog, *mag, *ang, *down;
    int dc;
    cudaStream_t s;
    // with a side stream, the octave's tail (layer 5, or the L4-L5 group) runs there after `fork`,
    // since the next octave needs only L3's downsample; `join` marks its end
    cudaStream_t side;
    cudaEvent_t fork, join;
    int* err;   // error word of the strip engine's bounded waits
};
int32_t run_octave_call(void* p, int v) {
    const OctaveCall* c = static_cast<const OctaveCall*>(p);
    const long long RC = (long long)c->R * c->C;
    cudaStream_t ts = c->s;   // stream of the tail
    auto fork = [&]() -> int32_t {
        if (!c->side) return FSB_OK;
        FSB_CUDA(cudaEventRecord(c->fork, c->s));
        FSB_CUDA(cudaStreamWaitEvent(c->side, c->fork, 0));
        ts = c->side;
        return FSB_OK;
    };
    if (v == 2) {
        // the whole octave in one launch: no tail to move to the side stream
        FSB_TRY(launch_octave_strip(c->src, c->R, c->C, c->dog, c->mag, c->ang, c->down, c->dc, c->err, c->s));
        if (c->side) FSB_CUDA(cudaEventRecord(c->join, c->s));
        return FSB_OK;
    }
    if (v == 1) {
        FSB_TRY(launch_group_lower(c->src, c->R, c->C, c->dog, c->mag, c->ang, c->x, c->down, c->dc, c->s));
        FSB_TRY(fork());
        FSB_TRY(launch_group_upper(c->x, c->R, c->C, c->dog + 3 * RC, ts));
    } else {
        FSB_TRY(tuned_layer(1, c->src, c->R, c->C, c->x, c->dog, nullptr, nullptr, nullptr, 0, c->err, c->s));
        FSB_TRY(tuned_layer(2, c->x, c->R, c->C, c->y, c->dog + RC, c->mag, c->ang, nullptr, 0, c->err, c->s));
        FSB_TRY(tuned_layer(3, c->y, c->R, c->C, c->x, c->dog + 2 * RC, c->mag + RC, c->ang + RC, nullptr, 0, c->err,
                            c->s));
        FSB_TRY(tuned_layer(4, c->x, c->R, c->C, c->y, c->dog + 3 * RC, c->mag + 2 * RC, c->ang + 2 * RC, c->down,
                            c->dc, c->err, c->s));
        FSB_TRY(fork());
        FSB_TRY(tuned_layer(5, c->y, c->R, c->C, nullptr, c->dog + 4 * RC, nullptr, nullptr, nullptr, 0, c->err, ts));
    }
    if (c->side) FSB_CUDA(cudaEventRecord(c->join, c->side));
    return FSB_OK;
}
}  // namespace

int32_t run_pyramid(Workspace& ws, const uint8_t* d_img, int img_stride, bool exact, cudaStream_t s, cudaStream_t side,
                    cudaEvent_t* ev) {
    const Geometry& g = ws.g;
    float* P[3] = {ws.plane[0].as<float>(), ws.plane[1].as<float>(), ws.plane[2].as<float>()};
    int* err = ws.counters.as<int>() + PYR_ERR_WORD;
    FSB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    float* DF = ws.dog.as<float>();
    float* MAG = ws.mag.as<float>();
    float* ANG = ws.ang.as<float>();
    BlurArgs a{};
    a.img = d_img;
    a.img_stride = img_stride;
    a.ih = g.h;
    a.iw = g.w;
    a.rows = g.R[0];
    a.cols = g.C[0];
    a.dst = P[0];
    if (exact) {
        launch<0, 5, true>(exact, a, s);
    } else {
        BaseCall bc{d_img, img_stride, g.h, g.w, P[0], s};
        char key[64];
        std::snprintf(key, sizeof(key), "k_base_%dx%d", g.h, g.w);
        int v = 0;
        FSB_TRY(autotune(key, 2, run_base_call, &bc, s, &v));
    }
    const Engine eng = exact ? Engine::Layer : pyramid_engine();
    if (!exact && eng != Engine::Fused) {
        // octave o reads its base from P[0] (o = 0) or one half of next_base and writes the next
        // base into the other half; two of P[0..2] hold its layers in flight. With a side stream,
        // an octave's tail (reading one of those planes) overlaps the next octave, which then takes
        // the other two planes; before an octave starts, the tail two octaves back has ended, so at
        // most one tail is in flight. While an octave size is being tuned its tail stays on s (the
        // tuner times s only).
        float* NB = ws.next_base.as<float>();
        const long long half = g.n_oct > 1 ? ((long long)g.R[1] * g.C[1] + 63) / 64 * 64 : 0;
        const float* cur = P[0];
        const float* tail_plane = nullptr;    // plane the latest side-stream tail reads
        int prev_tail = -1, last_tail = -1;   // the two latest octaves whose tails ran on the side
        for (int o = 0; o < g.n_oct; ++o) {
            const bool last = o + 1 == g.n_oct;
            // before this octave: every side tail has ended except the previous octave's (the side
            // stream runs its tails in order, so one wait covers the earlier ones)
            const float* busy = nullptr;
            if (last_tail >= 0 && last_tail < o - 1) {
                FSB_CUDA(cudaStreamWaitEvent(s, ev[2 * last_tail + 1], 0));
            } else if (last_tail == o - 1 && last_tail >= 0) {
                busy = tail_plane;
                if (prev_tail >= 0) FSB_CUDA(cudaStreamWaitEvent(s, ev[2 * prev_tail + 1], 0));
            }
            float* pl[2];
            for (int k = 0, n = 0; k < 3 && n < 2; ++k)
                if (P[k] != cur && P[k] != busy) pl[n++] = P[k];
            OctaveCall c{cur, g.R[o], g.C[o], pl[0], pl[1], DF + g.dog_off[o], MAG + g.grad_off[o],
                         ANG + g.grad_off[o], last ? nullptr : NB + (o & 1) * half, last ? 0 : g.C[o + 1], s,
                         nullptr, side ? ev[2 * o] : nullptr, side ? ev[2 * o + 1] : nullptr, err};
            int v = eng == Engine::Group ? 1 : eng == Engine::Strip ? 2 : 0;
            char key[64];
            std::snprintf(key, sizeof(key), "k_octave3_%dx%d", g.R[o], g.C[o]);
            const bool known = eng != Engine::Auto || autotune_cached(key, 3, &v);
            if (known && side && v != 2) c.side = side;
            if (eng == Engine::Auto && !known) {
                FSB_TRY(autotune(key, 3, run_octave_call, &c, s, &v));
            } else {
                FSB_TRY(run_octave_call(&c, v));
            }
            if (c.side) {
                tail_plane = v == 1 ? c.x : c.y;
                prev_tail = last_tail;
                last_tail = o;
            }
            cur = c.down;
        }
        if (last_tail >= 0) FSB_CUDA(cudaStreamWaitEvent(s, ev[2 * last_tail + 1], 0));
        FSB_CUDA(cudaGetLastError());
        return FSB_OK;
    }
    float* cur = P[0];   // base of the current octave
    for (int o = 0; o < g.n_oct; ++o) {
        const long long RC = (long long)g.R[o] * g.C[o];
        float* dog = DF + g.dog_off[o];
        float* mag = MAG + g.grad_off[o];
        float* ang = ANG + g.grad_off[o];
        float* other[2];
        for (int k = 0, n = 0; k < 3; ++k)
            if (P[k] != cur) other[n++] = P[k];
        if (!exact && g.C[o] >= kFusedMinCols) {
            // fused octave: reads cur, writes the next base into another plane
            float* down = o + 1 < g.n_oct ? other[0] : nullptr;
            FSB_TRY(launch_octave_fused(cur, g.R[o], g.C[o], dog, mag, ang, down, o + 1 < g.n_oct ? g.C[o + 1] : 0, s));
            cur = other[0];
            continue;
        }
        if (!exact) {
            const int R = g.R[o], C = g.C[o];
            float* down = o + 1 < g.n_oct ? cur : nullptr;
            const int dc = o + 1 < g.n_oct ? g.C[o + 1] : 0;
            FSB_TRY(tuned_layer(1, cur, R, C, other[0], dog, nullptr, nullptr, nullptr, 0, err, s));
            FSB_TRY(tuned_layer(2, other[0], R, C, other[1], dog + RC, mag, ang, nullptr, 0, err, s));
            FSB_TRY(tuned_layer(3, other[1], R, C, other[0], dog + 2 * RC, mag + RC, ang + RC, nullptr, 0, err, s));
            FSB_TRY(tuned_layer(4, other[0], R, C, other[1], dog + 3 * RC, mag + 2 * RC, ang + 2 * RC, down, dc,
                                err, s));
            FSB_TRY(tuned_layer(5, other[1], R, C, nullptr, dog + 4 * RC, nullptr, nullptr, nullptr, 0, err, s));
            continue;   // the next base is in `cur` (the dead L0 plane)
        }
        BlurArgs b{};
        b.rows = g.R[o];
        b.cols = g.C[o];
        // layer 1: L0 -> X, DoG 0
        b.src = cur; b.dst = other[0]; b.dog = dog;
        launch<1, 5, false>(exact, b, s);
        // layer 2: L1 (X) -> Y, DoG 1, gradient of L1
        b.src = other[0]; b.dst = other[1]; b.dog = dog + RC; b.mag = mag; b.ang = ang;
        launch<2, 6, false>(exact, b, s);
        // layer 3: L2 (Y) -> X, DoG 2, gradient of L2
        b.src = other[1]; b.dst = other[0]; b.dog = dog + 2 * RC; b.mag = mag + RC; b.ang = ang + RC;
        launch<3, 8, false>(exact, b, s);
        // layer 4: L3 (X) -> Y, DoG 3, gradient of L3, L3[::2, ::2] -> the (dead) base plane
        b.src = other[0]; b.dst = other[1]; b.dog = dog + 3 * RC; b.mag = mag + 2 * RC; b.ang = ang + 2 * RC;
        if (o + 1 < g.n_oct) { b.down = cur; b.down_cols = g.C[o + 1]; }
        launch<4, 10, false>(exact, b, s);
        // layer 5: L4 (Y) -> DoG 4 only
        b.src = other[1]; b.dst = nullptr; b.dog = dog + 4 * RC; b.mag = nullptr; b.ang = nullptr; b.down = nullptr;
        launch<5, 13, false>(exact, b, s);
    }
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

}  // namespace fsb
