// Contrast equalisation of the feature pre-step (features.prepare, app/planesite/features.py:60-71):
// CLAHE with OpenCV's definition (cv2.createCLAHE(clipLimit, tileGridSize).apply on uint8), as
// restated in oracle/clahe_ref.py and checked there bit for bit against OpenCV:
//   * the image is split into tx x ty tiles; when either side is not a multiple of its tile count,
//     both sides are extended at the far edge by reflect-101 (a divisible side by a whole tile);
//   * per tile: 256-bin histogram, clipped at max(int(clip * area / 256), 1); the clipped excess is
//     spread evenly, the remainder one count every max(256 / remainder, 1) bins from bin 0; the LUT
//     is round-half-even(cumulative count * (255 / area)) in float32;
//   * per pixel: bilinear blend of the four nearest tiles' LUT values at tile-centre coordinates
//     (x / tile_w - 0.5), float32 operations in a fixed order without fused multiply-add, rounded
//     half to even.
//   k_clahe_lut    one CTA per tile: shared-memory histogram over the (virtually extended) tile,
//                  clip / redistribute / LUT by one warp.
//   k_clahe_apply  one thread per pixel (4 rows per thread), LUTs staged in shared memory.
#include "fsb_internal.cuh"

namespace fsb {
namespace {

// reflect-101 index (repeated reflection: a side of a few pixels may be extended by a whole tile)
__device__ __forceinline__ int refl101(int p, int n) {
    if (n == 1) return 0;
    while (p < 0 || p >= n) p = p < 0 ? -p : 2 * n - 2 - p;
    return p;
}

__global__ void __launch_bounds__(512) k_clahe_lut(const uint8_t* __restrict__ img, int h, int w, int stride, int tw,
                                                   int th, int tiles_x, int climit, float lut_scale,
                                                   uint8_t* __restrict__ lut) {
    __shared__ int hist[256];
    const int tile = blockIdx.x, bx = tile % tiles_x, by = tile / tiles_x;
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const int x0 = bx * tw, y0 = by * th;
    for (int k = threadIdx.x; k < tw * th; k += blockDim.x) {
        const int y = y0 + k / tw, x = x0 + k % tw;
        atomicAdd(&hist[img[(size_t)refl101(y, h) * stride + refl101(x, w)]], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int v[8], excess = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            v[q] = hist[lane * 8 + q];
            if (v[q] > climit) {
                excess += v[q] - climit;
                v[q] = climit;
            }
        }
#pragma unroll
        for (int sh = 16; sh; sh >>= 1) excess += __shfl_xor_sync(0xffffffffu, excess, sh);
        const int batch = excess / 256;
        const int resid = excess - batch * 256;
        const int step = resid ? max(256 / resid, 1) : 256;
        // bins step * m (m < resid, below 256) take one more count
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int b = lane * 8 + q;
            v[q] += batch + ((resid && b % step == 0 && b / step < resid) ? 1 : 0);
        }
        // inclusive prefix over the 256 bins (8 per lane, lanes in order)
        int run = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) run += v[q];
        int incl = run;
#pragma unroll
        for (int sh = 1; sh < 32; sh <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, sh);
            if (lane >= sh) incl += t;
        }
        int sum = incl - run;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            sum += v[q];
            const int r = __float2int_rn(__fmul_rn((float)sum, lut_scale));
            lut[(size_t)tile * 256 + lane * 8 + q] = (uint8_t)min(max(r, 0), 255);
        }
    }
}

__global__ void __launch_bounds__(256) k_clahe_apply(const uint8_t* __restrict__ img, int h, int w, int stride,
                                                     const uint8_t* __restrict__ lut, int tiles_x, int tiles_y,
                                                     float inv_tw, float inv_th, uint8_t* __restrict__ out,
                                                     int out_stride) {
    extern __shared__ uint8_t s_lut[];
    const int n_lut = tiles_x * tiles_y * 256;
    for (int i = threadIdx.x * 4; i < n_lut; i += blockDim.x * 4)
        *reinterpret_cast<uint32_t*>(s_lut + i) = *reinterpret_cast<const uint32_t*>(lut + i);
    __syncthreads();
    const int x = blockIdx.x * 64 + (threadIdx.x & 63);
    const int y0 = blockIdx.y * 16 + (threadIdx.x >> 6) * 4;
    if (x >= w) return;
    const float txf = __fsub_rn(__fmul_rn((float)x, inv_tw), 0.5f);
    const int tx1r = (int)floorf(txf);
    const float xa = __fsub_rn(txf, (float)tx1r), xa1 = __fsub_rn(1.0f, xa);
    const int tx1 = max(tx1r, 0), tx2 = min(tx1r + 1, tiles_x - 1);
    for (int y = y0; y < min(y0 + 4, h); ++y) {
        const float tyf = __fsub_rn(__fmul_rn((float)y, inv_th), 0.5f);
        const int ty1r = (int)floorf(tyf);
        const float ya = __fsub_rn(tyf, (float)ty1r), ya1 = __fsub_rn(1.0f, ya);
        const int ty1 = max(ty1r, 0), ty2 = min(ty1r + 1, tiles_y - 1);
        const int v = img[(size_t)y * stride + x];
        const uint8_t* l1 = s_lut + (ty1 * tiles_x) * 256 + v;
        const uint8_t* l2 = s_lut + (ty2 * tiles_x) * 256 + v;
        const float a = l1[tx1 * 256], b = l1[tx2 * 256], c = l2[tx1 * 256], d = l2[tx2 * 256];
        const float r1 = __fadd_rn(__fmul_rn(a, xa1), __fmul_rn(b, xa));
        const float r2 = __fadd_rn(__fmul_rn(c, xa1), __fmul_rn(d, xa));
        const float res = __fadd_rn(__fmul_rn(r1, ya1), __fmul_rn(r2, ya));
        out[(size_t)y * out_stride + x] = (uint8_t)min(max(__float2int_rn(res), 0), 255);
    }
}

}  // namespace

int32_t run_clahe(const uint8_t* d_img, int h, int w, int stride, double clip, int tiles_x, int tiles_y,
                  uint8_t* d_lut, uint8_t* d_out, int out_stride, cudaStream_t s) {
    const bool even = w % tiles_x == 0 && h % tiles_y == 0;
    const int ew = even ? w : w + tiles_x - w % tiles_x;   // OpenCV extends both sides when either is ragged
    const int eh = even ? h : h + tiles_y - h % tiles_y;
    const int tw = ew / tiles_x, th = eh / tiles_y, area = tw * th;
    if (tw < 1 || th < 1) {
        set_error("image %dx%d too small for %dx%d tiles", w, h, tiles_x, tiles_y);
        return FSB_ERR_ARG;
    }
    int climit = (int)(clip * area / 256.0);
    if (climit < 1) climit = 1;
    if (clip <= 0.0) climit = 1 << 30;   // no clipping
    const float lut_scale = 255.0f / (float)area;
    k_clahe_lut<<<tiles_x * tiles_y, 512, 0, s>>>(d_img, h, w, stride, tw, th, tiles_x, climit, lut_scale, d_lut);
    const float inv_tw = 1.0f / (float)tw, inv_th = 1.0f / (float)th;
    const dim3 grid((w + 63) / 64, (h + 15) / 16);
    const int smem = tiles_x * tiles_y * 256;
    if (smem > 48 * 1024) {
        static std::atomic<int> attr[64];
        FSB_TRY(smem_attr((const void*)k_clahe_apply, 64 * 1024, attr));
    }
    k_clahe_apply<<<grid, 256, smem, s>>>(d_img, h, w, stride, d_lut, tiles_x, tiles_y, inv_tw, inv_th, d_out,
                                          out_stride);
    note_launch(2);
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

}  // namespace fsb
