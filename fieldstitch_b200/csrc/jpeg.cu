// JPEG decoding of the feature pre-step (features.decode / prepare, app/planesite/features.py:18-71)
// on the device through nvJPEG (a library call, loaded with dlopen on first use so that the library
// itself loads where nvJPEG is absent; the decode entries then report it):
//   * the luma plane of the JPEG (what a grayscale read of a colour JPEG yields) at full size;
//   * reduce 2, 4, 8 (the reference's reduced-size reads): each output pixel is the rounded mean of
//     its reduce x reduce block (sizes rounded up, edge blocks clipped). OpenCV's reduced reads scale
//     inside libjpeg's inverse DCT instead, so reduced images agree with OpenCV's approximately
//     (the tests state the bound), full-size ones to the IDCT's rounding.
#include <dlfcn.h>

#include <mutex>
#include <nvjpeg.h>

#include "fsb_internal.cuh"

namespace fsb {
namespace {

struct Nvjpeg {
    bool tried = false, ok = false;
    nvjpegStatus_t (*create_simple)(nvjpegHandle_t*) = nullptr;
    nvjpegStatus_t (*destroy)(nvjpegHandle_t) = nullptr;
    nvjpegStatus_t (*state_create)(nvjpegHandle_t, nvjpegJpegState_t*) = nullptr;
    nvjpegStatus_t (*state_destroy)(nvjpegJpegState_t) = nullptr;
    nvjpegStatus_t (*info)(nvjpegHandle_t, const unsigned char*, size_t, int*, nvjpegChromaSubsampling_t*, int*,
                           int*) = nullptr;
    nvjpegStatus_t (*decode)(nvjpegHandle_t, nvjpegJpegState_t, const unsigned char*, size_t, nvjpegOutputFormat_t,
                             nvjpegImage_t*, cudaStream_t) = nullptr;
};

Nvjpeg& nvj() {
    static Nvjpeg n;
    static std::mutex m;
    std::lock_guard<std::mutex> lk(m);
    if (n.tried) return n;
    n.tried = true;
    void* h = nullptr;
    for (const char* name : {"libnvjpeg.so.12", "libnvjpeg.so", "/usr/local/cuda/lib64/libnvjpeg.so.12"})
        if ((h = dlopen(name, RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) return n;
    n.create_simple = reinterpret_cast<decltype(n.create_simple)>(dlsym(h, "nvjpegCreateSimple"));
    n.destroy = reinterpret_cast<decltype(n.destroy)>(dlsym(h, "nvjpegDestroy"));
    n.state_create = reinterpret_cast<decltype(n.state_create)>(dlsym(h, "nvjpegJpegStateCreate"));
    n.state_destroy = reinterpret_cast<decltype(n.state_destroy)>(dlsym(h, "nvjpegJpegStateDestroy"));
    n.info = reinterpret_cast<decltype(n.info)>(dlsym(h, "nvjpegGetImageInfo"));
    n.decode = reinterpret_cast<decltype(n.decode)>(dlsym(h, "nvjpegDecode"));
    n.ok = n.create_simple && n.destroy && n.state_create && n.state_destroy && n.info && n.decode;
    return n;
}

// rounded mean of the r x r block (clipped at the image edge) of the full-size plane
__global__ void k_block_mean(const uint8_t* __restrict__ src, int h, int w, int pitch, int r, uint8_t* __restrict__ dst,
                             int oh, int ow, int out_pitch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= ow || y >= oh) return;
    const int x0 = x * r, y0 = y * r, x1 = min(x0 + r, w), y1 = min(y0 + r, h);
    int sum = 0;
    for (int yy = y0; yy < y1; ++yy)
        for (int xx = x0; xx < x1; ++xx) sum += src[(size_t)yy * pitch + xx];
    const int n = (x1 - x0) * (y1 - y0);
    dst[(size_t)y * out_pitch + x] = (uint8_t)((sum + n / 2) / n);
}

}  // namespace

int32_t jpeg_release(fsb_ctx* ctx) {
    Nvjpeg& n = nvj();
    if (n.ok) {
        if (ctx->jpeg_state) n.state_destroy(static_cast<nvjpegJpegState_t>(ctx->jpeg_state));
        if (ctx->jpeg_handle) n.destroy(static_cast<nvjpegHandle_t>(ctx->jpeg_handle));
    }
    ctx->jpeg_state = ctx->jpeg_handle = nullptr;
    return FSB_OK;
}

// Decodes the luma plane of a JPEG held in host memory, reduced by `reduce` (1, 2, 4, 8), into
// d_out (capacity out_cap bytes, row pitch = the output width); *h, *w receive the output size.
int32_t run_jpeg_gray(fsb_ctx* ctx, const uint8_t* data, size_t len, int reduce, uint8_t* d_out, size_t out_cap,
                      int* h, int* w) {
    Nvjpeg& n = nvj();
    if (!n.ok) {
        set_error("nvJPEG (libnvjpeg.so.12) could not be loaded");
        return FSB_ERR_UNSUPPORTED;
    }
    cudaStream_t s = ctx->stream;
    if (!ctx->jpeg_handle) {
        nvjpegHandle_t jh;
        nvjpegJpegState_t js;
        if (n.create_simple(&jh) != NVJPEG_STATUS_SUCCESS) {
            set_error("nvjpegCreateSimple failed");
            return FSB_ERR_CUDA;
        }
        if (n.state_create(jh, &js) != NVJPEG_STATUS_SUCCESS) {
            n.destroy(jh);
            set_error("nvjpegJpegStateCreate failed");
            return FSB_ERR_CUDA;
        }
        ctx->jpeg_handle = jh;
        ctx->jpeg_state = js;
    }
    int nc = 0, ws[NVJPEG_MAX_COMPONENT] = {}, hs[NVJPEG_MAX_COMPONENT] = {};
    nvjpegChromaSubsampling_t sub;
    if (n.info(static_cast<nvjpegHandle_t>(ctx->jpeg_handle), data, len, &nc, &sub, ws, hs) != NVJPEG_STATUS_SUCCESS ||
        ws[0] <= 0 || hs[0] <= 0) {
        set_error("not a decodable JPEG");
        return FSB_ERR_ARG;
    }
    const int W = ws[0], H = hs[0];
    const int ow = (W + reduce - 1) / reduce, oh = (H + reduce - 1) / reduce;
    *w = ow;
    *h = oh;
    if ((size_t)ow * oh > out_cap) {
        set_error("output buffer holds %zu bytes, the image needs %d x %d", out_cap, ow, oh);
        return FSB_ERR_ARG;
    }
    uint8_t* full = d_out;
    if (reduce > 1) {
        FSB_TRY(ctx->s_u8b.ensure((size_t)W * H + 256));
        full = ctx->s_u8b.as<uint8_t>();
    }
    nvjpegImage_t img{};
    img.channel[0] = full;
    img.pitch[0] = (size_t)W;
    if (n.decode(static_cast<nvjpegHandle_t>(ctx->jpeg_handle), static_cast<nvjpegJpegState_t>(ctx->jpeg_state), data,
                 len, NVJPEG_OUTPUT_Y, &img, s) != NVJPEG_STATUS_SUCCESS) {
        set_error("nvjpegDecode failed");
        return FSB_ERR_CUDA;
    }
    if (reduce > 1) {
        k_block_mean<<<dim3((ow + 127) / 128, oh), 128, 0, s>>>(full, H, W, W, reduce, d_out, oh, ow, ow);
        note_launch();
    }
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

}  // namespace fsb
