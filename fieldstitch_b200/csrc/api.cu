// C ABI of libfsb200: contexts, detect states, and the host-memory entry points declared in
// include/fsb200.h.
#include <time.h>

#include <cmath>
#include <cstring>
#include <atomic>
#include <string>

#include "fsb_internal.cuh"

namespace fsb {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

int32_t DevBuf::ensure(size_t n) {
    if (n <= bytes && p) return FSB_OK;
    // geometric growth: buffers sized by data (keypoint and match counts) settle after a few calls;
    // each regrowth frees, and cudaFree waits for the whole device (every stream of every context)
    size_t want = n < 256 ? 256 : n;
    if (p && want < bytes + bytes / 2) want = bytes + bytes / 2;
    if (want > ((size_t)1 << 20)) want = (want + ((size_t)1 << 20) - 1) & ~(((size_t)1 << 20) - 1);
    release();
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        bytes = 0;
        cudaGetLastError();
        set_error("cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
        return FSB_ERR_OOM;
    }
    bytes = want;
    return FSB_OK;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

size_t Workspace::bytes() const {
    size_t t = dog.bytes + mag.bytes + ang.bytes + img.bytes + cand.bytes + refined.bytes + oriented.bytes +
               keys_a.bytes + keys_b.bytes + vals_a.bytes + vals_b.bytes + sort_tmp.bytes + counters.bytes +
               kx.bytes + ky.bytes + ksize.bytes + kangle.bytes + kresp.bytes + koct.bytes + klayer.bytes +
               spread.bytes + take.bytes;
    for (const auto& b : plane) t += b.bytes;
    return t + next_base.bytes;
}

void Workspace::release() {
    DevBuf* all[] = {&dog, &mag, &ang, &img, &cand, &refined, &oriented, &keys_a, &keys_b, &vals_a, &vals_b,
                     &sort_tmp, &counters, &kx, &ky, &ksize, &kangle, &kresp, &koct, &klayer,
                     &plane[0], &plane[1], &plane[2], &next_base, &spread, &take};
    for (DevBuf* b : all) b->release();
}

// Sizes a workspace for an h x w image.
static int32_t prepare_workspace(Workspace& ws, int h, int w) {
    ws.g = make_geometry(h, w);
    const Geometry& g = ws.g;
    const size_t sum = (size_t)g.grad_off[g.n_oct] / 3;   // sum of octave pixels
    const size_t p0 = (size_t)g.R[0] * g.C[0];
    FSB_TRY(ws.dog.ensure(5 * sum * 4));
    FSB_TRY(ws.mag.ensure(3 * sum * 4));
    FSB_TRY(ws.ang.ensure(3 * sum * 4));
    for (auto& b : ws.plane) FSB_TRY(b.ensure(p0 * 4));
    if (g.n_oct > 1) FSB_TRY(ws.next_base.ensure(2 * (((size_t)g.R[1] * g.C[1] + 63) / 64 * 64) * 4));
    FSB_TRY(ws.img.ensure((size_t)h * w));
    if (ws.cap_cand < 65536) ws.cap_cand = 65536;
    if (ws.cap_cand < sum / 64) ws.cap_cand = sum / 64;
    FSB_TRY(ws.cand.ensure(ws.cap_cand * 4));
    FSB_TRY(ws.counters.ensure(64));
    return FSB_OK;
}

static Workspace* acquire(fsb_ctx* ctx) {
    if (!ctx->pool.empty()) {
        Workspace* w = ctx->pool.back();
        ctx->pool.pop_back();
        return w;
    }
    return new Workspace();
}

static void give_back(fsb_ctx* ctx, Workspace* w) {
    if (ctx->pool.size() >= 2) {
        w->release();
        delete w;
        return;
    }
    ctx->pool.push_back(w);
}

static int32_t use_device(fsb_ctx* ctx) {
    FSB_CUDA(cudaSetDevice(ctx->device));
    return FSB_OK;
}

// Host side of the host-buffer entry points. Page-locked user memory is copied directly; pageable
// memory goes through the context's own page-locked staging buffer (a CPU copy on the calling
// thread), so contexts driven by several host threads do not queue behind one another in the
// driver's shared staging of pageable copies. Within a call the staged inputs and outputs share
// the buffer: the device-to-host copies follow the host-to-device ones on the context's stream,
// and every host-buffer call ends synchronised.
static bool host_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

static int32_t stage_ensure(fsb_ctx* ctx, size_t bytes) {
    if (ctx->pinned_bytes >= bytes) return FSB_OK;
    FSB_CUDA(cudaStreamSynchronize(ctx->stream));   // no copy in flight uses the old buffer
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
    size_t nb = (size_t)4 << 20;
    while (nb < bytes) nb <<= 1;
    FSB_CUDA(cudaHostAlloc(&ctx->pinned, nb, cudaHostAllocDefault));
    ctx->pinned_bytes = nb;
    return FSB_OK;
}

struct HostCopy {
    void* host;
    void* dev;
    size_t bytes;
};

static size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// host -> device copies of k buffers, enqueued on the context's stream
static int32_t copy_in(fsb_ctx* ctx, const HostCopy* c, int k) {
    size_t total = 0;
    bool direct[16];
    for (int i = 0; i < k; ++i) {
        direct[i] = c[i].bytes == 0 || host_pinned(c[i].host);
        if (!direct[i]) total += al256(c[i].bytes);
    }
    if (total) FSB_TRY(stage_ensure(ctx, total));
    char* st = static_cast<char*>(ctx->pinned);
    for (int i = 0; i < k; ++i) {
        if (c[i].bytes == 0) continue;
        const void* src = c[i].host;
        if (!direct[i]) {
            std::memcpy(st, c[i].host, c[i].bytes);
            src = st;
            st += al256(c[i].bytes);
        }
        FSB_CUDA(cudaMemcpyAsync(c[i].dev, src, c[i].bytes, cudaMemcpyHostToDevice, ctx->stream));
    }
    return FSB_OK;
}

// device -> host copies of k buffers; returns with the data in the host buffers
static int32_t copy_out(fsb_ctx* ctx, const HostCopy* c, int k) {
    size_t total = 0;
    bool direct[16];
    for (int i = 0; i < k; ++i) {
        direct[i] = c[i].bytes == 0 || host_pinned(c[i].host);
        if (!direct[i]) total += al256(c[i].bytes);
    }
    if (total) FSB_TRY(stage_ensure(ctx, total));
    char* st = static_cast<char*>(ctx->pinned);
    char* at[16];
    for (int i = 0; i < k; ++i) {
        if (c[i].bytes == 0) continue;
        void* dst = c[i].host;
        if (!direct[i]) {
            at[i] = st;
            dst = st;
            st += al256(c[i].bytes);
        }
        FSB_CUDA(cudaMemcpyAsync(dst, c[i].dev, c[i].bytes, cudaMemcpyDeviceToHost, ctx->stream));
    }
    FSB_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < k; ++i)
        if (c[i].bytes && !direct[i]) std::memcpy(c[i].host, at[i], c[i].bytes);
    return FSB_OK;
}

template <class T>
static int32_t to_dev(DevBuf& b, const T* h, size_t n, cudaStream_t s) {
    FSB_TRY(b.ensure(n * sizeof(T) + 16));
    if (n) FSB_CUDA(cudaMemcpyAsync(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return FSB_OK;
}

// detect on an image already in device memory (the workspace must be prepared for h x w)
static int32_t detect_dev(fsb_ctx* ctx, Workspace& ws, const uint8_t* d_img, int stride, const fsb_sift_params* p,
                          int max_kp) {
    const bool exact = (p->flags & FSB_SIFT_EXACT_BLUR) != 0;
    ctx->stage_begin(ST_PYRAMID);
    FSB_TRY(run_pyramid(ws, d_img, stride, exact, ctx->stream, ctx->side, ctx->pyr_ev));
    ctx->stage_end(ST_PYRAMID);
    FSB_TRY(run_detect(ctx, ws, p->contrast, p->edge, max_kp, exact));
    return FSB_OK;
}

// detect into a workspace; the image is copied from host memory with its row stride
static int32_t detect_into(fsb_ctx* ctx, Workspace& ws, const uint8_t* img, int h, int w, int stride,
                           const fsb_sift_params* p, int max_kp) {
    cudaStream_t s = ctx->stream;
    FSB_TRY(prepare_workspace(ws, h, w));
    ctx->stage_begin(ST_UPLOAD);
    if (host_pinned(img)) {
        FSB_CUDA(cudaMemcpy2DAsync(ws.img.p, (size_t)w, img, (size_t)stride, (size_t)w, (size_t)h,
                                   cudaMemcpyHostToDevice, s));
    } else {
        // rows gathered into the context's page-locked buffer, one contiguous copy
        FSB_TRY(stage_ensure(ctx, (size_t)h * w));
        uint8_t* st = static_cast<uint8_t*>(ctx->pinned);
        for (int r = 0; r < h; ++r) std::memcpy(st + (size_t)r * w, img + (size_t)r * stride, (size_t)w);
        FSB_CUDA(cudaMemcpyAsync(ws.img.p, st, (size_t)h * w, cudaMemcpyHostToDevice, s));
    }
    ctx->stage_end(ST_UPLOAD);
    return detect_dev(ctx, ws, ws.img.as<uint8_t>(), w, p, max_kp);
}

// selected keypoints -> describe inputs (tx..tly) and optional interleaved xy / response outputs
// d_n (nullable): the selection count on the device, n a capacity
__global__ void k_take(const int32_t* __restrict__ sel, int n, const int* __restrict__ d_n, const float* x,
                       const float* y, const float* sz, const float* an, const float* rs, const int32_t* oc,
                       const int32_t* ly, float* ox, float* oy, float* osz, float* oan, float* ors, int32_t* ooc,
                       int32_t* oly, float* oxy, float* oresp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (d_n) n = min(*d_n, n);
    if (i >= n) return;
    const int k = sel[i];
    ox[i] = x[k]; oy[i] = y[k]; osz[i] = sz[k]; oan[i] = an[k]; ors[i] = rs[k]; ooc[i] = oc[k]; oly[i] = ly[k];
    if (oxy) { oxy[2 * i] = x[k]; oxy[2 * i + 1] = y[k]; }
    if (oresp) oresp[i] = rs[k];
}

// features.sift_gpu after detection: spread, stable response order, describe; device outputs
// (d_xy n*2 interleaved, d_resp, d_desc, d_u8; each nullable). *n_out = 0 below 10 keypoints.
static int32_t features_dev(fsb_ctx* ctx, Workspace& ws, int nfeat, bool exact, float* d_xy, float* d_resp,
                            float* d_desc, uint8_t* d_u8, int* n_out, float* d_size = nullptr,
                            float* d_angle = nullptr, int32_t* d_oct = nullptr) {
    cudaStream_t s = ctx->stream;
    *n_out = 0;
    if (ws.n_kp < 10) return FSB_OK;
    FSB_TRY(ctx->s_i64.ensure((size_t)ws.n_kp * 4 + 256));
    int32_t* sel = ctx->s_i64.as<int32_t>();
    int n_sel = 0;
    ctx->stage_begin(ST_SPREAD);
    FSB_TRY(run_spread(ws, nfeat, sel, &n_sel, ctx, s));
    if (n_sel == 0) return FSB_OK;
    FSB_TRY(ctx->s_f32a.ensure((size_t)n_sel * 4 * 7 + 256));
    float* tx = ctx->s_f32a.as<float>();
    float* ty = tx + n_sel;
    float* tsz = ty + n_sel;
    float* tan_ = tsz + n_sel;
    float* trs = tan_ + n_sel;
    int32_t* toc = reinterpret_cast<int32_t*>(trs + n_sel);
    int32_t* tly = toc + n_sel;
    k_take<<<(n_sel + 255) / 256, 256, 0, s>>>(sel, n_sel, nullptr, ws.kx.as<float>(), ws.ky.as<float>(),
                                               ws.ksize.as<float>(), ws.kangle.as<float>(), ws.kresp.as<float>(),
                                               ws.koct.as<int32_t>(), ws.klayer.as<int32_t>(), tx, ty, tsz, tan_,
                                               trs, toc, tly, d_xy, d_resp);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    ctx->stage_end(ST_SPREAD);
    ctx->stage_begin(ST_DESCRIBE);
    FSB_TRY(run_describe_mode(ws, n_sel, tx, ty, tsz, tan_, toc, tly, d_desc, d_u8, exact, s));
    ctx->stage_end(ST_DESCRIBE);
    if (d_size) FSB_CUDA(cudaMemcpyAsync(d_size, tsz, (size_t)n_sel * 4, cudaMemcpyDeviceToDevice, s));
    if (d_angle) FSB_CUDA(cudaMemcpyAsync(d_angle, tan_, (size_t)n_sel * 4, cudaMemcpyDeviceToDevice, s));
    if (d_oct) FSB_CUDA(cudaMemcpyAsync(d_oct, toc, (size_t)n_sel * 4, cudaMemcpyDeviceToDevice, s));
    *n_out = n_sel;
    return FSB_OK;
}

static std::atomic<long long> g_launches{0};

}  // namespace fsb

void fsb::note_launch(int n) { fsb::g_launches.fetch_add(n, std::memory_order_relaxed); }
long long fsb::launch_mark() { return fsb::g_launches.load(std::memory_order_relaxed); }

namespace {
cudaEvent_t take_event(std::vector<cudaEvent_t>& free_list) {
    cudaEvent_t e = nullptr;
    if (!free_list.empty()) {
        e = free_list.back();
        free_list.pop_back();
    } else if (cudaEventCreate(&e) != cudaSuccess) {
        e = nullptr;
    }
    return e;
}
}  // namespace

void fsb_ctx::stage_begin(int st) {
    if (!timing) return;
    if (ev_open[st]) ev_free.push_back(ev_open[st]);
    ev_open[st] = take_event(ev_free);
    if (ev_open[st]) cudaEventRecord(ev_open[st], stream);
}

void fsb_ctx::stage_end(int st) {
    if (!timing || !ev_open[st]) return;
    cudaEvent_t e1 = take_event(ev_free);
    if (!e1) return;
    cudaEventRecord(e1, stream);
    ev_pending.push_back({st, ev_open[st], e1});
    ev_open[st] = nullptr;
    // the oldest pairs finished long ago in a busy pipeline: reading them back does not wait
    if (ev_pending.size() >= 512) stage_resolve(64);
}

void fsb_ctx::stage_resolve(size_t keep) {
    if (ev_pending.size() <= keep) return;
    const size_t n = ev_pending.size() - keep;
    for (size_t i = 0; i < n; ++i) {
        const StageMark& m = ev_pending[i];
        float ms = 0.f;
        if (cudaEventSynchronize(m.e1) == cudaSuccess && cudaEventElapsedTime(&ms, m.e0, m.e1) == cudaSuccess) {
            stage_ms[m.st] += ms;
            stage_n[m.st] += 1;
        }
        ev_free.push_back(m.e0);
        ev_free.push_back(m.e1);
    }
    ev_pending.erase(ev_pending.begin(), ev_pending.begin() + (std::ptrdiff_t)n);
}

void fsb_ctx::stage_release() {
    stage_resolve(0);
    for (cudaEvent_t& e : ev_open)
        if (e) {
            ev_free.push_back(e);
            e = nullptr;
        }
    for (cudaEvent_t e : ev_free) cudaEventDestroy(e);
    ev_free.clear();
}

using namespace fsb;

// ---- sync-free batched extraction: one CUDA graph per batch
namespace fsb {
namespace {
// per image after its chain ran: the feature count and the flags (ASYNC_*, 8 = pyramid timeout)
__global__ void k_batch_status(const uint32_t* cnt, int32_t* count, uint32_t* status) {
    if (threadIdx.x != 0) return;
    *count = (int32_t)cnt[6];
    *status = cnt[7] | (cnt[PYR_ERR_WORD] ? 8u : 0u);
}

struct BatchCall {
    int n_img;
    const uint8_t* const* imgs;
    const uint8_t* const* h_imgs;   // page-locked host images uploaded by the graph, or null
    int h, w, stride;
    const fsb_sift_params* p;
    const int32_t* nfeats;
    float* const* xy;
    float* const* resp;
    uint8_t* const* u8;
    int32_t* d_counts;
};

// the stream work of the batch (captured): image i on chain i mod chains
int32_t batch_body(fsb_ctx* ctx, const BatchCall& b) {
    auto& x = ctx->xb;
    const int chains = (int)x.streams.size();
    const bool exact = (b.p->flags & FSB_SIFT_EXACT_BLUR) != 0;
    FSB_CUDA(cudaEventRecord(x.fork, ctx->stream));
    for (int c = 0; c < chains; ++c) FSB_CUDA(cudaStreamWaitEvent(x.streams[c], x.fork, 0));
    if (b.h_imgs) {
        // the uploads on their own stream, in image order: image i's chain waits for image i only,
        // so later uploads overlap the extraction of earlier images
        x.copy_nodes.assign(b.n_img, nullptr);
        FSB_CUDA(cudaStreamWaitEvent(x.upload, x.fork, 0));
        const size_t bytes = (size_t)b.h * b.stride;
        for (int i = 0; i < b.n_img; ++i) {
            FSB_CUDA(cudaMemcpyAsync(const_cast<uint8_t*>(b.imgs[i]), b.h_imgs[i], bytes, cudaMemcpyHostToDevice,
                                     x.upload));
            cudaStreamCaptureStatus cs;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            FSB_CUDA(cudaStreamGetCaptureInfo(x.upload, &cs, nullptr, nullptr, &deps, &nd));
            if (cs != cudaStreamCaptureStatusActive || nd != 1) {
                set_error("capture of the image uploads: unexpected capture state");
                return FSB_ERR_CUDA;
            }
            x.copy_nodes[i] = deps[0];
            FSB_CUDA(cudaEventRecord(x.uploaded[i], x.upload));
        }
    }
    uint32_t* status = x.status.as<uint32_t>();
    for (int i = 0; i < b.n_img; ++i) {
        const int c = i % chains;
        cudaStream_t s = x.streams[c];
        Workspace& ws = *x.ws[c];
        const int nfeat = b.nfeats[i];
        if (b.h_imgs) FSB_CUDA(cudaStreamWaitEvent(s, x.uploaded[i], 0));
        FSB_TRY(run_pyramid(ws, b.imgs[i], b.stride, exact, s, nullptr, nullptr));
        FSB_TRY(run_detect_async(ws, b.p->contrast, b.p->edge, x.caps, (int)((double)nfeat * 2.2), exact, s));
        const int nf = x.caps.nfeat;
        float* tx = ws.take.as<float>();
        float* ty = tx + nf;
        float* tsz = ty + nf;
        float* tan_ = tsz + nf;
        float* trs = tan_ + nf;
        int32_t* toc = reinterpret_cast<int32_t*>(trs + nf);
        int32_t* tly = toc + nf;
        int32_t* sel = tly + nf;
        FSB_TRY(spread_async(ws, x.caps, nfeat, sel, s));
        const int* d_nsel = reinterpret_cast<const int*>(ws.counters.as<uint32_t>() + 6);
        k_take<<<(nf + 255) / 256, 256, 0, s>>>(sel, nf, d_nsel, ws.kx.as<float>(), ws.ky.as<float>(),
                                               ws.ksize.as<float>(), ws.kangle.as<float>(), ws.kresp.as<float>(),
                                               ws.koct.as<int32_t>(), ws.klayer.as<int32_t>(), tx, ty, tsz, tan_, trs,
                                               toc, tly, b.xy[i], b.resp ? b.resp[i] : nullptr);
        FSB_TRY(run_describe_dev(ws, nf, d_nsel, tx, ty, tsz, tan_, toc, tly, nullptr, b.u8[i], exact, s));
        k_batch_status<<<1, 32, 0, s>>>(ws.counters.as<uint32_t>(), b.d_counts + i, status + i);
        note_launch(2);
        FSB_CUDA(cudaGetLastError());
    }
    for (int c = 0; c < chains; ++c) {
        FSB_CUDA(cudaEventRecord(x.join[c], x.streams[c]));
        FSB_CUDA(cudaStreamWaitEvent(ctx->stream, x.join[c], 0));
    }
    if (b.h_imgs) {   // the upload stream rejoins too (its last node precedes every chain anyway)
        FSB_CUDA(cudaEventRecord(x.uploaded[b.n_img - 1], x.upload));
        FSB_CUDA(cudaStreamWaitEvent(ctx->stream, x.uploaded[b.n_img - 1], 0));
    }
    return FSB_OK;
}

template <class T>
void key_put(std::vector<char>& k, const T& v) {
    const char* p = reinterpret_cast<const char*>(&v);
    k.insert(k.end(), p, p + sizeof(T));
}
}  // namespace
}  // namespace fsb

extern "C" {

int32_t fsb_version(void) { return 100; }

const char* fsb_last_error(void) { return g_err.c_str(); }

int32_t fsb_create(int32_t device, fsb_ctx** out) {
    FSB_ARG(out != nullptr, "out is null");
    *out = nullptr;
    int n = 0;
    FSB_CUDA(cudaGetDeviceCount(&n));
    FSB_ARG(device >= 0 && device < n, "device index out of range");
    cudaDeviceProp prop;
    FSB_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10 || prop.minor != 0) {
        set_error("device %d is sm_%d%d; this library is built for sm_100a (B200)", device, prop.major, prop.minor);
        return FSB_ERR_UNSUPPORTED;
    }
    FSB_CUDA(cudaSetDevice(device));
    fsb_ctx* ctx = new fsb_ctx();
    ctx->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx;
        set_error("cudaStreamCreate failed: %s", cudaGetErrorString(e));
        return FSB_ERR_CUDA;
    }
    bool ok = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) == cudaSuccess;
    for (auto& ev : ctx->pyr_ev) ok = ok && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
    int32_t st = ok ? upload_taps() : FSB_ERR_CUDA;
    if (st != FSB_OK) {
        if (!ok) set_error("side stream / event creation failed");
        for (auto& ev : ctx->pyr_ev)
            if (ev) cudaEventDestroy(ev);
        if (ctx->side) cudaStreamDestroy(ctx->side);
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return st;
    }
    *out = ctx;
    return FSB_OK;
}

int32_t fsb_destroy(fsb_ctx* ctx) {
    if (!ctx) return FSB_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (Workspace* w : ctx->pool) {
        w->release();
        delete w;
    }
    ctx->pool.clear();
    DevBuf* all[] = {&ctx->s_u8a, &ctx->s_u8b, &ctx->s_f32a, &ctx->s_f32b, &ctx->s_i32, &ctx->s_i64,
                     &ctx->s_u64, &ctx->s_misc, &ctx->s_misc2, &ctx->s_host_stage, &ctx->s_cub,
                     &ctx->s_tc_pack, &ctx->s_tc_part, &ctx->s_tc_aux, &ctx->s_count, &ctx->s_gb};
    for (DevBuf* b : all) b->release();
    if (ctx->gb_graph.exec) cudaGraphExecDestroy(ctx->gb_graph.exec);
    if (ctx->gb_graph.graph) cudaGraphDestroy(ctx->gb_graph.graph);
    {
        auto& x = ctx->xb;
        for (cudaStream_t cs : x.streams) cudaStreamSynchronize(cs);
        if (x.upload) cudaStreamSynchronize(x.upload);
        if (x.graph.exec) cudaGraphExecDestroy(x.graph.exec);
        if (x.graph.graph) cudaGraphDestroy(x.graph.graph);
        if (x.pyr_graph.exec) cudaGraphExecDestroy(x.pyr_graph.exec);
        if (x.pyr_graph.graph) cudaGraphDestroy(x.pyr_graph.graph);
        for (Workspace* w : x.ws) {
            w->release();
            delete w;
        }
        for (cudaStream_t cs : x.streams) cudaStreamDestroy(cs);
        for (cudaEvent_t e : x.join) cudaEventDestroy(e);
        if (x.fork) cudaEventDestroy(x.fork);
        for (cudaEvent_t e : x.uploaded) cudaEventDestroy(e);
        if (x.upload) cudaStreamDestroy(x.upload);
        x.status.release();
    }
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->stage_release();
    if (ctx->side) cudaStreamSynchronize(ctx->side);
    jpeg_release(ctx);
    for (auto& e : ctx->pyr_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return FSB_OK;
}

int32_t fsb_sync(fsb_ctx* ctx, int32_t timeout_ms) {
    FSB_ARG(ctx, "ctx is null");
    FSB_TRY(use_device(ctx));
    cudaEvent_t ev;
    FSB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, ctx->stream);
    if (e != cudaSuccess) {
        cudaEventDestroy(ev);
        set_error("cudaEventRecord failed: %s", cudaGetErrorString(e));
        return FSB_ERR_CUDA;
    }
    // bounded poll: the host gives up after timeout_ms instead of blocking forever
    const long long limit = timeout_ms <= 0 ? 0 : (long long)timeout_ms * 1000;
    long long waited = 0;
    while ((e = cudaEventQuery(ev)) == cudaErrorNotReady) {
        if (waited >= limit) {
            cudaEventDestroy(ev);
            set_error("stream did not drain within %d ms", timeout_ms);
            return FSB_ERR_TIMEOUT;
        }
        struct timespec ts = {0, 50000};
        nanosleep(&ts, nullptr);
        waited += 50;
    }
    cudaEventDestroy(ev);
    if (e != cudaSuccess) {
        set_error("stream error: %s", cudaGetErrorString(e));
        return FSB_ERR_CUDA;
    }
    return FSB_OK;
}

void* fsb_stream(fsb_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int64_t fsb_device_bytes(fsb_ctx* ctx) {
    if (!ctx) return 0;
    int64_t t = 0;
    for (Workspace* w : ctx->pool) t += (int64_t)w->bytes();
    const DevBuf* all[] = {&ctx->s_u8a, &ctx->s_u8b, &ctx->s_f32a, &ctx->s_f32b, &ctx->s_i32, &ctx->s_i64,
                           &ctx->s_u64, &ctx->s_misc, &ctx->s_misc2, &ctx->s_host_stage, &ctx->s_cub,
                     &ctx->s_tc_pack, &ctx->s_tc_part, &ctx->s_tc_aux, &ctx->s_count, &ctx->s_gb};
    for (const DevBuf* b : all) t += (int64_t)b->bytes;
    return t;
}

int32_t fsb_detect(fsb_ctx* ctx, const uint8_t* img, int32_t h, int32_t w, int32_t stride,
                   const fsb_sift_params* p, fsb_state** state, int32_t* n_kp) {
    FSB_ARG(ctx && img && p && state && n_kp, "null pointer");
    FSB_ARG(h > 0 && w > 0 && stride >= w, "bad image size or stride");
    FSB_ARG(h <= 32768 && w <= 32768, "image larger than 32768 pixels on a side");
    FSB_ARG(p->max_kp >= 0, "max_kp < 0");
    *state = nullptr;
    *n_kp = 0;
    FSB_TRY(use_device(ctx));
    Workspace* ws = acquire(ctx);
    int32_t st = detect_into(ctx, *ws, img, h, w, stride, p, p->max_kp);
    if (st == FSB_OK) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            set_error("detect: %s", cudaGetErrorString(e));
            st = FSB_ERR_CUDA;
        }
    }
    if (st != FSB_OK) {
        give_back(ctx, ws);
        return st;
    }
    ws->g.h = h;
    fsb_state* s = new fsb_state();
    s->ctx = ctx;
    s->ws = ws;
    s->magic = STATE_MAGIC;
    s->exact = (p->flags & FSB_SIFT_EXACT_BLUR) != 0;
    ctx->live_states++;
    *state = s;
    *n_kp = ws->n_kp;
    return FSB_OK;
}

int32_t fsb_state_keypoints(fsb_state* st, float* x, float* y, float* size, float* angle, float* response,
                            int32_t* octave, int32_t* layer) {
    FSB_ARG(st && st->magic == STATE_MAGIC, "invalid state");
    fsb_ctx* ctx = st->ctx;
    FSB_TRY(use_device(ctx));
    const Workspace& ws = *st->ws;
    const size_t n = (size_t)ws.n_kp;
    cudaStream_t s = ctx->stream;
    struct { void* h; const DevBuf* d; } out[] = {{x, &ws.kx}, {y, &ws.ky}, {size, &ws.ksize}, {angle, &ws.kangle},
                                                 {response, &ws.kresp}, {octave, &ws.koct}, {layer, &ws.klayer}};
    for (auto& o : out)
        if (o.h && n) FSB_CUDA(cudaMemcpyAsync(o.h, o.d->p, n * 4, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    return FSB_OK;
}

int32_t fsb_describe(fsb_ctx* ctx, fsb_state* st, int32_t n, const float* x, const float* y, const float* size,
                     const float* angle, const int32_t* octave, const int32_t* layer, float* desc,
                     uint8_t* rootsift) {
    FSB_ARG(ctx && st && st->magic == STATE_MAGIC, "invalid context or state");
    if (st->ctx != ctx) {
        set_error("state belongs to another context");
        return FSB_ERR_STATE;
    }
    FSB_ARG(n >= 0, "n < 0");
    if (n == 0) return FSB_OK;
    FSB_ARG(x && y && size && angle && octave && layer, "null keypoint array");
    const Workspace& ws = *st->ws;
    for (int i = 0; i < n; ++i) {
        if (octave[i] < 0 || octave[i] >= ws.g.n_oct || layer[i] < 1 || layer[i] > N_LAYERS) {
            set_error("keypoint %d has octave %d / layer %d outside the detected pyramid", i, octave[i], layer[i]);
            return FSB_ERR_ARG;
        }
    }
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    FSB_TRY(ctx->s_f32a.ensure((size_t)n * 4 * 6 + 256));
    float* dx = ctx->s_f32a.as<float>();
    float* dy = dx + n;
    float* ds = dy + n;
    float* da = ds + n;
    int32_t* dout = reinterpret_cast<int32_t*>(da + n);
    int32_t* dl = dout + n;
    FSB_CUDA(cudaMemcpyAsync(dx, x, n * 4, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(dy, y, n * 4, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(ds, size, n * 4, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(da, angle, n * 4, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(dout, octave, n * 4, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(dl, layer, n * 4, cudaMemcpyHostToDevice, s));
    FSB_TRY(ctx->s_f32b.ensure((size_t)n * 128 * 4 + 256));
    FSB_TRY(ctx->s_u8a.ensure((size_t)n * 128 + 256));
    float* dd = desc ? ctx->s_f32b.as<float>() : nullptr;
    uint8_t* du = rootsift ? ctx->s_u8a.as<uint8_t>() : nullptr;
    FSB_TRY(run_describe_mode(ws, n, dx, dy, ds, da, dout, dl, dd, du, st->exact, s));
    if (desc) FSB_CUDA(cudaMemcpyAsync(desc, dd, (size_t)n * 128 * 4, cudaMemcpyDeviceToHost, s));
    if (rootsift) FSB_CUDA(cudaMemcpyAsync(rootsift, du, (size_t)n * 128, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    return FSB_OK;
}

int32_t fsb_state_geometry(fsb_state* st, int32_t* n_oct, int32_t* rows, int32_t* cols) {
    FSB_ARG(st && st->magic == STATE_MAGIC, "invalid state");
    const Geometry& g = st->ws->g;
    if (n_oct) *n_oct = g.n_oct;
    for (int o = 0; o < g.n_oct; ++o) {
        if (rows) rows[o] = g.R[o];
        if (cols) cols[o] = g.C[o];
    }
    return FSB_OK;
}

int32_t fsb_state_atlas(fsb_state* st, int32_t which, float* out, int64_t n_floats) {
    FSB_ARG(st && st->magic == STATE_MAGIC, "invalid state");
    FSB_ARG(out && which >= 0 && which <= 2, "bad atlas request");
    const Geometry& g = st->ws->g;
    const int64_t want = which == 0 ? g.dog_off[g.n_oct] : g.grad_off[g.n_oct];
    if (n_floats != want) {
        set_error("invalid argument: atlas %d holds %lld floats, %lld requested", which, (long long)want,
                  (long long)n_floats);
        return FSB_ERR_ARG;
    }
    FSB_TRY(use_device(st->ctx));
    const DevBuf& b = which == 0 ? st->ws->dog : which == 1 ? st->ws->mag : st->ws->ang;
    if (want) FSB_CUDA(cudaMemcpyAsync(out, b.p, (size_t)want * 4, cudaMemcpyDeviceToHost, st->ctx->stream));
    FSB_CUDA(cudaStreamSynchronize(st->ctx->stream));
    return FSB_OK;
}

int32_t fsb_state_free(fsb_state* st) {
    if (!st) return FSB_OK;
    FSB_ARG(st->magic == STATE_MAGIC, "invalid state (double free?)");
    fsb_ctx* ctx = st->ctx;
    st->magic = 0;
    cudaSetDevice(ctx->device);
    give_back(ctx, st->ws);
    ctx->live_states--;
    delete st;
    return FSB_OK;
}

int32_t fsb_sift_features(fsb_ctx* ctx, const uint8_t* img, int32_t h, int32_t w, int32_t stride,
                          const fsb_sift_params* p, int32_t nfeat, float* xy, float* resp, float* desc,
                          uint8_t* rootsift, int32_t* n_out) {
    FSB_ARG(ctx && img && p && n_out, "null pointer");
    FSB_ARG(h > 0 && w > 0 && stride >= w, "bad image size or stride");
    FSB_ARG(h <= 32768 && w <= 32768, "image larger than 32768 pixels on a side");
    FSB_ARG(nfeat >= 0, "nfeat < 0");
    *n_out = 0;
    FSB_TRY(use_device(ctx));
    Workspace* ws = acquire(ctx);
    struct Guard {
        fsb_ctx* c;
        Workspace* w;
        ~Guard() { give_back(c, w); }
    } guard{ctx, ws};
    const int max_kp = (int)((double)nfeat * 2.2);
    FSB_TRY(detect_into(ctx, *ws, img, h, w, stride, p, max_kp));
    const size_t cap = (size_t)(nfeat > 0 ? nfeat : 1);
    FSB_TRY(ctx->s_f32b.ensure(cap * (128 * 4 + 12) + 1024));
    FSB_TRY(ctx->s_u8a.ensure(cap * 128 + 256));
    float* dd = ctx->s_f32b.as<float>();
    float* dxy = dd + cap * 128;
    float* drs = dxy + cap * 2;
    int n = 0;
    FSB_TRY(features_dev(ctx, *ws, nfeat, (p->flags & FSB_SIFT_EXACT_BLUR) != 0, dxy, drs, desc ? dd : nullptr,
                         rootsift ? ctx->s_u8a.as<uint8_t>() : nullptr, &n));
    HostCopy out[4];
    int k = 0;
    if (n) {
        if (xy) out[k++] = {xy, dxy, (size_t)n * 8};
        if (resp) out[k++] = {resp, drs, (size_t)n * 4};
        if (desc) out[k++] = {desc, dd, (size_t)n * 512};
        if (rootsift) out[k++] = {rootsift, ctx->s_u8a.p, (size_t)n * 128};
    }
    FSB_TRY(copy_out(ctx, out, k));
    *n_out = n;
    return FSB_OK;
}

int32_t fsb_sift_features_d(fsb_ctx* ctx, const uint8_t* d_img, int32_t h, int32_t w, int32_t stride,
                            const fsb_sift_params* p, int32_t nfeat, float* d_xy, float* d_resp, float* d_desc,
                            uint8_t* d_rootsift, int32_t* n_out) {
    FSB_ARG(ctx && d_img && p && n_out, "null pointer");
    FSB_ARG(h > 0 && w > 0 && stride >= w, "bad image size or stride");
    FSB_ARG(h <= 32768 && w <= 32768, "image larger than 32768 pixels on a side");
    FSB_ARG(nfeat >= 0, "nfeat < 0");
    *n_out = 0;
    FSB_TRY(use_device(ctx));
    Workspace* ws = acquire(ctx);
    struct Guard {
        fsb_ctx* c;
        Workspace* w;
        ~Guard() { give_back(c, w); }
    } guard{ctx, ws};
    FSB_TRY(prepare_workspace(*ws, h, w));
    FSB_TRY(detect_dev(ctx, *ws, d_img, stride, p, (int)((double)nfeat * 2.2)));
    int n = 0;
    FSB_TRY(features_dev(ctx, *ws, nfeat, (p->flags & FSB_SIFT_EXACT_BLUR) != 0, d_xy, d_resp, d_desc, d_rootsift,
                         &n));
    FSB_CUDA(cudaStreamSynchronize(ctx->stream));
    *n_out = n;
    return FSB_OK;
}

int32_t fsb_sift_features_ex_d(fsb_ctx* ctx, const uint8_t* d_img, int32_t h, int32_t w, int32_t stride,
                               const fsb_sift_params* p, int32_t nfeat, float* d_xy, float* d_resp, float* d_desc,
                               uint8_t* d_rootsift, float* d_size, float* d_angle, int32_t* d_octave,
                               int32_t* n_out) {
    FSB_ARG(ctx && d_img && p && n_out, "null pointer");
    FSB_ARG(h > 0 && w > 0 && stride >= w, "bad image size or stride");
    FSB_ARG(h <= 32768 && w <= 32768, "image larger than 32768 pixels on a side");
    FSB_ARG(nfeat >= 0, "nfeat < 0");
    *n_out = 0;
    FSB_TRY(use_device(ctx));
    Workspace* ws = acquire(ctx);
    struct Guard {
        fsb_ctx* c;
        Workspace* w;
        ~Guard() { give_back(c, w); }
    } guard{ctx, ws};
    FSB_TRY(prepare_workspace(*ws, h, w));
    FSB_TRY(detect_dev(ctx, *ws, d_img, stride, p, (int)((double)nfeat * 2.2)));
    int n = 0;
    FSB_TRY(features_dev(ctx, *ws, nfeat, (p->flags & FSB_SIFT_EXACT_BLUR) != 0, d_xy, d_resp, d_desc, d_rootsift,
                         &n, d_size, d_angle, d_octave));
    FSB_CUDA(cudaStreamSynchronize(ctx->stream));
    *n_out = n;
    return FSB_OK;
}


}  // extern "C"

namespace fsb {
namespace {
// fsb_sift_features_batch_d and, with h_imgs, fsb_sift_features_batch_hd
int32_t sift_features_batch(fsb_ctx* ctx, int32_t n_img, const uint8_t* const* h_imgs, const uint8_t* const* d_imgs,
                            int32_t h, int32_t w, int32_t stride, const fsb_sift_params* p, const int32_t* nfeats,
                            float* const* d_xy, float* const* d_resp, uint8_t* const* d_rootsift, int32_t* d_counts,
                            int32_t* h_counts, int32_t chains) {
    FSB_ARG(ctx && p, "null pointer");
    FSB_ARG(n_img >= 0, "n_img < 0");
    if (n_img == 0) return FSB_OK;
    FSB_ARG(d_imgs && nfeats && d_xy && d_rootsift && d_counts, "null array");
    FSB_ARG(h > 0 && w > 0 && stride >= w, "bad image size or stride");
    FSB_ARG(h <= 32768 && w <= 32768, "image larger than 32768 pixels on a side");
    FSB_ARG(chains >= 1 && chains <= 32, "chains must be 1..32");
    int nf_max = 0;
    for (int i = 0; i < n_img; ++i) {
        FSB_ARG(nfeats[i] >= 0 && nfeats[i] <= (1 << 24), "nfeat out of range");
        FSB_ARG(d_imgs[i] && d_xy[i] && d_rootsift[i], "null image or output pointer");
        nf_max = nfeats[i] > nf_max ? nfeats[i] : nf_max;
    }
    FSB_TRY(use_device(ctx));
    if (h_imgs) {
        for (int i = 0; i < n_img; ++i) {
            FSB_ARG(h_imgs[i], "null host image");
            cudaPointerAttributes at{};
            FSB_CUDA(cudaPointerGetAttributes(&at, h_imgs[i]));
            FSB_ARG(at.type == cudaMemoryTypeHost, "host images must be page-locked (cudaHostAlloc / registered)");
        }
    }
    auto& x = ctx->xb;
    cudaStream_t s = ctx->stream;
    const bool timing = ctx->timing;
    ctx->timing = false;   // stage events are not captured
    struct Restore {
        fsb_ctx* c;
        bool t;
        ~Restore() { c->timing = t; }
    } restore{ctx, timing};
    // first batch of a geometry: image 0 by the host-driven path (autotunes the pyramid for the
    // geometry, and its refined-extremum count sizes the sort capacity)
    if (x.h != h || x.w != w || x.warm_ref == 0) {
        Workspace* ws = acquire(ctx);
        struct Guard {
            fsb_ctx* c;
            Workspace* w;
            ~Guard() { give_back(c, w); }
        } guard{ctx, ws};
        FSB_TRY(prepare_workspace(*ws, h, w));
        if (h_imgs)
            FSB_CUDA(cudaMemcpyAsync(const_cast<uint8_t*>(d_imgs[0]), h_imgs[0], (size_t)h * stride,
                                     cudaMemcpyHostToDevice, s));
        FSB_TRY(detect_dev(ctx, *ws, d_imgs[0], stride, p, (int)((double)nfeats[0] * 2.2)));
        int n0 = 0;
        FSB_TRY(features_dev(ctx, *ws, nfeats[0], (p->flags & FSB_SIFT_EXACT_BLUR) != 0, d_xy[0],
                             d_resp ? d_resp[0] : nullptr, nullptr, d_rootsift[0], &n0));
        FSB_CUDA(cudaStreamSynchronize(s));
        x.h = h;
        x.w = w;
        x.warm_ref = (int)std::min<size_t>(ws->cap_ref, (size_t)1 << 30);
    }
    // chains: streams, events, workspaces sized for the geometry and the capacities
    while ((int)x.streams.size() < chains) {
        cudaStream_t cs;
        cudaEvent_t ev;
        FSB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        FSB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        x.streams.push_back(cs);
        x.join.push_back(ev);
        x.ws.push_back(new Workspace());
    }
    if (!x.fork) FSB_CUDA(cudaEventCreateWithFlags(&x.fork, cudaEventDisableTiming));
    if (h_imgs) {
        if (!x.upload) FSB_CUDA(cudaStreamCreateWithFlags(&x.upload, cudaStreamNonBlocking));
        while ((int)x.uploaded.size() < n_img) {
            cudaEvent_t ev;
            FSB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            x.uploaded.push_back(ev);
        }
    }
    AsyncCaps caps{};
    Workspace probe;
    probe.g = make_geometry(h, w);
    probe.cap_ref = (size_t)x.warm_ref + (size_t)x.warm_ref / 2;
    FSB_TRY(async_caps(probe, (int)((double)nf_max * 2.2), nf_max, &caps));
    const bool regrow = caps.kp > x.caps.kp || caps.nfeat > x.caps.nfeat || caps.ref > x.caps.ref ||
                        caps.cand != x.caps.cand;
    if (regrow || (int)x.ws.size() != (int)x.streams.size()) {
        caps.kp = std::max(caps.kp, x.caps.kp);
        caps.nfeat = std::max(caps.nfeat, x.caps.nfeat);
        caps.ref = std::max(caps.ref, x.caps.ref);
        caps.rank = (uint32_t)(2 * caps.kp + 32);
        x.caps = caps;
    }
    // the streams the capture uses are the first `chains`; the others idle
    std::vector<cudaStream_t> all_streams = x.streams;
    std::vector<cudaEvent_t> all_join = x.join;
    std::vector<Workspace*> all_ws = x.ws;
    x.streams.resize(chains);
    x.join.resize(chains);
    x.ws.resize(chains);
    struct Back {
        fsb_ctx::ExtractBatch& x;
        std::vector<cudaStream_t> s;
        std::vector<cudaEvent_t> j;
        std::vector<Workspace*> w;
        ~Back() { x.streams = s; x.join = j; x.ws = w; }
    } back{x, all_streams, all_join, all_ws};
    for (Workspace* ws : x.ws) {
        if (ws->g.h != h || ws->g.w != w) FSB_TRY(prepare_workspace(*ws, h, w));
        FSB_TRY(prepare_async(*ws, x.caps, s));
    }
    FSB_TRY(x.status.ensure((size_t)n_img * 4 + 64));
    // the captured graph is replayed while every argument and buffer address is unchanged
    std::vector<char> key;
    key_put(key, n_img);
    key_put(key, h_imgs != nullptr);   // the uploads' sources are set per launch, not keyed
    key_put(key, h);
    key_put(key, w);
    key_put(key, stride);
    key_put(key, chains);
    key_put(key, *p);
    key_put(key, x.caps);
    key_put(key, d_counts);
    key_put(key, x.status.p);
    for (int i = 0; i < n_img; ++i) {
        key_put(key, d_imgs[i]);
        key_put(key, nfeats[i]);
        key_put(key, d_xy[i]);
        key_put(key, d_resp ? d_resp[i] : nullptr);
        key_put(key, d_rootsift[i]);
    }
    for (Workspace* ws : x.ws) {
        const void* ptrs[] = {ws->dog.p, ws->mag.p, ws->ang.p, ws->plane[0].p, ws->plane[1].p, ws->plane[2].p,
                              ws->next_base.p, ws->cand.p, ws->refined.p, ws->oriented.p, ws->keys_a.p, ws->keys_b.p,
                              ws->vals_a.p, ws->sort_tmp.p, ws->counters.p, ws->kx.p, ws->ky.p, ws->ksize.p,
                              ws->kangle.p, ws->kresp.p, ws->koct.p, ws->klayer.p, ws->spread.p, ws->take.p};
        for (const void* q : ptrs) key_put(key, q);
        key_put(key, ws->sort_tmp.bytes);
    }
    if (!x.graph.exec || key != x.graph.key) {
        if (x.graph.exec) cudaGraphExecDestroy(x.graph.exec);
        if (x.graph.graph) cudaGraphDestroy(x.graph.graph);
        x.graph.exec = nullptr;
        x.graph.graph = nullptr;
        BatchCall bc{n_img, d_imgs, h_imgs, h, w, stride, p, nfeats, d_xy, d_resp, d_rootsift, d_counts};
        const long long m0 = launch_mark();
        FSB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const int32_t st = batch_body(ctx, bc);
        x.graph.n_kernels = (int)(launch_mark() - m0);
        note_launch(-x.graph.n_kernels);   // the kernels run (and count) at each replay
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &g);
        if (st != FSB_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            set_error("capture of the extraction batch failed: %s", cudaGetErrorString(e));
            return FSB_ERR_CUDA;
        }
        x.graph.graph = g;
        FSB_CUDA(cudaGraphInstantiate(&x.graph.exec, g, 0));
        x.graph.key = key;
    }
    if (h_imgs) {
        for (int i = 0; i < n_img; ++i)
            FSB_CUDA(cudaGraphExecMemcpyNodeSetParams1D(x.graph.exec, x.copy_nodes[i], const_cast<uint8_t*>(d_imgs[i]),
                                                        h_imgs[i], (size_t)h * stride, cudaMemcpyHostToDevice));
    }
    FSB_CUDA(cudaGraphLaunch(x.graph.exec, s));
    note_launch(x.graph.n_kernels);
    // one wait per batch: the flags say which images (if any) exceeded a capacity
    FSB_TRY(stage_ensure(ctx, (size_t)n_img * 8 + 64));
    uint32_t* h_status = static_cast<uint32_t*>(ctx->pinned);
    int32_t* h_cnt = reinterpret_cast<int32_t*>(h_status + n_img);
    FSB_CUDA(cudaMemcpyAsync(h_status, x.status.p, (size_t)n_img * 4, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaMemcpyAsync(h_cnt, d_counts, (size_t)n_img * 4, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < n_img; ++i) {
        if (h_status[i] & 8u) {
            set_error("pyramid: a TMA copy of the pyramid did not complete in time, image %d", i);
            return FSB_ERR_TIMEOUT;
        }
        if (h_status[i] == 0) continue;
        // a capacity was exceeded: this image again by the host-driven path
        Workspace* ws = acquire(ctx);
        struct Guard {
            fsb_ctx* c;
            Workspace* w;
            ~Guard() { give_back(c, w); }
        } guard{ctx, ws};
        FSB_TRY(prepare_workspace(*ws, h, w));
        FSB_TRY(detect_dev(ctx, *ws, d_imgs[i], stride, p, (int)((double)nfeats[i] * 2.2)));
        int n = 0;
        FSB_TRY(features_dev(ctx, *ws, nfeats[i], (p->flags & FSB_SIFT_EXACT_BLUR) != 0, d_xy[i],
                             d_resp ? d_resp[i] : nullptr, nullptr, d_rootsift[i], &n));
        h_cnt[i] = n;
        FSB_CUDA(cudaMemcpyAsync(d_counts + i, &h_cnt[i], 4, cudaMemcpyHostToDevice, s));
        FSB_CUDA(cudaStreamSynchronize(s));
        x.redone += 1;
    }
    if (h_counts) std::memcpy(h_counts, h_cnt, (size_t)n_img * 4);
    return FSB_OK;
}
}  // namespace
}  // namespace fsb

extern "C" {

int32_t fsb_sift_features_batch_d(fsb_ctx* ctx, int32_t n_img, const uint8_t* const* d_imgs, int32_t h, int32_t w,
                                  int32_t stride, const fsb_sift_params* p, const int32_t* nfeats, float* const* d_xy,
                                  float* const* d_resp, uint8_t* const* d_rootsift, int32_t* d_counts,
                                  int32_t* h_counts, int32_t chains) {
    return fsb::sift_features_batch(ctx, n_img, nullptr, d_imgs, h, w, stride, p, nfeats, d_xy, d_resp, d_rootsift,
                                    d_counts, h_counts, chains);
}

int32_t fsb_sift_features_batch_hd(fsb_ctx* ctx, int32_t n_img, const uint8_t* const* h_imgs,
                                   uint8_t* const* d_imgs, int32_t h, int32_t w, int32_t stride,
                                   const fsb_sift_params* p, const int32_t* nfeats, float* const* d_xy,
                                   float* const* d_resp, uint8_t* const* d_rootsift, int32_t* d_counts,
                                   int32_t* h_counts, int32_t chains) {
    FSB_ARG(n_img <= 0 || h_imgs, "null host image array");
    return fsb::sift_features_batch(ctx, n_img, h_imgs, d_imgs, h, w, stride, p, nfeats, d_xy, d_resp, d_rootsift,
                                    d_counts, h_counts, chains);
}

int32_t fsb_pyramid_batch_d(fsb_ctx* ctx, int32_t n_img, const uint8_t* const* d_imgs, int32_t h, int32_t w,
                            int32_t stride, int32_t flags, int32_t chains) {
    FSB_ARG(ctx, "null context");
    FSB_ARG(n_img >= 0, "n_img < 0");
    if (n_img == 0) return FSB_OK;
    FSB_ARG(d_imgs, "null image array");
    FSB_ARG(h > 0 && w > 0 && stride >= w, "bad image size or stride");
    FSB_ARG(h <= 32768 && w <= 32768, "image larger than 32768 pixels on a side");
    FSB_ARG(chains >= 1 && chains <= 32, "chains must be 1..32");
    for (int i = 0; i < n_img; ++i) FSB_ARG(d_imgs[i], "null image pointer");
    FSB_TRY(use_device(ctx));
    const bool exact = (flags & FSB_SIFT_EXACT_BLUR) != 0;
    auto& x = ctx->xb;
    cudaStream_t s = ctx->stream;
    while ((int)x.streams.size() < chains) {
        cudaStream_t cs;
        cudaEvent_t ev;
        FSB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        FSB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        x.streams.push_back(cs);
        x.join.push_back(ev);
        x.ws.push_back(new Workspace());
    }
    if (!x.fork) FSB_CUDA(cudaEventCreateWithFlags(&x.fork, cudaEventDisableTiming));
    for (int c = 0; c < chains; ++c)
        if (x.ws[c]->g.h != h || x.ws[c]->g.w != w) FSB_TRY(prepare_workspace(*x.ws[c], h, w));
    const bool timing = ctx->timing;
    ctx->timing = false;
    struct Restore {
        fsb_ctx* c;
        bool t;
        ~Restore() { c->timing = t; }
    } restore{ctx, timing};
    // a geometry's first pyramid runs outside any capture: the autotuner times its variants then
    if (x.pyr_h != h || x.pyr_w != w) {
        FSB_TRY(run_pyramid(*x.ws[0], d_imgs[0], stride, exact, s, nullptr, nullptr));
        FSB_CUDA(cudaStreamSynchronize(s));
        x.pyr_h = h;
        x.pyr_w = w;
    }
    std::vector<char> key;
    key_put(key, n_img);
    key_put(key, h);
    key_put(key, w);
    key_put(key, stride);
    key_put(key, chains);
    key_put(key, exact);
    for (int i = 0; i < n_img; ++i) key_put(key, d_imgs[i]);
    for (int c = 0; c < chains; ++c) {
        const Workspace* ws = x.ws[c];
        const void* ptrs[] = {ws->dog.p, ws->mag.p, ws->ang.p, ws->plane[0].p, ws->plane[1].p, ws->plane[2].p,
                              ws->next_base.p, ws->counters.p};
        for (const void* q : ptrs) key_put(key, q);
    }
    if (!x.pyr_graph.exec || key != x.pyr_graph.key) {
        if (x.pyr_graph.exec) cudaGraphExecDestroy(x.pyr_graph.exec);
        if (x.pyr_graph.graph) cudaGraphDestroy(x.pyr_graph.graph);
        x.pyr_graph.exec = nullptr;
        x.pyr_graph.graph = nullptr;
        const long long m0 = launch_mark();
        FSB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int32_t st = FSB_OK;
        [&]() {
            auto chk = [&](cudaError_t e) {
                if (e != cudaSuccess && st == FSB_OK) {
                    set_error("capture of the pyramid batch: %s", cudaGetErrorString(e));
                    st = FSB_ERR_CUDA;
                }
                return st == FSB_OK;
            };
            if (!chk(cudaEventRecord(x.fork, s))) return;
            for (int c = 0; c < chains; ++c)
                if (!chk(cudaStreamWaitEvent(x.streams[c], x.fork, 0))) return;
            for (int i = 0; i < n_img; ++i) {
                const int c = i % chains;
                st = run_pyramid(*x.ws[c], d_imgs[i], stride, exact, x.streams[c], nullptr, nullptr);
                if (st != FSB_OK) return;
            }
            for (int c = 0; c < chains; ++c) {
                if (!chk(cudaEventRecord(x.join[c], x.streams[c]))) return;
                if (!chk(cudaStreamWaitEvent(s, x.join[c], 0))) return;
            }
        }();
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &g);
        x.pyr_graph.n_kernels = (int)(launch_mark() - m0);
        note_launch(-x.pyr_graph.n_kernels);
        if (st != FSB_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            if (st == FSB_OK) {
                set_error("capture of the pyramid batch failed: %s", cudaGetErrorString(e));
                st = FSB_ERR_CUDA;
            }
            return st;
        }
        x.pyr_graph.graph = g;
        FSB_CUDA(cudaGraphInstantiate(&x.pyr_graph.exec, g, 0));
        x.pyr_graph.key = key;
    }
    FSB_CUDA(cudaGraphLaunch(x.pyr_graph.exec, s));
    note_launch(x.pyr_graph.n_kernels);
    // the error words of the chains' bounded waits (strip engine)
    const int used = chains < n_img ? chains : n_img;
    FSB_TRY(stage_ensure(ctx, (size_t)used * 4 + 64));
    int32_t* h_err = static_cast<int32_t*>(ctx->pinned);
    for (int c = 0; c < used; ++c)
        FSB_CUDA(cudaMemcpyAsync(h_err + c, x.ws[c]->counters.as<int32_t>() + PYR_ERR_WORD, 4, cudaMemcpyDeviceToHost,
                                 s));
    FSB_CUDA(cudaStreamSynchronize(s));
    for (int c = 0; c < used; ++c)
        if (h_err[c]) {
            set_error("pyramid: a TMA copy of the pyramid did not complete in time, chain %d", c);
            return FSB_ERR_TIMEOUT;
        }
    return FSB_OK;
}

int32_t fsb_project_d(fsb_ctx* ctx, const float* d_xy, int32_t n, const double* hm9, const float* d_offset,
                      double* d_out) {
    FSB_ARG(ctx && hm9, "null pointer");
    FSB_ARG(n >= 0 && (n == 0 || (d_xy && d_out)), "bad points");
    if (n == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    FSB_TRY(run_project(d_xy, n, hm9, d_offset, d_out, ctx->stream));
    FSB_CUDA(cudaStreamSynchronize(ctx->stream));
    return FSB_OK;
}

int32_t fsb_project_batch_d(fsb_ctx* ctx, int32_t n_sets, const float* const* d_xy, const int32_t* n,
                            const double* hm9, const float* const* d_offset, double* const* d_out) {
    FSB_ARG(ctx && (n_sets == 0 || (d_xy && n && hm9 && d_out)), "null pointer");
    FSB_ARG(n_sets >= 0, "n_sets < 0");
    for (int k = 0; k < n_sets; ++k) FSB_ARG(n[k] >= 0 && (n[k] == 0 || (d_xy[k] && d_out[k])), "bad points");
    if (n_sets == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    for (int k = 0; k < n_sets; ++k)
        if (n[k] > 0)
            FSB_TRY(run_project(d_xy[k], n[k], hm9 + 9 * (size_t)k, d_offset ? d_offset[k] : nullptr, d_out[k],
                                ctx->stream));
    return FSB_OK;
}

int32_t fsb_match_guided_d(fsb_ctx* ctx, const double* d_pred, const uint8_t* d_a, int32_t na, const double* d_bxy,
                           const uint8_t* d_b, int32_t nb, double w_b, double h_b, double radius, int32_t kc,
                           float ratio, int64_t* d_q, int64_t* d_t, int32_t* n_out) {
    FSB_ARG(ctx && n_out, "null pointer");
    FSB_ARG(na >= 0 && nb >= 0, "negative size");
    FSB_ARG((na == 0 || (d_a && d_pred && d_q && d_t)) && (nb == 0 || (d_b && d_bxy)), "null array");
    FSB_ARG(std::isfinite(radius) && std::isfinite(w_b) && std::isfinite(h_b), "non-finite frame or radius");
    *n_out = 0;
    if (na == 0 || nb == 0 || !(radius > 0.0)) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    FSB_TRY(ctx->s_count.ensure(64));
    int* dn = ctx->s_count.as<int>();
    ctx->stage_begin(ST_MATCH);
    FSB_TRY(run_match_guided(ctx, d_pred, d_a, na, d_bxy, d_b, nb, w_b, h_b, radius, kc, ratio, d_q, d_t, dn, s));
    int n = 0;
    FSB_CUDA(cudaMemcpyAsync(&n, dn, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    ctx->stage_end(ST_MATCH);
    *n_out = n;
    return FSB_OK;
}

int32_t fsb_match_bf_d(fsb_ctx* ctx, const uint8_t* d_a, int32_t na, const uint8_t* d_b, int32_t nb, float ratio,
                       int32_t precision, int64_t* d_q, int64_t* d_t, int32_t* n_out) {
    FSB_ARG(ctx && n_out, "null pointer");
    FSB_ARG(na >= 0 && nb >= 0, "negative size");
    FSB_ARG((na == 0 || (d_a && d_q && d_t)) && (nb == 0 || d_b), "null array");
    FSB_ARG(precision >= FSB_PREC_FP32 && precision <= FSB_PREC_FP8, "unknown precision");
    *n_out = 0;
    if (na < 2 || nb < 2) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    FSB_TRY(ctx->s_count.ensure(64));
    int* dn = ctx->s_count.as<int>();
    ctx->stage_begin(ST_MATCH);
    FSB_TRY(run_match_bf(ctx, d_a, na, d_b, nb, ratio, precision, d_q, d_t, dn, s));
    int n = 0;
    FSB_CUDA(cudaMemcpyAsync(&n, dn, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    ctx->stage_end(ST_MATCH);
    *n_out = n;
    return FSB_OK;
}

int32_t fsb_match_bf_batch_d(fsb_ctx* ctx, int32_t n_pairs, const uint8_t* const* d_a, const int32_t* na,
                             const uint8_t* const* d_b, const int32_t* nb, float ratio, int32_t precision,
                             int64_t* const* d_q, int64_t* const* d_t, int32_t* n_out) {
    FSB_ARG(ctx && n_out && n_pairs >= 0, "bad arguments");
    FSB_ARG(n_pairs == 0 || (d_a && na && d_b && nb && d_q && d_t), "null array");
    FSB_ARG(precision >= FSB_PREC_FP32 && precision <= FSB_PREC_FP8, "unknown precision");
    for (int p = 0; p < n_pairs; ++p) {
        FSB_ARG(na[p] >= 0 && nb[p] >= 0, "negative size");
        FSB_ARG((na[p] == 0 || (d_a[p] && d_q[p] && d_t[p])) && (nb[p] == 0 || d_b[p]), "null array");
        n_out[p] = 0;
    }
    if (n_pairs == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    std::vector<int> live;
    for (int p = 0; p < n_pairs; ++p)
        if (na[p] >= 2 && nb[p] >= 2) live.push_back(p);
    if (live.empty()) return FSB_OK;
    ctx->stage_begin(ST_MATCH);
    std::vector<int> cnt(n_pairs, 0);
    FSB_TRY(ctx->s_count.ensure((size_t)n_pairs * 4 + 64));
    int* dn_all = ctx->s_count.as<int>();
    FSB_CUDA(cudaMemsetAsync(dn_all, 0, (size_t)n_pairs * 4, s));
    if (precision == FSB_PREC_FP32) {
        for (int p : live)
            FSB_TRY(run_match_bf(ctx, d_a[p], na[p], d_b[p], nb[p], ratio, precision, d_q[p], d_t[p], dn_all + p, s));
    } else {
        std::vector<const uint8_t*> pa, pb;
        std::vector<int64_t*> pq, pt;
        std::vector<int> ra, rb;
        for (int p : live) {
            pa.push_back(d_a[p]);
            pb.push_back(d_b[p]);
            pq.push_back(d_q[p]);
            pt.push_back(d_t[p]);
            ra.push_back(na[p]);
            rb.push_back(nb[p]);
        }
        int32_t* dn_live = dn_all;
        FSB_TRY(run_match_bf_tc(ctx, (int)live.size(), pa.data(), ra.data(), pb.data(), rb.data(), ratio, precision,
                                pq.data(), pt.data(), dn_live, &ctx->tc_stats, s));
        std::vector<int> cl(live.size(), 0);
        FSB_CUDA(cudaMemcpyAsync(cl.data(), dn_live, cl.size() * 4, cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaStreamSynchronize(s));
        for (size_t i = 0; i < live.size(); ++i) cnt[live[i]] = cl[i];
        ctx->stage_end(ST_MATCH);
        for (int p = 0; p < n_pairs; ++p) n_out[p] = cnt[p];
        return FSB_OK;
    }
    FSB_CUDA(cudaMemcpyAsync(cnt.data(), dn_all, (size_t)n_pairs * 4, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    ctx->stage_end(ST_MATCH);
    for (int p = 0; p < n_pairs; ++p) n_out[p] = cnt[p];
    return FSB_OK;
}

int32_t fsb_match_tc_stats(fsb_ctx* ctx, int64_t* rows, int64_t* fallback_rows, double* max_abs_err,
                           double* mean_abs_err) {
    FSB_ARG(ctx, "ctx is null");
    if (rows) *rows = ctx->tc_stats.rows;
    if (fallback_rows) *fallback_rows = ctx->tc_stats.fallback_rows;
    if (max_abs_err) *max_abs_err = ctx->tc_stats.max_abs_err;
    if (mean_abs_err) *mean_abs_err = ctx->tc_stats.mean_abs_err;
    return FSB_OK;
}

int32_t fsb_match_guided_cand_d(fsb_ctx* ctx, const double* d_pred, const uint8_t* d_a, int32_t na,
                                const double* d_bxy, const uint8_t* d_b, int32_t nb, double w_b, double h_b,
                                double radius, int32_t kc, int32_t* d_t1, float* d_b12) {
    FSB_ARG(ctx, "null pointer");
    FSB_ARG(na >= 0 && nb >= 0, "negative size");
    FSB_ARG((na == 0 || (d_a && d_pred && d_t1 && d_b12)) && (nb == 0 || (d_b && d_bxy)), "null array");
    FSB_ARG(std::isfinite(radius) && std::isfinite(w_b) && std::isfinite(h_b), "non-finite frame or radius");
    if (na == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    ctx->stage_begin(ST_MATCH);
    FSB_TRY(run_match_guided(ctx, d_pred, d_a, na, d_bxy, d_b, nb, w_b, h_b, radius, kc, 1.f, nullptr, nullptr,
                             nullptr, s, d_t1, d_b12));
    FSB_CUDA(cudaStreamSynchronize(s));
    ctx->stage_end(ST_MATCH);
    return FSB_OK;
}

int32_t fsb_match_guided_batch_d(fsb_ctx* ctx, int32_t n_pairs, const double* const* d_pred, const uint8_t* const* d_a,
                                 const int32_t* na, const double* const* d_bxy, const uint8_t* const* d_b,
                                 const int32_t* nb, const double* w_b, const double* h_b, double radius, int32_t kc,
                                 float ratio, int64_t* const* d_q, int64_t* const* d_t, int32_t* n_out) {
    FSB_ARG(ctx && n_out && n_pairs >= 0, "bad arguments");
    FSB_ARG(n_pairs == 0 || (d_pred && d_a && na && d_bxy && d_b && nb && w_b && h_b && d_q && d_t), "null array");
    FSB_ARG(std::isfinite(radius), "non-finite radius");
    std::vector<int> live;
    for (int p = 0; p < n_pairs; ++p) {
        FSB_ARG(na[p] >= 0 && nb[p] >= 0, "negative size");
        FSB_ARG(na[p] == 0 || (d_a[p] && d_pred[p] && d_q[p] && d_t[p]), "null array");
        FSB_ARG(nb[p] == 0 || (d_b[p] && d_bxy[p]), "null array");
        FSB_ARG(std::isfinite(w_b[p]) && std::isfinite(h_b[p]), "non-finite frame");
        n_out[p] = 0;
        if (na[p] > 0 && nb[p] > 0 && radius > 0.0) live.push_back(p);
    }
    if (live.empty()) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    const size_t L = live.size();
    std::vector<const double*> pr(L), bx(L);
    std::vector<const uint8_t*> pa(L), pb(L);
    std::vector<int> ra(L), rb(L);
    std::vector<double> wv(L), hv(L);
    std::vector<int64_t*> pq(L), pt(L);
    for (size_t i = 0; i < L; ++i) {
        const int p = live[i];
        pr[i] = d_pred[p];
        pa[i] = d_a[p];
        ra[i] = na[p];
        bx[i] = d_bxy[p];
        pb[i] = d_b[p];
        rb[i] = nb[p];
        wv[i] = w_b[p];
        hv[i] = h_b[p];
        pq[i] = d_q[p];
        pt[i] = d_t[p];
    }
    FSB_TRY(ctx->s_count.ensure(L * 4 + 64));
    int32_t* dn = ctx->s_count.as<int32_t>();
    ctx->stage_begin(ST_MATCH);
    FSB_TRY(run_match_guided_batch(ctx, (int)L, pr.data(), pa.data(), ra.data(), bx.data(), pb.data(), rb.data(),
                                   wv.data(), hv.data(), radius, kc, ratio, pq.data(), pt.data(), dn, s));
    std::vector<int> cnt(L, 0);
    FSB_CUDA(cudaMemcpyAsync(cnt.data(), dn, L * 4, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    ctx->stage_end(ST_MATCH);
    for (size_t i = 0; i < L; ++i) n_out[live[i]] = cnt[i];
    return FSB_OK;
}

int32_t fsb_mlp_param_count(void) { return mlp_param_count(); }
int32_t fsb_mlp_trainable_count(void) { return mlp_trainable_count(); }

int32_t fsb_mlp_features_d(fsb_ctx* ctx, int32_t n, const int32_t* d_t1, const float* d_b12, const double* d_pred,
                           const float* d_xy_b, const float* d_size_a, const float* d_angle_a, const float* d_resp_a,
                           const int32_t* d_oct_a, const float* d_size_b, const float* d_angle_b,
                           const float* d_resp_b, float radius, float* d_feat) {
    FSB_ARG(ctx && n >= 0, "bad arguments");
    FSB_ARG(n == 0 || (d_t1 && d_b12 && d_pred && d_xy_b && d_size_a && d_angle_a && d_resp_a && d_oct_a && d_size_b &&
                       d_angle_b && d_resp_b && d_feat), "null array");
    FSB_ARG(radius > 0.f, "radius must be positive");
    if (n == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    FSB_TRY(run_mlp_features(n, d_t1, d_b12, d_pred, d_xy_b, d_size_a, d_angle_a, d_resp_a, d_oct_a, d_size_b,
                             d_angle_b, d_resp_b, radius, d_feat, ctx->stream));
    FSB_CUDA(cudaStreamSynchronize(ctx->stream));
    return FSB_OK;
}

int32_t fsb_mlp_grad_d(fsb_ctx* ctx, const float* d_params, int32_t n, const float* d_feat, const float* d_label,
                       float* d_grad, double* loss) {
    FSB_ARG(ctx && d_params && d_grad && n > 0 && d_feat && d_label, "bad arguments");
    FSB_TRY(use_device(ctx));
    return run_mlp_grad(ctx, d_params, n, d_feat, d_label, d_grad, loss, ctx->stream);
}

int32_t fsb_mlp_train_d(fsb_ctx* ctx, float* d_params, float* d_m, float* d_v, int32_t n, const float* d_feat,
                        const float* d_label, int32_t epochs, int32_t batch, float lr, uint32_t seed, double* losses) {
    FSB_ARG(ctx && d_params && d_m && d_v && d_feat && d_label, "null pointer");
    FSB_ARG(n > 0 && epochs >= 0 && batch > 0 && lr > 0.f, "bad training arguments");
    FSB_TRY(use_device(ctx));
    return run_mlp_train(ctx, d_params, d_m, d_v, n, d_feat, d_label, epochs, batch, lr, seed, losses, ctx->stream);
}

int32_t fsb_mlp_infer_d(fsb_ctx* ctx, const float* d_params, int32_t n, const float* d_feat, int32_t bf16,
                        float* d_prob) {
    FSB_ARG(ctx && d_params && n >= 0 && (n == 0 || (d_feat && d_prob)), "bad arguments");
    if (n == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    FSB_TRY(run_mlp_infer(d_params, n, d_feat, bf16 != 0, d_prob, ctx->stream));
    FSB_CUDA(cudaStreamSynchronize(ctx->stream));
    return FSB_OK;
}

int32_t fsb_mlp_filter_d(fsb_ctx* ctx, int32_t na, const int32_t* d_t1, const float* d_b12, const float* d_prob,
                         float threshold, float ratio, int32_t nb, int64_t* d_q, int64_t* d_t, int32_t* n_out) {
    FSB_ARG(ctx && n_out && na >= 0 && nb >= 0, "bad arguments");
    FSB_ARG(na == 0 || (d_t1 && d_b12 && d_q && d_t), "null array");
    *n_out = 0;
    if (na == 0 || nb == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    FSB_TRY(ctx->s_i32.ensure((size_t)na * 8 + 64));
    int32_t* t_row = ctx->s_i32.as<int32_t>();
    uint32_t* d_row = reinterpret_cast<uint32_t*>(t_row + na);
    FSB_TRY(ctx->s_count.ensure(64));
    int* dn = ctx->s_count.as<int>();
    FSB_TRY(run_mlp_accept(na, d_t1, d_b12, d_prob, threshold, ratio, t_row, d_row, s));
    FSB_TRY(run_unique_rows(ctx, t_row, d_row, na, nb, d_q, d_t, dn, s));
    int n = 0;
    FSB_CUDA(cudaMemcpyAsync(&n, dn, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    *n_out = n;
    return FSB_OK;
}

int64_t fsb_launch_count(void) { return fsb::g_launches.load(); }

int32_t fsb_timing(fsb_ctx* ctx, int32_t on) {
    FSB_ARG(ctx, "ctx is null");
    FSB_TRY(use_device(ctx));
    // events for the stage marks are created here, not inside the timed pipeline
    if (on)
        while (ctx->ev_free.size() < 1024) {
            cudaEvent_t e = nullptr;
            FSB_CUDA(cudaEventCreate(&e));
            ctx->ev_free.push_back(e);
        }
    ctx->timing = on != 0;
    return FSB_OK;
}

int32_t fsb_stage_times(fsb_ctx* ctx, double* ms, int64_t* calls, int32_t n) {
    FSB_ARG(ctx && n >= 0, "bad arguments");
    FSB_TRY(use_device(ctx));
    ctx->stage_resolve(0);
    for (int i = 0; i < n && i < ST_COUNT; ++i) {
        if (ms) ms[i] = ctx->stage_ms[i];
        if (calls) calls[i] = ctx->stage_n[i];
    }
    for (int i = 0; i < ST_COUNT; ++i) {
        ctx->stage_ms[i] = 0.0;
        ctx->stage_n[i] = 0;
    }
    return FSB_OK;
}

int32_t fsb_match_bf(fsb_ctx* ctx, const uint8_t* a, int32_t na, const uint8_t* b, int32_t nb, float ratio,
                     int32_t precision, int64_t* q, int64_t* t, int32_t* n_out) {
    FSB_ARG(ctx && n_out, "null pointer");
    FSB_ARG(na >= 0 && nb >= 0, "negative size");
    FSB_ARG((na == 0 || a) && (nb == 0 || b), "null descriptor array");
    FSB_ARG(na == 0 || (q && t), "null output array");
    FSB_ARG(precision >= FSB_PREC_FP32 && precision <= FSB_PREC_FP8, "unknown precision");
    *n_out = 0;
    if (na < 2 || nb < 2) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    FSB_TRY(to_dev(ctx->s_u8a, a, (size_t)na * 128, s));
    FSB_TRY(to_dev(ctx->s_u8b, b, (size_t)nb * 128, s));
    FSB_TRY(ctx->s_i64.ensure((size_t)na * 16 + 64));
    int64_t* dq = ctx->s_i64.as<int64_t>();
    int64_t* dt = dq + na;
    FSB_TRY(ctx->s_count.ensure(64));
    int* dn = ctx->s_count.as<int>();
    FSB_TRY(run_match_bf(ctx, ctx->s_u8a.as<uint8_t>(), na, ctx->s_u8b.as<uint8_t>(), nb, ratio, precision, dq, dt,
                         dn, s));
    int n = 0;
    FSB_CUDA(cudaMemcpyAsync(&n, dn, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    if (n) {
        FSB_CUDA(cudaMemcpyAsync(q, dq, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaMemcpyAsync(t, dt, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaStreamSynchronize(s));
    }
    *n_out = n;
    return FSB_OK;
}

int32_t fsb_match_guided(fsb_ctx* ctx, const double* pred_xy, const uint8_t* a, int32_t na, const double* b_xy,
                         const uint8_t* b, int32_t nb, double w_b, double h_b, double radius, int32_t kc,
                         float ratio, int64_t* q, int64_t* t, int32_t* n_out) {
    FSB_ARG(ctx && n_out, "null pointer");
    FSB_ARG(na >= 0 && nb >= 0, "negative size");
    FSB_ARG((na == 0 || (a && pred_xy && q && t)) && (nb == 0 || (b && b_xy)), "null array");
    FSB_ARG(std::isfinite(radius) && std::isfinite(w_b) && std::isfinite(h_b), "non-finite frame or radius");
    *n_out = 0;
    if (na == 0 || nb == 0 || !(radius > 0.0)) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    FSB_TRY(ctx->s_u8a.ensure((size_t)na * 128 + 16));
    FSB_TRY(ctx->s_u8b.ensure((size_t)nb * 128 + 16));
    FSB_TRY(ctx->s_f32a.ensure((size_t)(na + nb) * 16 + 256));
    double* dp = ctx->s_f32a.as<double>();
    double* dbx = dp + 2 * (size_t)na;
    const HostCopy in[4] = {{(void*)a, ctx->s_u8a.p, (size_t)na * 128},
                            {(void*)b, ctx->s_u8b.p, (size_t)nb * 128},
                            {(void*)pred_xy, dp, (size_t)na * 16},
                            {(void*)b_xy, dbx, (size_t)nb * 16}};
    FSB_TRY(copy_in(ctx, in, 4));
    FSB_TRY(ctx->s_i64.ensure((size_t)na * 16 + 64));
    int64_t* dq = ctx->s_i64.as<int64_t>();
    int64_t* dt = dq + na;
    FSB_TRY(ctx->s_count.ensure(64));
    int* dn = ctx->s_count.as<int>();
    FSB_TRY(run_match_guided(ctx, dp, ctx->s_u8a.as<uint8_t>(), na, dbx, ctx->s_u8b.as<uint8_t>(), nb, w_b, h_b, radius,
                             kc, ratio, dq, dt, dn, s));
    int n = 0;
    FSB_CUDA(cudaMemcpyAsync(&n, dn, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    const HostCopy out[2] = {{q, dq, (size_t)n * 8}, {t, dt, (size_t)n * 8}};
    FSB_TRY(copy_out(ctx, out, n ? 2 : 0));
    *n_out = n;
    return FSB_OK;
}

int32_t fsb_unique(fsb_ctx* ctx, const int64_t* q, const int64_t* t, const float* dd, int32_t n, int64_t* q_out,
                   int64_t* t_out, int32_t* n_out) {
    FSB_ARG(ctx && n_out, "null pointer");
    FSB_ARG(n >= 0 && (n == 0 || (q && t && dd && q_out && t_out)), "bad arrays");
    *n_out = 0;
    if (n == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    FSB_TRY(ctx->s_i64.ensure((size_t)n * 8 * 4 + (size_t)n * 4 + 64));
    int64_t* dq = ctx->s_i64.as<int64_t>();
    int64_t* dt = dq + n;
    int64_t* dqo = dt + n;
    int64_t* dto = dqo + n;
    float* ddd = reinterpret_cast<float*>(dto + n);
    FSB_TRY(ctx->s_count.ensure(64));
    int* dn = ctx->s_count.as<int>();
    FSB_CUDA(cudaMemcpyAsync(dq, q, (size_t)n * 8, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(dt, t, (size_t)n * 8, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(ddd, dd, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    FSB_TRY(run_unique_general(ctx, dq, dt, ddd, n, dqo, dto, dn, s));
    int m = 0;
    FSB_CUDA(cudaMemcpyAsync(&m, dn, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    if (m) {
        FSB_CUDA(cudaMemcpyAsync(q_out, dqo, (size_t)m * 8, cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaMemcpyAsync(t_out, dto, (size_t)m * 8, cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaStreamSynchronize(s));
    }
    *n_out = m;
    return FSB_OK;
}

int32_t fsb_build_tracks(fsb_ctx* ctx, const int64_t* u, const int64_t* v, int64_t n_edges, const int64_t* offsets,
                         int32_t n_img, int64_t* tid, int64_t* img, int64_t* feat, int64_t* n_obs, int64_t* n_tracks) {
    FSB_ARG(ctx && offsets && n_obs && n_tracks, "null pointer");
    FSB_ARG(n_img >= 1 && n_edges >= 0, "bad sizes");
    FSB_ARG(n_edges == 0 || (u && v && tid && img && feat), "null edge or output pointer");
    for (int i = 0; i < n_img; ++i) FSB_ARG(offsets[i] >= 0 && offsets[i] <= offsets[i + 1], "offsets must ascend");
    const long long T = offsets[n_img];
    FSB_ARG(T < (1ll << 31) - 1, "at most 2^31 - 2 features in all");
    for (int64_t e = 0; e < n_edges; ++e) FSB_ARG(u[e] >= 0 && u[e] < T && v[e] >= 0 && v[e] < T, "node out of range");
    *n_obs = 0;
    *n_tracks = 0;
    if (n_edges == 0 || T == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    const size_t E = (size_t)n_edges;
    FSB_TRY(ctx->s_i64.ensure(E * 16 + (size_t)(n_img + 1) * 8 + 64));
    FSB_TRY(ctx->s_u64.ensure(E * 48 + 64));
    long long* du = ctx->s_i64.as<long long>();
    long long* dv = du + E;
    long long* doff = dv + E;
    long long* dtid = ctx->s_u64.as<long long>();
    long long* dimg = dtid + 2 * E;
    long long* dfeat = dimg + 2 * E;
    FSB_CUDA(cudaMemcpyAsync(du, u, E * 8, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(dv, v, E * 8, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(doff, offsets, (size_t)(n_img + 1) * 8, cudaMemcpyHostToDevice, s));
    int no = 0, nt = 0;
    FSB_TRY(run_build_tracks(ctx, du, dv, n_edges, doff, n_img, (int)T, dtid, dimg, dfeat, &no, &nt, s));
    if (no) {
        FSB_CUDA(cudaMemcpyAsync(tid, dtid, (size_t)no * 8, cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaMemcpyAsync(img, dimg, (size_t)no * 8, cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaMemcpyAsync(feat, dfeat, (size_t)no * 8, cudaMemcpyDeviceToHost, s));
    }
    FSB_CUDA(cudaStreamSynchronize(s));
    *n_obs = no;
    *n_tracks = nt;
    return FSB_OK;
}

int32_t fsb_find_homography_batch(fsb_ctx* ctx, int32_t n_pairs, const int64_t* offsets, const double* src,
                                  const double* dst, double thr, int32_t iters, uint64_t seed, double* H, uint8_t* mask,
                                  int32_t* n_inliers) {
    FSB_ARG(ctx && offsets && H && n_inliers, "null pointer");
    FSB_ARG(n_pairs >= 0 && iters >= 1 && iters <= (1 << 20) && thr > 0.0, "bad arguments");
    FSB_ARG(offsets[0] == 0, "offsets must start at 0");
    for (int p = 0; p < n_pairs; ++p) FSB_ARG(offsets[p + 1] >= offsets[p], "offsets must ascend");
    if (n_pairs == 0) return FSB_OK;
    const size_t N = (size_t)offsets[n_pairs];
    FSB_ARG(N == 0 || (src && dst && mask), "null point or mask array");
    FSB_TRY(use_device(ctx));
    FSB_TRY(ctx->s_f32a.ensure(N * 32 + 256));
    FSB_TRY(ctx->s_i64.ensure((size_t)(n_pairs + 1) * 8 + 256));
    FSB_TRY(ctx->s_f32b.ensure((size_t)n_pairs * 76 + N + 512));
    double* dsrc = ctx->s_f32a.as<double>();
    double* ddst = dsrc + 2 * N;
    long long* doff = ctx->s_i64.as<long long>();
    double* dH = ctx->s_f32b.as<double>();
    int* dn = reinterpret_cast<int*>(dH + 9 * (size_t)n_pairs);
    uint8_t* dm = reinterpret_cast<uint8_t*>(dn + n_pairs);
    const HostCopy in[3] = {{(void*)src, dsrc, N * 16}, {(void*)dst, ddst, N * 16},
                            {(void*)offsets, doff, (size_t)(n_pairs + 1) * 8}};
    FSB_TRY(copy_in(ctx, in, 3));
    FSB_TRY(run_ransac_h(doff, n_pairs, reinterpret_cast<const double2*>(dsrc), reinterpret_cast<const double2*>(ddst),
                         thr, iters, seed, dH, dm, dn, ctx->stream));
    const HostCopy out[3] = {{H, dH, (size_t)n_pairs * 72}, {n_inliers, dn, (size_t)n_pairs * 4}, {mask, dm, N}};
    return copy_out(ctx, out, 3);
}

int32_t fsb_find_fundamental_batch(fsb_ctx* ctx, int32_t n_pairs, const int64_t* offsets, const double* src,
                                   const double* dst, double thr, int32_t iters, uint64_t seed, double* F, uint8_t* mask,
                                   int32_t* n_inliers) {
    FSB_ARG(ctx && offsets && F && n_inliers, "null pointer");
    FSB_ARG(n_pairs >= 0 && iters >= 1 && iters <= (1 << 20) && thr > 0.0, "bad arguments");
    FSB_ARG(offsets[0] == 0, "offsets must start at 0");
    for (int p = 0; p < n_pairs; ++p) FSB_ARG(offsets[p + 1] >= offsets[p], "offsets must ascend");
    if (n_pairs == 0) return FSB_OK;
    const size_t N = (size_t)offsets[n_pairs];
    FSB_ARG(N == 0 || (src && dst && mask), "null point or mask array");
    FSB_TRY(use_device(ctx));
    FSB_TRY(ctx->s_f32a.ensure(N * 32 + 256));
    FSB_TRY(ctx->s_i64.ensure((size_t)(n_pairs + 1) * 8 + 256));
    FSB_TRY(ctx->s_f32b.ensure((size_t)n_pairs * 76 + N + 512));
    double* dsrc = ctx->s_f32a.as<double>();
    double* ddst = dsrc + 2 * N;
    long long* doff = ctx->s_i64.as<long long>();
    double* dF = ctx->s_f32b.as<double>();
    int* dn = reinterpret_cast<int*>(dF + 9 * (size_t)n_pairs);
    uint8_t* dm = reinterpret_cast<uint8_t*>(dn + n_pairs);
    const HostCopy in[3] = {{(void*)src, dsrc, N * 16}, {(void*)dst, ddst, N * 16},
                            {(void*)offsets, doff, (size_t)(n_pairs + 1) * 8}};
    FSB_TRY(copy_in(ctx, in, 3));
    FSB_TRY(run_ransac_f(doff, n_pairs, reinterpret_cast<const double2*>(dsrc), reinterpret_cast<const double2*>(ddst),
                         thr, iters, seed, dF, dm, dn, ctx->stream));
    const HostCopy out[3] = {{F, dF, (size_t)n_pairs * 72}, {n_inliers, dn, (size_t)n_pairs * 4}, {mask, dm, N}};
    return copy_out(ctx, out, 3);
}

int32_t fsb_spread(fsb_ctx* ctx, const float* x, const float* y, const float* resp, int32_t n, int32_t W, int32_t H,
                   int32_t nfeat, int32_t order, int32_t* sel, int32_t* n_out) {
    FSB_ARG(ctx && n_out, "null pointer");
    FSB_ARG(n >= 0 && nfeat >= 0, "negative size");
    FSB_ARG(n <= (1 << 30), "at most 2^30 keypoints");
    FSB_ARG(W > 0 && H > 0, "image size must be positive");
    FSB_ARG(order == FSB_SPREAD_SELECTION || order == FSB_SPREAD_RESPONSE, "order must be 0 or 1");
    FSB_ARG(n == 0 || (x && y && resp && sel), "null keypoint or output array");
    *n_out = 0;
    for (int32_t i = 1; i < n; ++i)
        FSB_ARG(resp[i] <= resp[i - 1], "keypoints must be in response-descending order (as detect returns them)");
    if (n == 0 || nfeat == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    const size_t N = (size_t)n;
    FSB_TRY(ctx->s_f32b.ensure(al256(N * 4) * 3));
    FSB_TRY(ctx->s_i32.ensure(N * 4 + 256));
    float* dx = ctx->s_f32b.as<float>();
    float* dy = dx + al256(N * 4) / 4;
    float* dr = dy + al256(N * 4) / 4;
    int32_t* ds = ctx->s_i32.as<int32_t>();
    const HostCopy in[3] = {{(void*)x, dx, N * 4}, {(void*)y, dy, N * 4}, {(void*)resp, dr, N * 4}};
    FSB_TRY(copy_in(ctx, in, 3));
    int n_sel = 0;
    FSB_TRY(spread_dev(ctx, dx, dy, dr, n, (float)W, (float)H, nfeat, order == FSB_SPREAD_SELECTION, ds, &n_sel,
                       ctx->stream));
    const HostCopy out[1] = {{sel, ds, (size_t)n_sel * 4}};
    FSB_TRY(copy_out(ctx, out, 1));
    *n_out = n_sel;
    return FSB_OK;
}

int32_t fsb_decode_gray_d(fsb_ctx* ctx, const uint8_t* data, int64_t len, int32_t reduce, uint8_t* d_out,
                          int64_t out_cap, int32_t* h, int32_t* w) {
    FSB_ARG(ctx && data && d_out && h && w, "null pointer");
    FSB_ARG(len > 0 && out_cap > 0, "empty buffer");
    FSB_ARG(reduce == 1 || reduce == 2 || reduce == 4 || reduce == 8, "reduce must be 1, 2, 4 or 8");
    FSB_TRY(use_device(ctx));
    return run_jpeg_gray(ctx, data, (size_t)len, reduce, d_out, (size_t)out_cap, h, w);
}

int32_t fsb_prepare_gray(fsb_ctx* ctx, const uint8_t* data, int64_t len, int32_t reduce, double clip, uint8_t* out,
                         int64_t out_cap, int32_t* h, int32_t* w) {
    FSB_ARG(ctx && data && out && h && w, "null pointer");
    FSB_ARG(len > 0 && out_cap > 0, "empty buffer");
    FSB_ARG(reduce == 1 || reduce == 2 || reduce == 4 || reduce == 8, "reduce must be 1, 2, 4 or 8");
    FSB_TRY(use_device(ctx));
    // decoded plane, then its equalised copy, in one scratch buffer
    const size_t cap = (size_t)out_cap;
    FSB_TRY(ctx->s_u8a.ensure(2 * cap + 512));
    uint8_t* dg = ctx->s_u8a.as<uint8_t>();
    uint8_t* de = dg + ((cap + 255) & ~size_t(255));
    FSB_TRY(run_jpeg_gray(ctx, data, (size_t)len, reduce, dg, cap, h, w));
    FSB_TRY(ctx->s_misc.ensure(64 * 256));
    FSB_TRY(run_clahe(dg, *h, *w, *w, clip, 8, 8, ctx->s_misc.as<uint8_t>(), de, *w, ctx->stream));
    const HostCopy o[1] = {{out, de, (size_t)(*h) * (*w)}};
    return copy_out(ctx, o, 1);
}

int32_t fsb_clahe_d(fsb_ctx* ctx, const uint8_t* d_img, int32_t h, int32_t w, int32_t stride, double clip,
                    int32_t tiles_x, int32_t tiles_y, uint8_t* d_out, int32_t out_stride) {
    FSB_ARG(ctx && d_img && d_out, "null pointer");
    FSB_ARG(h > 0 && w > 0 && stride >= w && out_stride >= w, "bad image size");
    FSB_ARG(tiles_x >= 1 && tiles_y >= 1 && tiles_x * tiles_y <= 256, "tiles must be 1..256 in all");
    FSB_TRY(use_device(ctx));
    FSB_TRY(ctx->s_misc.ensure((size_t)tiles_x * tiles_y * 256));
    return run_clahe(d_img, h, w, stride, clip, tiles_x, tiles_y, ctx->s_misc.as<uint8_t>(), d_out, out_stride,
                     ctx->stream);
}

int32_t fsb_clahe(fsb_ctx* ctx, const uint8_t* img, int32_t h, int32_t w, int32_t stride, double clip,
                  int32_t tiles_x, int32_t tiles_y, uint8_t* out, int32_t out_stride) {
    FSB_ARG(ctx && img && out, "null pointer");
    FSB_ARG(h > 0 && w > 0 && stride >= w && out_stride >= w, "bad image size");
    FSB_ARG(tiles_x >= 1 && tiles_y >= 1 && tiles_x * tiles_y <= 256, "tiles must be 1..256 in all");
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)h * w;
    FSB_TRY(ctx->s_u8a.ensure(2 * n + 64));
    uint8_t* din = ctx->s_u8a.as<uint8_t>();
    uint8_t* dout = din + ((n + 63) & ~size_t(63));
    FSB_CUDA(cudaMemcpy2DAsync(din, (size_t)w, img, (size_t)stride, (size_t)w, (size_t)h, cudaMemcpyHostToDevice, s));
    FSB_TRY(ctx->s_misc.ensure((size_t)tiles_x * tiles_y * 256));
    FSB_TRY(run_clahe(din, h, w, w, clip, tiles_x, tiles_y, ctx->s_misc.as<uint8_t>(), dout, w, s));
    FSB_CUDA(cudaMemcpy2DAsync(out, (size_t)out_stride, dout, (size_t)w, (size_t)w, (size_t)h, cudaMemcpyDeviceToHost,
                               s));
    FSB_CUDA(cudaStreamSynchronize(s));
    return FSB_OK;
}

int32_t fsb_undistort_pixels(fsb_ctx* ctx, const double* uv, int32_t n, const double* k8, double* out) {
    FSB_ARG(ctx && k8, "null pointer");
    FSB_ARG(n >= 0 && (n == 0 || (uv && out)), "bad points");
    FSB_ARG(k8[0] != 0.0, "focal length 0");
    if (n == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    FSB_TRY(ctx->s_f32a.ensure((size_t)n * 32 + 256));
    double* du = ctx->s_f32a.as<double>();
    double* dout = du + 2 * (size_t)n;
    FSB_CUDA(cudaMemcpyAsync(du, uv, (size_t)n * 16, cudaMemcpyHostToDevice, s));
    FSB_TRY(run_undistort(du, n, k8, dout, s));
    FSB_CUDA(cudaMemcpyAsync(out, dout, (size_t)n * 16, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    return FSB_OK;
}

int32_t fsb_predict_ground(fsb_ctx* ctx, const double* u, int32_t n, const double* kinv_i, const double* r_i,
                           const double* c_i, const double* k_j, const double* r_j, const double* c_j, double zg,
                           double* pred, uint8_t* ok) {
    FSB_ARG(ctx && kinv_i && r_i && c_i && k_j && r_j && c_j, "null pointer");
    FSB_ARG(n >= 0 && (n == 0 || (u && pred && ok)), "bad points");
    if (n == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    FSB_TRY(ctx->s_f32a.ensure((size_t)n * 33 + 256));
    double* du = ctx->s_f32a.as<double>();
    double* dp = du + 2 * (size_t)n;
    uint8_t* dok = reinterpret_cast<uint8_t*>(dp + 2 * (size_t)n);
    FSB_CUDA(cudaMemcpyAsync(du, u, (size_t)n * 16, cudaMemcpyHostToDevice, s));
    FSB_TRY(run_predict(du, n, kinv_i, r_i, c_i, k_j, r_j, c_j, zg, dp, dok, s));
    FSB_CUDA(cudaMemcpyAsync(pred, dp, (size_t)n * 16, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaMemcpyAsync(ok, dok, (size_t)n, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    return FSB_OK;
}

int32_t fsb_perspective(fsb_ctx* ctx, const double* xy, int32_t n, const double* hm9, double* out) {
    FSB_ARG(ctx && hm9, "null pointer");
    FSB_ARG(n >= 0 && (n == 0 || (xy && out)), "bad points");
    if (n == 0) return FSB_OK;
    FSB_TRY(use_device(ctx));
    cudaStream_t s = ctx->stream;
    FSB_TRY(ctx->s_f32a.ensure((size_t)n * 32 + 256));
    double* dx = ctx->s_f32a.as<double>();
    double* dout = dx + 2 * (size_t)n;
    FSB_TRY(ctx->s_misc.ensure(128));
    double* dh = ctx->s_misc.as<double>();
    FSB_CUDA(cudaMemcpyAsync(dx, xy, (size_t)n * 16, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(dh, hm9, 72, cudaMemcpyHostToDevice, s));
    FSB_TRY(run_perspective(dx, n, dh, dout, s));
    FSB_CUDA(cudaMemcpyAsync(out, dout, (size_t)n * 16, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    return FSB_OK;
}

}  // extern "C"
