// Internal declarations shared by the CUDA translation units of libfsb200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/fsb200.h"

namespace fsb {

// ---------------------------------------------------------------------------------- errors
void set_error(const char* fmt, ...);

// Count of kernel launches issued by this library (observability; read by fsb_launch_count).
void note_launch(int n = 1);
long long launch_mark();   // the running count of note_launch

// Per-stage device timers (CUDA events on the context stream), enabled by fsb_timing().
enum Stage { ST_UPLOAD = 0, ST_PYRAMID, ST_EXTREMA, ST_REFINE, ST_ORIENT, ST_SORT, ST_SPREAD, ST_DESCRIBE,
             ST_MATCH, ST_TC_DENSE, ST_COUNT };

#define FSB_CUDA(call)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            ::fsb::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),        \
                             __FILE__, __LINE__);                                           \
            return e_ == cudaErrorMemoryAllocation ? FSB_ERR_OOM : FSB_ERR_CUDA;           \
        }                                                                                   \
    } while (0)

#define FSB_TRY(expr)                   \
    do {                                \
        int32_t s_ = (expr);            \
        if (s_ != FSB_OK) return s_;    \
    } while (0)

#define FSB_ARG(cond, msg)                                  \
    do {                                                    \
        if (!(cond)) {                                      \
            ::fsb::set_error("invalid argument: %s", msg);  \
            return FSB_ERR_ARG;                             \
        }                                                   \
    } while (0)

// Raises a kernel's dynamic shared-memory limit to `bytes` on the current device once per device
// (`done` holds the largest value set, per device; two threads meeting a device first may both set
// it, which is harmless). carveout >= 0 also sets the preferred shared-memory carveout.
inline int32_t smem_attr(const void* func, int bytes, std::atomic<int> (&done)[64], int carveout = -1) {
    int dev = 0;
    FSB_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && done[dev].load(std::memory_order_acquire) >= bytes) return FSB_OK;
    FSB_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if (carveout >= 0) FSB_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout, carveout));
    if (dev >= 0 && dev < 64) done[dev].store(bytes, std::memory_order_release);
    return FSB_OK;
}

// ------------------------------------------------------------------------ SIFT constants
// app/planesite/gsift.py:13-25, 224
constexpr int N_LAYERS = 3;
constexpr float SIGMA = 1.6f;
constexpr int BORDER = 5;
constexpr int MAX_INTERP = 5;
constexpr int ORI_BINS = 36;
constexpr int ORI_SLOTS = ORI_BINS / 2;   // peaks of one extremum: local maxima of 36 circular bins
constexpr float ORI_RADIUS = 4.5f;
constexpr float ORI_SIG = 1.5f;
constexpr int ORI_R_MAX = 16;
constexpr int D_WIDTH = 4;
constexpr int D_BINS = 8;
constexpr int MAXO = 16;

// Octave geometry of one image: octave o is R[o] x C[o]; DoG layers 0..4 of octave o start at
// dog_off[o] in the DoG atlas, gradient layers 1..3 (magnitude and angle) at grad_off[o].
struct Geometry {
    int h, w, n_oct;
    int R[MAXO], C[MAXO];
    long long dog_off[MAXO + 1];
    long long grad_off[MAXO + 1];
};
Geometry make_geometry(int h, int w);

// A refined extremum (one per surviving candidate).
struct Refined {
    uint32_t f;     // flat DoG-atlas index of the originating extremum (sort tie-break)
    int16_t o, l;   // octave, layer 1..3 (after refinement)
    int32_t r, c;   // integer position after refinement
    float x0, x1, x2;  // sub-pixel offset (column, row, layer)
    float resp;     // |contrast| at the fitted position
};

// One orientation peak of a refined extremum.
struct Oriented {
    uint32_t ri;    // index into the Refined array
    int32_t j;      // histogram bin of the peak (0..35)
    float angle;    // degrees
};

// ------------------------------------------------------------------- device buffers
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int32_t ensure(size_t n);   // grows (never shrinks); contents are not preserved
    void release();
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// Capacities of the sync-free extraction (fixed per geometry and keypoint cap; an image that exceeds
// one is flagged and redone by the host-driven path).
struct AsyncCaps {
    uint32_t cand, ref, rank;   // extrema candidates, refined extrema (sorted), ranks oriented
    int kp, nfeat;              // keypoint cap (largest max_kp of the batch), features selected
};

// Outcome of one tensor-core dense match (all pairs of the call).
struct TcStats {
    long long rows = 0;            // query rows
    long long fallback_rows = 0;   // rows recomputed exactly because the certificate did not hold
    float max_abs_err = 0.f;       // |approximate - exact| best distance, largest over rows
    float mean_abs_err = 0.f;      // and its mean
};

// A captured guided-batch graph and the exact inputs it was captured for.
struct GuidedGraph {
    std::vector<char> key;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int n_kernels = 0;   // this library's kernels in the graph (counted per replay, not at capture)
};

// Pyramid + detection workspace sized for one image geometry.
struct Workspace {
    Geometry g{};
    DevBuf dog, mag, ang;        // atlases
    DevBuf plane[3];             // gauss-layer scratch planes (octave-0 size)
    DevBuf next_base;            // two octave-1-sized halves: the next octave's base, alternating
    DevBuf img;                  // uploaded uint8 image
    DevBuf cand, refined, oriented;
    DevBuf keys_a, keys_b, vals_a, vals_b, sort_tmp;
    DevBuf spread, take;         // sync-free extraction: spread scratch, selected keypoint fields
    DevBuf counters;             // [0] candidates, [1] refined, [2] oriented
    size_t cap_cand = 0, cap_ref = 0;
    // sorted, capped keypoints (structure of arrays)
    DevBuf kx, ky, ksize, kangle, kresp, koct, klayer;
    int n_kp = 0;
    size_t bytes() const;
    void release();
};

}  // namespace fsb

struct fsb_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;                  // pyramid: each octave's last layers overlap the next octave
    cudaEvent_t pyr_ev[2 * fsb::MAXO] = {};       // its fork / join events
    void* jpeg_handle = nullptr;                  // nvJPEG decoder of this context (created on first use)
    void* jpeg_state = nullptr;
    std::vector<fsb::Workspace*> pool;   // idle workspaces
    int live_states = 0;
    // scratch for description and matching (grown on demand)
    fsb::DevBuf s_u8a, s_u8b, s_f32a, s_f32b, s_i32, s_i64, s_u64, s_misc, s_misc2, s_host_stage;
    fsb::DevBuf s_cub;   // CUB temporary storage (one primitive at a time)
    fsb::DevBuf s_tc_pack, s_tc_part, s_tc_aux;   // tensor-core matcher: packed operands, candidates, tables
    fsb::DevBuf s_count;   // result counts of the API calls; never grown by the internal stages
    fsb::DevBuf s_gb;      // guided batch scratch (addresses captured in gb_graph)
    fsb::GuidedGraph gb_graph;
    fsb::TcStats tc_stats{};                      // of the last tensor-core dense match
    // sync-free batched extraction (fsb_sift_features_batch_d): chains of images, each with its own
    // stream and workspace, captured as one CUDA graph and replayed while the call is unchanged
    struct ExtractBatch {
        std::vector<cudaStream_t> streams;
        std::vector<fsb::Workspace*> ws;
        std::vector<cudaEvent_t> join;
        cudaEvent_t fork = nullptr;
        cudaStream_t upload = nullptr;            // host-image batches: the uploads, in image order
        std::vector<cudaEvent_t> uploaded;        // image i on the device (captured edges)
        std::vector<cudaGraphNode_t> copy_nodes;  // the upload of image i in the captured graph
        fsb::GuidedGraph graph;
        fsb::GuidedGraph pyr_graph;   // fsb_pyramid_batch_d
        int pyr_h = 0, pyr_w = 0;     // geometry whose pyramid ran once outside a capture (autotuned)
        fsb::DevBuf status;
        fsb::AsyncCaps caps{};
        int h = 0, w = 0, warm_ref = 0;
        long long redone = 0;   // images redone by the host-driven path
    } xb;
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    // stage timers: event pairs recorded at stage boundaries while timing is on, read back lazily
    // (when many are pending, and when the times are queried), so timing adds no host wait
    struct StageMark { int st; cudaEvent_t e0, e1; };
    bool timing = false;
    std::vector<cudaEvent_t> ev_free;
    std::vector<StageMark> ev_pending;
    cudaEvent_t ev_open[fsb::ST_COUNT] = {};
    double stage_ms[fsb::ST_COUNT] = {};
    long long stage_n[fsb::ST_COUNT] = {};
    void stage_begin(int st);
    void stage_end(int st);
    void stage_resolve(size_t keep);   // accumulates all but the newest `keep` pending pairs
    void stage_release();
};

struct fsb_state {
    fsb_ctx* ctx = nullptr;
    fsb::Workspace* ws = nullptr;
    uint32_t magic = 0;
    bool exact = false;   // detect ran with FSB_SIFT_EXACT_BLUR; describe uses float64 sample math
};

namespace fsb {
constexpr uint32_t STATE_MAGIC = 0x51f7b200u;

// ---------------------------------------------------------------- pyramid.cu
int32_t upload_taps();
// side / ev (2 MAXO events) may be null: then every octave runs on s alone
int32_t run_pyramid(Workspace& ws, const uint8_t* d_img, int img_stride, bool exact, cudaStream_t s,
                    cudaStream_t side = nullptr, cudaEvent_t* ev = nullptr);
// octave.cu
int32_t upload_octave_taps(const float* taps, int stride, const int* counts);
int32_t launch_octave_fused(const float* L0, int R, int C, float* dog, float* mag, float* ang, float* down,
                            int down_cols, cudaStream_t s);
int layer_tile_variants();
int layer_tile_height(int variant);
int32_t launch_layer_fast(int layer, const float* src, int R, int C, float* dst, float* dog, float* mag, float* ang,
                          float* down, int down_cols, int variant, int* err, cudaStream_t s);
int32_t launch_base_fast(const uint8_t* img, int stride, int ih, int iw, float* dst, int variant, cudaStream_t s);
int32_t launch_group_lower(const float* src, int R, int C, float* dog, float* mag, float* ang, float* l3, float* down,
                           int down_cols, cudaStream_t s);
int32_t launch_group_upper(const float* src, int R, int C, float* dog3, cudaStream_t s);
// strip engine: the whole float32 octave in one launch (err: device word set when a TMA wait gives up)
int32_t launch_octave_strip(const float* L0, int R, int C, float* dog, float* mag, float* ang, float* down,
                            int down_cols, int* err, cudaStream_t s);
constexpr int PYR_ERR_WORD = 8;   // index of the pyramid's error word in Workspace::counters
// autotune.cu: the fastest of n_variants launches of `run` for `key` (timed once per process and
// device on `s`, then cached; FSB_AUTOTUNE=0 returns variant 0, FSB_AUTOTUNE_FILE persists choices)
bool autotune_cached(const char* key, int n_variants, int* variant);
int32_t autotune(const char* key, int n_variants, int32_t (*run)(void*, int), void* arg, cudaStream_t s, int* variant);

// ---------------------------------------------------------------- detect.cu / describe.cu
int32_t run_orient(const Workspace& ws, const Refined* ref, const uint32_t* order, uint32_t k0, uint32_t k1,
                   Oriented* slots, uint32_t* cnt, uint32_t* d_total, bool exact, cudaStream_t s);
int32_t run_detect(fsb_ctx* ctx, Workspace& ws, double contrast, double edge, int max_kp, bool exact);
int32_t run_describe_mode(const Workspace& ws, int n, const float* d_x, const float* d_y, const float* d_size,
                          const float* d_angle, const int32_t* d_oct, const int32_t* d_layer, float* d_desc,
                          uint8_t* d_u8, bool exact, cudaStream_t s);
int32_t run_describe(const Workspace& ws, int n, const float* d_x, const float* d_y, const float* d_size,
                     const float* d_angle, const int32_t* d_oct, const int32_t* d_layer, float* d_desc,
                     uint8_t* d_u8, cudaStream_t s);
int32_t run_spread(const Workspace& ws, int nfeat, int32_t* d_sel, int* n_sel, fsb_ctx* ctx, cudaStream_t s);
// Sync-free extraction (every count on the device; stream-capturable). Capacities are fixed per
// geometry and keypoint cap; an image that exceeds one is flagged in counters[7] (ASYNC_*).
constexpr uint32_t ASYNC_CAND_OVERFLOW = 1, ASYNC_REF_OVERFLOW = 2, ASYNC_ORIENT_INCOMPLETE = 4;
constexpr int ASYNC_ORIENT_PASSES = 3;
int32_t async_caps(const Workspace& ws, int max_kp, int nfeat, AsyncCaps* c);
int32_t prepare_async(Workspace& ws, const AsyncCaps& c, cudaStream_t s);
// max_kp (<= c.kp) is this image's keypoint cap
int32_t run_detect_async(Workspace& ws, double contrast, double edge, const AsyncCaps& c, int max_kp, bool exact,
                         cudaStream_t s);
int32_t spread_async(Workspace& ws, const AsyncCaps& c, int nfeat, int32_t* d_sel, cudaStream_t s);
int32_t run_orient_dev(const Workspace& ws, const Refined* ref, const uint32_t* order, uint32_t max_ranks,
                       const uint32_t* d_range, Oriented* slots, uint32_t* cnt, uint32_t* d_total, bool exact,
                       cudaStream_t s);
int32_t run_describe_dev(const Workspace& ws, int cap, const int* d_n, const float* d_x, const float* d_y,
                         const float* d_size, const float* d_angle, const int32_t* d_oct, const int32_t* d_layer,
                         float* d_desc, uint8_t* d_u8, bool exact, cudaStream_t s);
int32_t spread_dev(fsb_ctx* ctx, const float* d_x, const float* d_y, const float* d_resp, int n, float W, float H,
                   int nfeat, bool by_position, int32_t* d_sel, int* n_sel, cudaStream_t s);

// ---------------------------------------------------------------- match.cu
int32_t run_match_bf(fsb_ctx* ctx, const uint8_t* d_a, int na, const uint8_t* d_b, int nb, float ratio,
                     int precision, int64_t* d_q, int64_t* d_t, int* d_n, cudaStream_t s);
// d_n null: candidates only (c_t, c_b12: best target or -1, b1, b2 per query; no ratio test, no _unique)
int32_t run_match_guided(fsb_ctx* ctx, const double* d_pred, const uint8_t* d_a, int na, const double* d_bxy,
                         const uint8_t* d_b, int nb, double wb, double hb, double radius, int kc, float ratio,
                         int64_t* d_q, int64_t* d_t, int* d_n, cudaStream_t s, int32_t* c_t = nullptr,
                         float* c_b12 = nullptr);
int32_t run_match_guided_batch(fsb_ctx* ctx, int n_pairs, const double* const* d_pred, const uint8_t* const* d_a,
                               const int* na, const double* const* d_bxy, const uint8_t* const* d_b, const int* nb,
                               const double* wb, const double* hb, double radius, int kc, float ratio,
                               int64_t* const* d_q, int64_t* const* d_t, int32_t* counts, cudaStream_t s);
int32_t run_unique_rows(fsb_ctx* ctx, const int32_t* t_row, const uint32_t* d_row, int na, int nb, int64_t* d_q,
                        int64_t* d_t, int* d_n, cudaStream_t s);
// mlp.cu
int mlp_param_count();
int mlp_trainable_count();
int32_t run_mlp_features(int n, const int32_t* t1, const float* b12, const double* pred, const float* xy_b,
                         const float* size_a, const float* angle_a, const float* resp_a, const int32_t* oct_a,
                         const float* size_b, const float* angle_b, const float* resp_b, float radius, float* feat,
                         cudaStream_t s);
int32_t run_mlp_infer(const float* prm, int n, const float* feat, bool bf16, float* prob, cudaStream_t s);
int32_t run_mlp_accept(int n, const int32_t* t1, const float* b12, const float* prob, float thr, float ratio,
                       int32_t* t_row, uint32_t* d_row, cudaStream_t s);
int32_t run_mlp_grad(fsb_ctx* ctx, const float* prm, int n, const float* feat, const float* label, float* grad,
                     double* loss, cudaStream_t s);
int32_t run_mlp_train(fsb_ctx* ctx, float* prm, float* m, float* v, int n, const float* feat, const float* label,
                      int epochs, int batch, float lr, uint32_t seed, double* losses, cudaStream_t s);
// tc_match.cu: tensor-core dense matching of a batch of pairs (na, nb >= 1), _unique included;
// counts (device, one per pair), q_out/t_out device arrays of capacity na[p]
int32_t run_match_bf_tc(fsb_ctx* ctx, int n_pairs, const uint8_t* const* d_a, const int* na,
                        const uint8_t* const* d_b, const int* nb, float ratio, int precision, int64_t* const* q_out,
                        int64_t* const* t_out, int32_t* counts, TcStats* stats, cudaStream_t s);
// ransac.cu
int32_t run_ransac_h(const long long* d_off, int n_pairs, const double2* d_src, const double2* d_dst, double thr,
                     int iters, unsigned long long seed, double* d_H, uint8_t* d_mask, int* d_ninl, cudaStream_t s);
int32_t run_ransac_f(const long long* d_off, int n_pairs, const double2* d_src, const double2* d_dst, double thr,
                     int iters, unsigned long long seed, double* d_F, uint8_t* d_mask, int* d_ninl, cudaStream_t s);
// jpeg.cu
int32_t run_jpeg_gray(fsb_ctx* ctx, const uint8_t* data, size_t len, int reduce, uint8_t* d_out, size_t out_cap,
                      int* h, int* w);
int32_t jpeg_release(fsb_ctx* ctx);
// tracks.cu
int32_t run_build_tracks(fsb_ctx* ctx, const long long* d_u, const long long* d_v, long long ne, const long long* d_off,
                         int n_img, int n_nodes, long long* d_tid, long long* d_img, long long* d_feat, int* n_obs,
                         int* n_tracks, cudaStream_t s);
// prep.cu
int32_t run_clahe(const uint8_t* d_img, int h, int w, int stride, double clip, int tiles_x, int tiles_y,
                  uint8_t* d_lut, uint8_t* d_out, int out_stride, cudaStream_t s);
// geom.cu
int32_t run_undistort(const double* d_uv, int n, const double* k8, double* d_out, cudaStream_t s);
int32_t run_predict(const double* d_u, int n, const double* kinv_i, const double* r_i, const double* c_i,
                    const double* k_j, const double* r_j, const double* c_j, double zg, double* d_pred, uint8_t* d_ok,
                    cudaStream_t s);
int32_t run_perspective(const double* d_xy, int n, const double* hm9, double* d_out, cudaStream_t s);
int32_t run_project(const float* d_xy, int n, const double* hm9_host, const float* d_off, double* d_out,
                    cudaStream_t s);
int32_t run_unique_general(fsb_ctx* ctx, const int64_t* d_q, const int64_t* d_t, const float* d_dd, int n,
                           int64_t* d_qo, int64_t* d_to, int* d_n, cudaStream_t s);

}  // namespace fsb
