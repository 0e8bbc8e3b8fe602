/*
 * fsb200.h - C ABI of the B200 (sm_100a) SIFT + guided-matching front end.
 *
 * Plain C types only (pointers, sizes, status codes). Every function returns FSB_OK (0) or a
 * non-zero status; fsb_last_error() returns a message for the calling thread. Unless a
 * function's comment says "device pointers", array arguments are HOST memory and the call
 * returns once its results are in host memory.
 *
 * Each entry point replaces a function of PlaneSite (Edko01/FieldStitch); the citation names the
 * reference file:line whose behaviour it reproduces. A context (fsb_ctx) owns one CUDA stream on
 * one device and is not thread-safe: use one context per thread, or guard it.
 */
#ifndef FSB200_H
#define FSB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FSB_OK 0
#define FSB_ERR_ARG 1         /* invalid argument (null pointer, bad size, unknown mode) */
#define FSB_ERR_OOM 2         /* device allocation failed */
#define FSB_ERR_CUDA 3        /* a CUDA runtime call failed */
#define FSB_ERR_TIMEOUT 4     /* a bounded device wait gave up */
#define FSB_ERR_STATE 5       /* a detect state was used with another context or after free */
#define FSB_ERR_UNSUPPORTED 6 /* the device is not sm_100 or the mode is not built */
#define FSB_ERR_OVERFLOW 7    /* an internal capacity was exceeded and could not be grown */

/* dense matcher precision (fsb_match_bf) */
#define FSB_PREC_FP32 0 /* CUDA-core FP32 distances: the plain path */
#define FSB_PREC_BF16 1 /* tcgen05 BF16 x BF16 -> FP32 (exact for uint8 rows), exact integer re-rank */
#define FSB_PREC_FP8 2  /* tcgen05 E4M3 (per-row power-of-two scale) -> FP32, exact integer re-rank of
                           the best 4 x 32 columns, certified ratio test, exact fallback rows */

typedef struct fsb_ctx fsb_ctx;
typedef struct fsb_state fsb_state;

/* SIFT parameters (gsift.detect keyword arguments, app/planesite/gsift.py:435). */
typedef struct {
    double contrast; /* contrast threshold (default 0.015; OpenCV default 0.04) */
    double edge;     /* edge threshold (default 12; OpenCV default 10) */
    int32_t max_kp;  /* keep at most this many keypoints, strongest first (default 12000) */
    int32_t flags;   /* FSB_SIFT_* bits */
} fsb_sift_params;

/* blur accumulates in float64 and rounds once to float32 per pass, as scipy.ndimage does in the
   reference's CPU path: the pyramid is then bit-identical to it (slower). Default: float32 FMA. */
#define FSB_SIFT_EXACT_BLUR 1

/* ---- library / context ------------------------------------------------------------------- */
int32_t fsb_version(void);
const char* fsb_last_error(void);
/* Creates a context on CUDA device `device` (the CuPy device/stream the reference's GPU worker
   uses, app/planesite/features.py:258-267). Fails with FSB_ERR_UNSUPPORTED unless sm_100. */
int32_t fsb_create(int32_t device, fsb_ctx** out);
int32_t fsb_destroy(fsb_ctx* ctx);
/* Waits, for at most timeout_ms, for the context's stream; FSB_ERR_TIMEOUT if it did not drain. */
int32_t fsb_sync(fsb_ctx* ctx, int32_t timeout_ms);
/* The context's cudaStream_t, as an opaque pointer (for callers that share the stream). */
void* fsb_stream(fsb_ctx* ctx);
/* Bytes of device memory the context holds (workspaces and scratch). */
int64_t fsb_device_bytes(fsb_ctx* ctx);
/* Number of kernel launches this library has issued in the process (all contexts). */
int64_t fsb_launch_count(void);
/* Per-stage device timing, the counterpart of gsift.detect(timings=dict)
   (app/planesite/gsift.py:441-446): while on, CUDA events bracket each stage on the context
   stream; they are read back lazily, so timing adds no host wait to the pipeline (the reference
   synchronises at each stage instead). fsb_stage_times waits for the pending ones, copies the accumulated milliseconds and call counts of the FSB_STAGE_*
   stages (n entries each, nullable) and resets them. */
int32_t fsb_timing(fsb_ctx* ctx, int32_t on);
int32_t fsb_stage_times(fsb_ctx* ctx, double* ms, int64_t* calls, int32_t n);
#define FSB_STAGE_UPLOAD 0
#define FSB_STAGE_PYRAMID 1
#define FSB_STAGE_EXTREMA 2
#define FSB_STAGE_REFINE 3
#define FSB_STAGE_ORIENT 4
#define FSB_STAGE_SORT 5
#define FSB_STAGE_SPREAD 6
#define FSB_STAGE_DESCRIBE 7
#define FSB_STAGE_MATCH 8
#define FSB_STAGE_TC_DENSE 9 /* the tensor-core contraction kernel alone (inside FSB_STAGE_MATCH) */
#define FSB_STAGE_COUNT 10

/* ---- SIFT detection / description ---------------------------------------------------------- */
/* gsift.detect (app/planesite/gsift.py:435-477): 2x upsample, Gaussian/DoG pyramid, 3x3x3
   extrema, sub-pixel refinement with contrast and edge tests, 36-bin orientations, strongest
   first (ties: octave, layer, row, column of the extremum, then orientation bin), at most
   p->max_kp. `img` is a uint8 grey image with `stride` bytes per row. On success *state holds
   the gradient atlas for fsb_describe and *n_kp the keypoint count. */
int32_t fsb_detect(fsb_ctx* ctx, const uint8_t* img, int32_t h, int32_t w, int32_t stride,
                   const fsb_sift_params* p, fsb_state** state, int32_t* n_kp);
/* Copies the detected keypoints (n_kp entries each) into host arrays: x, y in input-image
   pixels, size, angle (degrees), response, 0-based octave of the upsampled image, layer 1..3
   (the dict returned by gsift.detect, app/planesite/gsift.py:473-474). Null outputs are skipped. */
int32_t fsb_state_keypoints(fsb_state* st, float* x, float* y, float* size, float* angle,
                            float* response, int32_t* octave, int32_t* layer);
/* gsift.describe (app/planesite/gsift.py:480-525): 128-d descriptors of n keypoints given by
   their x, y, size, angle, octave, layer (usually kps[sel] of fsb_detect). desc (n*128 float32,
   L2 norm 512, unrounded) and/or rootsift (n*128 uint8, the feature-file encoding of
   app/planesite/features.py:80-82) may be null. */
int32_t fsb_describe(fsb_ctx* ctx, fsb_state* st, int32_t n, const float* x, const float* y,
                     const float* size, const float* angle, const int32_t* octave,
                     const int32_t* layer, float* desc, uint8_t* rootsift);
int32_t fsb_state_free(fsb_state* st);
/* The detect state's atlases (gsift's `_Atlas`, app/planesite/gsift.py:227-267): octave count and
   per-octave rows/cols (capacity 16 each), then a copy of one atlas into host memory:
   which = 0 DoG [octave][layer 0..4][R][C], 1 gradient magnitude, 2 gradient angle (degrees)
   [octave][layer 1..3][R][C]; n_floats must equal the atlas size. */
int32_t fsb_state_geometry(fsb_state* st, int32_t* n_oct, int32_t* rows, int32_t* cols);
int32_t fsb_state_atlas(fsb_state* st, int32_t which, float* out, int64_t n_floats);

/* features._spread (app/planesite/features.py:38-57) on the device: n keypoints (x, y, response;
   host arrays, responses non-increasing as detect returns them, else FSB_ERR_ARG) of a W x H
   image; keeps min(n, nfeat) spread over a 12 x 9 grid (per cell the strongest first, at most
   ceil(nfeat / 108) per cell, then the strongest of the rest, ties by index). order
   FSB_SPREAD_SELECTION returns the indices in _spread's order, FSB_SPREAD_RESPONSE after the
   stable response sort that follows it (features.py:126). sel holds min(n, nfeat) int32. */
#define FSB_SPREAD_SELECTION 0
#define FSB_SPREAD_RESPONSE 1
int32_t fsb_spread(fsb_ctx* ctx, const float* x, const float* y, const float* resp, int32_t n, int32_t W, int32_t H,
                   int32_t nfeat, int32_t order, int32_t* sel, int32_t* n_out);

/* features.sift_gpu (app/planesite/features.py:115-129) in one device pass: detect with
   max_kp = int(2.2 nfeat) (p->max_kp is ignored), grid-spread selection of nfeat keypoints
   (features.py:38-57, ties by index), stable sort by response, describe, RootSIFT. Outputs hold
   up to nfeat rows: xy (n*2 float32), resp (n float32), desc (n*128 float32, nullable),
   rootsift (n*128 uint8, nullable). *n_out = 0 when fewer than 10 keypoints were found
   (features.py:121-122). */
int32_t fsb_sift_features(fsb_ctx* ctx, const uint8_t* img, int32_t h, int32_t w, int32_t stride,
                          const fsb_sift_params* p, int32_t nfeat, float* xy, float* resp,
                          float* desc, uint8_t* rootsift, int32_t* n_out);

/* ---- device-pointer variants ---------------------------------------------------------------
   Same computations with inputs and outputs in device memory of the context's device (the
   caller keeps them resident across calls); counts are returned to the host and the call returns
   once its outputs are written. */
/* fsb_sift_features on an image in device memory. d_xy (nfeat*2), d_resp (nfeat),
   d_desc (nfeat*128 float32) and d_rootsift (nfeat*128 uint8) are device pointers (nullable). */
int32_t fsb_sift_features_d(fsb_ctx* ctx, const uint8_t* d_img, int32_t h, int32_t w, int32_t stride,
                            const fsb_sift_params* p, int32_t nfeat, float* d_xy, float* d_resp,
                            float* d_desc, uint8_t* d_rootsift, int32_t* n_out);
/* fsb_sift_features_d plus the selected keypoints' size (float32, pixels of the input image),
   angle (float32, degrees) and octave (int32, 0 = the 2x upsampled octave), each nullable: the
   keypoint attributes of gsift.detect (app/planesite/gsift.py:435-477) for the selected set,
   which the learned match filter's features use. */
int32_t fsb_sift_features_ex_d(fsb_ctx* ctx, const uint8_t* d_img, int32_t h, int32_t w, int32_t stride,
                               const fsb_sift_params* p, int32_t nfeat, float* d_xy, float* d_resp,
                               float* d_desc, uint8_t* d_rootsift, float* d_size, float* d_angle,
                               int32_t* d_octave, int32_t* n_out);
/* fsb_sift_features_d over a batch of n_img same-size images in device memory (the per-photo
   feature step of the reference's GPU worker, app/planesite/features.py:115-129 and 343-378, for a
   batch), with no host wait inside the batch: every count stays on the device and each launch is
   sized by a capacity fixed for the geometry, so the whole batch is one CUDA graph - `chains`
   images in flight, each chain with its own stream and workspace - captured on the first call and
   replayed while the arguments and buffers are unchanged. Image i: d_imgs[i] (h x w, row pitch
   stride), nfeats[i] features; outputs d_xy[i] (nfeat*2 float32), d_resp[i] (nfeat float32,
   nullable array), d_rootsift[i] (nfeat*128 uint8); d_counts (device, n_img int32) receives the
   feature counts, h_counts (host, nullable) too. The first call for a geometry runs image 0 by
   the host-driven path first (autotuning, capacities). The call waits once, at the end; an image
   that exceeded a capacity is redone by the host-driven path, so the outputs always equal
   fsb_sift_features_d's. */
int32_t fsb_sift_features_batch_d(fsb_ctx* ctx, int32_t n_img, const uint8_t* const* d_imgs, int32_t h, int32_t w,
                                  int32_t stride, const fsb_sift_params* p, const int32_t* nfeats, float* const* d_xy,
                                  float* const* d_resp, uint8_t* const* d_rootsift, int32_t* d_counts,
                                  int32_t* h_counts, int32_t chains);
/* fsb_sift_features_batch_d from host images: h_imgs[i] (page-locked host memory, h rows of
   `stride` bytes) is uploaded into d_imgs[i] by the same graph, on a copy stream in image order,
   and image i's extraction waits for its own upload only, so the uploads of later images overlap
   the extraction of earlier ones. The graph is keyed like fsb_sift_features_batch_d's (device
   buffers, not host addresses): a later call with other host buffers replays it with the uploads
   re-pointed. Pageable host memory is rejected (FSB_ERR_ARG). The end-to-end form of the
   reference's per-photo worker loop (app/planesite/features.py:115-129 over a spawn queue). */
int32_t fsb_sift_features_batch_hd(fsb_ctx* ctx, int32_t n_img, const uint8_t* const* h_imgs,
                                   uint8_t* const* d_imgs, int32_t h, int32_t w, int32_t stride,
                                   const fsb_sift_params* p, const int32_t* nfeats, float* const* d_xy,
                                   float* const* d_resp, uint8_t* const* d_rootsift, int32_t* d_counts,
                                   int32_t* h_counts, int32_t chains);
/* The Gaussian / DoG pyramid stage alone (gsift.py `_pyramid`, app/planesite/gsift.py:158-179, and
   the gradient atlases of `_Atlas`, :227-267) for n_img device images of one size, on `chains`
   streams (image i on chain i mod chains) captured as one CUDA graph and replayed while the image
   pointers are unchanged; the same chains and workspaces as fsb_sift_features_batch_d. The
   atlases stay in the chain workspaces (each chain holds the last image it processed), so this is
   the stage that fsb_sift_features_batch_d runs first, exposed to time the pyramid in the batch
   configuration. A geometry's first call runs one pyramid outside the capture (autotuning).
   flags: FSB_SIFT_EXACT_BLUR or 0. Waits for the batch. */
int32_t fsb_pyramid_batch_d(fsb_ctx* ctx, int32_t n_img, const uint8_t* const* d_imgs, int32_t h, int32_t w,
                            int32_t stride, int32_t flags, int32_t chains);
/* Prior prediction: projects n float32 points (d_xy, n*2) through the homography hm9 (host,
   row-major 3x3) into float64 positions d_out (n*2), adding the float32 offsets d_offset (n*2,
   nullable) - e.g. a GNSS/gimbal prior and its error. Identity hm9 converts to float64. */
int32_t fsb_project_d(fsb_ctx* ctx, const float* d_xy, int32_t n, const double* hm9,
                      const float* d_offset, double* d_out);
/* fsb_project_d for n_sets point sets (set k: d_xy[k], n[k] points, homography hm9 + 9k, offsets
   d_offset[k] or none when d_offset is null, output d_out[k]), queued on the context's stream with
   no host wait (later work on the same context sees the results). */
int32_t fsb_project_batch_d(fsb_ctx* ctx, int32_t n_sets, const float* const* d_xy, const int32_t* n,
                            const double* hm9, const float* const* d_offset, double* const* d_out);
/* fsb_match_guided with every array in device memory; d_q, d_t capacity na. */
int32_t fsb_match_guided_d(fsb_ctx* ctx, const double* d_pred, const uint8_t* d_a, int32_t na,
                           const double* d_bxy, const uint8_t* d_b, int32_t nb, double w_b, double h_b,
                           double radius, int32_t kc, float ratio, int64_t* d_q, int64_t* d_t,
                           int32_t* n_out);
/* A batch of fsb_match_guided_d problems in one call (pointer and size arrays on the host,
   data in device memory): pair p matches d_a[p] (na[p] queries, predicted positions d_pred[p])
   against d_b[p] (nb[p] targets at d_bxy[p], frame w_b[p] x h_b[p]) and writes n_out[p] pairs
   into d_q[p], d_t[p]. All pairs share one set of launches (one grid build, one guided kernel
   over every query of every pair, one batched _unique), issued as a CUDA graph that is captured
   on the first call and replayed while the pair table and the context's scratch are unchanged.
   Replaces a loop over matching._guided (app/planesite/matching.py:113-152); results are
   identical to per-pair calls. */
int32_t fsb_match_guided_batch_d(fsb_ctx* ctx, int32_t n_pairs, const double* const* d_pred,
                                 const uint8_t* const* d_a, const int32_t* na, const double* const* d_bxy,
                                 const uint8_t* const* d_b, const int32_t* nb, const double* w_b,
                                 const double* h_b, double radius, int32_t kc, float ratio,
                                 int64_t* const* d_q, int64_t* const* d_t, int32_t* n_out);
/* The guided matcher's candidates before its ratio test: per query the best target within the
   radius (kc rule as fsb_match_guided; -1 when there is none) in d_t1 (na int32) and its squared
   distance b1 and the second-best b2 (+inf for a single candidate) in d_b12 (na x 2 float32).
   The inputs of matching._guided's ratio test (app/planesite/matching.py:137-146). */
int32_t fsb_match_guided_cand_d(fsb_ctx* ctx, const double* d_pred, const uint8_t* d_a, int32_t na,
                                const double* d_bxy, const uint8_t* d_b, int32_t nb, double w_b, double h_b,
                                double radius, int32_t kc, int32_t* d_t1, float* d_b12);
/* fsb_match_bf with every array in device memory; d_q, d_t capacity na. */
int32_t fsb_match_bf_d(fsb_ctx* ctx, const uint8_t* d_a, int32_t na, const uint8_t* d_b, int32_t nb,
                       float ratio, int32_t precision, int64_t* d_q, int64_t* d_t, int32_t* n_out);

/* A batch of independent fsb_match_bf_d problems in one call: pair p matches d_a[p] (na[p] x 128)
   against d_b[p] (nb[p] x 128) and writes n_out[p] pairs into d_q[p], d_t[p] (device, capacity
   na[p]). The pointer and size arrays are host arrays; the descriptors and outputs are device
   memory. With FSB_PREC_BF16 / FSB_PREC_FP8 all pairs share one persistent tensor-core launch
   (work items of 256 query rows, uneven sizes allowed); FSB_PREC_FP32 runs the pairs one after
   another. Replaces a Python loop over matching._ratio_match_bf (app/planesite/matching.py:86-100);
   every precision returns the same pairs. */
int32_t fsb_match_bf_batch_d(fsb_ctx* ctx, int32_t n_pairs, const uint8_t* const* d_a, const int32_t* na,
                             const uint8_t* const* d_b, const int32_t* nb, float ratio, int32_t precision,
                             int64_t* const* d_q, int64_t* const* d_t, int32_t* n_out);
/* Statistics of the last tensor-core dense match on ctx (fsb_match_bf* with FSB_PREC_BF16 or
   FSB_PREC_FP8): query rows, rows whose ratio-test decision the rounding-error certificate could
   not settle and that were recomputed exactly, and the largest and mean absolute difference
   between the approximate and the exact best squared distance of a row. Any pointer may be null. */
int32_t fsb_match_tc_stats(fsb_ctx* ctx, int64_t* rows, int64_t* fallback_rows, double* max_abs_err,
                           double* mean_abs_err);

/* Launch-variant autotuner report: the choices made so far in this process, one "key variant"
   line each (key = device name / ordinal / kernel and size; for the per-layer pyramid kernel the
   variant indexes the tile heights 32, 16, 64). Returns the bytes needed including the final
   zero; writes at most len of them into buf (nullable). Set FSB_AUTOTUNE=0 to disable tuning,
   FSB_AUTOTUNE_FILE=path to keep choices across processes. No counterpart in the reference. */
int32_t fsb_autotune_table(char* buf, int32_t len);

/* ---- learned match filter (no counterpart in the reference: it replaces the ratio test of
   matching._guided, app/planesite/matching.py:142-146, by an 8-64-64-1 MLP whose labels come
   from the plain pipeline's own RANSAC verification, matching.py:205-233) --------------------
   Parameters: one float32 device vector of fsb_mlp_param_count() values: W1[64][8], b1[64],
   W2[64][64], b2[64], w3[64], b3 (the first fsb_mlp_trainable_count() values, trained), then
   the input normalisation mu[8], sigma[8]. Features (n x 8 float32) of a query's best candidate:
   ratio sqrt(b1)/sqrt(b2) (0 for a single candidate), sqrt(b1)/512, log2(size_b/size_a), signed
   angle difference/180, |pred_a - xy_b|/radius, response_a, response_b, octave_a; queries without
   a candidate get zeros. */
int32_t fsb_mlp_param_count(void);
int32_t fsb_mlp_trainable_count(void);
int32_t fsb_mlp_features_d(fsb_ctx* ctx, int32_t n, const int32_t* d_t1, const float* d_b12,
                           const double* d_pred, const float* d_xy_b, const float* d_size_a,
                           const float* d_angle_a, const float* d_resp_a, const int32_t* d_oct_a,
                           const float* d_size_b, const float* d_angle_b, const float* d_resp_b,
                           float radius, float* d_feat);
/* Gradient (d_grad, trainable count) and mean binary cross-entropy (*loss, nullable) of the
   network over n labelled samples (d_label: 0 or 1). */
int32_t fsb_mlp_grad_d(fsb_ctx* ctx, const float* d_params, int32_t n, const float* d_feat,
                       const float* d_label, float* d_grad, double* loss);
/* Mini-batch Adam (beta 0.9 / 0.999) on the GPU: each epoch shuffles the samples on the device
   (seeded) and takes floor(n / batch) steps; the epoch runs as one captured CUDA graph. d_m, d_v:
   Adam moments (trainable count each, reset here). losses (host, nullable) receives the mean
   loss of each of the `epochs` epochs. */
int32_t fsb_mlp_train_d(fsb_ctx* ctx, float* d_params, float* d_m, float* d_v, int32_t n,
                        const float* d_feat, const float* d_label, int32_t epochs, int32_t batch,
                        float lr, uint32_t seed, double* losses);
/* Probabilities (n float32); bf16 != 0: BF16 weights, inputs and hidden activations with FP32
   accumulation. */
int32_t fsb_mlp_infer_d(fsb_ctx* ctx, const float* d_params, int32_t n, const float* d_feat, int32_t bf16,
                        float* d_prob);
/* Accept the candidates (d_t1, d_b12 from fsb_match_guided_cand_d) whose probability exceeds
   threshold, or - d_prob null, the fallback - those passing the ratio test of matching._guided;
   then the one-to-one filter of _unique. Writes *n_out pairs ordered by target (capacity na). */
int32_t fsb_mlp_filter_d(fsb_ctx* ctx, int32_t na, const int32_t* d_t1, const float* d_b12, const float* d_prob,
                         float threshold, float ratio, int32_t nb, int64_t* d_q, int64_t* d_t, int32_t* n_out);

/* Allocation-free variant of fsb_match_bf_d (FP32 distances), for callers that cannot call
   cudaMalloc: processes that reserve their whole device-memory budget up front, host frameworks
   that own the CUDA allocator, real-time loops that must not block or fail in an allocation.
   No counterpart in the reference (PlaneSite allocates through CuPy/NumPy). All scratch lives in
   one fixed device array inside the library (about 1.9 MiB, held on every GPU that loads the
   library until exit); na and nb must be <= 16384, larger sizes are rejected with FSB_ERR_ARG.
   Inputs d_a (na x 128), d_b (nb x 128) and outputs d_q, d_t (capacity na, int64) and d_n (one
   int32, the number of pairs, ordered by target) are device pointers; the work is queued on
   `stream` (a cudaStream_t; null = the legacy default stream) and the call does not wait for it.
   The first call on a device looks up the array's device address (cudaGetSymbolAddress) with
   that device current, and so does the first call in any other CUDA context of that device (after
   a cudaDeviceReset, or in a driver-API context other than the primary one); make that first call
   before any stream capture. Calls share the array:
   calls whose work can overlap on the GPU race and must be serialised by the caller. */
int32_t fsb_match_bf_noalloc(const uint8_t* d_a, int32_t na, const uint8_t* d_b, int32_t nb, float ratio,
                             int64_t* d_q, int64_t* d_t, int32_t* d_n, void* stream);

/* ---- matching ------------------------------------------------------------------------------- */
/* matching._ratio_match_bf + _unique (app/planesite/matching.py:86-110) on uint8 descriptors
   (na x 128, nb x 128, row-major): nearest and second-nearest squared L2 distance over all of B,
   ratio test sqrt(b1) < ratio * sqrt(b2) in float32, then one match per target keeping the
   smallest distance (ties: smaller query index). Writes *n_out pairs ordered by target into
   q, t (capacity na each). precision: FSB_PREC_*; every precision returns the same pairs. */
int32_t fsb_match_bf(fsb_ctx* ctx, const uint8_t* a, int32_t na, const uint8_t* b, int32_t nb,
                     float ratio, int32_t precision, int64_t* q, int64_t* t, int32_t* n_out);
/* matching._guided + _unique (app/planesite/matching.py:113-152) given predicted positions
   pred_xy (na x 2 float64) of A's keypoints in B: predictions outside B's w_b x h_b frame
   widened by radius are skipped; candidates are B keypoints (b_xy, nb x 2 float64) strictly
   within radius; kc > 0 keeps only the kc nearest (ties: smaller B index), kc <= 0 keeps all;
   exact squared descriptor distances; top-2 ratio test (a single candidate passes); one match
   per target. Writes *n_out pairs ordered by target. */
int32_t fsb_match_guided(fsb_ctx* ctx, const double* pred_xy, const uint8_t* a, int32_t na,
                         const double* b_xy, const uint8_t* b, int32_t nb, double w_b, double h_b,
                         double radius, int32_t kc, float ratio, int64_t* q, int64_t* t,
                         int32_t* n_out);
/* matching._unique (app/planesite/matching.py:103-110) for n candidate pairs (q, t, dd): per
   target t keeps the entry with the smallest dd (ties: earlier position), output ordered by t
   (q_out, t_out capacity n; *n_out entries written). */
int32_t fsb_unique(fsb_ctx* ctx, const int64_t* q, const int64_t* t, const float* dd, int32_t n,
                   int64_t* q_out, int64_t* t_out, int32_t* n_out);
/* cv2.perspectiveTransform of app/planesite/matching.py:115 on the device (float64):
   out = (H [x y 1]^T)_{xy} / (H [x y 1]^T)_z. */
int32_t fsb_perspective(fsb_ctx* ctx, const double* xy, int32_t n, const double* hm9, double* out);
/* recon.build_tracks (app/planesite/recon.py:14-54) on the device: feature tracks over the match
   graph. Nodes are global feature indices (offsets[photo] + feature; offsets has n_img + 1
   ascending entries, at most 2^31 - 2 features in all); every match is an edge u[e] - v[e]. A track
   is a connected component of at least two matched features with no two features of the same
   photo, numbered in the order of its smallest node; the observations (tid, img, feat; capacity
   2 n_edges) are listed by track, then node. Same output as the reference. */
int32_t fsb_build_tracks(fsb_ctx* ctx, const int64_t* u, const int64_t* v, int64_t n_edges, const int64_t* offsets,
                         int32_t n_img, int64_t* tid, int64_t* img, int64_t* feat, int64_t* n_obs, int64_t* n_tracks);
/* The stage-1 homography of matching.match_pair (app/planesite/matching.py:226,
   cv2.findHomography(src, dst, cv2.RANSAC, thr)) for n_pairs pairs in one launch: pair p's
   correspondences are src / dst rows offsets[p] .. offsets[p+1] - 1 (float64 (x, y)); `iters`
   hypotheses per pair from 4-point samples (seeded, deterministic); inliers: squared reprojection
   error <= thr^2; the homography (9 per pair, row-major, h33 = 1; zeros when a pair has fewer than
   4 correspondences or no usable sample) is refined by least squares over the best hypothesis's
   inliers; mask (one byte per correspondence) and n_inliers as OpenCV returns them. Random samples
   differ from OpenCV's: results agree statistically. */
int32_t fsb_find_homography_batch(fsb_ctx* ctx, int32_t n_pairs, const int64_t* offsets, const double* src,
                                  const double* dst, double thr, int32_t iters, uint64_t seed, double* H, uint8_t* mask,
                                  int32_t* n_inliers);
/* The fundamental-matrix verification of matching.match_pair (matching._verify,
   app/planesite/matching.py:175-191, cv2.findFundamentalMat(pi, pj, USAC_MAGSAC, thr, 0.999,
   10000)) for n_pairs pairs in one launch: pair p's correspondences are src (image i) / dst
   (image j) rows offsets[p] .. offsets[p+1] - 1 (float64 (x, y)); `iters` seven-point samples per
   pair (seeded, deterministic); inliers: Sampson distance <= thr (OpenCV's USAC_MAGSAC mask rule);
   the best candidate refined by eight-point least squares over its inliers. F (9 per pair,
   row-major, x_j^T F x_i = 0, F33 = 1 or unit norm; zeros when a pair has fewer than 8
   correspondences or no candidate with 8 inliers), mask (one byte per correspondence) and
   n_inliers. Random samples and the consensus rule differ from MAGSAC's: results agree
   statistically. */
int32_t fsb_find_fundamental_batch(fsb_ctx* ctx, int32_t n_pairs, const int64_t* offsets, const double* src,
                                   const double* dst, double thr, int32_t iters, uint64_t seed, double* F,
                                   uint8_t* mask, int32_t* n_inliers);
/* features.decode / prepare (app/planesite/features.py:18-71) on the device: the luma plane of a
   JPEG held in host memory (data, len bytes), read at full size (reduce 1) or reduced by 2, 4, 8
   (block means; OpenCV's reduced reads scale inside the inverse DCT, so those agree with OpenCV
   approximately). fsb_decode_gray_d writes the plane to device memory (capacity out_cap, pitch =
   width); fsb_prepare_gray also equalises it with CLAHE (clip, 8 x 8 tiles) and returns it in host
   memory. *h, *w receive the output size. nvJPEG is loaded on first use (FSB_ERR_UNSUPPORTED
   without it). */
int32_t fsb_decode_gray_d(fsb_ctx* ctx, const uint8_t* data, int64_t len, int32_t reduce, uint8_t* d_out,
                          int64_t out_cap, int32_t* h, int32_t* w);
int32_t fsb_prepare_gray(fsb_ctx* ctx, const uint8_t* data, int64_t len, int32_t reduce, double clip, uint8_t* out,
                         int64_t out_cap, int32_t* h, int32_t* w);
/* Contrast equalisation of features.prepare (app/planesite/features.py:60-71):
   cv2.createCLAHE(clipLimit = clip, tileGridSize = (tiles_x, tiles_y)).apply(img) on a uint8 image,
   identical output (OpenCV's tile extension, clipping, redistribution, LUT rounding and bilinear
   blend); clip <= 0 disables clipping; tiles_x * tiles_y <= 256.
   fsb_clahe takes host buffers, fsb_clahe_d device buffers (enqueued on the context's stream). */
int32_t fsb_clahe(fsb_ctx* ctx, const uint8_t* img, int32_t h, int32_t w, int32_t stride, double clip,
                  int32_t tiles_x, int32_t tiles_y, uint8_t* out, int32_t out_stride);
int32_t fsb_clahe_d(fsb_ctx* ctx, const uint8_t* d_img, int32_t h, int32_t w, int32_t stride, double clip,
                    int32_t tiles_x, int32_t tiles_y, uint8_t* d_out, int32_t out_stride);
/* camera.undistort_pixels (app/planesite/camera.py:5-31) on the device, float64: distorted pixels
   uv (n,2) -> ideal pinhole pixels with the same f, cx, cy; k8 = f, cx, cy, k1, k2, p1, p2, k3;
   25 fixed-point iterations in the reference's operation order (no fused multiply-add). */
int32_t fsb_undistort_pixels(fsb_ctx* ctx, const double* uv, int32_t n, const double* k8, double* out);
/* matching._predict (app/planesite/matching.py:155-172) on the device, float64: where the
   undistorted pixels u (n,2) of image i land in image j under the ground-plane prior z = zg.
   kinv_i = inverse of K_i, r_i / r_j world-to-camera rotations, c_i / c_j camera centres, k_j the
   intrinsics of j (3x3 row-major). pred (n,2); ok[k] = 1 where the ray meets the plane in front of
   camera i and the point lies in front of camera j. */
int32_t fsb_predict_ground(fsb_ctx* ctx, const double* u, int32_t n, const double* kinv_i, const double* r_i,
                           const double* c_i, const double* k_j, const double* r_j, const double* c_j, double zg,
                           double* pred, uint8_t* ok);

#ifdef __cplusplus
}
#endif
#endif /* FSB200_H */
