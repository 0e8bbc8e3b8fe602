// Learned match filter: an 8-64-64-1 MLP over per-correspondence features, trained on the GPU.
//
// The plain guided matcher (matching._guided, app/planesite/matching.py:113-152) accepts a
// query's best candidate when it passes the ratio test; the pipeline then verifies the accepted
// set geometrically (RANSAC homography, matching.py:205-233). Here the candidates that the plain
// matcher sees (best target, b1, b2 for every query) are described by 8 features and scored by
// a small MLP trained on labels that the plain pipeline's own verification produces; the plain
// ratio test remains the fallback.
//
//   k_mlp_features    features of every query's best candidate:
//                     0 ratio sqrt(b1) / sqrt(b2) (0 for a single candidate), 1 sqrt(b1) / 512,
//                     2 log2(size_b / size_a), 3 signed angle difference / 180 (wrapped),
//                     4 prior residual |pred_a - xy_b| / radius, 5 response_a, 6 response_b,
//                     7 octave_a
//   k_mlp_fwd_bwd     one mini-batch slice per block (128 samples): forward (ReLU, sigmoid),
//                     mean binary cross-entropy gradient; activations and deltas staged in shared
//                     memory, per-block partial gradients (fixed summation order)
//   k_mlp_adam        sums the partials in block order and applies one Adam step
//   k_mlp_infer       inference, FP32 or BF16 (BF16 weights, inputs and hidden activations,
//                     FP32 accumulation)
//   k_mlp_accept      probability > threshold (or the ratio test when no network is given)
//                     -> (target, distance) rows for the one-to-one filter
//
// Parameter vector (float32): W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3, then the input
// normalisation mu[8], sigma[8] (not trained). An epoch (device-side shuffle + every step) is
// captured once as a CUDA graph and replayed.
#include <cub/cub.cuh>
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "fsb_internal.cuh"

namespace fsb {
namespace {

constexpr int NF = 8, H = 64;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * NF, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H, N_TRAIN = OFF_B3 + 1, OFF_MU = N_TRAIN,
              OFF_SIG = OFF_MU + NF, N_PARAM = OFF_SIG + NF;
constexpr int MB = 128;          // samples per block in k_mlp_fwd_bwd
constexpr int HP = H + 1;        // padded row of the shared activation tiles

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// ------------------------------------------------------------------------ features
__global__ void k_mlp_features(int n, const int32_t* __restrict__ t1, const float* __restrict__ b12,
                               const double* __restrict__ pred, const float* __restrict__ xy_b,
                               const float* __restrict__ size_a, const float* __restrict__ angle_a,
                               const float* __restrict__ resp_a, const int32_t* __restrict__ oct_a,
                               const float* __restrict__ size_b, const float* __restrict__ angle_b,
                               const float* __restrict__ resp_b, float radius, float* __restrict__ feat) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float f[NF] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const int t = t1[i];
    if (t >= 0) {
        const float b1 = fmaxf(b12[2 * i], 0.f), b2 = b12[2 * i + 1];
        f[0] = isinf(b2) ? 0.f : sqrtf(b1) / fmaxf(sqrtf(fmaxf(b2, 0.f)), 1e-6f);
        f[1] = sqrtf(b1) * (1.f / 512.f);
        f[2] = log2f(fmaxf(size_b[t], 1e-6f) / fmaxf(size_a[i], 1e-6f));
        float da = angle_b[t] - angle_a[i];
        da = da - 360.f * floorf((da + 180.f) / 360.f);
        f[3] = da * (1.f / 180.f);
        const double dx = pred[2 * i] - (double)xy_b[2 * t], dy = pred[2 * i + 1] - (double)xy_b[2 * t + 1];
        f[4] = (float)sqrt(dx * dx + dy * dy) / radius;
        f[5] = resp_a[i];
        f[6] = resp_b[t];
        f[7] = (float)oct_a[i];
    }
#pragma unroll
    for (int k = 0; k < NF; ++k) feat[(size_t)i * NF + k] = f[k];
}

// ------------------------------------------------------------------------ training
__device__ __forceinline__ float sigmoidf_(float z) { return 1.f / (1.f + __expf(-z)); }

// Per-block partial gradient of mean BCE over `count` samples (sample = idx[base + s]); part has
// N_TRAIN floats per block. loss_sum (nullable) accumulates the summed loss.
__global__ void __launch_bounds__(MB) k_mlp_fwd_bwd(const float* __restrict__ prm, const float* __restrict__ feat,
                                                    const float* __restrict__ label,
                                                    const int32_t* __restrict__ idx, int base, int count,
                                                    float inv_batch, float* __restrict__ part,
                                                    double* __restrict__ loss_sum) {
    extern __shared__ float sm[];
    float* sW1 = sm;                       // H*NF
    float* sB1 = sW1 + H * NF;             // H
    float* sW2 = sB1 + H;                  // H*H
    float* sB2 = sW2 + H * H;              // H
    float* sW3 = sB2 + H;                  // H
    float* sX = sW3 + H;                   // MB*NF
    float* sH1 = sX + MB * NF;             // MB*HP
    float* sH2 = sH1 + MB * HP;            // MB*HP
    float* sD2 = sH2 + MB * HP;            // MB*HP
    float* sD1 = sD2 + MB * HP;            // MB*HP
    float* sDz = sD1 + MB * HP;            // MB
    __shared__ float s_loss[MB / 32];
    const int tid = threadIdx.x;
    for (int i = tid; i < OFF_B3; i += MB) sm[i] = prm[i];
    const float b3 = prm[OFF_B3];
    __syncthreads();
    const int s = tid;
    const int gi = blockIdx.x * MB + s;
    const bool live = gi < count;
    float loss = 0.f;
    {
        float x[NF];
        const int id = live ? idx[base + gi] : 0;
#pragma unroll
        for (int k = 0; k < NF; ++k) {
            x[k] = live ? (feat[(size_t)id * NF + k] - prm[OFF_MU + k]) / prm[OFF_SIG + k] : 0.f;
            sX[s * NF + k] = x[k];
        }
        for (int i = 0; i < H; ++i) {
            float a = sB1[i];
#pragma unroll
            for (int k = 0; k < NF; ++k) a = fmaf(sW1[i * NF + k], x[k], a);
            sH1[s * HP + i] = fmaxf(a, 0.f);
        }
        float z = b3;
        for (int i = 0; i < H; ++i) {
            float a = sB2[i];
            for (int j = 0; j < H; ++j) a = fmaf(sW2[i * H + j], sH1[s * HP + j], a);
            a = fmaxf(a, 0.f);
            sH2[s * HP + i] = a;
            z = fmaf(sW3[i], a, z);
        }
        const float y = live ? label[id] : 0.f;
        const float p = sigmoidf_(z);
        // BCE with logits: max(z, 0) - z y + log(1 + exp(-|z|))
        loss = live ? fmaxf(z, 0.f) - z * y + log1pf(__expf(-fabsf(z))) : 0.f;
        const float dz = live ? (p - y) * inv_batch : 0.f;
        sDz[s] = dz;
        for (int i = 0; i < H; ++i) sD2[s * HP + i] = sH2[s * HP + i] > 0.f ? dz * sW3[i] : 0.f;
        for (int j = 0; j < H; ++j) {
            float a = 0.f;
            if (sH1[s * HP + j] > 0.f)
                for (int i = 0; i < H; ++i) a = fmaf(sW2[i * H + j], sD2[s * HP + i], a);
            sD1[s * HP + j] = a;
        }
    }
    for (int o = 16; o; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if ((tid & 31) == 0) s_loss[tid >> 5] = loss;
    __syncthreads();
    if (tid == 0 && loss_sum) {
        float l = 0.f;
        for (int w = 0; w < MB / 32; ++w) l += s_loss[w];
        atomicAdd(loss_sum, (double)l);
    }
    // partial gradients, one output per thread and loop step, summed over the block's samples in order
    float* out = part + (size_t)blockIdx.x * N_TRAIN;
    for (int e = tid; e < N_TRAIN; e += MB) {
        float g = 0.f;
        if (e < OFF_B1) {                       // W1[i][k] = sum d1[s][i] x[s][k]
            const int i = e / NF, k = e - i * NF;
            for (int q = 0; q < MB; ++q) g = fmaf(sD1[q * HP + i], sX[q * NF + k], g);
        } else if (e < OFF_W2) {                // b1[i]
            const int i = e - OFF_B1;
            for (int q = 0; q < MB; ++q) g += sD1[q * HP + i];
        } else if (e < OFF_B2) {                // W2[i][j] = sum d2[s][i] h1[s][j]
            const int r = e - OFF_W2, i = r / H, j = r - i * H;
            for (int q = 0; q < MB; ++q) g = fmaf(sD2[q * HP + i], sH1[q * HP + j], g);
        } else if (e < OFF_W3) {                // b2[i]
            const int i = e - OFF_B2;
            for (int q = 0; q < MB; ++q) g += sD2[q * HP + i];
        } else if (e < OFF_B3) {                // w3[i] = sum dz[s] h2[s][i]
            const int i = e - OFF_W3;
            for (int q = 0; q < MB; ++q) g = fmaf(sDz[q], sH2[q * HP + i], g);
        } else {                                // b3
            for (int q = 0; q < MB; ++q) g += sDz[q];
        }
        out[e] = g;
    }
}

// Sum of the partial gradients (block order) and one Adam step. step_ctr holds the number of
// steps taken so far; k_mlp_step_done increments it after the update.
__global__ void k_mlp_adam(float* __restrict__ prm, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ part, int nparts, const int* __restrict__ step_ctr, float lr,
                           float* __restrict__ grad_out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= N_TRAIN) return;
    float g = 0.f;
    for (int b = 0; b < nparts; ++b) g += part[(size_t)b * N_TRAIN + e];
    if (grad_out) grad_out[e] = g;
    if (!m) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const int t = *step_ctr + 1;
    const float mm = b1 * m[e] + (1.f - b1) * g;
    const float vv = b2 * v[e] + (1.f - b2) * g * g;
    m[e] = mm;
    v[e] = vv;
    const float mh = mm / (1.f - powf(b1, (float)t)), vh = vv / (1.f - powf(b2, (float)t));
    prm[e] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void k_mlp_step_done(int* step_ctr) { ++*step_ctr; }

__global__ void k_mlp_perm_keys(int n, const int* __restrict__ epoch_ctr, uint32_t seed, uint32_t* __restrict__ key,
                                int32_t* __restrict__ val) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // splitmix-style 32-bit hash of (seed, epoch, i)
    uint32_t h = seed ^ (0x9E3779B9u * (uint32_t)(*epoch_ctr + 1)) ^ (0x85EBCA6Bu * (uint32_t)i);
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    key[i] = h;
    val[i] = i;
}

__global__ void k_mlp_epoch_done(int* epoch_ctr) { ++*epoch_ctr; }

// ------------------------------------------------------------------------ inference
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

template <bool BF16>
__global__ void __launch_bounds__(256) k_mlp_infer(const float* __restrict__ prm, int n, const float* __restrict__ feat,
                                                   float* __restrict__ prob) {
    __shared__ float sW[OFF_B3 + 1];
    for (int i = threadIdx.x; i <= OFF_B3; i += blockDim.x) {
        const bool weight = i < OFF_B1 || (i >= OFF_W2 && i < OFF_B2) || (i >= OFF_W3 && i < OFF_B3);
        sW[i] = BF16 && weight ? bf16r(prm[i]) : prm[i];
    }
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[NF];
#pragma unroll
    for (int k = 0; k < NF; ++k) {
        x[k] = (feat[(size_t)s * NF + k] - prm[OFF_MU + k]) / prm[OFF_SIG + k];
        if (BF16) x[k] = bf16r(x[k]);
    }
    float h1[H];
#pragma unroll
    for (int i = 0; i < H; ++i) {
        float a = sW[OFF_B1 + i];
#pragma unroll
        for (int k = 0; k < NF; ++k) a = fmaf(sW[OFF_W1 + i * NF + k], x[k], a);
        a = fmaxf(a, 0.f);
        h1[i] = BF16 ? bf16r(a) : a;
    }
    float z = sW[OFF_B3];
    for (int i = 0; i < H; ++i) {
        float a = sW[OFF_B2 + i];
#pragma unroll
        for (int j = 0; j < H; ++j) a = fmaf(sW[OFF_W2 + i * H + j], h1[j], a);
        a = fmaxf(a, 0.f);
        if (BF16) a = bf16r(a);
        z = fmaf(sW[OFF_W3 + i], a, z);
    }
    prob[s] = sigmoidf_(z);
}

__global__ void k_mlp_accept(int n, const int32_t* __restrict__ t1, const float* __restrict__ b12,
                             const float* __restrict__ prob, float thr, float ratio, int32_t* __restrict__ t_row,
                             uint32_t* __restrict__ d_row) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int t = t1[i];
    bool ok = false;
    if (t >= 0) {
        if (prob) {
            ok = prob[i] > thr;
        } else {   // plain ratio test (app/planesite/matching.py:142-146; a single candidate passes)
            ok = __fsqrt_rn(fmaxf(b12[2 * i], 0.f)) < __fmul_rn(ratio, __fsqrt_rn(b12[2 * i + 1]));
        }
    }
    t_row[i] = ok ? t : -1;
    d_row[i] = ok ? (uint32_t)b12[2 * i] : 0u;
}

size_t fwd_bwd_smem() { return sizeof(float) * (size_t)(OFF_B3 + MB * NF + 4 * MB * HP + MB); }

int32_t configure_fwd_bwd() {
    static std::atomic<int> done[64];
    return smem_attr((const void*)k_mlp_fwd_bwd, (int)fwd_bwd_smem(), done);
}

}  // namespace

int mlp_param_count() { return N_PARAM; }
int mlp_trainable_count() { return N_TRAIN; }

int32_t run_mlp_features(int n, const int32_t* t1, const float* b12, const double* pred, const float* xy_b,
                         const float* size_a, const float* angle_a, const float* resp_a, const int32_t* oct_a,
                         const float* size_b, const float* angle_b, const float* resp_b, float radius, float* feat,
                         cudaStream_t s) {
    if (n <= 0) return FSB_OK;
    k_mlp_features<<<nblk(n, 256), 256, 0, s>>>(n, t1, b12, pred, xy_b, size_a, angle_a, resp_a, oct_a, size_b,
                                                angle_b, resp_b, radius, feat);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

int32_t run_mlp_infer(const float* prm, int n, const float* feat, bool bf16, float* prob, cudaStream_t s) {
    if (n <= 0) return FSB_OK;
    if (bf16) k_mlp_infer<true><<<nblk(n, 256), 256, 0, s>>>(prm, n, feat, prob);
    else k_mlp_infer<false><<<nblk(n, 256), 256, 0, s>>>(prm, n, feat, prob);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

int32_t run_mlp_accept(int n, const int32_t* t1, const float* b12, const float* prob, float thr, float ratio,
                       int32_t* t_row, uint32_t* d_row, cudaStream_t s) {
    if (n <= 0) return FSB_OK;
    k_mlp_accept<<<nblk(n, 256), 256, 0, s>>>(n, t1, b12, prob, thr, ratio, t_row, d_row);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

// Mean-BCE gradient over samples idx[0..n) (identity when idx is null) into grad (N_TRAIN floats).
int32_t run_mlp_grad(fsb_ctx* ctx, const float* prm, int n, const float* feat, const float* label, float* grad,
                     double* loss, cudaStream_t s) {
    FSB_TRY(configure_fwd_bwd());
    const int nb = (int)nblk(n, MB);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    FSB_TRY(ctx->s_misc.ensure(al((size_t)nb * N_TRAIN * 4) + al((size_t)n * 4) + al(64)));
    uint8_t* base = ctx->s_misc.as<uint8_t>();
    float* part = reinterpret_cast<float*>(base);
    int32_t* idx = reinterpret_cast<int32_t*>(base + al((size_t)nb * N_TRAIN * 4));
    double* dl = reinterpret_cast<double*>(base + al((size_t)nb * N_TRAIN * 4) + al((size_t)n * 4));
    std::vector<int32_t> iota(n);
    for (int i = 0; i < n; ++i) iota[i] = i;
    FSB_CUDA(cudaMemcpyAsync(idx, iota.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemsetAsync(dl, 0, 8, s));
    k_mlp_fwd_bwd<<<nb, MB, fwd_bwd_smem(), s>>>(prm, feat, label, idx, 0, n, 1.f / (float)n, part, dl);
    k_mlp_adam<<<nblk(N_TRAIN, 256), 256, 0, s>>>(nullptr, nullptr, nullptr, part, nb, nullptr, 0.f, grad);
    note_launch(2);
    FSB_CUDA(cudaGetLastError());
    double h = 0.0;
    FSB_CUDA(cudaMemcpyAsync(&h, dl, 8, cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = h / (double)n;
    return FSB_OK;
}

// Mini-batch Adam over n samples for `epochs` epochs. prm (N_PARAM), m, v (N_TRAIN) in device memory.
// Each epoch: shuffle (hash keys + radix sort), then floor(n / batch) steps (one step of n when
// n < batch). The epoch is captured once as a CUDA graph and replayed. losses (host, nullable,
// `epochs` entries) receives the mean training loss of every epoch.
int32_t run_mlp_train(fsb_ctx* ctx, float* prm, float* m, float* v, int n, const float* feat, const float* label,
                      int epochs, int batch, float lr, uint32_t seed, double* losses, cudaStream_t s) {
    FSB_TRY(configure_fwd_bwd());
    batch = std::max(MB, (batch / MB) * MB);
    const int bsz = n < batch ? n : batch;
    const int steps = n < batch ? 1 : n / batch;
    const int nb = (int)nblk(bsz, MB);
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, (uint32_t*)nullptr, (uint32_t*)nullptr, (int32_t*)nullptr,
                                    (int32_t*)nullptr, n, 0, 32, s);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t need = al((size_t)nb * N_TRAIN * 4) + 4 * al((size_t)n * 4) + al(tb) + 2 * al(64);
    FSB_TRY(ctx->s_misc.ensure(need));
    uint8_t* cur = ctx->s_misc.as<uint8_t>();
    auto take = [&](size_t bytes) {
        uint8_t* p = cur;
        cur += (bytes + 255) & ~size_t(255);
        return p;
    };
    float* part = reinterpret_cast<float*>(take((size_t)nb * N_TRAIN * 4));
    uint32_t* keys = reinterpret_cast<uint32_t*>(take((size_t)n * 4));
    uint32_t* keys2 = reinterpret_cast<uint32_t*>(take((size_t)n * 4));
    int32_t* vals = reinterpret_cast<int32_t*>(take((size_t)n * 4));
    int32_t* perm = reinterpret_cast<int32_t*>(take((size_t)n * 4));
    void* tmp = take(tb);
    int* ctr = reinterpret_cast<int*>(take(64));      // [0] steps, [1] epochs
    double* dl = reinterpret_cast<double*>(take(64));
    FSB_CUDA(cudaMemsetAsync(ctr, 0, 64, s));
    FSB_CUDA(cudaMemsetAsync(dl, 0, 64, s));
    FSB_CUDA(cudaMemsetAsync(m, 0, (size_t)N_TRAIN * 4, s));
    FSB_CUDA(cudaMemsetAsync(v, 0, (size_t)N_TRAIN * 4, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    // capture one epoch
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    FSB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    k_mlp_perm_keys<<<nblk(n, 256), 256, 0, s>>>(n, ctr + 1, seed, keys, vals);
    cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, vals, perm, n, 0, 32, s);
    for (int st = 0; st < steps; ++st) {
        k_mlp_fwd_bwd<<<nb, MB, fwd_bwd_smem(), s>>>(prm, feat, label, perm, st * bsz, bsz, 1.f / (float)bsz, part, dl);
        k_mlp_adam<<<nblk(N_TRAIN, 256), 256, 0, s>>>(prm, m, v, part, nb, ctr, lr, nullptr);
        k_mlp_step_done<<<1, 1, 0, s>>>(ctr);
    }
    k_mlp_epoch_done<<<1, 1, 0, s>>>(ctr + 1);
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ce != cudaSuccess) {
        set_error("graph capture of the training epoch failed: %s", cudaGetErrorString(ce));
        return FSB_ERR_CUDA;
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        set_error("graph instantiation failed: %s", cudaGetErrorString(ce));
        return FSB_ERR_CUDA;
    }
    int32_t rc = FSB_OK;
    for (int e = 0; e < epochs && rc == FSB_OK; ++e) {
        if (cudaMemsetAsync(dl, 0, 8, s) != cudaSuccess || cudaGraphLaunch(exec, s) != cudaSuccess) {
            set_error("training epoch launch failed: %s", cudaGetErrorString(cudaGetLastError()));
            rc = FSB_ERR_CUDA;
            break;
        }
        note_launch(3 * steps + 3);
        if (losses) {
            double h = 0.0;
            cudaMemcpyAsync(&h, dl, 8, cudaMemcpyDeviceToHost, s);
            if (cudaStreamSynchronize(s) != cudaSuccess) {
                set_error("training epoch failed: %s", cudaGetErrorString(cudaGetLastError()));
                rc = FSB_ERR_CUDA;
                break;
            }
            losses[e] = h / ((double)steps * bsz);
        }
    }
    if (rc == FSB_OK && cudaStreamSynchronize(s) != cudaSuccess) {
        set_error("training failed: %s", cudaGetErrorString(cudaGetLastError()));
        rc = FSB_ERR_CUDA;
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    return rc;
}

}  // namespace fsb
