// Descriptor matching on uint8 RootSIFT descriptors.
//
//   k_bf_fp32     exhaustive nearest / second-nearest squared distance, CUDA-core FP32 tiles
//                 (the plain path of matching._ratio_match_bf, app/planesite/matching.py:86-100)
//   k_bf_merge    merge of the per-split top-2, float32 ratio test
//   k_guided      prior-guided candidates within a radius on a uniform grid, exact integer
//                 distances (matching._guided, app/planesite/matching.py:113-152)
//   k_unique      one match per target: atomicMin on (distance << 32 | query) keys
//                 (matching._unique, app/planesite/matching.py:103-110), then target-ordered
//                 compaction
//
// Exactness: descriptors are uint8 and every squared distance na + nb - 2 a.b is an integer below
// 2^24, so FP32 FMA accumulation in any order, integer dp4a, and BF16 x BF16 -> FP32 tensor-core
// products all give the same values as the reference's float32 BLAS. Results therefore depend only
// on the values and the tie rules, which follow the reference.
#include <cub/cub.cuh>

#include <mutex>

#include "fsb_internal.cuh"

namespace fsb {
namespace {

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// squared L2 norm of each uint8 row (exact integer)
__global__ void k_norms(const uint8_t* __restrict__ d, int n, int32_t* __restrict__ out) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const uint32_t w = reinterpret_cast<const uint32_t*>(d + (size_t)row * 128)[lane];
    int s = (int)__dp4a(w, w, 0u);
    for (int sh = 16; sh; sh >>= 1) s += __shfl_xor_sync(0xffffffffu, s, sh);
    if (lane == 0) out[row] = s;
}

// ------------------------------------------------------------------------- FP32 dense tiles
constexpr int BM = 128, BN = 128, BK = 32, TM = 8, TN = 8, BF_THREADS = 256;

struct Top2 {
    float b1, b2;
    int i1;
};

__device__ __forceinline__ void top2_push(Top2& t, float d, int j) {
    if (d < t.b1) {
        t.b2 = t.b1;
        t.b1 = d;
        t.i1 = j;
    } else if (d < t.b2) {
        t.b2 = d;
    }
}

__device__ __forceinline__ Top2 top2_merge(Top2 a, Top2 b) {
    Top2 r;
    if (a.b1 < b.b1 || (a.b1 == b.b1 && a.i1 <= b.i1)) {
        r.b1 = a.b1; r.i1 = a.i1; r.b2 = fminf(a.b2, b.b1);
    } else {
        r.b1 = b.b1; r.i1 = b.i1; r.b2 = fminf(b.b2, a.b1);
    }
    return r;
}

// grid: (row blocks, splits of B). Each CTA sweeps B rows [n0, n1) for 128 A rows and writes the
// per-row top-2 of its split.
__global__ void __launch_bounds__(BF_THREADS) k_bf_fp32(const uint8_t* __restrict__ A, int na,
                                                        const uint8_t* __restrict__ B, int nb,
                                                        const int32_t* __restrict__ nA, const int32_t* __restrict__ nB,
                                                        int split_len, Top2* __restrict__ part) {
    // operand tiles during the sweep; the same bytes hold the row merge afterwards
    constexpr size_t kTileBytes = 2 * sizeof(float) * BK * (BM + 4);
    constexpr size_t kRedBytes = sizeof(Top2) * 16 * BM;
    __shared__ __align__(16) unsigned char smem[kTileBytes > kRedBytes ? kTileBytes : kRedBytes];
    float (*As)[BM + 4] = reinterpret_cast<float (*)[BM + 4]>(smem);
    float (*Bs)[BN + 4] = reinterpret_cast<float (*)[BN + 4]>(smem + sizeof(float) * BK * (BM + 4));
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.x * BM;
    const int n_begin = blockIdx.y * split_len;
    const int n_end = min(nb, n_begin + split_len);
    Top2 best[TM];
#pragma unroll
    for (int i = 0; i < TM; ++i) best[i] = Top2{INFINITY, INFINITY, -1};
    float rn[TM];
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int r = m0 + ty + 16 * i;
        rn[i] = r < na ? (float)nA[r] : 0.f;
    }
    for (int n0 = n_begin; n0 < n_end; n0 += BN) {
        float acc[TM][TN];
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) acc[i][j] = 0.f;
        for (int k0 = 0; k0 < 128; k0 += BK) {
            // stage 128 x 32 bytes of A and B as float, transposed (k-major)
            for (int e = tid; e < BM * (BK / 4); e += BF_THREADS) {
                const int r = e / (BK / 4), q = e - r * (BK / 4);
                uint32_t wa = 0, wb = 0;
                if (m0 + r < na) wa = reinterpret_cast<const uint32_t*>(A + (size_t)(m0 + r) * 128 + k0)[q];
                if (n0 + r < n_end) wb = reinterpret_cast<const uint32_t*>(B + (size_t)(n0 + r) * 128 + k0)[q];
#pragma unroll
                for (int b = 0; b < 4; ++b) {
                    As[q * 4 + b][r] = (float)((wa >> (8 * b)) & 255u);
                    Bs[q * 4 + b][r] = (float)((wb >> (8 * b)) & 255u);
                }
            }
            __syncthreads();
#pragma unroll 4
            for (int kk = 0; kk < BK; ++kk) {
                float a[TM], b[TN];
#pragma unroll
                for (int i = 0; i < TM; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
                for (int j = 0; j < TN; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
                for (int i = 0; i < TM; ++i)
#pragma unroll
                    for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
            }
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int c = n0 + tx + 16 * j;
            if (c >= n_end) continue;
            const float cn = (float)nB[c];
#pragma unroll
            for (int i = 0; i < TM; ++i) top2_push(best[i], (rn[i] + cn) - 2.f * acc[i][j], c);
        }
    }
    // merge the 16 column groups of each row through shared memory
    Top2 (*red)[BM] = reinterpret_cast<Top2 (*)[BM]>(smem);
#pragma unroll
    for (int i = 0; i < TM; ++i) red[tx][ty + 16 * i] = best[i];
    __syncthreads();
    if (tid < BM) {
        Top2 t = red[0][tid];
        for (int g = 1; g < 16; ++g) t = top2_merge(t, red[g][tid]);
        const int r = m0 + tid;
        if (r < na) part[(size_t)blockIdx.y * na + r] = t;
    }
}

// merge the splits, ratio test (float32, app/planesite/matching.py:96-99)
__global__ void k_bf_merge(const Top2* __restrict__ part, int na, int splits, float ratio,
                           int32_t* __restrict__ t_row, uint32_t* __restrict__ d_row) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= na) return;
    Top2 t = part[r];
    for (int s = 1; s < splits; ++s) t = top2_merge(t, part[(size_t)s * na + r]);
    const float b1 = fmaxf(t.b1, 0.f), b2 = fmaxf(t.b2, 0.f);
    const bool ok = __fsqrt_rn(b1) < __fmul_rn(ratio, __fsqrt_rn(b2));
    t_row[r] = ok ? t.i1 : -1;
    d_row[r] = (uint32_t)b1;
}

// ------------------------------------------------------------------------------ one-to-one
__global__ void k_fill_u64(unsigned long long* p, int n, unsigned long long v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void k_unique_keys(const int32_t* __restrict__ t_row, const uint32_t* __restrict__ d_row, int na,
                              unsigned long long* __restrict__ key) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= na) return;
    const int t = t_row[r];
    if (t >= 0) atomicMin(key + t, ((unsigned long long)d_row[r] << 32) | (unsigned)r);
}

__global__ void k_unique_flags(const unsigned long long* __restrict__ key, int nb, uint8_t* __restrict__ flag,
                               int32_t* __restrict__ iota) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    flag[t] = key[t] != ~0ull;
    iota[t] = t;
}

__global__ void k_unique_emit(const unsigned long long* __restrict__ key, const int32_t* __restrict__ tsel,
                              const int* __restrict__ n, int64_t* __restrict__ q, int64_t* __restrict__ t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *n) return;
    const int tt = tsel[i];
    q[i] = (int64_t)(key[tt] & 0xffffffffull);
    t[i] = tt;
}

// ------------------------------------------------------------------------------ guided
struct GridSpec {
    double x0, y0, cs;   // origin and cell size
    int gw, gh;
};

__device__ __forceinline__ int cell_of(double v, double o, double cs, int n) {
    const double f = floor((v - o) / cs);
    return f < 0.0 ? 0 : (f >= (double)(n - 1) ? n - 1 : (int)f);
}

__global__ void k_grid_count(const double* __restrict__ bxy, int nb, GridSpec gs, int32_t* __restrict__ cell,
                             int32_t* __restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const int cx = cell_of(bxy[2 * i], gs.x0, gs.cs, gs.gw), cy = cell_of(bxy[2 * i + 1], gs.y0, gs.cs, gs.gh);
    const int c = cy * gs.gw + cx;
    cell[i] = c;
    atomicAdd(count + c, 1);
}

__global__ void k_grid_fill(const int32_t* __restrict__ cell, int nb, const int32_t* __restrict__ start,
                            int32_t* __restrict__ cursor, int32_t* __restrict__ items) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const int c = cell[i];
    items[start[c] + atomicAdd(cursor + c, 1)] = i;
}

constexpr int G_WARPS = 4, G_CAND = 512;

__device__ __forceinline__ int exact_d2(const uint32_t* __restrict__ qa, const uint8_t* __restrict__ B, int j,
                                        int qn, const int32_t* __restrict__ nB) {
    const uint4* pb = reinterpret_cast<const uint4*>(B + (size_t)j * 128);
    unsigned dot = 0;
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        const uint4 w = __ldg(pb + v);
        dot = __dp4a(qa[4 * v + 0], w.x, dot);
        dot = __dp4a(qa[4 * v + 1], w.y, dot);
        dot = __dp4a(qa[4 * v + 2], w.z, dot);
        dot = __dp4a(qa[4 * v + 3], w.w, dot);
    }
    return (qn + nB[j]) - 2 * (int)dot;
}

// One query of the guided matcher (one warp): candidates of the prior window, exact distances,
// top-2, ratio test; writes t_row/d_row (nullable) and the pre-ratio candidate (c_t, nullable).
__device__ __forceinline__ void guided_query(int q, const double* __restrict__ pred, const uint8_t* __restrict__ A,
                                             int na, const double* __restrict__ bxy,
                                             const uint8_t* __restrict__ B, int nb,
                                             const int32_t* __restrict__ nA, const int32_t* __restrict__ nB,
                                             GridSpec gs, const int32_t* __restrict__ start,
                                             const int32_t* __restrict__ items, double wb, double hb,
                                             double radius, int kc, float ratio,
                                             int32_t* __restrict__ t_row, uint32_t* __restrict__ d_row,
                                             int32_t* __restrict__ c_t, float* __restrict__ c_b12,
                                             int* __restrict__ overflow, uint32_t (*s_q)[32],
                                             double (*s_cd)[G_CAND], int32_t (*s_ci)[G_CAND]) {
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (q >= na) return;
    const double px = pred[2 * q], py = pred[2 * q + 1];
    int32_t res_t = -1;
    uint32_t res_d = 0;
    int32_t cand_t = -1;
    float cand_b1 = INFINITY, cand_b2 = INFINITY;
    const bool inside = px > -radius && px < wb + radius && py > -radius && py < hb + radius;
    if (inside) {
        s_q[wid][lane] = reinterpret_cast<const uint32_t*>(A + (size_t)q * 128)[lane];
        __syncwarp();
        uint32_t qa[32];
#pragma unroll
        for (int v = 0; v < 32; ++v) qa[v] = s_q[wid][v];
        const int qn = nA[q];
        const double r2 = radius * radius;
        const int cx = cell_of(px, gs.x0, gs.cs, gs.gw), cy = cell_of(py, gs.y0, gs.cs, gs.gh);
        Top2 best{INFINITY, INFINITY, -1};
        if (kc <= 0) {
            // every B keypoint strictly within the radius is a candidate
            for (int yy = max(cy - 1, 0); yy <= min(cy + 1, gs.gh - 1); ++yy)
                for (int xx = max(cx - 1, 0); xx <= min(cx + 1, gs.gw - 1); ++xx) {
                    const int c = yy * gs.gw + xx;
                    const int s0 = start[c], s1 = start[c + 1];
                    for (int p = s0 + lane; p < s1; p += 32) {
                        const int j = items[p];
                        const double dx = __dsub_rn(bxy[2 * j], px), dy = __dsub_rn(bxy[2 * j + 1], py);
                        const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
                        if (d2 < r2) top2_push(best, (float)exact_d2(qa, B, j, qn, nB), j);
                    }
                }
        } else {
            // collect candidates (spatial distance, index) in shared memory
            int cnt = 0;
            for (int yy = max(cy - 1, 0); yy <= min(cy + 1, gs.gh - 1); ++yy)
                for (int xx = max(cx - 1, 0); xx <= min(cx + 1, gs.gw - 1); ++xx) {
                    const int c = yy * gs.gw + xx;
                    const int s0 = start[c], s1 = start[c + 1];
                    for (int p0 = s0; p0 < s1; p0 += 32) {
                        const int p = p0 + lane;
                        bool hit = false;
                        double d2 = 0.0;
                        int j = 0;
                        if (p < s1) {
                            j = items[p];
                            const double dx = __dsub_rn(bxy[2 * j], px), dy = __dsub_rn(bxy[2 * j + 1], py);
                            d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
                            hit = d2 < r2;
                        }
                        const unsigned m = __ballot_sync(0xffffffffu, hit);
                        if (hit) {
                            const int pos = cnt + __popc(m & ((1u << lane) - 1u));
                            if (pos < G_CAND) {
                                s_cd[wid][pos] = d2;
                                s_ci[wid][pos] = j;
                            }
                        }
                        cnt += __popc(m);
                    }
                }
            __syncwarp();
            if (cnt > G_CAND) {
                if (lane == 0) atomicExch(overflow, 1);
                cnt = G_CAND;
            }
            // keep the kc nearest (ties: smaller B index)
            for (int e = lane; e < cnt; e += 32) {
                const double de = s_cd[wid][e];
                const int ie = s_ci[wid][e];
                int rank = 0;
                if (cnt > kc)
                    for (int f = 0; f < cnt; ++f) {
                        const double df = s_cd[wid][f];
                        rank += (df < de || (df == de && s_ci[wid][f] < ie)) ? 1 : 0;
                    }
                if (rank < kc) top2_push(best, (float)exact_d2(qa, B, ie, qn, nB), ie);
            }
        }
        // warp merge of the per-lane top-2
#pragma unroll
        for (int sh = 16; sh; sh >>= 1) {
            Top2 o;
            o.b1 = __shfl_xor_sync(0xffffffffu, best.b1, sh);
            o.b2 = __shfl_xor_sync(0xffffffffu, best.b2, sh);
            o.i1 = __shfl_xor_sync(0xffffffffu, best.i1, sh);
            best = top2_merge(best, o);
        }
        cand_t = best.i1;
        cand_b1 = best.b1;
        cand_b2 = best.b2;
        if (best.i1 >= 0) {
            // single candidate: b2 = inf passes (app/planesite/matching.py:142-146)
            const bool ok = __fsqrt_rn(best.b1) < __fmul_rn(ratio, __fsqrt_rn(best.b2));
            if (ok) {
                res_t = best.i1;
                res_d = (uint32_t)best.b1;
            }
        }
    }
    if (lane == 0) {
        if (t_row) {
            t_row[q] = res_t;
            d_row[q] = res_d;
        }
        if (c_t) {   // the best candidate before the ratio test (learned filter input)
            c_t[q] = cand_t;
            c_b12[2 * q] = cand_b1;
            c_b12[2 * q + 1] = cand_b2;
        }
    }
}

__global__ void __launch_bounds__(G_WARPS * 32) k_guided(const double* __restrict__ pred, const uint8_t* __restrict__ A,
                                                         int na, const double* __restrict__ bxy,
                                                         const uint8_t* __restrict__ B, int nb,
                                                         const int32_t* __restrict__ nA, const int32_t* __restrict__ nB,
                                                         GridSpec gs, const int32_t* __restrict__ start,
                                                         const int32_t* __restrict__ items, double wb, double hb,
                                                         double radius, int kc, float ratio,
                                                         int32_t* __restrict__ t_row, uint32_t* __restrict__ d_row,
                                                         int32_t* __restrict__ c_t, float* __restrict__ c_b12,
                                                         int* __restrict__ overflow) {
    __shared__ uint32_t s_q[G_WARPS][32];
    __shared__ double s_cd[G_WARPS][G_CAND];
    __shared__ int32_t s_ci[G_WARPS][G_CAND];
    guided_query(blockIdx.x * G_WARPS + (threadIdx.x >> 5), pred, A, na, bxy, B, nb, nA, nB, gs, start, items, wb, hb,
                 radius, kc, ratio, t_row, d_row, c_t, c_b12, overflow, s_q, s_cd, s_ci);
}

__global__ void k_perspective(const double* __restrict__ xy, int n, const double* __restrict__ hm,
                              double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = xy[2 * i], y = xy[2 * i + 1];
    double w = __dadd_rn(__dadd_rn(__dmul_rn(hm[6], x), __dmul_rn(hm[7], y)), hm[8]);
    double u = 0.0, v = 0.0;
    if (fabs(w) > 1.1920928955078125e-07) {
        w = 1.0 / w;
        u = __dmul_rn(__dadd_rn(__dadd_rn(__dmul_rn(hm[0], x), __dmul_rn(hm[1], y)), hm[2]), w);
        v = __dmul_rn(__dadd_rn(__dadd_rn(__dmul_rn(hm[3], x), __dmul_rn(hm[4], y)), hm[5]), w);
    }
    out[2 * i] = u;
    out[2 * i + 1] = v;
}

// one-to-one filter + compaction ordered by target: q[i], t[i], *d_n
int32_t run_unique(fsb_ctx* ctx, const int32_t* t_row, const uint32_t* d_row, int na, int nb, int64_t* d_q,
                   int64_t* d_t, int* d_n, cudaStream_t s) {
    FSB_TRY(ctx->s_u64.ensure((size_t)nb * 8 + 64));
    FSB_TRY(ctx->s_misc2.ensure((size_t)nb * 9 + 1024));
    unsigned long long* key = ctx->s_u64.as<unsigned long long>();
    uint8_t* flag = ctx->s_misc2.as<uint8_t>();
    int32_t* iota = reinterpret_cast<int32_t*>(flag + ((nb + 255) / 256) * 256);
    int32_t* tsel = iota + nb;
    k_fill_u64<<<blocks(nb, 256), 256, 0, s>>>(key, nb, ~0ull);
    k_unique_keys<<<blocks(na, 256), 256, 0, s>>>(t_row, d_row, na, key);
    k_unique_flags<<<blocks(nb, 256), 256, 0, s>>>(key, nb, flag, iota);
    size_t tb = 0;
    cub::DeviceSelect::Flagged(nullptr, tb, iota, flag, tsel, d_n, nb, s);
    FSB_TRY(ctx->s_cub.ensure(tb + 16));
    FSB_CUDA(cub::DeviceSelect::Flagged(ctx->s_cub.p, tb, iota, flag, tsel, d_n, nb, s));
    k_unique_emit<<<blocks(nb, 256), 256, 0, s>>>(key, tsel, d_n, d_q, d_t);
    note_launch(4);
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

__device__ __forceinline__ uint32_t orderable(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__global__ void k_uq_keys1(const float* __restrict__ dd, int n, uint32_t* __restrict__ key, uint32_t* __restrict__ val) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    key[i] = orderable(dd[i]);
    val[i] = (uint32_t)i;
}

__global__ void k_uq_keys2(const int64_t* __restrict__ t, const uint32_t* __restrict__ perm, int n,
                           unsigned long long* __restrict__ key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    key[i] = (unsigned long long)t[perm[i]] ^ 0x8000000000000000ull;
}

__global__ void k_uq_first(const unsigned long long* __restrict__ key, int n, uint8_t* __restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flag[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

__global__ void k_uq_emit(const uint32_t* __restrict__ pos, const int* __restrict__ n, const int64_t* __restrict__ q,
                          const int64_t* __restrict__ t, int64_t* __restrict__ qo, int64_t* __restrict__ to) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *n) return;
    qo[i] = q[pos[i]];
    to[i] = t[pos[i]];
}


// ------------------------------------------------------------------------------ guided batch
// Many guided problems in one set of launches (blockIdx.y = pair): concatenated norms, one grid
// per pair in one concatenated cell array (one prefix sum for all), one guided kernel over every
// query of every pair, and _unique per pair over concatenated target keys.
struct GPair {
    const double* pred;
    const uint8_t* a;
    const double* bxy;
    const uint8_t* b;
    int na, nb;
    double wb, hb;
    GridSpec gs;
    int cell0;   // first cell of this pair's grid
    int item0;   // first target (B row) in the concatenated target arrays
    int row0;    // first query (A row) in the concatenated query arrays
    int64_t* q_out;
    int64_t* t_out;
};

__global__ void k_gb_norms(const GPair* __restrict__ pairs, int which, int32_t* __restrict__ out) {
    const GPair& P = pairs[blockIdx.y];
    const int n = which ? P.nb : P.na;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const uint8_t* d = which ? P.b : P.a;
    const uint32_t w = reinterpret_cast<const uint32_t*>(d + (size_t)row * 128)[lane];
    int s = (int)__dp4a(w, w, 0u);
    for (int sh = 16; sh; sh >>= 1) s += __shfl_xor_sync(0xffffffffu, s, sh);
    if (lane == 0) out[(which ? P.item0 : P.row0) + row] = s;
}

__global__ void k_gb_count(const GPair* __restrict__ pairs, int32_t* __restrict__ cell, int32_t* __restrict__ count) {
    const GPair& P = pairs[blockIdx.y];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P.nb) return;
    const int cx = cell_of(P.bxy[2 * j], P.gs.x0, P.gs.cs, P.gs.gw), cy = cell_of(P.bxy[2 * j + 1], P.gs.y0, P.gs.cs, P.gs.gh);
    const int c = P.cell0 + cy * P.gs.gw + cx;
    cell[P.item0 + j] = c;
    atomicAdd(count + c, 1);
}

__global__ void k_gb_fill(const GPair* __restrict__ pairs, const int32_t* __restrict__ cell,
                          const int32_t* __restrict__ start, int32_t* __restrict__ cursor, int32_t* __restrict__ items) {
    const GPair& P = pairs[blockIdx.y];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P.nb) return;
    const int c = cell[P.item0 + j];
    items[start[c] + atomicAdd(cursor + c, 1)] = j;   // local target index
}

__global__ void __launch_bounds__(G_WARPS * 32) k_gb_guided(const GPair* __restrict__ pairs, const int32_t* __restrict__ nA,
                                                            const int32_t* __restrict__ nB,
                                                            const int32_t* __restrict__ start,
                                                            const int32_t* __restrict__ items, double radius, int kc,
                                                            float ratio, int32_t* __restrict__ t_row,
                                                            uint32_t* __restrict__ d_row, int* __restrict__ overflow) {
    __shared__ uint32_t s_q[G_WARPS][32];
    __shared__ double s_cd[G_WARPS][G_CAND];
    __shared__ int32_t s_ci[G_WARPS][G_CAND];
    const GPair& P = pairs[blockIdx.y];
    guided_query(blockIdx.x * G_WARPS + (threadIdx.x >> 5), P.pred, P.a, P.na, P.bxy, P.b, P.nb, nA + P.row0,
                 nB + P.item0, P.gs, start + P.cell0, items, P.wb, P.hb, radius, kc, ratio, t_row + P.row0,
                 d_row + P.row0, nullptr, nullptr, overflow, s_q, s_cd, s_ci);
}

__global__ void k_gb_fill_keys(unsigned long long* __restrict__ key, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) key[i] = ~0ull;
}

__global__ void k_gb_keys(const GPair* __restrict__ pairs, const int32_t* __restrict__ t_row,
                          const uint32_t* __restrict__ d_row, unsigned long long* __restrict__ key) {
    const GPair& P = pairs[blockIdx.y];
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.na) return;
    const int t = t_row[P.row0 + q];
    if (t >= 0) atomicMin(key + P.item0 + t, ((unsigned long long)d_row[P.row0 + q] << 32) | (unsigned)q);
}

__global__ void k_gb_flags(const unsigned long long* __restrict__ key, int n, int32_t* __restrict__ flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n) flag[i] = i < n && key[i] != ~0ull;
}

__global__ void k_gb_emit(const GPair* __restrict__ pairs, const unsigned long long* __restrict__ key,
                          const int32_t* __restrict__ pos, int32_t* __restrict__ counts) {
    const GPair& P = pairs[blockIdx.y];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= P.nb) return;
    const int i = P.item0 + j;
    if (j == P.nb - 1) counts[blockIdx.y] = pos[P.item0 + P.nb] - pos[P.item0];
    const unsigned long long k = key[i];
    if (k == ~0ull) return;
    const int o = pos[i] - pos[P.item0];
    P.q_out[o] = (int64_t)(k & 0xffffffffull);
    P.t_out[o] = j;
}

}  // namespace

// General one-to-one filter (matching._unique) for arbitrary int64 targets and float distances:
// stable sorts by distance then by target give (t, dd, position) order; the first of each target
// run is kept.
int32_t run_unique_general(fsb_ctx* ctx, const int64_t* d_q, const int64_t* d_t, const float* d_dd, int n,
                           int64_t* d_qo, int64_t* d_to, int* d_n, cudaStream_t s) {
    const size_t N = (size_t)n;
    FSB_TRY(ctx->s_misc.ensure(N * (4 * 4 + 8 * 2 + 1 + 4) + 256));
    uint32_t* k1 = ctx->s_misc.as<uint32_t>();
    uint32_t* k1o = k1 + N;
    uint32_t* v1 = k1o + N;
    uint32_t* v1o = v1 + N;
    unsigned long long* k2 = reinterpret_cast<unsigned long long*>(v1o + N);
    unsigned long long* k2o = k2 + N;
    uint32_t* v2o = reinterpret_cast<uint32_t*>(k2o + N);
    uint8_t* flag = reinterpret_cast<uint8_t*>(v2o + N);
    uint32_t* sel = v1;   // reused after the second sort
    size_t t1 = 0, t2 = 0, t3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, k1, k1o, v1, v1o, n, 0, 32, s);
    cub::DeviceRadixSort::SortPairs(nullptr, t2, k2, k2o, v1o, v2o, n, 0, 64, s);
    cub::DeviceSelect::Flagged(nullptr, t3, v2o, flag, sel, d_n, n, s);
    size_t tmax = t1 > t2 ? t1 : t2;
    tmax = tmax > t3 ? tmax : t3;
    FSB_TRY(ctx->s_cub.ensure(tmax + 16));
    k_uq_keys1<<<blocks(n, 256), 256, 0, s>>>(d_dd, n, k1, v1);
    size_t tb = tmax;
    FSB_CUDA(cub::DeviceRadixSort::SortPairs(ctx->s_cub.p, tb, k1, k1o, v1, v1o, n, 0, 32, s));
    k_uq_keys2<<<blocks(n, 256), 256, 0, s>>>(d_t, v1o, n, k2);
    tb = tmax;
    FSB_CUDA(cub::DeviceRadixSort::SortPairs(ctx->s_cub.p, tb, k2, k2o, v1o, v2o, n, 0, 64, s));
    k_uq_first<<<blocks(n, 256), 256, 0, s>>>(k2o, n, flag);
    tb = tmax;
    FSB_CUDA(cub::DeviceSelect::Flagged(ctx->s_cub.p, tb, v2o, flag, sel, d_n, n, s));
    k_uq_emit<<<blocks(n, 256), 256, 0, s>>>(sel, d_n, d_q, d_t, d_qo, d_to);
    note_launch(4);
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

struct H9 {
    double h[9];
};

// float32 points -> float64 positions through a homography, plus optional float32 offsets
__global__ void k_project(const float* __restrict__ xy, int n, H9 H, const float* __restrict__ off,
                          double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = (double)xy[2 * i], y = (double)xy[2 * i + 1];
    const double* hm = H.h;
    double w = __dadd_rn(__dadd_rn(__dmul_rn(hm[6], x), __dmul_rn(hm[7], y)), hm[8]);
    double u = 0.0, v = 0.0;
    if (fabs(w) > 1.1920928955078125e-07) {
        w = 1.0 / w;
        u = __dmul_rn(__dadd_rn(__dadd_rn(__dmul_rn(hm[0], x), __dmul_rn(hm[1], y)), hm[2]), w);
        v = __dmul_rn(__dadd_rn(__dadd_rn(__dmul_rn(hm[3], x), __dmul_rn(hm[4], y)), hm[5]), w);
    }
    if (off) {
        u += (double)off[2 * i];
        v += (double)off[2 * i + 1];
    }
    out[2 * i] = u;
    out[2 * i + 1] = v;
}

int32_t run_project(const float* d_xy, int n, const double* hm9, const float* d_off, double* d_out, cudaStream_t s) {
    if (n <= 0) return FSB_OK;
    H9 H;
    for (int i = 0; i < 9; ++i) H.h[i] = hm9[i];
    k_project<<<blocks(n, 256), 256, 0, s>>>(d_xy, n, H, d_off, d_out);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

int32_t run_perspective(const double* d_xy, int n, const double* d_hm9, double* d_out, cudaStream_t s) {
    if (n <= 0) return FSB_OK;
    k_perspective<<<blocks(n, 256), 256, 0, s>>>(d_xy, n, d_hm9, d_out);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

int32_t run_match_bf(fsb_ctx* ctx, const uint8_t* d_a, int na, const uint8_t* d_b, int nb, float ratio,
                     int precision, int64_t* d_q, int64_t* d_t, int* d_n, cudaStream_t s) {
    if (na < 2 || nb < 2) {
        FSB_CUDA(cudaMemsetAsync(d_n, 0, sizeof(int), s));
        return FSB_OK;
    }
    if (precision != FSB_PREC_FP32)
        return run_match_bf_tc(ctx, 1, &d_a, &na, &d_b, &nb, ratio, precision, &d_q, &d_t, d_n, &ctx->tc_stats, s);
    const int row_blocks = (na + BM - 1) / BM;
    int splits = 1;
    while (row_blocks * splits < 2 * 148 && (nb + splits * 2 - 1) / (splits * 2) >= BN) splits *= 2;
    int split_len = (nb + splits - 1) / splits;
    split_len = ((split_len + BN - 1) / BN) * BN;
    splits = (nb + split_len - 1) / split_len;
    FSB_TRY(ctx->s_i32.ensure((size_t)(na + nb) * 4 + (size_t)na * 8 + 64));
    int32_t* nA = ctx->s_i32.as<int32_t>();
    int32_t* nB = nA + na;
    int32_t* t_row = nB + nb;
    uint32_t* d_row = reinterpret_cast<uint32_t*>(t_row + na);
    FSB_TRY(ctx->s_misc.ensure((size_t)splits * na * sizeof(Top2) + 64));
    Top2* part = ctx->s_misc.as<Top2>();
    k_norms<<<blocks(na, 8), 256, 0, s>>>(d_a, na, nA);
    k_norms<<<blocks(nb, 8), 256, 0, s>>>(d_b, nb, nB);
    k_bf_fp32<<<dim3(row_blocks, splits), BF_THREADS, 0, s>>>(d_a, na, d_b, nb, nA, nB, split_len, part);
    k_bf_merge<<<blocks(na, 256), 256, 0, s>>>(part, na, splits, ratio, t_row, d_row);
    note_launch(4);
    FSB_CUDA(cudaGetLastError());
    return run_unique(ctx, t_row, d_row, na, nb, d_q, d_t, d_n, s);
}

int32_t run_unique_rows(fsb_ctx* ctx, const int32_t* t_row, const uint32_t* d_row, int na, int nb, int64_t* d_q,
                        int64_t* d_t, int* d_n, cudaStream_t s) {
    return run_unique(ctx, t_row, d_row, na, nb, d_q, d_t, d_n, s);
}

int32_t run_match_guided(fsb_ctx* ctx, const double* d_pred, const uint8_t* d_a, int na, const double* d_bxy,
                         const uint8_t* d_b, int nb, double wb, double hb, double radius, int kc, float ratio,
                         int64_t* d_q, int64_t* d_t, int* d_n, cudaStream_t s, int32_t* c_t, float* c_b12) {
    if (na < 1 || nb < 1 || !(radius > 0.0)) {
        if (d_n) FSB_CUDA(cudaMemsetAsync(d_n, 0, sizeof(int), s));
        if (c_t && na > 0) FSB_CUDA(cudaMemsetAsync(c_t, 0xff, (size_t)na * 4, s));
        return FSB_OK;
    }
    GridSpec gs;
    gs.x0 = 0.0;
    gs.y0 = 0.0;
    gs.cs = radius;
    double gwd = (wb > 0 ? wb : 1.0) / radius + 1.0, ghd = (hb > 0 ? hb : 1.0) / radius + 1.0;
    while (gwd * ghd > 4.0e6) {
        gs.cs *= 2.0;
        gwd = (wb > 0 ? wb : 1.0) / gs.cs + 1.0;
        ghd = (hb > 0 ? hb : 1.0) / gs.cs + 1.0;
    }
    gs.gw = (int)gwd;
    gs.gh = (int)ghd;
    const int ncell = gs.gw * gs.gh;
    FSB_TRY(ctx->s_i32.ensure((size_t)(na + nb) * 4 + (size_t)na * 8 + (size_t)nb * 8 + (size_t)ncell * 12 + 256));
    int32_t* nA = ctx->s_i32.as<int32_t>();
    int32_t* nB = nA + na;
    int32_t* t_row = nB + nb;
    uint32_t* d_row = reinterpret_cast<uint32_t*>(t_row + na);
    int32_t* cell = reinterpret_cast<int32_t*>(d_row + na);
    int32_t* items = cell + nb;
    int32_t* count = items + nb;      // ncell + 1
    int32_t* start = count + ncell + 1;
    int32_t* cursor = start + ncell + 1;
    int* overflow = cursor + ncell;
    FSB_CUDA(cudaMemsetAsync(count, 0, (size_t)(ncell + 1) * 4, s));
    FSB_CUDA(cudaMemsetAsync(cursor, 0, (size_t)ncell * 4 + 4, s));
    k_norms<<<blocks(na, 8), 256, 0, s>>>(d_a, na, nA);
    k_norms<<<blocks(nb, 8), 256, 0, s>>>(d_b, nb, nB);
    k_grid_count<<<blocks(nb, 256), 256, 0, s>>>(d_bxy, nb, gs, cell, count);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, count, start, ncell + 1, s);
    FSB_TRY(ctx->s_cub.ensure(tb + 16));
    FSB_CUDA(cub::DeviceScan::ExclusiveSum(ctx->s_cub.p, tb, count, start, ncell + 1, s));
    k_grid_fill<<<blocks(nb, 256), 256, 0, s>>>(cell, nb, start, cursor, items);
    note_launch(5);
    k_guided<<<blocks(na, G_WARPS), G_WARPS * 32, 0, s>>>(d_pred, d_a, na, d_bxy, d_b, nb, nA, nB, gs, start, items,
                                                          wb, hb, radius, kc, ratio, d_n ? t_row : nullptr,
                                                          d_row, c_t, c_b12, overflow);
    FSB_CUDA(cudaGetLastError());
    int h_over = 0;
    FSB_CUDA(cudaMemcpyAsync(&h_over, overflow, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    if (h_over) {
        set_error("more than %d B keypoints within the radius of one prediction (kc mode)", G_CAND);
        return FSB_ERR_OVERFLOW;
    }
    if (!d_n) return FSB_OK;   // candidates only
    return run_unique(ctx, t_row, d_row, na, nb, d_q, d_t, d_n, s);
}


// Guided matching of a batch of pairs (each na, nb >= 1, radius > 0) with _unique, as one CUDA
// graph on the context's stream: captured on the first call with a given pair table and replayed
// while the table (pointers, sizes, frames) and the scratch addresses stay the same. counts:
// device, one per pair.
int32_t run_match_guided_batch(fsb_ctx* ctx, int n_pairs, const double* const* d_pred, const uint8_t* const* d_a,
                               const int* na, const double* const* d_bxy, const uint8_t* const* d_b, const int* nb,
                               const double* wb, const double* hb, double radius, int kc, float ratio,
                               int64_t* const* d_q, int64_t* const* d_t, int32_t* counts, cudaStream_t s) {
    if (n_pairs <= 0) return FSB_OK;
    std::vector<GPair> hp(n_pairs);
    long long cells = 0, rows = 0, items = 0;
    int max_na = 0, max_nb = 0;
    for (int p = 0; p < n_pairs; ++p) {
        GPair& P = hp[p];
        P.pred = d_pred[p];
        P.a = d_a[p];
        P.bxy = d_bxy[p];
        P.b = d_b[p];
        P.na = na[p];
        P.nb = nb[p];
        P.wb = wb[p];
        P.hb = hb[p];
        GridSpec gs;
        gs.x0 = 0.0;
        gs.y0 = 0.0;
        gs.cs = radius;
        double gwd = (wb[p] > 0 ? wb[p] : 1.0) / radius + 1.0, ghd = (hb[p] > 0 ? hb[p] : 1.0) / radius + 1.0;
        while (gwd * ghd > 4.0e6) {
            gs.cs *= 2.0;
            gwd = (wb[p] > 0 ? wb[p] : 1.0) / gs.cs + 1.0;
            ghd = (hb[p] > 0 ? hb[p] : 1.0) / gs.cs + 1.0;
        }
        gs.gw = (int)gwd;
        gs.gh = (int)ghd;
        P.gs = gs;
        P.cell0 = (int)cells;
        P.item0 = (int)items;
        P.row0 = (int)rows;
        P.q_out = d_q[p];
        P.t_out = d_t[p];
        cells += (long long)gs.gw * gs.gh;
        rows += na[p];
        items += nb[p];
        max_na = std::max(max_na, na[p]);
        max_nb = std::max(max_nb, nb[p]);
    }
    if (cells + items + rows > 0x7fffffffLL) {
        set_error("guided batch too large (%lld cells, %lld targets, %lld queries)", cells, items, rows);
        return FSB_ERR_ARG;
    }
    size_t tb1 = 0, tb2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb1, (int32_t*)nullptr, (int32_t*)nullptr, (int)(cells + 1), s);
    cub::DeviceScan::ExclusiveSum(nullptr, tb2, (int32_t*)nullptr, (int32_t*)nullptr, (int)(items + 1), s);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t b_pairs = al((size_t)n_pairs * sizeof(GPair)), b_rows = al((size_t)rows * 4), b_items = al((size_t)items * 4);
    const size_t b_cells = al((size_t)(cells + 1) * 4), b_keys = al((size_t)items * 8), b_flag = al((size_t)(items + 1) * 4);
    const size_t need = b_pairs + 3 * b_rows + 3 * b_items + 3 * b_cells + b_keys + 2 * b_flag + al(std::max(tb1, tb2)) + 512;
    void* before = ctx->s_gb.p;
    FSB_TRY(ctx->s_gb.ensure(need));
    uint8_t* cur = ctx->s_gb.as<uint8_t>();
    auto take = [&](size_t bytes) {
        uint8_t* p = cur;
        cur += bytes;
        return p;
    };
    GPair* d_pairs = reinterpret_cast<GPair*>(take(b_pairs));
    int32_t* nA = reinterpret_cast<int32_t*>(take(b_rows));
    int32_t* t_row = reinterpret_cast<int32_t*>(take(b_rows));
    uint32_t* d_row = reinterpret_cast<uint32_t*>(take(b_rows));
    int32_t* nB = reinterpret_cast<int32_t*>(take(b_items));
    int32_t* cell = reinterpret_cast<int32_t*>(take(b_items));
    int32_t* gitems = reinterpret_cast<int32_t*>(take(b_items));
    int32_t* count = reinterpret_cast<int32_t*>(take(b_cells));
    int32_t* start = reinterpret_cast<int32_t*>(take(b_cells));
    int32_t* cursor = reinterpret_cast<int32_t*>(take(b_cells));
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(take(b_keys));
    int32_t* flag = reinterpret_cast<int32_t*>(take(b_flag));
    int32_t* pos = reinterpret_cast<int32_t*>(take(b_flag));
    void* tmp = take(al(std::max(tb1, tb2)));
    int* overflow = reinterpret_cast<int*>(take(256));
    // the graph is valid for exactly this table, these scratch addresses and parameters
    GuidedGraph& G = ctx->gb_graph;
    std::vector<char> key(sizeof(GPair) * n_pairs + 64);
    memcpy(key.data(), hp.data(), sizeof(GPair) * n_pairs);
    {
        char* k = key.data() + sizeof(GPair) * n_pairs;
        memcpy(k, &radius, 8);
        memcpy(k + 8, &kc, 4);
        memcpy(k + 12, &ratio, 4);
        memcpy(k + 16, &counts, 8);
        void* base = ctx->s_gb.p;
        memcpy(k + 24, &base, 8);
        const size_t nb_ = ctx->s_gb.bytes;
        memcpy(k + 32, &nb_, 8);
    }
    const bool reuse = G.exec && before == ctx->s_gb.p && G.key == key;
    if (!reuse) {
        if (G.exec) cudaGraphExecDestroy(G.exec);
        if (G.graph) cudaGraphDestroy(G.graph);
        G.exec = nullptr;
        G.graph = nullptr;
        G.key.clear();
        FSB_CUDA(cudaMemcpyAsync(d_pairs, hp.data(), (size_t)n_pairs * sizeof(GPair), cudaMemcpyHostToDevice, s));
        FSB_CUDA(cudaStreamSynchronize(s));
        FSB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const unsigned py = (unsigned)n_pairs;
        cudaMemsetAsync(count, 0, (size_t)(cells + 1) * 4, s);
        cudaMemsetAsync(cursor, 0, (size_t)(cells + 1) * 4, s);
        cudaMemsetAsync(overflow, 0, 4, s);
        k_gb_norms<<<dim3(blocks(max_na, 8), py), 256, 0, s>>>(d_pairs, 0, nA);
        k_gb_norms<<<dim3(blocks(max_nb, 8), py), 256, 0, s>>>(d_pairs, 1, nB);
        k_gb_count<<<dim3(blocks(max_nb, 256), py), 256, 0, s>>>(d_pairs, cell, count);
        cub::DeviceScan::ExclusiveSum(tmp, tb1, count, start, (int)(cells + 1), s);
        k_gb_fill<<<dim3(blocks(max_nb, 256), py), 256, 0, s>>>(d_pairs, cell, start, cursor, gitems);
        k_gb_guided<<<dim3(blocks(max_na, G_WARPS), py), G_WARPS * 32, 0, s>>>(d_pairs, nA, nB, start, gitems, radius,
                                                                             kc, ratio, t_row, d_row, overflow);
        k_gb_fill_keys<<<blocks(items, 256), 256, 0, s>>>(keys, (int)items);
        k_gb_keys<<<dim3(blocks(max_na, 256), py), 256, 0, s>>>(d_pairs, t_row, d_row, keys);
        k_gb_flags<<<blocks(items + 1, 256), 256, 0, s>>>(keys, (int)items, flag);
        cub::DeviceScan::ExclusiveSum(tmp, tb2, flag, pos, (int)(items + 1), s);
        k_gb_emit<<<dim3(blocks(max_nb, 256), py), 256, 0, s>>>(d_pairs, keys, pos, counts);
        cudaError_t ce = cudaStreamEndCapture(s, &G.graph);
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&G.exec, G.graph, 0);
        if (ce != cudaSuccess) {
            if (G.graph) cudaGraphDestroy(G.graph);
            G.graph = nullptr;
            G.exec = nullptr;
            cudaGetLastError();
            set_error("guided batch graph: %s", cudaGetErrorString(ce));
            return FSB_ERR_CUDA;
        }
        G.key = key;
    }
    FSB_CUDA(cudaGraphLaunch(G.exec, s));
    note_launch(13);
    int h_over = 0;
    FSB_CUDA(cudaMemcpyAsync(&h_over, overflow, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    if (h_over) {
        set_error("more than %d B keypoints within the radius of one prediction (kc mode)", G_CAND);
        return FSB_ERR_OVERFLOW;
    }
    return FSB_OK;
}

}  // namespace fsb

// ---------------------------------------------------------------------------------------------
// Allocation-free dense ratio matcher (fsb_match_bf_noalloc).
//
// Some callers cannot call cudaMalloc: services that reserve their whole device-memory budget
// when they start (a fixed pool handed to them by a host application, as in multi-tenant
// serving), host frameworks that own the CUDA allocator and forbid allocations behind their back,
// and real-time loops where an allocation may block or fail in the middle of a frame. For them
// this entry point runs the FP32 dense matcher with all of its scratch in one file-scope device
// array of fixed size (kNoAllocScratchBytes, about 1.9 MiB), so a call allocates nothing: the
// caller passes device inputs and outputs and a stream.
//
// The array lives in every GPU that loads this library until the process exits. Host code may
// not use its name as an address (on the host it is only a stand-in symbol), so its device
// address is looked up with cudaGetSymbolAddress, with that device current, by the first call made
// on the device (and again by the first call in another context of that device, e.g. after a
// cudaDeviceReset); that first call should come before any stream capture.
// Every call shares the array and it keeps the last call's contents: the per-target key table is
// re-filled at the start of each call, everything else is fully overwritten. Calls whose work
// overlaps on the GPU (different streams, or host threads using the same device) race on the
// array and must be serialised by the caller.
namespace fsb {
namespace {

constexpr int kNoAllocMaxRows = 16384;
constexpr int kNoAllocSplitRows = 8 * kNoAllocMaxRows;   // capacity of the per-split top-2 table
constexpr size_t kNoAllocScratchBytes =
    4 * sizeof(int32_t) * kNoAllocMaxRows +                // norms of A and B, best target, distance
    sizeof(unsigned long long) * kNoAllocMaxRows +         // one-to-one keys per target
    sizeof(Top2) * (size_t)kNoAllocSplitRows;              // per-split top-2 of every A row

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[256] = {};
void* g_noalloc_ctx[256] = {};   // the CUDA context the cached address belongs to

// The current CUDA context (driver-level handle), through the runtime's driver entry point so the
// library needs no link against libcuda; null if it cannot be queried.
void* current_context() {
    typedef int (*CtxGetCurrent)(void**);
    static CtxGetCurrent fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrent>(f);
    }();
    void* c = nullptr;
    if (fn == nullptr || fn(&c) != 0) return nullptr;
    return c;
}

// Device address of g_noalloc_scratch in the current device's current context. It is looked up
// on the first call in a context and cached with that context's handle; a different context on
// the same device (the module loaded again after cudaDeviceReset, or a driver-API context other
// than the primary one) looks it up again.
int32_t noalloc_scratch(void** out) {
    int dev = 0;
    FSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) {
        set_error("device ordinal %d out of range", dev);
        return FSB_ERR_ARG;
    }
    void* ctx = current_context();
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev] || ctx == nullptr || ctx != g_noalloc_ctx[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            set_error("cudaGetSymbolAddress(scratch) failed on device %d: %s", dev, cudaGetErrorString(e));
            return FSB_ERR_CUDA;
        }
        g_noalloc_addr[dev] = p;
        g_noalloc_ctx[dev] = ctx;
    }
    *out = g_noalloc_addr[dev];
    return FSB_OK;
}

// single-CTA, target-ordered compaction of the one-to-one keys (nb <= kNoAllocMaxRows)
constexpr int kCompactThreads = 1024;
__global__ void __launch_bounds__(kCompactThreads) k_noalloc_compact(const unsigned long long* __restrict__ key, int nb,
                                                                      int64_t* __restrict__ q, int64_t* __restrict__ t,
                                                                      int32_t* __restrict__ n_out) {
    typedef cub::BlockScan<int, kCompactThreads> Scan;
    __shared__ typename Scan::TempStorage tmp;
    const int per = (nb + kCompactThreads - 1) / kCompactThreads;
    const int t0 = threadIdx.x * per, t1 = min(nb, t0 + per);
    int cnt = 0;
    for (int i = t0; i < t1; ++i) cnt += key[i] != ~0ull;
    int off = 0, total = 0;
    Scan(tmp).ExclusiveSum(cnt, off, total);
    for (int i = t0; i < t1; ++i) {
        const unsigned long long k = key[i];
        if (k != ~0ull) {
            q[off] = (int64_t)(k & 0xffffffffull);
            t[off] = i;
            ++off;
        }
    }
    if (threadIdx.x == 0) *n_out = total;
}

}  // namespace
}  // namespace fsb

extern "C" int32_t fsb_match_bf_noalloc(const uint8_t* d_a, int32_t na, const uint8_t* d_b, int32_t nb,
                                        float ratio, int64_t* d_q, int64_t* d_t, int32_t* d_n, void* stream) {
    using namespace fsb;
    FSB_ARG(d_n != nullptr, "n_out is null");
    FSB_ARG(na >= 0 && nb >= 0, "negative size");
    if (na > kNoAllocMaxRows || nb > kNoAllocMaxRows) {
        set_error("invalid argument: na=%d, nb=%d exceeds the %d-row limit of the allocation-free matcher "
                  "(use fsb_match_bf_d)", na, nb, kNoAllocMaxRows);
        return FSB_ERR_ARG;
    }
    FSB_ARG((na == 0 || (d_a && d_q && d_t)) && (nb == 0 || d_b), "null device array");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (na < 2 || nb < 2) {
        FSB_CUDA(cudaMemsetAsync(d_n, 0, sizeof(int32_t), s));
        return FSB_OK;
    }
    void* base = nullptr;
    FSB_TRY(noalloc_scratch(&base));
    int32_t* nA = static_cast<int32_t*>(base);
    int32_t* nB = nA + kNoAllocMaxRows;
    int32_t* t_row = nB + kNoAllocMaxRows;
    uint32_t* d_row = reinterpret_cast<uint32_t*>(t_row + kNoAllocMaxRows);
    unsigned long long* key = reinterpret_cast<unsigned long long*>(d_row + kNoAllocMaxRows);
    Top2* part = reinterpret_cast<Top2*>(key + kNoAllocMaxRows);
    // same split rule as the allocating matcher, bounded by the top-2 table's capacity
    const int row_blocks = (na + BM - 1) / BM;
    const int max_splits = kNoAllocSplitRows / na;
    int splits = 1;
    while (row_blocks * splits < 2 * 148 && (nb + splits * 2 - 1) / (splits * 2) >= BN && splits * 2 <= max_splits)
        splits *= 2;
    int split_len = (nb + splits - 1) / splits;
    split_len = ((split_len + BN - 1) / BN) * BN;
    splits = (nb + split_len - 1) / split_len;
    k_norms<<<blocks(na, 8), 256, 0, s>>>(d_a, na, nA);
    k_norms<<<blocks(nb, 8), 256, 0, s>>>(d_b, nb, nB);
    k_bf_fp32<<<dim3(row_blocks, splits), BF_THREADS, 0, s>>>(d_a, na, d_b, nb, nA, nB, split_len, part);
    k_bf_merge<<<blocks(na, 256), 256, 0, s>>>(part, na, splits, ratio, t_row, d_row);
    k_fill_u64<<<blocks(nb, 256), 256, 0, s>>>(key, nb, ~0ull);
    k_unique_keys<<<blocks(na, 256), 256, 0, s>>>(t_row, d_row, na, key);
    k_noalloc_compact<<<1, kCompactThreads, 0, s>>>(key, nb, d_q, d_t, d_n);
    note_launch(7);
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}
