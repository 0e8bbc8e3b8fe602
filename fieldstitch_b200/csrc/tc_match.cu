// Dense descriptor matching on the tcgen05 tensor cores (sm_100a).
//
// matching._ratio_match_bf (app/planesite/matching.py:86-100) needs, for every query row a_q, the
// smallest and second-smallest d2(q, j) = |a_q|^2 + |b_j|^2 - 2 a_q.b_j over all target rows b_j
// and the index of the smallest; _unique (matching.py:103-110) then keeps one query per target.
// Here the contraction runs as K-major GEMMs with the accumulators in tensor memory:
//
//   k_tc_pack    uint8 rows of every pair (one launch) -> operand rows in the canonical no-swizzle
//                core-matrix layout (8 rows x 16 bytes per core matrix, one block per 128 rows).
//                Each row ends with 16 BF16 "norm slots": query slots -s*32768, -s*128, -s*0.5,
//                target slots the three bytes of |b|^2, so one extra K=16 MMA step adds
//                -s*|b|^2/2 and the accumulator holds s * (a.b - |b|^2/2): its largest value over
//                j is the smallest d2 of the row.
//                BF16: the 128 values are exact (uint8 fits the 8-bit significand) and every partial
//                      sum is a multiple of 1/2 below 2^23, so the FP32 accumulation is exact; s = 1.
//                E4M3: round to nearest with a per-query power-of-two scale s (max * s <= 448);
//                      targets are not scaled (uint8 never exceeds the E4M3 range). A power-of-two
//                      scale moves only the exponent, so for uint8 values it changes no rounded
//                      value; it is kept for inputs whose range needs it.
//   k_tc_dense   persistent warp-specialised kernel. Warp 0 streams 128-row target tiles into a
//                shared-memory ring with bulk asynchronous copies (no tensor map, no multicast);
//                warp 1 issues the MMAs (M=128, N=128) for the two 128-row halves of a 256-row
//                query block into double-buffered FP32 accumulators (4 x 128 of the 512 TMEM
//                columns); warps 2-9 read the accumulators with tcgen05.ld (a 128-column row per wait)
//                and keep, per query row, the two largest 32-column maxima and their chunks.
//   k_tc_finish  per query row: the two best chunks over all column splits and the exact integer
//                distances (dp4a) of their columns (BF16: the best chunk only; the second chunk's
//                maximum is already exact), top-2, the float32 ratio test of the reference, and a
//                certificate that no other column can change the decision. BF16: the best chunk's
//                tensor-core maximum must equal the exact best (otherwise the row is recomputed).
//                E4M3: the bound on the rounding error decides; unsettled rows are recomputed by
//                k_tc_exact_rows over every target.
//   k_tcu_*      _unique for every pair of the batch at once (one key per target, atomicMin on
//                (distance << 32 | query), target-ordered compaction by a prefix sum).
//
// The best target, the exact best distance and the accept decision are therefore the same as
// those of the CUDA-core FP32 path and of the reference, for every precision.
#include <cub/cub.cuh>
#include <cuda_fp8.h>

#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "fsb_internal.cuh"

namespace fsb {
namespace {

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

constexpr int TC_THREADS = 320;      // producer warp, MMA warp, 8 epilogue warps
constexpr int TC_ROWS = 256;         // query rows per work item (two M=128 halves)
constexpr int TC_N = 128;            // target rows per tile (MMA N)
constexpr int TC_CHUNK = 32;         // columns per tcgen05.ld
constexpr int TC_MAX_SPLITS = 8;
constexpr long long TC_TIMEOUT_CYCLES = 4000000000ll;   // about two seconds at full clock

// kind::f16 descriptor: F32 accumulator (bit 4), A and B BF16 (bits 7, 10), K-major, N>>3 at 17, M>>4 at 24
constexpr uint32_t IDESC_BF16 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                                ((uint32_t)(128 >> 4) << 24);
// kind::f8f6f4 descriptor: F32 accumulator, A and B E4M3 (format 0), K-major
constexpr uint32_t IDESC_E4M3 = (1u << 4) | ((uint32_t)(TC_N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);

template <int PREC> struct TcTraits;
template <> struct TcTraits<FSB_PREC_BF16> {
    static constexpr int ROW_BYTES = 288;   // 128 + 16 BF16 values
    static constexpr int MAIN_STEPS = 8;    // K = 16 BF16 per MMA (32 bytes)
    static constexpr int STAGES = 4;
    static constexpr int TOPK = 2;
};
template <> struct TcTraits<FSB_PREC_FP8> {
    static constexpr int ROW_BYTES = 160;   // 128 E4M3 + 16 BF16 values
    static constexpr int MAIN_STEPS = 4;    // K = 32 E4M3 per MMA (32 bytes)
    static constexpr int STAGES = 8;
    static constexpr int TOPK = 2;
};

template <int PREC> constexpr int tile_bytes() { return 128 * TcTraits<PREC>::ROW_BYTES; }
template <int PREC> constexpr int smem_bytes() {
    return 2 * tile_bytes<PREC>() + TcTraits<PREC>::STAGES * tile_bytes<PREC>() + 2048;
}

// Byte offset of (row, k-byte) inside a 128-row block: core matrix (row / 8, kb / 16) at
// (row / 8) * SBO + (kb / 16) * 128 with SBO = ROW_BYTES * 8; the descriptor's LBO is 128.
__host__ __device__ constexpr int core_off(int row, int kb, int row_bytes) {
    return (row >> 3) * (row_bytes * 8) + (kb >> 4) * 128 + (row & 7) * 16 + (kb & 15);
}

// ------------------------------------------------------------------------ per-pair tables
struct TcPair {
    const uint8_t* a;      // uint8 query rows (na x 128)
    const uint8_t* b;      // uint8 target rows (nb x 128)
    const uint8_t* pa;     // packed query blocks (nrb x 256 rows)
    const uint8_t* pb;     // packed target tiles (ntiles x 128 rows)
    const float* rowsc;    // E4M3: per query (s, 1 / s, |a|, |alpha|)
    const float* bmax;     // E4M3: (max |b|, max |beta|) over the targets
    const int32_t* nA;     // |a|^2
    const int32_t* nB;     // |b|^2
    int64_t* q_out;        // _unique output (capacity na)
    int64_t* t_out;
    int na, nb, nrb, ntiles, splits, tps;   // tps: tiles per split
    int item0;             // first work item
    int row0;              // first row in the concatenated row arrays
    long long part0;       // first candidate record
    long long key0;        // first target in the concatenated key array
};

struct Cand {
    float v;   // largest s * (a.b - |b|^2 / 2) of a 32-column chunk, as computed by the tensor cores
    int j;     // the chunk (column / 32), -1 when empty
};

// Packing job: `n` rows of `src` (padded with zero rows to n_pad) into `dst`.
struct PackSeg {
    const uint8_t* src;
    uint8_t* dst;
    int32_t* norms;
    float* rowsc;   // E4M3 queries
    float* bmax;    // E4M3 targets
    int n, n_pad, role;   // role 0: query, 1: target
};

template <class T, class F>
__device__ __forceinline__ int upper_index(const T* __restrict__ arr, int n, long long key, F field) {
    int lo = 0, hi = n - 1;   // last element with field <= key
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (field(arr[mid]) <= key) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------------------------ packing
__device__ __forceinline__ uint16_t bf16_bits(float x) {
    return (uint16_t)(__float_as_uint(x) >> 16);   // exact for the integers 0..255 and powers of two
}

// One warp per packed row; blockIdx.y is the job.
template <int PREC>
__global__ void k_tc_pack(const PackSeg* __restrict__ segs) {
    constexpr int RB = TcTraits<PREC>::ROW_BYTES;
    constexpr int XB = RB - 32;   // byte offset of the norm slots
    const PackSeg& S = segs[blockIdx.y];
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= S.n_pad) return;
    uint8_t* blk = S.dst + (size_t)(row >> 7) * (128 * RB);
    const int r = row & 127;
    const bool live = row < S.n;
    const uint32_t w = live ? reinterpret_cast<const uint32_t*>(S.src + (size_t)row * 128)[lane] : 0u;
    int nrm = (int)__dp4a(w, w, 0u);
    for (int sh = 16; sh; sh >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, sh);
    if (lane == 0 && live) S.norms[row] = nrm;
    float s = 1.f;
    if constexpr (PREC == FSB_PREC_BF16) {
        uint2 v;
        v.x = (uint32_t)bf16_bits((float)(w & 255u)) | ((uint32_t)bf16_bits((float)((w >> 8) & 255u)) << 16);
        v.y = (uint32_t)bf16_bits((float)((w >> 16) & 255u)) | ((uint32_t)bf16_bits((float)(w >> 24)) << 16);
        *reinterpret_cast<uint2*>(blk + core_off(r, lane * 8, RB)) = v;
    } else {
        if (S.role == 0) {   // per-query power-of-two scale: the largest e <= 8 with max * 2^e <= 448
            uint32_t mx = max(max(w & 255u, (w >> 8) & 255u), max((w >> 16) & 255u, w >> 24));
            for (int sh = 16; sh; sh >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, sh));
            int e = 8;
            while (e > 0 && (mx << e) > 448u) --e;
            s = (float)(1 << e);
        }
        uint32_t packed = 0;
        float err2 = 0.f;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const float x = (float)((w >> (8 * b)) & 255u);
            const __nv_fp8_storage_t q = __nv_cvt_float_to_fp8(x * s, __NV_SATFINITE, __NV_E4M3);
            const float back = __half2float(__half(__nv_cvt_fp8_to_halfraw(q, __NV_E4M3))) / s;
            err2 = fmaf(back - x, back - x, err2);
            packed |= (uint32_t)q << (8 * b);
        }
        for (int sh = 16; sh; sh >>= 1) err2 += __shfl_xor_sync(0xffffffffu, err2, sh);
        *reinterpret_cast<uint32_t*>(blk + core_off(r, lane * 4, RB)) = packed;
        const float len = live ? sqrtf((float)nrm) * (1.f + 1e-6f) : 0.f;
        const float elen = live ? sqrtf(err2) * (1.f + 1e-6f) : 0.f;
        if (lane == 0 && live && S.role == 0)
            reinterpret_cast<float4*>(S.rowsc)[row] = make_float4(s, 1.f / s, len, elen);
        if (lane == 0 && live && S.role == 1) {
            // the largest |b| and |beta| of the job (non-negative floats order like their bit
            // patterns); the atomic is skipped once the running maximum is already larger
            int* bm = reinterpret_cast<int*>(S.bmax);
            if (__float_as_int(len) > *reinterpret_cast<volatile int*>(bm)) atomicMax(bm, __float_as_int(len));
            if (__float_as_int(elen) > *reinterpret_cast<volatile int*>(bm + 1)) atomicMax(bm + 1, __float_as_int(elen));
        }
    }
    if (lane < 4) {   // the 16 norm slots (32 bytes), 8 bytes per lane
        uint16_t e[4] = {0, 0, 0, 0};
        if (lane == 0 && live) {
            if (S.role == 0) {
                e[0] = bf16_bits(-32768.f * s);
                e[1] = bf16_bits(-128.f * s);
                e[2] = bf16_bits(-0.5f * s);
            } else {
                e[0] = bf16_bits((float)((nrm >> 16) & 255));
                e[1] = bf16_bits((float)((nrm >> 8) & 255));
                e[2] = bf16_bits((float)(nrm & 255));
            }
        }
        uint2 x;
        x.x = (uint32_t)e[0] | ((uint32_t)e[1] << 16);
        x.y = (uint32_t)e[2] | ((uint32_t)e[3] << 16);
        *reinterpret_cast<uint2*>(blk + core_off(r, XB + lane * 8, RB)) = x;
    }
}

// ------------------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(b)) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false (and the CTA-wide abort flag set) when the phase does not complete in time
// or another role already gave up.
__device__ __noinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
    if (mbar_test(b, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test(b, parity)) {
        if (*abort_flag) return false;
        if (clock64() - t0 > TC_TIMEOUT_CYCLES) {
            *abort_flag = 1;
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(saddr(dst)),
        "l"(src), "r"(bytes), "r"(saddr(bar))
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t sbo) {
    // start >> 4 at [0,14), LBO = 128 >> 4 at [16,30), SBO >> 4 at [32,46), version 1 at [46,48),
    // base offset 0, no swizzle (layout type 0 at [61,64))
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(IDESC_BF16), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_e4m3(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(IDESC_E4M3), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float max3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// v > t[K-1]: insert keeping t descending; among equal values the earlier chunk stays first
template <int K>
__device__ __forceinline__ void top_insert(float (&t)[K], int (&j)[K], float v, int col) {
#pragma unroll
    for (int i = K - 1; i >= 0; --i) {
        if (v > t[i]) {
            if (i > 0 && v > t[i - 1]) {
                t[i] = t[i - 1];
                j[i] = j[i - 1];
            } else {
                t[i] = v;
                j[i] = col;
            }
        }
    }
}

// ------------------------------------------------------------------------ the dense kernel
template <int PREC>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_tc_dense(const TcPair* __restrict__ pairs, int n_pairs, int n_items, Cand* __restrict__ part,
               int* __restrict__ err) {
    using T = TcTraits<PREC>;
    constexpr int TB = tile_bytes<PREC>();
    constexpr int NST = T::STAGES;
    constexpr int K = T::TOPK;
    constexpr uint32_t SBO = T::ROW_BYTES * 8;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem =
        reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    unsigned char* sA = smem;            // 2 x TB
    unsigned char* sB = smem + 2 * TB;   // NST x TB
    uint64_t* bars = reinterpret_cast<uint64_t*>(sB + NST * TB);
    uint64_t* b_full = bars;             // NST
    uint64_t* b_empty = bars + NST;      // NST
    uint64_t* a_full = bars + 2 * NST;
    uint64_t* a_empty = a_full + 1;
    uint64_t* acc_full = a_full + 2;     // 2
    uint64_t* acc_empty = a_full + 4;    // 2
    uint64_t* done_bar = a_full + 6;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(a_full + 8);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    auto item0_of = [](const TcPair& x) { return (long long)x.item0; };
    if (threadIdx.x == 0) {
        for (int i = 0; i < NST; ++i) {
            mbar_init(b_full + i, 1);
            mbar_init(b_empty + i, 1);
        }
        mbar_init(a_full, 1);
        mbar_init(a_empty, 1);
        for (int i = 0; i < 2; ++i) {
            mbar_init(acc_full + i, 1);
            mbar_init(acc_empty + i, 8);
        }
        mbar_init(done_bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(saddr(tmem_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ---------------------------------------------------------------- producer
        if (lane == 0) {
            uint32_t bit = 0;   // target tiles issued so far
            int wi = 0;
            bool ok = true;
            int pend[NST];
            for (int i = 0; i < NST; ++i) pend[i] = -1;
            int a_pend = -1;
            for (int item = blockIdx.x; item < n_items && ok; item += gridDim.x, ++wi) {
                const TcPair& P = pairs[upper_index(pairs, n_pairs, item, item0_of)];
                const int local = item - P.item0;
                const int rb = local / P.splits, sp = local - rb * P.splits;
                const int t0 = sp * P.tps, t1 = min(P.ntiles, t0 + P.tps);
                const int pre = min(t1 - t0, NST);
                // the first target tiles of this item do not depend on the query block
                for (int t = t0; t < t0 + pre && ok; ++t, ++bit) {
                    const int st = bit % NST;
                    ok = mbar_wait(b_empty + st, ((bit / NST) & 1) ^ 1, abort_flag);
                    if (!ok) break;
                    mbar_expect_tx(b_full + st, TB);
                    bulk_load(sB + st * TB, P.pb + (size_t)t * TB, TB, b_full + st);
                    pend[st] = (int)((bit / NST) & 1);
                }
                if (!ok) break;
                ok = mbar_wait(a_empty, (wi & 1) ^ 1, abort_flag);
                if (!ok) break;
                mbar_expect_tx(a_full, 2 * TB);
                bulk_load(sA, P.pa + (size_t)rb * 2 * TB, TB, a_full);
                bulk_load(sA + TB, P.pa + (size_t)rb * 2 * TB + TB, TB, a_full);
                a_pend = wi & 1;
                for (int t = t0 + pre; t < t1 && ok; ++t, ++bit) {
                    const int st = bit % NST;
                    ok = mbar_wait(b_empty + st, ((bit / NST) & 1) ^ 1, abort_flag);
                    if (!ok) break;
                    mbar_expect_tx(b_full + st, TB);
                    bulk_load(sB + st * TB, P.pb + (size_t)t * TB, TB, b_full + st);
                    pend[st] = (int)((bit / NST) & 1);
                }
            }
            if (!ok) {
                // let every copy already issued land before the CTA leaves (bounded)
                const long long c0 = clock64();
                for (int st = 0; st < NST; ++st)
                    if (pend[st] >= 0)
                        while (!mbar_test(b_full + st, (uint32_t)pend[st]) && clock64() - c0 < TC_TIMEOUT_CYCLES) {
                        }
                if (a_pend >= 0)
                    while (!mbar_test(a_full, (uint32_t)a_pend) && clock64() - c0 < TC_TIMEOUT_CYCLES) {
                    }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------------------------------------------------------- MMA issuer
        if (lane == 0) {
            uint32_t bit = 0, tit = 0;
            int wi = 0;
            bool ok = true, issued = false;
            const uint32_t a0 = saddr(sA), b0 = saddr(sB);
            for (int item = blockIdx.x; item < n_items && ok; item += gridDim.x, ++wi) {
                const TcPair& P = pairs[upper_index(pairs, n_pairs, item, item0_of)];
                const int local = item - P.item0;
                const int sp = local % P.splits;
                const int t0 = sp * P.tps, t1 = min(P.ntiles, t0 + P.tps);
                ok = mbar_wait(a_full, wi & 1, abort_flag);
                if (!ok) break;
                tc_fence_after();
                for (int t = t0; t < t1; ++t, ++bit, ++tit) {
                    const int st = bit % NST;
                    const int ac = tit & 1;
                    ok = mbar_wait(b_full + st, (bit / NST) & 1, abort_flag);
                    if (!ok) break;
                    ok = mbar_wait(acc_empty + ac, ((tit >> 1) & 1) ^ 1, abort_flag);
                    if (!ok) break;
                    tc_fence_after();
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const uint32_t d = tmem + (uint32_t)(ac * 256 + h * 128);
                        const uint32_t ra = a0 + h * TB, rb = b0 + st * TB;
#pragma unroll
                        for (int k = 0; k < T::MAIN_STEPS; ++k) {
                            if constexpr (PREC == FSB_PREC_BF16)
                                mma_bf16(d, smem_desc(ra + k * 256, SBO), smem_desc(rb + k * 256, SBO), k > 0);
                            else
                                mma_e4m3(d, smem_desc(ra + k * 256, SBO), smem_desc(rb + k * 256, SBO), k > 0);
                        }
                        mma_bf16(d, smem_desc(ra + T::MAIN_STEPS * 256, SBO), smem_desc(rb + T::MAIN_STEPS * 256, SBO),
                                 1u);
                    }
                    issued = true;
                    mma_commit(b_empty + st);
                    mma_commit(acc_full + ac);
                }
                if (!ok) break;
                mma_commit(a_empty);
            }
            // every MMA issued by this thread has completed before TMEM is released
            if (issued) {
                mma_commit(done_bar);
                const long long c0 = clock64();
                while (!mbar_test(done_bar, 0) && clock64() - c0 < TC_TIMEOUT_CYCLES) {
                }
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------------- epilogue
        const int ew = warp - 2;
        const int lq = warp & 3;   // TMEM lane quarter this warp may access
        const int h = ew >> 2;     // query half
        const int rloc = h * 128 + lq * 32 + lane;
        uint32_t tit = 0;
        bool ok = true;
        for (int item = blockIdx.x; item < n_items && ok; item += gridDim.x) {
            const TcPair& P = pairs[upper_index(pairs, n_pairs, item, item0_of)];
            const int local = item - P.item0;
            const int rb = local / P.splits, sp = local - rb * P.splits;
            const int t0 = sp * P.tps, t1 = min(P.ntiles, t0 + P.tps);
            const int q = rb * TC_ROWS + rloc;
            float tv[K];
            int tj[K];
#pragma unroll
            for (int i = 0; i < K; ++i) {
                tv[i] = -INFINITY;
                tj[i] = -1;
            }
            for (int t = t0; t < t1; ++t, ++tit) {
                const int ac = tit & 1;
                ok = mbar_wait(acc_full + ac, (tit >> 1) & 1, abort_flag);
                if (!ok) break;
                tc_fence_after();
                const uint32_t base = tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)(ac * 256 + h * 128);
                // the whole 128-column row at once (four loads, one wait), then the accumulator is free
                uint32_t r[TC_N / TC_CHUNK][32];
#pragma unroll
                for (int ch = 0; ch < TC_N / TC_CHUNK; ++ch) tmem_ld32(base + ch * TC_CHUNK, r[ch]);
                tmem_wait_ld();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(acc_empty + ac);
#pragma unroll
                for (int ch = 0; ch < TC_N / TC_CHUNK; ++ch) {
                    const int j0 = t * TC_N + ch * TC_CHUNK;
                    float v[32];
#pragma unroll
                    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[ch][i]);
                    if (j0 + TC_CHUNK > P.nb) {
#pragma unroll
                        for (int i = 0; i < 32; ++i)
                            if (j0 + i >= P.nb) v[i] = -INFINITY;
                    }
                    float a0 = max3(v[0], v[1], v[2]), a1 = max3(v[3], v[4], v[5]), a2 = max3(v[6], v[7], v[8]);
                    float a3 = max3(v[9], v[10], v[11]), a4 = max3(v[12], v[13], v[14]);
                    float a5 = max3(v[15], v[16], v[17]), a6 = max3(v[18], v[19], v[20]);
                    float a7 = max3(v[21], v[22], v[23]), a8 = max3(v[24], v[25], v[26]);
                    float a9 = max3(v[27], v[28], v[29]), a10 = fmaxf(v[30], v[31]);
                    a0 = max3(a0, a1, a2);
                    a3 = max3(a3, a4, a5);
                    a6 = max3(a6, a7, a8);
                    a9 = fmaxf(a9, a10);
                    const float mx = fmaxf(max3(a0, a3, a6), a9);
                    if (mx > tv[K - 1]) top_insert<K>(tv, tj, mx, j0 / TC_CHUNK);
                }
            }
            if (!ok) break;
            if (q < P.na) {
                Cand* out = part + P.part0 + ((size_t)q * P.splits + sp) * K;
#pragma unroll
                for (int i = 0; i < K; ++i) out[i] = Cand{tv[i], tj[i]};
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicExch(err, 1);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
    }
}

// ------------------------------------------------------------------------ finishing
__device__ __forceinline__ bool ratio_ok(float b1, float b2, float ratio) {
    // app/planesite/matching.py:96-99 on float32 values: sqrt(b1) < ratio * sqrt(b2)
    return __fsqrt_rn(fmaxf(b1, 0.f)) < __fmul_rn(ratio, __fsqrt_rn(fmaxf(b2, 0.f)));
}

__device__ __forceinline__ int exact_dot(const uint4 (&a)[8], const uint8_t* __restrict__ brow) {
    const uint4* b4 = reinterpret_cast<const uint4*>(brow);
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint4 b = __ldg(b4 + i);
        s = __dp4a(a[i].x, b.x, s);
        s = __dp4a(a[i].y, b.y, s);
        s = __dp4a(a[i].z, b.z, s);
        s = __dp4a(a[i].w, b.w, s);
    }
    return (int)s;
}

// warp-wide merge of per-lane (key1 = d << 32 | j, d2): smallest d first, smaller index among equal d
__device__ __forceinline__ void warp_top2(long long& k1, long long& d2) {
    for (int sh = 16; sh; sh >>= 1) {
        const long long ok1 = __shfl_xor_sync(0xffffffffu, k1, sh);
        const long long od2 = __shfl_xor_sync(0xffffffffu, d2, sh);
        const long long hi = max(k1, ok1);
        d2 = min(min(d2, od2), hi >> 32);
        k1 = min(k1, ok1);
    }
}

constexpr long long NO_D = LLONG_MAX >> 32;   // "no distance" (above every uint8 distance)

constexpr int FIN_PASSES = 2;   // a warp finishes 4 rows per pass

// Per-lane error statistics of the certificate (kept by the lane that finishes a row, summed per
// block, then one global update per block: a global atomic per row on one address serialises the
// whole kernel).
struct ErrAcc {
    float mx = 0.f, sum = 0.f;
    int n = 0;
};

// Top-2 merge of (key1 = d << 32 | j, d2) over the 8 lanes of a row group (xor 1, 2, 4).
__device__ __forceinline__ void group_top2(long long& k1, long long& d2) {
#pragma unroll
    for (int sh = 1; sh < 8; sh <<= 1) {
        const long long ok1 = __shfl_xor_sync(0xffffffffu, k1, sh);
        const long long od2 = __shfl_xor_sync(0xffffffffu, d2, sh);
        const long long hi = max(k1, ok1);
        d2 = min(min(d2, od2), hi >> 32);
        k1 = min(k1, ok1);
    }
}

// A warp finishes 4 query rows at a time, 8 lanes per row: lane = 8 * grp + seg, seg the 16-byte
// segment of the 128-byte rows that the lane multiplies. Per row:
//   1. the K best chunks over the column splits (value descending, chunk ascending; one split's
//      records are already in that order);
//   2. the exact distances of the re-ranked chunks' 32 columns each: 32 independent 16-byte loads
//      and dp4a per lane, then a transposed butterfly over seg (16 + 8 + 4 shuffles) leaves lane
//      seg the whole dots of columns 4 seg .. 4 seg + 3; top-2 over the row's lanes;
//   3. (lane seg 0) the certificate and the float32 ratio test of the reference: BF16, the best
//      chunk's tensor-core maximum must equal the exact best (the values are exact) and the next
//      chunk's maximum is the exact best outside it; E4M3, the rounding bound must settle the
//      decision. Unsettled rows go to k_tc_exact_rows.
template <int K>
__global__ void __launch_bounds__(256) k_tc_finish(const TcPair* __restrict__ pairs, const Cand* __restrict__ part,
                                                   float ratio, int prec, int32_t* __restrict__ t_row,
                                                   uint32_t* __restrict__ d_row, int32_t* __restrict__ flagged,
                                                   int* __restrict__ n_flagged, float* __restrict__ err_stat) {
    __shared__ float s_mx, s_sum;
    __shared__ int s_n;
    if (threadIdx.x == 0) {
        s_mx = 0.f;
        s_sum = 0.f;
        s_n = 0;
    }
    __syncthreads();
    const TcPair& P = pairs[blockIdx.y];
    const int lane = threadIdx.x & 31, seg = lane & 7, grp = lane >> 3;
    const int nre = prec == FSB_PREC_BF16 ? 1 : K;
    const bool h4 = seg & 4, h2 = seg & 2, h1 = seg & 1;
    ErrAcc acc;
    const int wq = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * (4 * FIN_PASSES);
    for (int pass = 0; pass < FIN_PASSES; ++pass) {
        const int q0 = wq + 4 * pass;
        if (q0 >= P.na) break;   // warp-uniform
        const int qr = q0 + grp;
        const bool live = qr < P.na;
        const int q = live ? qr : P.na - 1;   // dead groups repeat a live row and write nothing
        // 1. the K best chunks
        float sv[K];
        int sc[K];
        if (P.splits == 1) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const Cand c = part[P.part0 + (size_t)q * K + k];
                sv[k] = c.v;
                sc[k] = c.j;
            }
        } else {
            const int ne = P.splits * K;   // <= 32: at most 4 records per lane
            Cand e[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int idx = seg + 8 * t;
                e[t] = idx < ne ? part[P.part0 + (size_t)q * ne + idx] : Cand{-INFINITY, -1};
                if (e[t].j < 0) e[t] = Cand{-INFINITY, INT_MAX};
            }
#pragma unroll
            for (int k = 0; k < K; ++k) {
                float bv = e[0].v;
                int bc = e[0].j;
#pragma unroll
                for (int t = 1; t < 4; ++t)
                    if (e[t].v > bv || (e[t].v == bv && e[t].j < bc)) {
                        bv = e[t].v;
                        bc = e[t].j;
                    }
#pragma unroll
                for (int sh = 1; sh < 8; sh <<= 1) {
                    const float ov = __shfl_xor_sync(0xffffffffu, bv, sh);
                    const int oc = __shfl_xor_sync(0xffffffffu, bc, sh);
                    if (ov > bv || (ov == bv && oc < bc)) {
                        bv = ov;
                        bc = oc;
                    }
                }
                sv[k] = bv;
                sc[k] = bc == INT_MAX ? -1 : bc;
#pragma unroll
                for (int t = 0; t < 4; ++t)
                    if (e[t].j == bc && bc != INT_MAX) e[t] = Cand{-INFINITY, INT_MAX};
            }
        }
        const long long na = P.nA[q];
        double inv_s = 1.0, eps = 0.0;
        if (prec == FSB_PREC_FP8) {
            const float4 rs = reinterpret_cast<const float4*>(P.rowsc)[q];
            const double bl = P.bmax[0], be = P.bmax[1];
            inv_s = rs.y;
            eps = (double)rs.z * be + (double)rs.w * bl + (double)rs.w * be + (double)rs.z * bl * (1.0 / 512.0) +
                  4.0;
        }
        // 2. exact distances of the re-ranked chunks
        const uint4 a4 = __ldg(reinterpret_cast<const uint4*>(P.a + (size_t)q * 128) + seg);
        long long k1 = LLONG_MAX, d2 = NO_D;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (k >= nre) break;   // warp-uniform
            const int jc = sc[k] < 0 ? P.nb : sc[k] * TC_CHUNK;   // an empty chunk: no valid column
            uint32_t p[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int j = jc + i;
                uint32_t dot = 0;
                if (j < P.nb) {
                    const uint4 b4 = __ldg(reinterpret_cast<const uint4*>(P.b + (size_t)j * 128) + seg);
                    dot = __dp4a(a4.x, b4.x, dot);
                    dot = __dp4a(a4.y, b4.y, dot);
                    dot = __dp4a(a4.z, b4.z, dot);
                    dot = __dp4a(a4.w, b4.w, dot);
                }
                p[i] = dot;
            }
#pragma unroll
            for (int t = 0; t < 16; ++t)
                p[t] = (h4 ? p[t + 16] : p[t]) + __shfl_xor_sync(0xffffffffu, h4 ? p[t] : p[t + 16], 4);
#pragma unroll
            for (int t = 0; t < 8; ++t)
                p[t] = (h2 ? p[t + 8] : p[t]) + __shfl_xor_sync(0xffffffffu, h2 ? p[t] : p[t + 8], 2);
#pragma unroll
            for (int t = 0; t < 4; ++t)
                p[t] = (h1 ? p[t + 4] : p[t]) + __shfl_xor_sync(0xffffffffu, h1 ? p[t] : p[t + 4], 1);
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int j = jc + 4 * seg + t;
                if (j < P.nb) {
                    const long long d = na + __ldg(P.nB + j) - 2ll * (long long)p[t];
                    const long long key = (d << 32) | (unsigned)j;
                    if (key < k1) {
                        d2 = min(d2, k1 >> 32);
                        k1 = key;
                    } else {
                        d2 = min(d2, d);
                    }
                }
            }
        }
        group_top2(k1, d2);
        if (seg != 0 || !live) continue;
        // 3. certificate and ratio test
        const int g = P.row0 + q;
        const bool has1 = k1 != LLONG_MAX;
        const long long e1 = has1 ? (k1 >> 32) : NO_D;
        const int j1 = (int)(k1 & 0xffffffffll);
        long long e2 = d2;
        bool mismatch = false;
        float err = 0.f;
        if (has1) {
            const double approx = (double)na - 2.0 * (double)sv[0] * inv_s;   // the best chunk's maximum
            err = (float)fabs(approx - (double)e1);
            if (prec == FSB_PREC_BF16) {
                mismatch = err != 0.f;
                // BF16 values are exact: the best column outside the first chunk is the second chunk's maximum
                if (sv[1] > -INFINITY) e2 = min(e2, na - (long long)(2.0 * (double)sv[1]));
            }
        }
        // lower bound on the exact distance of every column outside the re-ranked chunks
        double L = INFINITY;
        const float vb = sv[nre < K ? nre : K - 1];
        if (vb > -INFINITY) {
            L = ceil((double)na - 2.0 * ((double)vb * inv_s + eps));
            if (L < 0.0) L = 0.0;
        }
        const float fL = L > 16777216.0 ? 16777216.f : (float)L;
        const float f1 = e1 > (1ll << 24) ? 16777216.f : (float)e1;
        const float f2 = e2 > (1ll << 24) ? 16777216.f : (float)e2;
        const bool accept = has1 && (double)e1 < L && ratio_ok(f1, fminf(f2, fL), ratio);
        const bool reject = !has1 || !ratio_ok(fminf(f1, fL), f2, ratio);
        if (has1) {
            acc.mx = fmaxf(acc.mx, err);
            acc.sum += err;
            ++acc.n;
        }
        if (!mismatch && accept) {
            t_row[g] = j1;
            d_row[g] = (uint32_t)e1;
        } else if (!mismatch && reject) {
            t_row[g] = -1;
            d_row[g] = has1 ? (uint32_t)e1 : 0u;
        } else {
            t_row[g] = -1;
            d_row[g] = 0u;
            flagged[atomicAdd(n_flagged, 1)] = g;
        }
    }
    if (acc.n) {   // err >= 0: its bits order like the values
        atomicMax(reinterpret_cast<int*>(&s_mx), __float_as_int(acc.mx));
        atomicAdd(&s_sum, acc.sum);
        atomicAdd(&s_n, acc.n);
    }
    __syncthreads();
    if (threadIdx.x == 0 && err_stat && s_n) {
        atomicMax(reinterpret_cast<int*>(err_stat), __float_as_int(s_mx));
        atomicAdd(err_stat + 1, s_sum);
        atomicAdd(reinterpret_cast<int*>(err_stat) + 2, s_n);
    }
}

// Exact fallback for rows the certificate could not settle: one CTA per row, every target.
__global__ void __launch_bounds__(256) k_tc_exact_rows(const TcPair* __restrict__ pairs, int n_pairs,
                                                       const int32_t* __restrict__ rows, const int* __restrict__ n_rows,
                                                       float ratio, int32_t* __restrict__ t_row,
                                                       uint32_t* __restrict__ d_row) {
    __shared__ long long s_k1[8], s_d2[8];
    const int nr = *n_rows;
    for (int ri = blockIdx.x; ri < nr; ri += gridDim.x) {
        const int g = rows[ri];
        const TcPair& P = pairs[upper_index(pairs, n_pairs, g, [](const TcPair& x) { return (long long)x.row0; })];
        const int q = g - P.row0;
        const uint4* ar = reinterpret_cast<const uint4*>(P.a + (size_t)q * 128);
        uint4 a[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = __ldg(ar + i);
        const long long na = P.nA[q];
        long long k1 = LLONG_MAX, d2 = NO_D;
        for (int j = threadIdx.x; j < P.nb; j += blockDim.x) {
            const long long d = na + P.nB[j] - 2ll * exact_dot(a, P.b + (size_t)j * 128);
            const long long key = (d << 32) | (unsigned)j;
            if (key < k1) {
                d2 = min(d2, k1 >> 32);
                k1 = key;
            } else {
                d2 = min(d2, d);
            }
        }
        warp_top2(k1, d2);
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) {
            s_k1[w] = k1;
            s_d2[w] = d2;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            long long b1 = s_k1[0], b2 = s_d2[0];
            for (int i = 1; i < 8; ++i) {
                const long long hi = max(b1, s_k1[i]);
                b2 = min(min(b2, s_d2[i]), hi >> 32);
                b1 = min(b1, s_k1[i]);
            }
            const long long e1 = b1 >> 32;
            const float f1 = (float)e1, f2 = b2 > (1ll << 24) ? 16777216.f : (float)b2;
            const bool ok = b1 != LLONG_MAX && ratio_ok(f1, f2, ratio);
            t_row[g] = ok ? (int32_t)(b1 & 0xffffffffll) : -1;
            d_row[g] = b1 != LLONG_MAX ? (uint32_t)e1 : 0u;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------ batched _unique
__global__ void k_tcu_fill(unsigned long long* __restrict__ key, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) key[i] = ~0ull;
}

__global__ void k_tcu_keys(const TcPair* __restrict__ pairs, const int32_t* __restrict__ t_row,
                           const uint32_t* __restrict__ d_row, unsigned long long* __restrict__ key) {
    const TcPair& P = pairs[blockIdx.y];
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.na) return;
    const int g = P.row0 + q;
    const int t = t_row[g];
    if (t >= 0) atomicMin(key + P.key0 + t, ((unsigned long long)d_row[g] << 32) | (unsigned)q);
}

__global__ void k_tcu_flags(const unsigned long long* __restrict__ key, long long n, int32_t* __restrict__ flag) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n) flag[i] = i < n && key[i] != ~0ull;
}

__global__ void k_tcu_emit(const TcPair* __restrict__ pairs, const unsigned long long* __restrict__ key,
                           const int32_t* __restrict__ pos, int32_t* __restrict__ counts) {
    const int p = blockIdx.y;
    const TcPair& P = pairs[p];
    const int local = blockIdx.x * blockDim.x + threadIdx.x;
    if (local >= P.nb) return;
    const long long i = P.key0 + local;
    if (local == P.nb - 1) counts[p] = pos[P.key0 + P.nb] - pos[P.key0];
    const unsigned long long k = key[i];
    if (k == ~0ull) return;
    const int o = pos[i] - pos[P.key0];
    P.q_out[o] = (int64_t)(k & 0xffffffffull);
    P.t_out[o] = local;
}

template <int PREC>
int32_t tc_launch_dense(const TcPair* d_pairs, int n_pairs, int n_items, Cand* part, int* err, int grid,
                        cudaStream_t s) {
    static std::atomic<int> configured[64];
    FSB_TRY(smem_attr((const void*)k_tc_dense<PREC>, (int)smem_bytes<PREC>(), configured));
    k_tc_dense<PREC><<<grid, TC_THREADS, smem_bytes<PREC>(), s>>>(d_pairs, n_pairs, n_items, part, err);
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

}  // namespace

// Tensor-core dense matching of a batch of pairs, _unique included: pair p writes counts[p]
// (device) matches into q_out[p], t_out[p] (device, capacity na[p]). Pairs need na, nb >= 1.
// Scratch comes from ctx; stats (nullable) receives the certificate and error statistics.
int32_t run_match_bf_tc(fsb_ctx* ctx, int n_pairs, const uint8_t* const* d_a, const int* na,
                        const uint8_t* const* d_b, const int* nb, float ratio, int precision, int64_t* const* q_out,
                        int64_t* const* t_out, int32_t* counts, TcStats* stats, cudaStream_t s) {
    if (precision != FSB_PREC_BF16 && precision != FSB_PREC_FP8) {
        set_error("precision %d has no tensor-core path", precision);
        return FSB_ERR_UNSUPPORTED;
    }
    if (n_pairs <= 0) return FSB_OK;
    const bool fp8 = precision == FSB_PREC_FP8;
    const int RB = fp8 ? TcTraits<FSB_PREC_FP8>::ROW_BYTES : TcTraits<FSB_PREC_BF16>::ROW_BYTES;
    const int K = fp8 ? TcTraits<FSB_PREC_FP8>::TOPK : TcTraits<FSB_PREC_BF16>::TOPK;
    int num_sms = 148;
    {
        int dev = 0;
        FSB_CUDA(cudaGetDevice(&dev));
        FSB_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    std::vector<TcPair> hp(n_pairs);
    size_t off_pa = 0, off_pb = 0, n_norm = 0, n_parts = 0;
    long long n_keys = 0, rb_total = 0;
    int items = 0, rows = 0;
    for (int p = 0; p < n_pairs; ++p) rb_total += (na[p] + TC_ROWS - 1) / TC_ROWS;
    for (int p = 0; p < n_pairs; ++p) {
        TcPair& P = hp[p];
        P.a = d_a[p];
        P.b = d_b[p];
        P.na = na[p];
        P.nb = nb[p];
        P.q_out = q_out[p];
        P.t_out = t_out[p];
        P.nrb = (na[p] + TC_ROWS - 1) / TC_ROWS;
        P.ntiles = (nb[p] + TC_N - 1) / TC_N;
        int splits = 1;
        if (rb_total < 2 * num_sms) {   // too few query blocks to fill the GPU: split the targets too
            splits = (int)((2 * num_sms + rb_total - 1) / rb_total);
            splits = std::max(1, std::min(std::min(splits, TC_MAX_SPLITS), std::min(32 / K, P.ntiles)));
        }
        P.tps = (P.ntiles + splits - 1) / splits;
        P.splits = (P.ntiles + P.tps - 1) / P.tps;
        P.item0 = items;
        P.row0 = rows;
        P.part0 = (long long)n_parts;
        P.key0 = n_keys;
        items += P.nrb * P.splits;
        rows += P.na;
        n_keys += P.nb;
        off_pa += (size_t)P.nrb * TC_ROWS * RB;
        off_pb += (size_t)P.ntiles * TC_N * RB;
        n_norm += (size_t)P.na + P.nb;
        n_parts += (size_t)P.na * P.splits * K;
    }
    size_t tb_scan = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, (int32_t*)nullptr, (int32_t*)nullptr, (int)(n_keys + 1), s);
    // scratch layout
    const size_t b_pairs = al((size_t)n_pairs * sizeof(TcPair)), b_segs = al((size_t)2 * n_pairs * sizeof(PackSeg));
    const size_t b_norm = al(n_norm * 4), b_rowsc = fp8 ? al((size_t)rows * 16) : 0, b_bmax = al((size_t)n_pairs * 8);
    const size_t b_rowi = al((size_t)rows * 4), b_keys = al((size_t)n_keys * 8), b_flag = al((size_t)(n_keys + 1) * 4);
    FSB_TRY(ctx->s_tc_pack.ensure(al(off_pa) + al(off_pb)));
    FSB_TRY(ctx->s_tc_part.ensure(al(n_parts * sizeof(Cand)) + 256));
    FSB_TRY(ctx->s_tc_aux.ensure(b_pairs + b_segs + b_norm + b_rowsc + b_bmax + 4 * b_rowi + b_keys + 2 * b_flag +
                                 al(tb_scan) + 512));
    uint8_t* pack = ctx->s_tc_pack.as<uint8_t>();
    uint8_t* cur = ctx->s_tc_aux.as<uint8_t>();
    auto take = [&](size_t bytes) {
        uint8_t* p = cur;
        cur += bytes;
        return p;
    };
    TcPair* d_pairs = reinterpret_cast<TcPair*>(take(b_pairs));
    PackSeg* d_segs = reinterpret_cast<PackSeg*>(take(b_segs));
    int32_t* norms = reinterpret_cast<int32_t*>(take(b_norm));
    float* rowsc = reinterpret_cast<float*>(take(b_rowsc));
    float* bmax = reinterpret_cast<float*>(take(b_bmax));
    int32_t* t_row = reinterpret_cast<int32_t*>(take(b_rowi));
    uint32_t* d_row = reinterpret_cast<uint32_t*>(take(b_rowi));
    int32_t* flagged = reinterpret_cast<int32_t*>(take(b_rowi));
    take(b_rowi);
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(take(b_keys));
    int32_t* flag = reinterpret_cast<int32_t*>(take(b_flag));
    int32_t* pos = reinterpret_cast<int32_t*>(take(b_flag));
    void* scan_tmp = take(al(tb_scan));
    int* small = reinterpret_cast<int*>(take(256));   // [0] abort, [1] flagged rows, [2..4] error statistics
    FSB_CUDA(cudaMemsetAsync(small, 0, 64, s));
    if (fp8) FSB_CUDA(cudaMemsetAsync(bmax, 0, (size_t)n_pairs * 8, s));
    std::vector<PackSeg> segs;
    segs.reserve(2 * n_pairs);
    size_t pa = 0, pb = 0, nn = 0, rr = 0;
    int max_pad = 0, max_na = 0, max_nb = 0;
    for (int p = 0; p < n_pairs; ++p) {
        TcPair& P = hp[p];
        P.pa = pack + pa;
        P.pb = pack + al(off_pa) + pb;
        P.nA = norms + nn;
        P.nB = norms + nn + P.na;
        P.rowsc = fp8 ? rowsc + 4 * rr : nullptr;
        P.bmax = bmax + 2 * p;
        const int pad_a = P.nrb * TC_ROWS, pad_b = P.ntiles * TC_N;
        max_pad = std::max(max_pad, std::max(pad_a, pad_b));
        max_na = std::max(max_na, P.na);
        max_nb = std::max(max_nb, P.nb);
        segs.push_back(PackSeg{P.a, const_cast<uint8_t*>(P.pa), const_cast<int32_t*>(P.nA), const_cast<float*>(P.rowsc),
                               nullptr, P.na, pad_a, 0});
        segs.push_back(PackSeg{P.b, const_cast<uint8_t*>(P.pb), const_cast<int32_t*>(P.nB), nullptr,
                               const_cast<float*>(P.bmax), P.nb, pad_b, 1});
        pa += (size_t)pad_a * RB;
        pb += (size_t)pad_b * RB;
        nn += (size_t)P.na + P.nb;
        rr += (size_t)P.na;
    }
    FSB_CUDA(cudaMemcpyAsync(d_pairs, hp.data(), (size_t)n_pairs * sizeof(TcPair), cudaMemcpyHostToDevice, s));
    FSB_CUDA(cudaMemcpyAsync(d_segs, segs.data(), segs.size() * sizeof(PackSeg), cudaMemcpyHostToDevice, s));
    const dim3 pack_grid(nblk(max_pad, 8), (unsigned)segs.size());
    if (fp8)
        k_tc_pack<FSB_PREC_FP8><<<pack_grid, 256, 0, s>>>(d_segs);
    else
        k_tc_pack<FSB_PREC_BF16><<<pack_grid, 256, 0, s>>>(d_segs);
    note_launch(1);
    FSB_CUDA(cudaGetLastError());
    Cand* part = ctx->s_tc_part.as<Cand>();
    ctx->stage_begin(ST_TC_DENSE);
    if (fp8) FSB_TRY(tc_launch_dense<FSB_PREC_FP8>(d_pairs, n_pairs, items, part, small, std::min(items, num_sms), s));
    else FSB_TRY(tc_launch_dense<FSB_PREC_BF16>(d_pairs, n_pairs, items, part, small, std::min(items, num_sms), s));
    note_launch(1);
    ctx->stage_end(ST_TC_DENSE);
    float* err_stat = stats ? reinterpret_cast<float*>(small + 2) : nullptr;
    const dim3 fin_grid(nblk(max_na, 8 * 4 * FIN_PASSES), (unsigned)n_pairs);
    if (fp8)
        k_tc_finish<TcTraits<FSB_PREC_FP8>::TOPK><<<fin_grid, 256, 0, s>>>(d_pairs, part, ratio, precision, t_row,
                                                                           d_row, flagged, small + 1, err_stat);
    else
        k_tc_finish<TcTraits<FSB_PREC_BF16>::TOPK><<<fin_grid, 256, 0, s>>>(d_pairs, part, ratio, precision, t_row,
                                                                            d_row, flagged, small + 1, err_stat);
    note_launch(1);
    FSB_CUDA(cudaGetLastError());
    int host_small[5] = {0, 0, 0, 0, 0};
    FSB_CUDA(cudaMemcpyAsync(host_small, small, sizeof(host_small), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    if (host_small[0]) {
        set_error("tensor-core matcher: a pipeline wait timed out");
        return FSB_ERR_CUDA;
    }
    if (host_small[1] > 0) {
        k_tc_exact_rows<<<std::min(host_small[1], 8 * num_sms), 256, 0, s>>>(d_pairs, n_pairs, flagged, small + 1,
                                                                            ratio, t_row, d_row);
        note_launch(1);
        FSB_CUDA(cudaGetLastError());
    }
    // _unique of every pair
    k_tcu_fill<<<nblk(n_keys, 256), 256, 0, s>>>(keys, n_keys);
    k_tcu_keys<<<dim3(nblk(max_na, 256), (unsigned)n_pairs), 256, 0, s>>>(d_pairs, t_row, d_row, keys);
    k_tcu_flags<<<nblk(n_keys + 1, 256), 256, 0, s>>>(keys, n_keys, flag);
    FSB_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, tb_scan, flag, pos, (int)(n_keys + 1), s));
    k_tcu_emit<<<dim3(nblk(max_nb, 256), (unsigned)n_pairs), 256, 0, s>>>(d_pairs, keys, pos, counts);
    note_launch(5);
    FSB_CUDA(cudaGetLastError());
    if (stats) {
        float mx, sum;
        memcpy(&mx, &host_small[2], 4);
        memcpy(&sum, &host_small[3], 4);
        stats->rows = rows;
        stats->fallback_rows = host_small[1];
        stats->max_abs_err = mx;
        stats->mean_abs_err = host_small[4] ? sum / (float)host_small[4] : 0.f;
    }
    return FSB_OK;
}

}  // namespace fsb
