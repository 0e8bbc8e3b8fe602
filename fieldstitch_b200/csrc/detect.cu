// Keypoint detection and description on the DoG / gradient atlases.
//
// Compiled with --fmad=false: every float32 expression below is evaluated with the reference's
// rounding (one rounding per operation, in the written order), so integer positions, sub-pixel
// offsets and responses follow app/planesite/gsift.py bit for bit given the same DoG values.
//
//   k_extrema   3x3x3 extrema of DoG layers 1..3 (gsift.py:293-319), warp-aggregated append
//   k_refine    sub-pixel fit, contrast and edge tests (gsift.py:322-369), thread per candidate
//   orientation peaks come from describe.cu (run_orient)
//   sort        rank of the refined extrema: stable radix sort by response, DoG index inside ties
//               (gsift.py:471)
//   k_gather    keypoint fields in input-image pixels (gsift.py:462-474)
//   spread      grid-spread selection of features.py:38-57
#include <cub/cub.cuh>

#include <cmath>

#include "fsb_internal.cuh"

namespace fsb {
namespace {

struct DetectConsts {
    Geometry g;
    float pthr, contrast, edge, e1sq;
    long long vox_off[MAXO + 1];
};


__device__ __forceinline__ int find_octave(const Geometry& g, long long f) {
    int o = 0;
    while (o + 1 < g.n_oct && f >= g.dog_off[o + 1]) ++o;
    return o;
}

// warp-aggregated append of `flag` entries into out[], counter shared by the grid
template <class T>
__device__ __forceinline__ void warp_append(bool flag, const T& v, T* out, uint32_t* counter, uint32_t cap) {
    const unsigned m = __ballot_sync(0xffffffffu, flag);
    if (!m) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (flag) {
        const uint32_t pos = base + __popc(m & ((1u << lane) - 1u));
        if (pos < cap) out[pos] = v;
    }
}

// k_extrema: a block is 8 warps side by side over 240 interior columns of an EX_ROWS-row chunk of
// one octave; each warp walks its chunk row by row (see the kernel).
constexpr int EX_T = 256;            // 8 warps per block
constexpr int EX_COLS = 30;          // output columns per warp (lanes 1..30; lanes 0 and 31 are halo)
constexpr int EX_ROWS = 64;          // rows per block (a chunk of the octave's interior rows)

struct ExTiles {
    int n_oct;
    int col_tiles[MAXO], row_tiles[MAXO];
    int first[MAXO + 1];     // first block of each octave
};

constexpr int EX_DEPTH = 9;          // rows in flight per lane (the shared-memory ring's slots)

// three-input maximum / minimum (one instruction on sm_100); exact, so the same values as two
// two-input ones
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

__device__ __forceinline__ void ex_cp_async4(float* dst, const float* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

// Streaming 3x3x3 extremum test: each warp walks down a chunk of rows of 30 interior columns;
// every DoG value is read once (coalesced, EX_DEPTH rows ahead through a shared-memory ring),
// horizontal neighbours come from the adjacent lanes,
// the 3-row vertical window of the horizontal maxima / minima stays in registers. A voxel is an
// extremum when it equals the maximum (minimum) of its 27-neighbourhood - ties count - and is
// beyond the threshold, as scipy's maximum_filter / minimum_filter test in the reference
// (gsift.py:293-319). Candidates of a row are appended with one warp-aggregated atomic.
__global__ void __launch_bounds__(EX_T, 4) k_extrema(const float* __restrict__ DF, DetectConsts k, ExTiles tl,
                                                  uint32_t* __restrict__ cand, uint32_t* counter, uint32_t cap) {
    __shared__ float ex_ring[EX_DEPTH * 5 * EX_T];
    int o = 0;
    while (o + 1 < tl.n_oct && (int)blockIdx.x >= tl.first[o + 1]) ++o;
    const int b = blockIdx.x - tl.first[o];
    const int ry = b / tl.col_tiles[o], cx = b - ry * tl.col_tiles[o];
    const int R = k.g.R[o], C = k.g.C[o];
    const long long RC = (long long)R * C;
    const float* base = DF + k.g.dog_off[o];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int c = BORDER + (cx * (EX_T / 32) + wid) * EX_COLS + lane - 1;   // this lane's column
    const int cc = min(max(c, 0), C - 1);                                    // clamped for loading
    const bool col_ok = lane >= 1 && lane <= EX_COLS && c >= BORDER && c < C - BORDER;
    const int y0 = BORDER + ry * EX_ROWS, y1 = min(y0 + EX_ROWS, R - BORDER);   // output rows [y0, y1)
    // one row of the 3-row window: horizontal max / min of the 5 layers and the centre values of
    // layers 1..3
    struct Row {
        float hx[5], hn[5], c[3];
    };
    // Row r's five layer values at this lane's column arrive by 4-byte cp.async into the lane's own
    // ring slot ((r - (y0 - 1)) % EX_DEPTH), EX_DEPTH rows ahead of the row being finished; only the
    // lane that copied a value reads it, so a lane waits on its own copy groups and no barrier is
    // needed. One commit group per row (empty past the last needed row) keeps the count uniform.
    float* ring = ex_ring + threadIdx.x;   // element (slot, l) at ring[(slot * 5 + l) * EX_T]
    const float* colp = base + cc;
    const int last_row = min(y1 + 1, R - 1);
    int next_row = y0 - 1, next_slot = 0, take_slot = 0;
    auto issue_next = [&]() {
        if (next_row <= last_row) {
            const float* src = colp + (long long)next_row * C;
#pragma unroll
            for (int l = 0; l < 5; ++l) ex_cp_async4(ring + (next_slot * 5 + l) * EX_T, src + l * RC);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        ++next_row;
        next_slot = next_slot + 1 == EX_DEPTH ? 0 : next_slot + 1;
    };
    // the oldest row in flight, once landed (EX_DEPTH groups outstanding -> wait for all but the
    // newest EX_DEPTH - 1), then its slot gets the next row
    auto take_row = [&](float (&raw)[5]) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(EX_DEPTH - 1) : "memory");
#pragma unroll
        for (int l = 0; l < 5; ++l) raw[l] = ring[(take_slot * 5 + l) * EX_T];
        take_slot = take_slot + 1 == EX_DEPTH ? 0 : take_slot + 1;
        issue_next();
    };
    auto finish_row = [&](Row& w, const float (&raw)[5]) {
#pragma unroll
        for (int l = 0; l < 5; ++l) {
            const float v = raw[l];
            const float vl = __shfl_up_sync(0xffffffffu, v, 1), vr = __shfl_down_sync(0xffffffffu, v, 1);
            w.hx[l] = max3f(vl, v, vr);
            w.hn[l] = min3f(vl, v, vr);
            if (l >= 1 && l <= N_LAYERS) w.c[l - 1] = v;
        }
    };
    auto load_row = [&](Row& w) {
        float raw[5];
        take_row(raw);
        finish_row(w, raw);
    };
    // test row y from the window (up, mid, dn), append its extrema, then finish row y + 2 into `up`
    // (no longer needed): the three windows rotate by name, not by register moves
    auto step = [&](Row& up, const Row& mid, const Row& dn, int y) {
        float vmx[5], vmn[5];
#pragma unroll
        for (int l = 0; l < 5; ++l) {
            vmx[l] = max3f(up.hx[l], mid.hx[l], dn.hx[l]);
            vmn[l] = min3f(up.hn[l], mid.hn[l], dn.hn[l]);
        }
        unsigned mask = 0;
        if (col_ok) {
#pragma unroll
            for (int l = 1; l <= N_LAYERS; ++l) {
                const float v = mid.c[l - 1];
                const float mx = max3f(vmx[l - 1], vmx[l], vmx[l + 1]);
                const float mn = min3f(vmn[l - 1], vmn[l], vmn[l + 1]);
                if ((v >= mx && v > k.pthr) || (v <= mn && v < -k.pthr)) mask |= 1u << (l - 1);
            }
        }
        const unsigned any = __ballot_sync(0xffffffffu, mask != 0);
        if (any) {
            const int cntv = __popc(mask);
            int incl = cntv;
#pragma unroll
            for (int sh = 1; sh < 32; sh <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, sh);
                if (lane >= sh) incl += t;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            uint32_t basepos = 0;
            if (lane == 31) basepos = atomicAdd(counter, (uint32_t)total);
            basepos = __shfl_sync(0xffffffffu, basepos, 31);
            uint32_t pos = basepos + (uint32_t)(incl - cntv);
            while (mask) {
                const int bit = __ffs(mask) - 1;
                mask &= mask - 1;
                if (pos < cap) cand[pos] = (uint32_t)(k.g.dog_off[o] + (bit + 1) * RC + (long long)y * C + c);
                ++pos;
            }
        }
        load_row(up);   // row y + 2
    };
    for (int i = 0; i < EX_DEPTH; ++i) issue_next();   // rows y0 - 1 .. y0 + EX_DEPTH - 2
    Row w0, w1, w2;
    load_row(w0);   // y0 - 1
    load_row(w1);   // y0
    load_row(w2);   // y0 + 1
    for (int y = y0; y < y1; y += 3) {
        step(w0, w1, w2, y);
        if (y + 1 >= y1) break;
        step(w1, w2, w0, y + 1);
        if (y + 2 >= y1) break;
        step(w2, w0, w1, y + 2);
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");   // no copy outlives the block
}

ExTiles make_tiles(const Geometry& g, int* total) {
    ExTiles t{};
    t.n_oct = g.n_oct;
    int acc = 0;
    for (int o = 0; o < g.n_oct; ++o) {
        t.first[o] = acc;
        const int inner_c = g.C[o] - 2 * BORDER, inner_r = g.R[o] - 2 * BORDER;
        t.col_tiles[o] = inner_c > 0 ? (inner_c + (EX_T / 32) * EX_COLS - 1) / ((EX_T / 32) * EX_COLS) : 0;
        t.row_tiles[o] = inner_r > 0 ? (inner_r + EX_ROWS - 1) / EX_ROWS : 0;
        acc += t.col_tiles[o] * t.row_tiles[o];
    }
    t.first[g.n_oct] = acc;
    *total = acc;
    return t;
}

// The extremum candidates of every octave in one launch, appended to `cand` through `cnt[0]`.
int32_t launch_extrema(const Geometry& g, const float* DF, const DetectConsts& k, uint32_t* cand, uint32_t* cnt,
                       uint32_t cap, cudaStream_t s) {
    int n = 0;
    const ExTiles t = make_tiles(g, &n);
    if (n > 0) {
        k_extrema<<<n, EX_T, 0, s>>>(DF, k, t, cand, cnt, cap);
        note_launch();
    }
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

struct Fit {
    float v, dx, dy, ds, dxx, dyy, dss, dxy, dxs, dys;
};

// finite-difference gradient and Hessian at an integer voxel (gsift.py:274-290)
__device__ __forceinline__ Fit local_fit(const float* __restrict__ D, long long k, long long C, long long RC) {
    Fit f;
    f.v = D[k];
    const float xp1 = D[k + 1], xm1 = D[k - 1], yp1 = D[k + C], ym1 = D[k - C];
    const float sp1 = D[k + RC], sm1 = D[k - RC];
    f.dx = (xp1 - xm1) * 0.5f;
    f.dy = (yp1 - ym1) * 0.5f;
    f.ds = (sp1 - sm1) * 0.5f;
    f.dxx = (xp1 + xm1) - 2.f * f.v;
    f.dyy = (yp1 + ym1) - 2.f * f.v;
    f.dss = (sp1 + sm1) - 2.f * f.v;
    f.dxy = (((D[k + C + 1] - D[k + C - 1]) - D[k - C + 1]) + D[k - C - 1]) * 0.25f;
    f.dxs = (((D[k + RC + 1] - D[k + RC - 1]) - D[k - RC + 1]) + D[k - RC - 1]) * 0.25f;
    f.dys = (((D[k + RC + C] - D[k + RC - C]) - D[k - RC + C]) + D[k - RC - C]) * 0.25f;
    return f;
}

__global__ void __launch_bounds__(128) k_refine(const float* __restrict__ DF, DetectConsts k,
                                                const uint32_t* __restrict__ cand, const uint32_t* n_cand,
                                                uint32_t cap_cand, Refined* __restrict__ out,
                                                uint32_t* counter, uint32_t cap) {
    const uint32_t n = min(*n_cand, cap_cand);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t i = base + threadIdx.x;
        bool good = false;
        Refined e{};
        if (i < n) {
            const uint32_t f = cand[i];
            const int o = find_octave(k.g, f);
            const int R = k.g.R[o], C = k.g.C[o];
            const long long RC = (long long)R * C, ob = k.g.dog_off[o];
            const long long loc = (long long)f - ob;
            int l = (int)(loc / RC);
            const long long rem = loc - (long long)l * RC;
            int r = (int)(rem / C);
            int c = (int)(rem - (long long)r * C);
            float X0 = 0.f, X1 = 0.f, X2 = 0.f;
            bool done = false;
            for (int it = 0; it < MAX_INTERP; ++it) {
                const Fit F = local_fit(DF, ob + l * RC + (long long)r * C + c, C, RC);
                // adjugate solve of H x = g (gsift.py:182-198); x = -H^-1 g
                const float a = F.dxx, b = F.dxy, cc = F.dxs, d = F.dxy, ee = F.dyy, ff = F.dys;
                const float gg = F.dxs, hh = F.dys, ii = F.dss;
                const float A = ee * ii - ff * hh, B = -(d * ii - ff * gg), Cc = d * hh - ee * gg;
                const float det = (a * A + b * B) + cc * Cc;
                if (!(fabsf(det) > 1e-20f)) break;
                const float i00 = A / det, i01 = -(b * ii - cc * hh) / det, i02 = (b * ff - cc * ee) / det;
                const float i10 = B / det, i11 = (a * ii - cc * gg) / det, i12 = -(a * ff - cc * d) / det;
                const float i20 = Cc / det, i21 = -(a * hh - b * gg) / det, i22 = (a * ee - b * d) / det;
                const float x0 = -((i00 * F.dx + i01 * F.dy) + i02 * F.ds);
                const float x1 = -((i10 * F.dx + i11 * F.dy) + i12 * F.ds);
                const float x2 = -((i20 * F.dx + i21 * F.dy) + i22 * F.ds);
                if (fabsf(x0) < 0.5f && fabsf(x1) < 0.5f && fabsf(x2) < 0.5f) {
                    X0 = x0; X1 = x1; X2 = x2;
                    done = true;
                    break;
                }
                if (!(fabsf(x0) <= 1e6f && fabsf(x1) <= 1e6f && fabsf(x2) <= 1e6f)) break;   // also NaN
                c += (int)rintf(x0);
                r += (int)rintf(x1);
                l += (int)rintf(x2);
                if (l < 1 || l > N_LAYERS || c < BORDER || c >= C - BORDER || r < BORDER || r >= R - BORDER) break;
            }
            if (done) {
                const Fit F = local_fit(DF, ob + l * RC + (long long)r * C + c, C, RC);
                const float contr = F.v + 0.5f * ((F.dx * X0 + F.dy * X1) + F.ds * X2);
                const float tr = F.dxx + F.dyy;
                const float dt = F.dxx * F.dyy - F.dxy * F.dxy;
                if (fabsf(contr) * (float)N_LAYERS >= k.contrast && dt > 0.f && (tr * tr) * k.edge < k.e1sq * dt) {
                    good = true;
                    e.f = f; e.o = (int16_t)o; e.l = (int16_t)l; e.r = r; e.c = c;
                    e.x0 = X0; e.x1 = X1; e.x2 = X2;
                    e.resp = fabsf(contr);
                }
            }
        }
        warp_append(good, e, out, counter, cap);
    }
}

// keypoint scale in octave pixels: 1.6 * 2^((l + x2) / 3) (gsift.py:462)
__device__ __forceinline__ float kp_scale(int l, float x2) {
    const float t = ((float)l + x2) / 3.f;
    return 1.6f * exp2f(t);
}

// rank key of a refined extremum: response descending (a positive finite float's bits order like
// its value); the DoG-atlas index breaks ties afterwards (k_rank_ties)
// d_n (nullable): the refined count on the device; entries from it up to n get the largest key, so
// a stable sort of n entries puts them last (n is then a capacity)
__global__ void k_rank_keys(const Refined* __restrict__ ref, uint32_t n, const uint32_t* __restrict__ d_n,
                            uint32_t* __restrict__ key, uint32_t* __restrict__ val) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t m = d_n ? min(*d_n, n) : n;
    key[i] = i < m ? 0x7fffffffu - __float_as_uint(ref[i].resp) : 0x7fffffffu;
    val[i] = i;
}

// ranks from the (stable) response sort: inside a run of equal responses the extrema are ordered
// by DoG-atlas index (their order in the refined list is the atomic append order), so an element
// goes to the run's start + the number of run members with a smaller index
__global__ void k_rank_ties(const uint32_t* __restrict__ key, const uint32_t* __restrict__ val,
                            const Refined* __restrict__ ref, uint32_t n, const uint32_t* __restrict__ d_n,
                            uint32_t* __restrict__ order) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (d_n) n = min(*d_n, n);
    if (t >= n) return;
    const uint32_t k = key[t], v = val[t];
    uint32_t a = t, b = t + 1;
    while (a > 0 && key[a - 1] == k) --a;
    while (b < n && key[b] == k) ++b;
    if (b - a == 1) {
        order[t] = v;
        return;
    }
    const uint32_t f = ref[v].f;
    uint32_t r = a;
    for (uint32_t u = a; u < b; ++u)
        if (ref[val[u]].f < f) ++r;
    order[r] = v;
}

// keypoints in final order: rank t's peaks (bin order) at pos[t] .. pos[t] + cnt[t] - 1, kept below
// n_keep
// d_rk (nullable): on the device, [0] the ranks oriented, [1] the keypoints kept (n_rank is then a
// capacity and n_keep unused)
__global__ void k_gather_ranked(const Oriented* __restrict__ slots, const uint32_t* __restrict__ cnt,
                                const uint32_t* __restrict__ pos, const Refined* __restrict__ ref, uint32_t n_rank,
                                uint32_t n_keep, const uint32_t* __restrict__ d_rk, float* kx, float* ky, float* ksize,
                                float* kang, float* kresp, int32_t* koct, int32_t* klayer) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (d_rk) {
        n_rank = min(d_rk[0], n_rank);
        n_keep = d_rk[1];
    }
    if (t >= n_rank) return;
    const uint32_t c = cnt[t], p = pos[t];
    for (uint32_t k = 0; k < c && p + k < n_keep; ++k) {
        const Oriented e = slots[(size_t)t * ORI_SLOTS + k];
        const Refined r = ref[e.ri];
        const float f = (float)(1 << r.o) * 0.5f;
        const float scl = kp_scale(r.l, r.x2);
        const uint32_t i = p + k;
        kx[i] = ((float)r.c + r.x0) * f;
        ky[i] = ((float)r.r + r.x1) * f;
        ksize[i] = (scl * 2.f) * f;
        kang[i] = e.angle;
        kresp[i] = r.resp;
        koct[i] = r.o;
        klayer[i] = r.l;
    }
}

// ------------------------------------------------------------------------------------ spread
// Grid-spread selection of features.py:38-57 on keypoints already in response-descending order
// (the detector's output order; ties in detection order), restated without sorts:
//   * cell = clip(int(x / W * 12), 0, 11) + 12 * clip(int(y / H * 9), 0, 8) in float32;
//   * the reference orders by (cell, response descending, index), which on this input is
//     (cell, index): an element's rank in its cell is the number of earlier elements of that cell;
//   * "group 0" = rank < cap = ceil(nfeat / 108); their selection position is the cell's start
//     (exclusive scan of min(count, cap) over cells) + rank; the others ("the rest", in index
//     order = response order) follow from position n1 = the group-0 total; positions >= nfeat are
//     dropped (sel[:n]);
//   * the stable response sort of features.py:126 orders the selection by (response descending,
//     selection position): index order, except inside a run of equal responses, where the
//     selection positions decide.
// The input is split into chunks of `ch` elements (a multiple of 1024; at most 64 chunks), one
// 1024-thread block each, one element per thread per step: k_sp_hist counts cells per chunk;
// k_sp_pos ranks elements in their cells (per-warp multi-split by __match_any_sync, warps in
// order through per-cell prefix sums, chunks in order through the histograms) and writes each
// element's selection position (or -1) and the number selected per 32-element group; k_sp_place
// (a warp per group) puts each selected index in its final slot.
constexpr int SP_GX = 12, SP_GY = 9, SP_CELLS = SP_GX * SP_GY;
constexpr int SP_T = 1024, SP_NW = SP_T / 32;

__device__ __forceinline__ int sp_cell(float x, float y, float W, float H) {
    int cx = (int)(x / W * (float)SP_GX), cy = (int)(y / H * (float)SP_GY);
    cx = min(max(cx, 0), SP_GX - 1);
    cy = min(max(cy, 0), SP_GY - 1);
    return cy * SP_GX + cx;
}

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
    for (int sh = 16; sh; sh >>= 1) v += __shfl_xor_sync(0xffffffffu, v, sh);
    return v;
}

__global__ void __launch_bounds__(SP_T) k_sp_hist(const float* __restrict__ x, const float* __restrict__ y, int n,
                                                  const int* __restrict__ d_n, float W, float H, int ch,
                                                  int* __restrict__ hist) {
    __shared__ int h[SP_CELLS];
    const int tid = threadIdx.x;
    if (d_n) n = min(*d_n, n);
    if (tid < SP_CELLS) h[tid] = 0;
    __syncthreads();
    const int i0 = blockIdx.x * ch, i1 = min(i0 + ch, n);
    for (int i = i0 + tid; i < i1; i += SP_T) atomicAdd(&h[sp_cell(x[i], y[i], W, H)], 1);
    __syncthreads();
    if (tid < SP_CELLS) hist[blockIdx.x * SP_CELLS + tid] = h[tid];
}

__global__ void __launch_bounds__(SP_T) k_sp_pos(const float* __restrict__ x, const float* __restrict__ y, int n,
                                                 const int* __restrict__ d_n, float W, float H, int ch, int nch,
                                                 const int* __restrict__ hist, int cap, int nfeat,
                                                 int* __restrict__ pos, int* __restrict__ grp_sel,
                                                 int* __restrict__ chunk_sel) {
    if (d_n) n = min(*d_n, n);
    __shared__ int run[SP_CELLS];          // elements of the cell before the current step (all chunks)
    __shared__ int start0[SP_CELLS];       // first selection position of the cell's group-0 elements
    __shared__ int wc[SP_NW][SP_CELLS];    // per warp and cell: count, then the warp's base
    __shared__ int wg1[SP_NW];             // per warp: elements outside group 0, then their base
    __shared__ int s_n1, s_g1, s_sel;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, k = blockIdx.x;
    const unsigned lt = (1u << lane) - 1u;
    if (w == 0) {
        // lane owns cells 4 lane .. 4 lane + 3 (lanes 27..31 none)
        int pre[4], tot[4], g0_pre = 0, g0_tot = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = 4 * lane + q;
            pre[q] = tot[q] = 0;
            if (c < SP_CELLS)
                for (int kk = 0; kk < nch; ++kk) {
                    const int v = hist[kk * SP_CELLS + c];
                    if (kk < k) pre[q] += v;
                    tot[q] += v;
                }
            g0_pre += min(pre[q], cap);
            g0_tot += min(tot[q], cap);
        }
        int incl = g0_tot;
#pragma unroll
        for (int sh = 1; sh < 32; sh <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, sh);
            if (lane >= sh) incl += t;
        }
        int st = incl - g0_tot;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int c = 4 * lane + q;
            if (c < SP_CELLS) {
                start0[c] = st;
                run[c] = pre[q];
            }
            st += min(tot[q], cap);
        }
        g0_pre = warp_sum(g0_pre);
        if (lane == 31) s_n1 = incl;
        // elements of earlier chunks outside group 0: every earlier element minus the group-0
        // ones, which are the first min(pre, cap) of each cell
        if (lane == 0) {
            s_g1 = k * ch - g0_pre;
            s_sel = 0;
        }
    }
    __syncthreads();
    const int n1 = s_n1;
    const int i0 = k * ch, i1 = min(i0 + ch, n);
    for (int base = i0; base < i1; base += SP_T) {
        const int i = base + tid;
        const bool v = i < i1;
        const int c = v ? sp_cell(x[i], y[i], W, H) : SP_CELLS + lane;   // idle lanes: a key of their own
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        const int rl = __popc(peers & lt);
        for (int q = lane; q < SP_CELLS; q += 32) wc[w][q] = 0;
        __syncwarp();
        if (v && rl == 0) wc[w][c] = __popc(peers);
        __syncthreads();
        if (tid < SP_CELLS) {
            int acc = run[tid];
            for (int ww = 0; ww < SP_NW; ++ww) {
                const int t = wc[ww][tid];
                wc[ww][tid] = acc;
                acc += t;
            }
            run[tid] = acc;
        }
        __syncthreads();
        const int rank = v ? wc[w][c] + rl : 0;
        const bool g0 = v && rank < cap;
        const unsigned g1m = __ballot_sync(0xffffffffu, v && !g0);
        if (lane == 0) wg1[w] = __popc(g1m);
        __syncthreads();
        if (w == 0) {
            const int cnt = wg1[lane];
            int incl = cnt;
#pragma unroll
            for (int sh = 1; sh < 32; sh <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, sh);
                if (lane >= sh) incl += t;
            }
            const int g1b = s_g1;
            wg1[lane] = g1b + incl - cnt;
            __syncwarp();
            if (lane == 31) s_g1 = g1b + incl;
        }
        __syncthreads();
        int p = -1;
        if (g0) p = start0[c] + rank;
        else if (v) p = n1 + wg1[w] + __popc(g1m & lt);
        const bool take = v && p < nfeat;
        if (v) pos[i] = take ? p : -1;
        const unsigned tm = __ballot_sync(0xffffffffu, take);
        if (lane == 0 && base + 32 * w < i1) {
            grp_sel[(base + 32 * w) >> 5] = __popc(tm);
            atomicAdd(&s_sel, __popc(tm));
        }
    }
    __syncthreads();
    if (tid == 0) chunk_sel[k] = s_sel;
}

// final slot of each selected element: selected elements before it (earlier chunks, earlier
// groups of its chunk, earlier lanes), corrected inside its run of equal responses (elements of
// the run after it with a smaller selection position come first, elements before it with a
// larger one come after). by_position: slot = selection position (the order _spread returns).
// d_n (nullable): the keypoint count on the device, n a capacity; at most nfeat keypoints are
// all selected, in their own order (features.py:39-40 returns range(n)), as k_iota does
__global__ void __launch_bounds__(256) k_sp_place(const float* __restrict__ resp, int n, const int* __restrict__ d_n,
                                                  int nfeat, int ch, const int* __restrict__ pos,
                                                  const int* __restrict__ grp_sel, const int* __restrict__ chunk_sel,
                                                  bool by_position, int32_t* __restrict__ sel) {
    const int lane = threadIdx.x & 31;
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;   // 32-element group
    if (d_n) {
        n = min(*d_n, n);
        if (n <= nfeat) {
            const int i = g * 32 + lane;
            if (i < n) sel[i] = i;
            return;
        }
    }
    if (g * 32 >= n) return;
    const int k = (g * 32) / ch;
    int before = 0;
    for (int kk = lane; kk < k; kk += 32) before += chunk_sel[kk];
    for (int gg = (k * ch >> 5) + lane; gg < g; gg += 32) before += grp_sel[gg];
    before = warp_sum(before);
    const int i = g * 32 + lane;
    const int p = i < n ? pos[i] : -1;
    const unsigned cm = __ballot_sync(0xffffffffu, p >= 0);
    if (p < 0) return;
    int f = before + __popc(cm & ((1u << lane) - 1u));
    if (by_position) {
        f = p;
    } else {
        const float r = resp[i];
        for (int j = i - 1; j >= 0 && resp[j] == r; --j)
            if (pos[j] > p) --f;
        for (int j = i + 1; j < n && resp[j] == r; ++j) {
            const int pj = pos[j];
            if (pj >= 0 && pj < p) ++f;
        }
    }
    sel[f] = i;
}

__global__ void k_iota(int32_t* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = i;
}

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

DetectConsts make_consts(const Geometry& g, double contrast, double edge) {
    DetectConsts k{};
    k.g = g;
    k.pthr = (float)(0.8 * 0.5 * contrast / N_LAYERS);
    k.contrast = (float)contrast;
    k.edge = (float)edge;
    k.e1sq = (float)((edge + 1.0) * (edge + 1.0));
    long long acc = 0;
    for (int o = 0; o < g.n_oct; ++o) {
        k.vox_off[o] = acc;
        acc += (long long)N_LAYERS * (g.R[o] - 2 * BORDER) * (g.C[o] - 2 * BORDER);
    }
    k.vox_off[g.n_oct] = acc;
    return k;
}

}  // namespace

// Full detection pipeline; contrast/edge in double as the reference's Python floats.
int32_t run_detect(fsb_ctx* ctx, Workspace& ws, double contrast, double edge, int max_kp, bool exact) {
    cudaStream_t s = ctx->stream;
    const Geometry& g = ws.g;
    const DetectConsts k = make_consts(g, contrast, edge);
    uint32_t* cnt = ws.counters.as<uint32_t>();
    const float* DF = ws.dog.as<float>();
    uint32_t h_cnt[3];
    ctx->stage_begin(ST_EXTREMA);
    for (int attempt = 0; attempt < 3; ++attempt) {
        FSB_CUDA(cudaMemsetAsync(cnt, 0, 3 * sizeof(uint32_t), s));
        FSB_TRY(launch_extrema(g, DF, k, ws.cand.as<uint32_t>(), cnt, (uint32_t)ws.cap_cand, s));
        uint32_t h_head[PYR_ERR_WORD + 1];
        FSB_CUDA(cudaMemcpyAsync(h_head, cnt, sizeof(h_head), cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaStreamSynchronize(s));
        if (h_head[PYR_ERR_WORD]) {
            set_error("pyramid: a TMA copy of the pyramid did not complete in time");
            return FSB_ERR_TIMEOUT;
        }

        h_cnt[0] = h_head[0];
        if (h_cnt[0] <= ws.cap_cand) break;
        ws.cap_cand = (size_t)h_cnt[0] + (h_cnt[0] >> 3) + 1024;
        FSB_TRY(ws.cand.ensure(ws.cap_cand * sizeof(uint32_t)));
    }
    ctx->stage_end(ST_EXTREMA);
    const uint32_t n_cand = h_cnt[0];
    if (n_cand == 0) { ws.n_kp = 0; return FSB_OK; }
    if (ws.cap_ref < n_cand) {
        ws.cap_ref = n_cand;
        FSB_TRY(ws.refined.ensure(ws.cap_ref * sizeof(Refined)));
    }
    ctx->stage_begin(ST_REFINE);
    k_refine<<<blocks(n_cand, 128), 128, 0, s>>>(DF, k, ws.cand.as<uint32_t>(), cnt, (uint32_t)ws.cap_cand,
                                                 ws.refined.as<Refined>(), cnt + 1, (uint32_t)ws.cap_ref);
    note_launch();
    FSB_CUDA(cudaGetLastError());
    FSB_CUDA(cudaMemcpyAsync(h_cnt + 1, cnt + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    ctx->stage_end(ST_REFINE);
    const uint32_t n_ref = h_cnt[1];
    if (n_ref == 0) { ws.n_kp = 0; return FSB_OK; }
    if (max_kp <= 0) { ws.n_kp = 0; return FSB_OK; }
    // The reference orients every refined extremum, orders the keypoints by response (stable, the
    // keypoints listed by extremum and bin) and keeps max_kp. All peaks of an extremum share its
    // response, so the kept keypoints are the peaks of the strongest extrema in the order
    // (response descending, DoG index ascending), each extremum's peaks in bin order: rank the
    // extrema once, orient them rank by rank until their peaks fill max_kp (an extremum may have
    // none), and lay the peaks out by an exclusive scan of the per-rank counts.
    ctx->stage_begin(ST_SORT);
    // a stable 31-bit sort by response, then the index order inside runs of equal responses:
    // (response descending, DoG index ascending) with half the radix passes of one 63-bit key
    FSB_TRY(ws.keys_a.ensure((size_t)n_ref * 4 * 2));
    FSB_TRY(ws.vals_a.ensure((size_t)n_ref * 4 * 2));
    FSB_TRY(ws.keys_b.ensure((size_t)n_ref * 4 * 2));
    uint32_t* ka = ws.keys_a.as<uint32_t>();
    uint32_t* va = ws.vals_a.as<uint32_t>();
    uint32_t* rcnt = ws.keys_b.as<uint32_t>();
    uint32_t* rpos = rcnt + n_ref;
    size_t t1 = 0, t2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, ka, ka + n_ref, va, va + n_ref, (int)n_ref, 0, 31, s);
    cub::DeviceScan::ExclusiveSum(nullptr, t2, rcnt, rpos, (int)n_ref, s);
    FSB_TRY(ws.sort_tmp.ensure(t1 > t2 ? t1 : t2));
    k_rank_keys<<<blocks(n_ref, 256), 256, 0, s>>>(ws.refined.as<Refined>(), n_ref, nullptr, ka, va);
    size_t tb = ws.sort_tmp.bytes;
    FSB_CUDA(cub::DeviceRadixSort::SortPairs(ws.sort_tmp.p, tb, ka, ka + n_ref, va, va + n_ref, (int)n_ref, 0, 31,
                                             s));
    uint32_t* order = va;   // the unsorted values are dead
    k_rank_ties<<<blocks(n_ref, 256), 256, 0, s>>>(ka + n_ref, va + n_ref, ws.refined.as<Refined>(), n_ref, nullptr,
                                                   order);
    note_launch(3);
    ctx->stage_end(ST_SORT);
    ctx->stage_begin(ST_ORIENT);
    FSB_TRY(ws.oriented.ensure((size_t)n_ref * ORI_SLOTS * sizeof(Oriented)));
    Oriented* slots = ws.oriented.as<Oriented>();
    FSB_CUDA(cudaMemsetAsync(cnt + 2, 0, sizeof(uint32_t), s));
    uint32_t k1 = 0, total = 0;
    while (true) {
        const uint32_t k0 = k1;
        const uint64_t want = (uint64_t)max_kp > total ? (uint64_t)max_kp - total : 1;
        k1 = (uint32_t)((uint64_t)k0 + want < n_ref ? (uint64_t)k0 + want : n_ref);
        FSB_TRY(run_orient(ws, ws.refined.as<Refined>(), order, k0, k1, slots, rcnt, cnt + 2, exact, s));
        FSB_CUDA(cudaMemcpyAsync(h_cnt + 2, cnt + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaStreamSynchronize(s));
        total = h_cnt[2];
        if (total >= (uint32_t)max_kp || k1 >= n_ref) break;
    }
    ctx->stage_end(ST_ORIENT);
    const uint32_t n_keep = total < (uint32_t)max_kp ? total : (uint32_t)max_kp;
    if (n_keep == 0) { ws.n_kp = 0; return FSB_OK; }
    ctx->stage_begin(ST_SORT);
    tb = ws.sort_tmp.bytes;
    FSB_CUDA(cub::DeviceScan::ExclusiveSum(ws.sort_tmp.p, tb, rcnt, rpos, (int)k1, s));
    const size_t nb4 = (size_t)n_keep * 4;
    FSB_TRY(ws.kx.ensure(nb4));
    FSB_TRY(ws.ky.ensure(nb4));
    FSB_TRY(ws.ksize.ensure(nb4));
    FSB_TRY(ws.kangle.ensure(nb4));
    FSB_TRY(ws.kresp.ensure(nb4));
    FSB_TRY(ws.koct.ensure(nb4));
    FSB_TRY(ws.klayer.ensure(nb4));
    k_gather_ranked<<<blocks(k1, 256), 256, 0, s>>>(slots, rcnt, rpos, ws.refined.as<Refined>(), k1, n_keep, nullptr,
                                                    ws.kx.as<float>(), ws.ky.as<float>(), ws.ksize.as<float>(),
                                                    ws.kangle.as<float>(), ws.kresp.as<float>(), ws.koct.as<int32_t>(),
                                                    ws.klayer.as<int32_t>());
    note_launch(2);
    FSB_CUDA(cudaGetLastError());
    ctx->stage_end(ST_SORT);
    ws.n_kp = (int)n_keep;
    return FSB_OK;
}

// grid-spread selection of nfeat keypoints out of n response-sorted ones (features.py:38-57),
// then (by_position false) the stable response sort of features.py:126: d_sel receives
// min(n, nfeat) keypoint indices. Three launches, no host wait.
int32_t spread_dev(fsb_ctx* ctx, const float* d_x, const float* d_y, const float* d_resp, int n, float W, float H,
                   int nfeat, bool by_position, int32_t* d_sel, int* n_sel, cudaStream_t s) {
    *n_sel = 0;
    if (n <= 0 || nfeat <= 0) return FSB_OK;
    if (n <= nfeat) {
        // every keypoint, already in stable response order (and _spread returns range(n))
        k_iota<<<blocks(n, 256), 256, 0, s>>>(d_sel, n);
        note_launch();
        FSB_CUDA(cudaGetLastError());
        *n_sel = n;
        return FSB_OK;
    }
    // at most 64 chunks of a multiple of 1024 elements
    const int ch = (int)(1024 * (((long long)n + 65535) / 65536));
    const int nch = (n + ch - 1) / ch;
    const int ngrp = (n + 31) / 32;
    FSB_TRY(ctx->s_misc.ensure(((size_t)nch * (SP_CELLS + 1) + (size_t)ngrp + (size_t)n) * 4 + 512));
    int* hist = ctx->s_misc.as<int>();
    int* chunk_sel = hist + (size_t)nch * SP_CELLS;
    int* grp_sel = chunk_sel + nch;
    int* pos = grp_sel + ngrp;
    const int cap = (nfeat + SP_CELLS - 1) / SP_CELLS;
    k_sp_hist<<<nch, SP_T, 0, s>>>(d_x, d_y, n, nullptr, W, H, ch, hist);
    k_sp_pos<<<nch, SP_T, 0, s>>>(d_x, d_y, n, nullptr, W, H, ch, nch, hist, cap, nfeat, pos, grp_sel, chunk_sel);
    k_sp_place<<<blocks((long long)ngrp * 32, 256), 256, 0, s>>>(d_resp, n, nullptr, nfeat, ch, pos, grp_sel,
                                                                   chunk_sel, by_position, d_sel);
    note_launch(3);
    FSB_CUDA(cudaGetLastError());
    *n_sel = nfeat;
    return FSB_OK;
}

int32_t run_spread(const Workspace& ws, int nfeat, int32_t* d_sel_out, int* n_sel, fsb_ctx* ctx, cudaStream_t s) {
    return spread_dev(ctx, ws.kx.as<float>(), ws.ky.as<float>(), ws.kresp.as<float>(), ws.n_kp, (float)ws.g.w,
                      (float)ws.g.h, nfeat, false, d_sel_out, n_sel, s);
}

}  // namespace fsb

// -------------------------------------------------------------------------------------------------
// Detection with every count on the device (no host wait; stream-capturable): the same stages and
// the same outputs as run_detect, each launch sized by a capacity fixed beforehand and reading its
// count from ws.counters. Status words (uint32) of ws.counters: [0] candidates, [1] refined,
// [2] orientation peaks, [3] / [4] the current orientation pass's rank range, [5] keypoints kept,
// [6] features selected, [7] flags (ASYNC_*). A flagged image must be redone by the host-driven path.
namespace fsb {
namespace {

// orientation pass `pass`: the next rank range, as run_detect's loop forms it (empty once the cap
// is met or every refined extremum is oriented)
__global__ void k_orient_range(uint32_t* cnt, int pass, uint32_t max_kp, uint32_t cap_ref, uint32_t cap_rank) {
    if (threadIdx.x != 0) return;
    const uint32_t n_ref = min(cnt[1], cap_ref), total = cnt[2], k1 = pass == 0 ? 0u : cnt[4];
    if (pass > 0 && (total >= max_kp || k1 >= n_ref)) {
        cnt[3] = k1;
        return;
    }
    const uint32_t want = max_kp > total ? max_kp - total : 1u;
    const unsigned long long e = (unsigned long long)k1 + want;
    uint32_t nk = (uint32_t)min(e, (unsigned long long)n_ref);
    nk = min(nk, cap_rank);
    cnt[3] = k1;
    cnt[4] = nk;
}

// after the passes: keypoints kept and the overflow / incomplete flags
__global__ void k_detect_finish(uint32_t* cnt, uint32_t max_kp, uint32_t cap_cand, uint32_t cap_ref) {
    if (threadIdx.x != 0) return;
    const uint32_t n_ref = min(cnt[1], cap_ref), total = cnt[2], k1 = cnt[4];
    uint32_t flags = cnt[7];
    if (cnt[0] > cap_cand) flags |= ASYNC_CAND_OVERFLOW;
    if (cnt[1] > cap_ref) flags |= ASYNC_REF_OVERFLOW;
    if (total < max_kp && k1 < n_ref) flags |= ASYNC_ORIENT_INCOMPLETE;
    cnt[7] = flags;
    cnt[5] = cnt[0] == 0 || n_ref == 0 ? 0u : min(total, max_kp);
}

// features selected: none below 10 keypoints (features.py:121-122), else min(n, nfeat)
__global__ void k_select_count(uint32_t* cnt, int nfeat) {
    if (threadIdx.x != 0) return;
    const uint32_t n = cnt[5];
    cnt[6] = n < 10u ? 0u : min(n, (uint32_t)nfeat);
}

}  // namespace

int32_t async_caps(const Workspace& ws, int max_kp, int nfeat, AsyncCaps* c) {
    const Geometry& g = ws.g;
    long long vox = 0;
    for (int o = 0; o < g.n_oct; ++o)
        vox += (long long)N_LAYERS * max(0, g.R[o] - 2 * BORDER) * max(0, g.C[o] - 2 * BORDER);
    c->cand = (uint32_t)std::min<long long>(std::max<long long>(vox, 1), 1ll << 22);
    c->ref = (uint32_t)std::min<long long>(std::max<long long>((long long)ws.cap_ref, 1ll << 16), c->cand);
    c->ref = (c->ref + 1023) / 1024 * 1024;
    c->kp = std::max(max_kp, 1);
    c->rank = (uint32_t)(2 * c->kp + 32);
    c->nfeat = std::max(nfeat, 1);
    return FSB_OK;
}

int32_t prepare_async(Workspace& ws, const AsyncCaps& c, cudaStream_t s) {
    if (ws.cap_cand < c.cand) {
        ws.cap_cand = c.cand;
        FSB_TRY(ws.cand.ensure((size_t)c.cand * sizeof(uint32_t)));
    }
    FSB_TRY(ws.refined.ensure((size_t)c.ref * sizeof(Refined)));
    FSB_TRY(ws.keys_a.ensure((size_t)c.ref * 4 * 2));
    FSB_TRY(ws.vals_a.ensure((size_t)c.ref * 4 * 2));
    FSB_TRY(ws.keys_b.ensure((size_t)c.rank * 4 * 2));
    FSB_TRY(ws.oriented.ensure((size_t)c.rank * ORI_SLOTS * sizeof(Oriented)));
    size_t t1 = 0, t2 = 0;
    uint32_t* k = ws.keys_a.as<uint32_t>();
    FSB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, k, k + c.ref, k, k + c.ref, (int)c.ref, 0, 31, s));
    FSB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, t2, k, k, (int)c.rank, s));
    FSB_TRY(ws.sort_tmp.ensure(t1 > t2 ? t1 : t2));
    const size_t kb = (size_t)c.kp * 4;
    FSB_TRY(ws.kx.ensure(kb));
    FSB_TRY(ws.ky.ensure(kb));
    FSB_TRY(ws.ksize.ensure(kb));
    FSB_TRY(ws.kangle.ensure(kb));
    FSB_TRY(ws.kresp.ensure(kb));
    FSB_TRY(ws.koct.ensure(kb));
    FSB_TRY(ws.klayer.ensure(kb));
    // spread scratch: chunk histograms, positions, group and chunk counts, the selection
    const int ch = (int)(1024 * (((long long)c.kp + 65535) / 65536));
    const int nch = (c.kp + ch - 1) / ch, ngrp = (c.kp + 31) / 32;
    FSB_TRY(ws.spread.ensure(((size_t)nch * (SP_CELLS + 1) + (size_t)ngrp + 2 * (size_t)c.kp) * 4 + 512));
    // the selected keypoints' fields for description (7 arrays of nfeat) and the selection (kp)
    FSB_TRY(ws.take.ensure(((size_t)c.nfeat * 7 + (size_t)c.kp) * 4 + 512));
    return FSB_OK;
}

int32_t run_detect_async(Workspace& ws, double contrast, double edge, const AsyncCaps& c, int max_kp, bool exact,
                         cudaStream_t s) {
    const uint32_t mk = (uint32_t)std::max(1, std::min(max_kp, c.kp));
    const Geometry& g = ws.g;
    const DetectConsts k = make_consts(g, contrast, edge);
    uint32_t* cnt = ws.counters.as<uint32_t>();
    const float* DF = ws.dog.as<float>();
    FSB_CUDA(cudaMemsetAsync(cnt, 0, 8 * sizeof(uint32_t), s));
    FSB_TRY(launch_extrema(g, DF, k, ws.cand.as<uint32_t>(), cnt, c.cand, s));
    const unsigned gr = std::min(blocks(c.cand, 128), 148u * 16u);
    k_refine<<<gr, 128, 0, s>>>(DF, k, ws.cand.as<uint32_t>(), cnt, c.cand, ws.refined.as<Refined>(), cnt + 1, c.ref);
    uint32_t* ka = ws.keys_a.as<uint32_t>();
    uint32_t* va = ws.vals_a.as<uint32_t>();
    k_rank_keys<<<blocks(c.ref, 256), 256, 0, s>>>(ws.refined.as<Refined>(), c.ref, cnt + 1, ka, va);
    size_t tb = ws.sort_tmp.bytes;
    FSB_CUDA(cub::DeviceRadixSort::SortPairs(ws.sort_tmp.p, tb, ka, ka + c.ref, va, va + c.ref, (int)c.ref, 0, 31,
                                             s));
    uint32_t* order = va;
    k_rank_ties<<<blocks(c.ref, 256), 256, 0, s>>>(ka + c.ref, va + c.ref, ws.refined.as<Refined>(), c.ref, cnt + 1,
                                                   order);
    uint32_t* rcnt = ws.keys_b.as<uint32_t>();
    uint32_t* rpos = rcnt + c.rank;
    FSB_CUDA(cudaMemsetAsync(rcnt, 0, (size_t)c.rank * 4, s));
    Oriented* slots = ws.oriented.as<Oriented>();
    for (int pass = 0; pass < ASYNC_ORIENT_PASSES; ++pass) {
        k_orient_range<<<1, 32, 0, s>>>(cnt, pass, mk, c.ref, c.rank);
        FSB_TRY(run_orient_dev(ws, ws.refined.as<Refined>(), order, (uint32_t)c.kp, cnt + 3, slots, rcnt, cnt + 2,
                               exact, s));
    }
    k_detect_finish<<<1, 32, 0, s>>>(cnt, mk, c.cand, c.ref);
    tb = ws.sort_tmp.bytes;
    FSB_CUDA(cub::DeviceScan::ExclusiveSum(ws.sort_tmp.p, tb, rcnt, rpos, (int)c.rank, s));
    k_gather_ranked<<<blocks(c.rank, 256), 256, 0, s>>>(slots, rcnt, rpos, ws.refined.as<Refined>(), c.rank, 0, cnt + 4,
                                                        ws.kx.as<float>(), ws.ky.as<float>(), ws.ksize.as<float>(),
                                                        ws.kangle.as<float>(), ws.kresp.as<float>(),
                                                        ws.koct.as<int32_t>(), ws.klayer.as<int32_t>());
    note_launch(5 + ASYNC_ORIENT_PASSES);   // k_extrema* and k_orient count themselves
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

int32_t spread_async(Workspace& ws, const AsyncCaps& c, int nfeat, int32_t* d_sel, cudaStream_t s) {
    uint32_t* cnt = ws.counters.as<uint32_t>();
    k_select_count<<<1, 32, 0, s>>>(cnt, nfeat);
    if (nfeat <= 0) return FSB_OK;
    const int* d_n = reinterpret_cast<const int*>(cnt + 5);
    const int n = c.kp;
    const int ch = (int)(1024 * (((long long)n + 65535) / 65536));
    const int nch = (n + ch - 1) / ch;
    const int ngrp = (n + 31) / 32;
    int* hist = ws.spread.as<int>();
    int* chunk_sel = hist + (size_t)nch * SP_CELLS;
    int* grp_sel = chunk_sel + nch;
    int* pos = grp_sel + ngrp;
    const int cap = (nfeat + SP_CELLS - 1) / SP_CELLS;
    const float W = (float)ws.g.w, H = (float)ws.g.h;
    k_sp_hist<<<nch, SP_T, 0, s>>>(ws.kx.as<float>(), ws.ky.as<float>(), n, d_n, W, H, ch, hist);
    k_sp_pos<<<nch, SP_T, 0, s>>>(ws.kx.as<float>(), ws.ky.as<float>(), n, d_n, W, H, ch, nch, hist, cap, nfeat, pos,
                                  grp_sel, chunk_sel);
    k_sp_place<<<blocks((long long)ngrp * 32, 256), 256, 0, s>>>(ws.kresp.as<float>(), n, d_n, nfeat, ch, pos, grp_sel,
                                                                   chunk_sel, false, d_sel);
    note_launch(4);
    FSB_CUDA(cudaGetLastError());
    return FSB_OK;
}

}  // namespace fsb
