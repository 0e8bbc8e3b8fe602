// Feature tracks over the match graph (recon.build_tracks, app/planesite/recon.py:14-54) on the
// device. Nodes are global feature indices (offset of the photo + feature index); every match (i,
// q) <-> (j, t) is an undirected edge. A track is a connected component of at least two matched
// features with no two features of the same photo; tracks are numbered in the order of their
// smallest node (the order in which scipy's connected_components labels the components of an
// undirected graph), observations listed by track, then node.
//   k_tr_hook      every edge joins the roots of its ends: the larger root is hooked under the
//                  smaller (atomicMin), so every tree's root stays the minimum of its nodes; the
//                  host repeats hook + compress until no edge joins two roots (bounded count)
//   k_tr_compress  pointer jumping to the root
//   k_tr_nodes     used flags, per-root sizes, (root, photo) keys of the used nodes
//   k_tr_dups      adjacent equal (root, photo) keys mark their root bad
//   k_tr_live      root flags of the kept components; an exclusive scan numbers them
//   k_tr_emit      (track, node) of every kept node, in node order; a stable sort by track follows
#include <cub/cub.cuh>

#include "fsb_internal.cuh"

namespace fsb {
namespace {

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ int root_of(const int* __restrict__ parent, int x) {
    while (true) {
        const int p = parent[x];
        if (p == x) return x;
        x = p;
    }
}

__global__ void k_tr_init(int* parent, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) parent[i] = i;
}

__global__ void k_tr_hook(const int* __restrict__ eu, const int* __restrict__ ev, long long ne, int* parent,
                          int* changed) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int ru = root_of(parent, eu[e]), rv = root_of(parent, ev[e]);
    if (ru == rv) return;
    const int lo = min(ru, rv), hi = max(ru, rv);
    atomicMin(&parent[hi], lo);
    *changed = 1;
}

__global__ void k_tr_compress(int* parent, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    parent[i] = root_of(parent, i);
}

// photo of global node x: the last offset <= x (offsets ascending, n_img + 1 entries)
__device__ __forceinline__ int photo_of(const long long* __restrict__ off, int n_img, long long x) {
    int lo = 0, hi = n_img;   // off[lo] <= x < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

__global__ void k_tr_used(const int* __restrict__ eu, const int* __restrict__ ev, long long ne, uint8_t* used) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    used[eu[e]] = 1;
    used[ev[e]] = 1;
}

// per used node: size of its root, (root, photo) key and the node itself (for the duplicate sort)
__global__ void k_tr_keys(const uint8_t* __restrict__ used, const int* __restrict__ parent, int n,
                          const long long* __restrict__ off, int n_img, int photo_bits, int* size,
                          unsigned long long* key, int* node, int* n_used) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool u = i < n && used[i];
    const unsigned m = __ballot_sync(0xffffffffu, u);
    int base = 0;
    if ((threadIdx.x & 31) == 0 && m) base = atomicAdd(n_used, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (!u) return;
    const int r = parent[i];
    atomicAdd(&size[r], 1);
    const int slot = base + __popc(m & ((1u << (threadIdx.x & 31)) - 1u));
    key[slot] = ((unsigned long long)r << photo_bits) | (unsigned long long)photo_of(off, n_img, i);
    node[slot] = i;
}

__global__ void k_tr_dups(const unsigned long long* __restrict__ key, int n, int photo_bits, uint8_t* bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 1 || i >= n) return;
    if (key[i] == key[i - 1]) bad[key[i] >> photo_bits] = 1;
}

__global__ void k_tr_live(const int* __restrict__ parent, const int* __restrict__ size, const uint8_t* __restrict__ bad,
                          int n, int* live) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    live[i] = (parent[i] == i && size[i] >= 2 && !bad[i]) ? 1 : 0;
}

// kept used nodes in ascending node order: track number and node
__global__ void k_tr_emit(const uint8_t* __restrict__ used, const int* __restrict__ parent,
                          const int* __restrict__ live, const int* __restrict__ rank, int n, unsigned* tkey,
                          int* tnode, int* n_kept) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool k = false;
    int r = 0;
    if (i < n && used[i]) {
        r = parent[i];
        k = live[r] != 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, k);
    int base = 0;
    if ((threadIdx.x & 31) == 0 && m) base = atomicAdd(n_kept, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (!k) return;
    const int slot = base + __popc(m & ((1u << (threadIdx.x & 31)) - 1u));
    tkey[slot] = (unsigned)rank[r];
    tnode[slot] = i;
}

// combined order key of a kept node: track above node (both below 2^31)
__global__ void k_tr_key64(const unsigned* __restrict__ tkey, const int* __restrict__ tnode, int n,
                           unsigned long long* __restrict__ key) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) key[i] = ((unsigned long long)tkey[i] << 32) | (unsigned)tnode[i];
}

__global__ void k_tr_out(const unsigned long long* __restrict__ key, int n, const long long* __restrict__ off,
                         int n_img, long long* tid, long long* img, long long* feat) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int x = (int)(key[i] & 0xffffffffull);
    const int p = photo_of(off, n_img, x);
    tid[i] = (long long)(key[i] >> 32);
    img[i] = p;
    feat[i] = x - off[p];
}

__global__ void k_tr_edges(const long long* __restrict__ u, const long long* __restrict__ v, long long ne, int* eu,
                           int* ev) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    eu[e] = (int)u[e];
    ev[e] = (int)v[e];
}

}  // namespace

// d_u, d_v: n_edges global node indices in [0, n_nodes); d_off: n_img + 1 photo offsets. Outputs
// (capacity 2 n_edges): track, photo, feature of every observation; *n_obs, *n_tracks.
int32_t run_build_tracks(fsb_ctx* ctx, const long long* d_u, const long long* d_v, long long ne, const long long* d_off,
                         int n_img, int n_nodes, long long* d_tid, long long* d_img, long long* d_feat, int* n_obs,
                         int* n_tracks, cudaStream_t s) {
    *n_obs = 0;
    *n_tracks = 0;
    if (ne == 0 || n_nodes == 0) return FSB_OK;
    const size_t N = (size_t)n_nodes, E = (size_t)ne;
    int photo_bits = 1;
    while ((1 << photo_bits) < n_img) ++photo_bits;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    size_t t1 = 0, t2 = 0, t3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t1, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                    (int*)nullptr, (int*)nullptr, n_nodes, 0, 31 + photo_bits, s);
    cub::DeviceScan::ExclusiveSum(nullptr, t2, (int*)nullptr, (int*)nullptr, n_nodes, s);
    cub::DeviceRadixSort::SortKeys(nullptr, t3, (unsigned long long*)nullptr, (unsigned long long*)nullptr, n_nodes,
                                   0, 64, s);
    const size_t tmp = std::max(t1, std::max(t2, t3));
    const size_t need = 4 * al(N * 4) + 2 * al(N) + 2 * al(N * 8) + 4 * al(N * 4) + 2 * al(E * 4) + al(64) + al(tmp);
    FSB_TRY(ctx->s_misc.ensure(need));
    char* b = static_cast<char*>(ctx->s_misc.p);
    auto take = [&](size_t bytes) {
        char* p = b;
        b += al(bytes);
        return p;
    };
    int* parent = (int*)take(N * 4);
    int* size = (int*)take(N * 4);
    int* live = (int*)take(N * 4);
    int* rank = (int*)take(N * 4);
    uint8_t* used = (uint8_t*)take(N);
    uint8_t* bad = (uint8_t*)take(N);
    unsigned long long* key = (unsigned long long*)take(N * 8);
    unsigned long long* key2 = (unsigned long long*)take(N * 8);
    int* node = (int*)take(N * 4);
    int* node2 = (int*)take(N * 4);
    unsigned* tkey = (unsigned*)take(N * 4);
    int* tnode = (int*)take(N * 4);
    int* eu = (int*)take(E * 4);
    int* ev = (int*)take(E * 4);
    int* cnt = (int*)take(64);   // [0] changed, [1] used, [2] kept
    void* ctmp = take(tmp);
    const unsigned gn = blocks(n_nodes, 256), ge = blocks(ne, 256);
    k_tr_edges<<<ge, 256, 0, s>>>(d_u, d_v, ne, eu, ev);
    k_tr_init<<<gn, 256, 0, s>>>(parent, n_nodes);
    note_launch(2);
    // union by hooking to the smaller root; each round joins every pair of trees an edge still spans
    int changed = 1, rounds = 0;
    while (changed) {
        if (++rounds > 64) {
            set_error("track union did not converge in 64 rounds");
            return FSB_ERR_CUDA;
        }
        FSB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), s));
        k_tr_hook<<<ge, 256, 0, s>>>(eu, ev, ne, parent, cnt);
        k_tr_compress<<<gn, 256, 0, s>>>(parent, n_nodes);
        note_launch(2);
        FSB_CUDA(cudaMemcpyAsync(&changed, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
        FSB_CUDA(cudaStreamSynchronize(s));
    }
    FSB_CUDA(cudaMemsetAsync(used, 0, N, s));
    FSB_CUDA(cudaMemsetAsync(bad, 0, N, s));
    FSB_CUDA(cudaMemsetAsync(size, 0, N * 4, s));
    FSB_CUDA(cudaMemsetAsync(cnt, 0, 64, s));
    k_tr_used<<<ge, 256, 0, s>>>(eu, ev, ne, used);
    k_tr_keys<<<gn, 256, 0, s>>>(used, parent, n_nodes, d_off, n_img, photo_bits, size, key, node, cnt + 1);
    note_launch(2);
    int h_used = 0;
    FSB_CUDA(cudaMemcpyAsync(&h_used, cnt + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    size_t tb = tmp;
    FSB_CUDA(cub::DeviceRadixSort::SortPairs(ctmp, tb, key, key2, node, node2, h_used, 0, 31 + photo_bits, s));
    k_tr_dups<<<blocks(h_used, 256), 256, 0, s>>>(key2, h_used, photo_bits, bad);
    k_tr_live<<<gn, 256, 0, s>>>(parent, size, bad, n_nodes, live);
    note_launch(3);
    tb = tmp;
    FSB_CUDA(cub::DeviceScan::ExclusiveSum(ctmp, tb, live, rank, n_nodes, s));
    k_tr_emit<<<gn, 256, 0, s>>>(used, parent, live, rank, n_nodes, tkey, tnode, cnt + 2);
    note_launch(2);
    int h_kept = 0, h_last_rank = 0, h_last_live = 0;
    FSB_CUDA(cudaMemcpyAsync(&h_kept, cnt + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaMemcpyAsync(&h_last_rank, rank + n_nodes - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaMemcpyAsync(&h_last_live, live + n_nodes - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    FSB_CUDA(cudaStreamSynchronize(s));
    if (h_kept > 0) {
        // warp-appended order -> (track, node) order; the keys are distinct
        k_tr_key64<<<blocks(h_kept, 256), 256, 0, s>>>(tkey, tnode, h_kept, key);
        tb = tmp;
        FSB_CUDA(cub::DeviceRadixSort::SortKeys(ctmp, tb, key, key2, h_kept, 0, 64, s));
        k_tr_out<<<blocks(h_kept, 256), 256, 0, s>>>(key2, h_kept, d_off, n_img, d_tid, d_img, d_feat);
        note_launch(3);
    }
    FSB_CUDA(cudaGetLastError());
    *n_obs = h_kept;
    *n_tracks = h_last_rank + h_last_live;
    return FSB_OK;
}

}  // namespace fsb
