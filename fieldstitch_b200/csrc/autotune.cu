// Launch-variant autotuner.
//
// Several kernels here come in variants that compute bit-identical results with different launch
// shapes (the per-layer pyramid kernel's tile height, for instance). The first time a problem key
// (kernel and size) is met on a device, autotune() runs every variant twice on the caller's
// stream (warm-up, then timed with CUDA events) and keeps the fastest; later calls run the kept
// variant directly. Because the variants agree bit for bit and the runs are idempotent, tuning
// inside a real call leaves that call's outputs as they would have been. A variant may itself call
// autotune() for its own launches (the lock is never held while a variant runs).
//   FSB_AUTOTUNE=0          always variant 0 (no timing)
//   FSB_AUTOTUNE_FILE=path  choices are read from and appended to `path` ("key variant" lines)
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <string>

#include "fsb_internal.cuh"

namespace fsb {
namespace {

std::mutex g_mu;
std::map<std::string, int> g_best;
bool g_loaded = false;

bool tuning_on() {
    const char* e = std::getenv("FSB_AUTOTUNE");
    return !(e && std::strcmp(e, "0") == 0);
}

void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    const char* f = std::getenv("FSB_AUTOTUNE_FILE");
    if (!f) return;
    std::ifstream in(f);
    std::string k;
    int v;
    while (in >> k >> v) g_best[k] = v;
}

// device name per ordinal, looked up once (cudaGetDeviceProperties is slow)
std::string device_tag(int dev) {
    static std::mutex m;
    static std::map<int, std::string> names;
    std::lock_guard<std::mutex> lk(m);
    auto it = names.find(dev);
    if (it != names.end()) return it->second;
    cudaDeviceProp p;
    std::string name = cudaGetDeviceProperties(&p, dev) == cudaSuccess ? p.name : "gpu";
    for (char& c : name)
        if (c == ' ') c = '_';
    name += "/" + std::to_string(dev) + "/";
    names[dev] = name;
    return name;
}

std::string full_key(const char* key) {
    int dev = 0;
    cudaGetDevice(&dev);
    return device_tag(dev) + key;
}

}  // namespace

int32_t autotune(const char* key, int n_variants, int32_t (*run)(void*, int), void* arg, cudaStream_t s, int* variant) {
    *variant = 0;
    if (n_variants <= 1 || !tuning_on()) return run(arg, 0);
    const std::string k = full_key(key);
    int cached = -1;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        load_locked();
        auto it = g_best.find(k);
        if (it != g_best.end()) cached = it->second < n_variants ? it->second : 0;
    }
    if (cached >= 0) {   // run outside the lock: a variant may tune its own launches
        *variant = cached;
        return run(arg, cached);
    }
    cudaEvent_t e0, e1;
    FSB_CUDA(cudaEventCreate(&e0));
    FSB_CUDA(cudaEventCreate(&e1));
    int best = 0;
    float best_ms = 0.f;
    int32_t rc = FSB_OK;
    for (int v = 0; v < n_variants && rc == FSB_OK; ++v) {
        rc = run(arg, v);   // warm-up (first launch of a variant sets its attributes)
        if (rc != FSB_OK) break;
        cudaEventRecord(e0, s);
        rc = run(arg, v);
        cudaEventRecord(e1, s);
        if (rc != FSB_OK || cudaEventSynchronize(e1) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (v == 0 || ms < best_ms) {
            best = v;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != FSB_OK) return rc;
    FSB_CUDA(cudaGetLastError());
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_best.emplace(k, best).second) {
        if (const char* f = std::getenv("FSB_AUTOTUNE_FILE")) {
            std::ofstream out(f, std::ios::app);
            out << k << " " << best << "\n";
        }
    }
    *variant = best;
    return FSB_OK;
}

// The kept variant of `key` when it is known (or tuning is off: variant 0); false while the key
// has not been tuned yet.
bool autotune_cached(const char* key, int n_variants, int* variant) {
    *variant = 0;
    if (n_variants <= 1 || !tuning_on()) return true;
    const std::string k = full_key(key);
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    auto it = g_best.find(k);
    if (it == g_best.end()) return false;
    *variant = it->second < n_variants ? it->second : 0;
    return true;
}

}  // namespace fsb

// "key variant" lines of every choice made so far in this process (for reports); returns the
// number of bytes needed, writes at most len - 1 of them and a terminating zero.
int32_t fsb_autotune_table(char* buf, int32_t len) {
    std::string t;
    {
        std::lock_guard<std::mutex> lk(fsb::g_mu);
        for (const auto& kv : fsb::g_best) t += kv.first + " " + std::to_string(kv.second) + "\n";
    }
    if (buf && len > 0) {
        const size_t n = t.size() < (size_t)(len - 1) ? t.size() : (size_t)(len - 1);
        std::memcpy(buf, t.data(), n);
        buf[n] = 0;
    }
    return (int32_t)t.size() + 1;
}
