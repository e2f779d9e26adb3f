// Kernel-variant autotuner; see b200_tune.h.
#include "b200_tune.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

namespace b200 {

namespace {

std::mutex g_mu;
std::map<std::tuple<int, int, int, int, int, int>, int> g_cache;

int env_int(const char* name, int fallback) {
    const char* v = std::getenv(name);
    if (!v || !*v) return fallback;
    return std::atoi(v);
}

// BEAGLE_B200_FORCE_VARIANT: one variant for every kind ("3"), or one per
// kind in TuneKind order ("1,1,4" = post-order walk, pre-order walk,
// derivative); -1 or a missing entry leaves that kind to the tuner.
int forced_variant(int kind) {
    const char* v = std::getenv("BEAGLE_B200_FORCE_VARIANT");
    if (!v || !*v) return -1;
    if (!std::strchr(v, ',')) return std::atoi(v);
    int k = 1;
    for (const char* q = v; q && *q; ++k) {
        if (k == kind) return std::atoi(q);
        q = std::strchr(q, ',');
        if (q) ++q;
    }
    return -1;
}

}  // namespace

int tune_count_class(int n) {
    int c = 0;
    while (n > 1) {
        n >>= 1;
        ++c;
    }
    return c;
}

int tune_pick(const TuneKey& k, int nvariants, bool may_time, cudaStream_t s,
              const std::function<cudaError_t(int)>& run) {
    if (nvariants <= 1) return -1;
    const int forced = forced_variant(k.kind);
    if (forced >= 0) return forced < nvariants ? forced : nvariants - 1;
    if (env_int("BEAGLE_B200_TUNE", 1) == 0) return -1;
    const auto key = std::make_tuple(k.kind, k.dbl, k.C, k.Pp, k.count_class, k.device);
    {
        std::lock_guard<std::mutex> g(g_mu);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) return it->second;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (!may_time || cudaStreamIsCapturing(s, &cap) != cudaSuccess ||
        cap != cudaStreamCaptureStatusNone)
        return -1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        (void)cudaGetLastError();
        return -1;
    }
    int best = -1;
    float best_ms = 0;
    for (int v = 0; v < nvariants; ++v) {
        // One untimed run (first-launch costs), then two timed runs.
        if (run(v) != cudaSuccess) {
            (void)cudaGetLastError();
            continue;
        }
        cudaEventRecord(e0, s);
        cudaError_t e = run(v);
        if (e == cudaSuccess) e = run(v);
        cudaEventRecord(e1, s);
        if (e != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
            (void)cudaGetLastError();
            continue;
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (env_int("BEAGLE_B200_TUNE_LOG", 0))
            std::fprintf(stderr, "beagle-b200 tune: kind %d dbl %d C %d Pp %d n~2^%d variant %d: %.4f ms\n",
                         k.kind, k.dbl, k.C, k.Pp, k.count_class, v, ms / 2);
        if (best < 0 || ms < best_ms) {
            best = v;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> g(g_mu);
    g_cache[key] = best;
    return best;
}

}  // namespace b200
