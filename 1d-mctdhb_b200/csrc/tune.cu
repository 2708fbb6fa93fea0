// tune.cu -- autotuner for the register-resident kernels.
//
// Each tuned kernel (the pair contraction of H.C, single-system and batched;
// the per-row H.C and density kernels) has a few launch variants (rows per
// tile, output tiles per pass; block size, barrier interval) that compute
// every output with the same instructions in the same order, so a choice
// changes speed, never results.  A launch function returning 1 marks a
// variant that does not exist for the shape (skipped).
// The first call for a (kernel, device, N, M) outside a stream capture times
// every variant on the caller's own data and keeps the fastest; the choice
// is cached in memory and, when MCTDHB_TUNE_CACHE names a file, appended to
// it ("kernel device N M variant" per line) and read back by later
// processes.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "kernels.h"

namespace mctdhb {

namespace {
std::mutex g_mu;
std::map<std::tuple<std::string, int, int, int>, int> g_choice;
bool g_loaded = false;

void load_cache() {
    if (g_loaded) return;
    g_loaded = true;
    const char* path = std::getenv("MCTDHB_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char name[64];
    int d, n, m, v;
    while (std::fscanf(f, "%63s %d %d %d %d", name, &d, &n, &m, &v) == 5)
        g_choice[{name, d, n, m}] = v;
    std::fclose(f);
}

void save(const char* kernel, int d, int n, int m, int v) {
    const char* path = std::getenv("MCTDHB_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%s %d %d %d %d\n", kernel, d, n, m, v);
    std::fclose(f);
}
}  // namespace

int tune_lookup(const char* kernel, int N, int M) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mu);
    load_cache();
    auto it = g_choice.find({kernel, dev, N, M});
    return it == g_choice.end() ? -1 : it->second;
}

void tune_set(const char* kernel, int N, int M, int variant) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mu);
    load_cache();
    g_choice[{kernel, dev, N, M}] = variant;
}

int tune_pick(const char* kernel, int N, int M, int nvariants, cudaStream_t st,
              int (*launch)(void* ctx, int v, cudaStream_t st), void* ctx) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mu);
    load_cache();
    const auto key = std::make_tuple(std::string(kernel), dev, N, M);
    auto it = g_choice.find(key);
    if (it != g_choice.end() && it->second >= 0 && it->second < nvariants) return it->second;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
        return 0;
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return 0;
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return 0;
    }
    int best = 0;
    float best_ms = 1e30f;
    bool ok = true;
    for (int v = 0; v < nvariants && ok; v++) {
        const int w = launch(ctx, v, st);  // warm-up (and attributes); 1: no such variant
        if (w == 1) continue;
        ok = w == 0;
        cudaEventRecord(a, st);
        for (int r = 0; r < 2 && ok; r++) ok = launch(ctx, v, st) == 0;
        cudaEventRecord(b, st);
        if (cudaEventSynchronize(b) != cudaSuccess) ok = false;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (ok && ms < best_ms) {
            best_ms = ms;
            best = v;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (!ok) return 0;
    g_choice[key] = best;
    save(kernel, dev, N, M, best);
    return best;
}

}  // namespace mctdhb

extern "C" {

int mctdhb_tune_get(const char* kernel, int npar, int norb) {
    if (!kernel) return -1;
    return mctdhb::tune_lookup(kernel, npar, norb);
}

int mctdhb_tune_set(const char* kernel, int npar, int norb, int variant) {
    if (!kernel || variant < 0 || variant >= 16) {
        mctdhb::set_error("mctdhb_tune_set: invalid argument");
        return -1;
    }
    mctdhb::tune_set(kernel, npar, norb, variant);
    return 0;
}

}  // extern "C"
