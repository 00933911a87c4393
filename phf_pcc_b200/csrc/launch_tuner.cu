// Per-shape launch tuner: the first evaluation of a plan created with autotune records every GEMM
// launch it makes (shape, layout, and a closure that can repeat the launch with another choice), then
// times each candidate choice of every shape not yet in the table -- two warm-up launches and the
// fastest of three timed ones, CUDA events on the tuning stream -- and keeps the fastest.  The table
// is shared by all plans of the process, so instances with the same shapes are timed once.
// Candidates never change results: the FP64 GEMM's tile shapes share one k order per output element,
// and the int8 GEMM's raster group only reorders the CTAs.
#include <cuda_runtime.h>

#include <mutex>
#include <unordered_map>

#include "phf_internal.h"

namespace phf {

thread_local std::vector<TuneCall> *t_tune_record = nullptr;

namespace {
struct KeyHash {
    size_t operator()(const TuneKey &k) const {
        size_t h = (size_t)k.kind * 0x9E3779B97F4A7C15ull;
        for (long long v : {k.a, k.b, k.c, k.d, k.e}) h = (h ^ (size_t)v) * 0x100000001B3ull + 0x9E3779B9ull;
        return h;
    }
};
std::mutex g_tune_mu;
std::unordered_map<TuneKey, int, KeyHash> g_tune_table;
}  // namespace

int tuned_choice(const TuneKey &key) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_table.find(key);
    return it == g_tune_table.end() ? -1 : it->second;
}

int tuned_entries() {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    return (int)g_tune_table.size();
}

int tune_recorded(std::vector<TuneCall> &calls, cudaStream_t st) {
    cudaEvent_t e0, e1;
    PHF_CUDA(cudaEventCreate(&e0));
    PHF_CUDA(cudaEventCreate(&e1));
    int status = PHF_OK;
    for (TuneCall &c : calls) {
        if (tuned_choice(c.key) >= 0) continue;
        int best = -1;
        float best_ms = 0.f;
        for (int cand : c.candidates) {
            bool ok = true;
            for (int w = 0; w < 2 && ok; ++w) ok = c.launch(cand, st) == PHF_OK;
            float t = 0.f;
            for (int r = 0; r < 3 && ok; ++r) {
                ok = cudaEventRecord(e0, st) == cudaSuccess && c.launch(cand, st) == PHF_OK &&
                     cudaEventRecord(e1, st) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
                float ms = 0.f;
                if (ok) ok = cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
                if (ok && (r == 0 || ms < t)) t = ms;
            }
            if (!ok) {  // a candidate that cannot launch this shape (grid limits) is skipped
                cudaGetLastError();
                continue;
            }
            if (best < 0 || t < best_ms) {
                best = cand;
                best_ms = t;
            }
        }
        if (best < 0) {
            set_error(PHF_ERR_CUDA, "launch tuner: no candidate could run a recorded launch");
            status = PHF_ERR_CUDA;
            break;
        }
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_table[c.key] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (status == PHF_OK) PHF_CUDA(cudaStreamSynchronize(st));
    return status;
}

}  // namespace phf
