// Launch accounting: every kernel launch of the library is counted by kind, and when
// event timing is switched on each launch is bracketed by CUDA events recorded on the
// launching stream, so per-kernel device time can be read back after a timed region.
#include <mutex>
#include <vector>

#include "profile.cuh"

namespace emusv {

namespace {
struct Rec {
    int kind;
    cudaEvent_t a, b;
};
std::mutex mu;
bool timing = false;
long long counts[PROF_KINDS] = {0};
std::vector<Rec> recs;
std::vector<cudaEvent_t> pool;
size_t pool_used = 0;

cudaEvent_t take_event() {
    if (pool_used < pool.size()) return pool[pool_used++];
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    pool.push_back(e);
    ++pool_used;
    return e;
}
}  // namespace

void prof_begin_launch(int kind, cudaStream_t s, void **token) {
    std::lock_guard<std::mutex> g(mu);
    if (kind >= 0 && kind < PROF_KINDS) ++counts[kind];
    *token = nullptr;
    if (!timing) return;
    cudaEvent_t a = take_event(), b = take_event();
    if (!a || !b) return;
    cudaEventRecord(a, s);
    recs.push_back({kind, a, b});
    *token = reinterpret_cast<void *>(recs.size());
}

void prof_end_launch(void *token, cudaStream_t s) {
    if (!token) return;
    std::lock_guard<std::mutex> g(mu);
    const size_t i = reinterpret_cast<size_t>(token) - 1;
    if (i < recs.size()) cudaEventRecord(recs[i].b, s);
}

}  // namespace emusv

using namespace emusv;

extern "C" {

void emusv_profile_begin(int event_timing) {
    std::lock_guard<std::mutex> g(mu);
    for (int k = 0; k < PROF_KINDS; ++k) counts[k] = 0;
    recs.clear();
    pool_used = 0;
    timing = event_timing != 0;
}

int emusv_profile_end(double *ms_by_kind, long long *launches_by_kind, int nkinds) {
    std::lock_guard<std::mutex> g(mu);
    const int nk = nkinds < PROF_KINDS ? nkinds : PROF_KINDS;
    for (int k = 0; k < nk; ++k) {
        if (ms_by_kind) ms_by_kind[k] = 0.0;
        if (launches_by_kind) launches_by_kind[k] = counts[k];
    }
    int st = EMUSV_OK;
    for (const Rec &r : recs) {
        if (cudaEventSynchronize(r.b) != cudaSuccess) {
            st = EMUSV_CUDA_ERROR;
            continue;
        }
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) {
            st = EMUSV_CUDA_ERROR;
            continue;
        }
        if (ms_by_kind && r.kind >= 0 && r.kind < nk) ms_by_kind[r.kind] += ms;
    }
    recs.clear();
    pool_used = 0;
    timing = false;
    return st;
}

}  // extern "C"
