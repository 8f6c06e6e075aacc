// Stage timers (see mpm_profile.h).
#include "mpm_profile.h"

#include "mpm_common.cuh"

#include <mutex>
#include <unordered_map>

namespace mpm {

void note_launch() { Profiler::get().count_launch(); }

void raise_smem_limit(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::unordered_map<const void*, size_t> set;
    std::lock_guard<std::mutex> g(mu);
    size_t& cur = set[kernel];
    if (bytes <= cur) return;
    MPM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    cur = bytes;
}

Profiler& Profiler::get() {
    static Profiler p;
    return p;
}

// Enabling pre-creates a pool of events so that recording during a timed
// region costs only cudaEventRecord; intervals are resolved in read().
void Profiler::enable(bool on) {
    std::lock_guard<std::mutex> g(mu_);
    if (on) {
        const size_t want = 1 << 16;
        while (pool_.size() < want) {
            cudaEvent_t e = nullptr;
            if (cudaEventCreate(&e) != cudaSuccess) break;
            pool_.push_back(e);
        }
    }
    enabled_ = on;
}

cudaEvent_t Profiler::take() {
    if (!pool_.empty()) {
        cudaEvent_t e = pool_.back();
        pool_.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void Profiler::begin(int stage, cudaStream_t s) {
    if (!enabled_) return;
    std::lock_guard<std::mutex> g(mu_);
    cudaEvent_t e = take();
    cudaEventRecord(e, s);
    open_[stage] = e;
}

void Profiler::end(int stage, cudaStream_t s) {
    if (!enabled_) return;
    std::lock_guard<std::mutex> g(mu_);
    if (!open_[stage]) return;
    cudaEvent_t e = take();
    cudaEventRecord(e, s);
    pending_.push_back({stage, open_[stage], e});
    open_[stage] = nullptr;
}

void Profiler::resolve() {
    for (auto& p : pending_) {
        cudaEventSynchronize(p.b);
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            ms_[p.stage] += ms;
            cnt_[p.stage] += 1;
        }
        pool_.push_back(p.a);
        pool_.push_back(p.b);
    }
    pending_.clear();
}

void Profiler::read(double* ms, long long* count, int n) {
    std::lock_guard<std::mutex> g(mu_);
    resolve();
    for (int i = 0; i < n && i < ST_COUNT; ++i) {
        if (ms) ms[i] = ms_[i];
        if (count) count[i] = cnt_[i];
    }
}

void Profiler::reset() {
    std::lock_guard<std::mutex> g(mu_);
    resolve();
    for (int i = 0; i < ST_COUNT; ++i) {
        ms_[i] = 0.0;
        cnt_[i] = 0;
    }
    launches_.store(0);
}

}  // namespace mpm
