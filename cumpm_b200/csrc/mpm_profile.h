// Stage timers and a launch counter for measurement.
//
// When enabled, each stage of the operator and of the Krylov solver is
// bracketed by CUDA events recorded on the stream it runs on; elapsed times
// are resolved lazily (one synchronisation at read time), so enabling it
// adds no host synchronisation to the solve.  The launch counter counts this
// library's own kernel launches (not cuFFT's).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <vector>

namespace mpm {

enum Stage {
    ST_SPREAD = 0,
    ST_FFT_FWD,
    ST_KSPACE,
    ST_FFT_INV,
    ST_CONTRACT,
    ST_REAL,
    ST_DIRECT,
    ST_KRYLOV,
    ST_PRECALC,
    ST_COUNT
};

class Profiler {
public:
    static Profiler& get();
    void enable(bool on);
    bool enabled() const { return enabled_; }
    void begin(int stage, cudaStream_t s);
    void end(int stage, cudaStream_t s);
    // milliseconds and number of intervals per stage
    void read(double* ms, long long* count, int n);
    void reset();
    void count_launch() { launches_.fetch_add(1, std::memory_order_relaxed); }
    long long launches() const { return launches_.load(); }

private:
    struct Pending { int stage; cudaEvent_t a, b; };
    bool enabled_ = false;
    std::mutex mu_;
    std::vector<Pending> pending_;
    cudaEvent_t open_[ST_COUNT] = {};
    double ms_[ST_COUNT] = {};
    long long cnt_[ST_COUNT] = {};
    std::vector<cudaEvent_t> pool_;
    std::atomic<long long> launches_{0};
    cudaEvent_t take();
    void resolve();
};

struct StageScope {
    int st;
    cudaStream_t s;
    StageScope(int stage, cudaStream_t stream) : st(stage), s(stream) { Profiler::get().begin(st, s); }
    ~StageScope() { Profiler::get().end(st, s); }
};

}  // namespace mpm
