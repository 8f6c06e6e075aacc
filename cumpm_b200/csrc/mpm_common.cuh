// Shared device/host helpers for the cuMPM-B200 operator and solvers.
//
// Complex numbers are float2/double2 (interleaved re/im) so that buffers can
// be handed to cuFFT without copies.  Every multi-right-hand-side buffer in
// this library uses the "RHS-innermost" layout [row][M]: the M right-hand
// sides of one unknown are contiguous, which makes every per-particle access
// a coalesced M-wide vector.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace mpm {

// ---------------------------------------------------------------- errors --

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        throw CudaError(std::string("CUDA error: ") + cudaGetErrorString(e) + " in " + what + " at " +
                        file + ":" + std::to_string(line));
    }
}
#define MPM_CUDA(x) ::mpm::cuda_check((x), #x, __FILE__, __LINE__)

// Raises a kernel's dynamic shared-memory limit to at least `bytes` and never
// lowers it.  The limit is one attribute per kernel for the whole process:
// fields solved at once from several host threads share it, and a lower
// value set for one would make another's larger launch fail.
void raise_smem_limit(const void* kernel, size_t bytes);
template <typename K>
inline void set_smem_limit(K* kernel, size_t bytes) {
    raise_smem_limit(reinterpret_cast<const void*>(kernel), bytes);
}
// count one of this library's kernel launches and check it
void note_launch();
#define MPM_LAUNCH() (::mpm::note_launch(), ::mpm::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__))

// --------------------------------------------------------------- complex --

template <typename R> struct CTraits;
template <> struct CTraits<float> { using T = float2; };
template <> struct CTraits<double> { using T = double2; };
template <typename R> using cplx = typename CTraits<R>::T;

template <typename R> __host__ __device__ __forceinline__ cplx<R> mk(R a, R b) {
    cplx<R> c; c.x = a; c.y = b; return c;
}
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float2 operator*(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ void operator+=(float2& a, float2 b) { a.x += b.x; a.y += b.y; }
__host__ __device__ __forceinline__ void operator-=(float2& a, float2 b) { a.x -= b.x; a.y -= b.y; }
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ void operator+=(double2& a, double2 b) { a.x += b.x; a.y += b.y; }
__host__ __device__ __forceinline__ void operator-=(double2& a, double2 b) { a.x -= b.x; a.y -= b.y; }

__host__ __device__ __forceinline__ double2 conjmul(double2 a, double2 b) {  // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

template <typename R> __device__ __forceinline__ cplx<R> to_r(double2 v);
template <> __device__ __forceinline__ float2 to_r<float>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <> __device__ __forceinline__ double2 to_r<double>(double2 v) { return v; }
__device__ __forceinline__ double2 to_d(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ double2 to_d(double2 v) { return v; }

// fused multiply-add of a real weight into a complex accumulator
__device__ __forceinline__ void fma_rc(float2& acc, float w, float2 v) {
    acc.x = fmaf(w, v.x, acc.x); acc.y = fmaf(w, v.y, acc.y);
}
__device__ __forceinline__ void fma_rc(double2& acc, double w, double2 v) {
    acc.x = fma(w, v.x, acc.x); acc.y = fma(w, v.y, acc.y);
}

// positive modulo for grid indices
__host__ __device__ __forceinline__ int pmod(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }

// signed cyclic distance a-b on a ring of n in (-n/2, n/2]
__host__ __device__ __forceinline__ int cyc_diff(int a, int b, int n) {
    int d = pmod(a - b, n);
    return (2 * d > n) ? d - n : d;
}

constexpr double kPi = 3.14159265358979323846;

// --------------------------------------------------------------- buffers --

// Minimal owning device buffer (cudaMalloc/cudaFree, no caching allocator).
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void ensure(size_t n) {
        if (n <= bytes && p) return;
        release();
        if (n == 0) return;
        MPM_CUDA(cudaMalloc(&p, n));
        bytes = n;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Page-locked host buffer (reused across calls, so host<->device copies run
// at full PCIe/C2C speed and never fault fresh pages).
struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    ~HostBuf() { release(); }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
    }
    void ensure(size_t n) {
        if (n <= bytes && p) return;
        release();
        if (n == 0) return;
        MPM_CUDA(cudaHostAlloc(&p, n, cudaHostAllocDefault));
        bytes = n;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace mpm
