// Small device helpers shared by the grid kernels of the field operator
// (spatial bins of particles over voxel tiles).  Included inside an
// anonymous namespace by each translation unit that needs them.
#pragma once

#include "mpm_common.cuh"

namespace mpm {
namespace {

__global__ void k_bin_keys(const int4* __restrict__ base, int n, int tx, int ty, int tz, int nbx, int nby,
                           int* __restrict__ key, int* __restrict__ idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 b = base[i];
    key[i] = (b.z / tz * nby + b.y / ty) * nbx + b.x / tx;
    idx[i] = i;
}

__global__ void k_fill_int(int* p, int n, int v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void k_bin_bounds(const int* __restrict__ skey, int n, int* __restrict__ start, int* __restrict__ end) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = skey[i];
    if (i == 0 || skey[i - 1] != k) start[k] = i;
    if (i == n - 1 || skey[i + 1] != k) end[k] = i + 1;
}

// Distinct bins whose index range can reach [lo, hi] (inclusive, possibly
// outside [0, n) and then wrapped when periodic).
__device__ int reach_bins(int lo, int hi, int n, int t, bool periodic, int* out) {
    int cnt = 0;
    for (int v = lo; v <= hi; ++v) {
        int w = v;
        if (periodic) w = pmod(v, n);
        else if (v < 0 || v >= n) continue;
        const int b = w / t;
        bool seen = false;
        for (int k = 0; k < cnt; ++k) seen |= (out[k] == b);
        if (!seen && cnt < 8) out[cnt++] = b;
    }
    return cnt;
}

}  // namespace
}  // namespace mpm
