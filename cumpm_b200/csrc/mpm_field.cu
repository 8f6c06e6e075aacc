// Field operator kernels and host orchestration (see mpm_field.h).
//
// Reciprocal space (periodic boxes) follows the reference algorithm
// (monodisperse_ewald_electric_field.cu:2211-2411: spread -> forward FFT ->
// k-space Green tensor -> inverse FFT -> contract) with a B200-first layout:
//
//  * The grid is stored [ix][iy][slot][b] with b = component*M + rhs, so all
//    M right-hand sides of a voxel are contiguous and every access is a
//    coalesced vector.
//  * Spreading is a gather over voxel tiles: each CTA owns a tile, pulls the
//    particles whose Gaussian stencil reaches it from a spatial bin index and
//    writes every voxel exactly once (no atomics, deterministic, no memset).
//  * Slab geometries (all particles within a few z planes, as in a monolayer
//    with a vacuum gap) use a pruned transform: 2-D FFTs on the occupied
//    planes only, and the z part of DFT -> Green tensor -> inverse DFT applied
//    per (kx, ky) column as a Toeplitz matrix over the occupied planes.  This
//    is the same discrete operator as the full 3-D FFT path, evaluated
//    without the zero planes.
//  * Contraction gathers each particle's stencil for all M columns at once.
//  * The real-space pair sum is a gather by target over a CSR neighbour list
//    built on the device from a cell list (no atomics); the self term, the
//    Jacobi scaling and the INTERACTION_FIELD sign are fused into it.
#include "mpm_field.h"
#include "mpm_bins.cuh"
#include "mpm_profile.h"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace mpm {

// ---------------------------------------------------------------- geometry

EwaldGeom make_ewald_geom(const double box[3], double errortol, double xi, const int* grid, int support) {
    EwaldGeom g;
    double rc = std::sqrt(-std::log(errortol)) / xi;
    if (rc < 2.0) rc = 2.0;
    if (rc > box[0] / 2.0 || rc > box[1] / 2.0 || rc > box[2] / 2.0) {
        throw std::runtime_error("Real space cutoff (" + std::to_string(rc) + ") larger than half the box length.");
    }
    g.rc = rc;
    g.kcut = 2.0 * xi * xi * rc;
    for (int d = 0; d < 3; ++d) {
        g.ng[d] = static_cast<int>(std::ceil(1.0 + box[d] * g.kcut / kPi));
        if (grid && grid[d] > 0) g.ng[d] = grid[d];
        g.h[d] = box[d] / g.ng[d];
    }
    g.P = static_cast<int>(std::ceil(-2.0 * std::log(errortol) / kPi));
    if (support > 0) g.P = support;
    g.off = g.P / 2;
    for (int d = 0; d < 3; ++d) g.eta[d] = g.P * std::pow(g.h[d] * xi, 2) / kPi;
    g.spread_const = std::pow(2.0 * xi * xi / kPi, 1.5) * std::sqrt(1.0 / (g.eta[0] * g.eta[1] * g.eta[2]));
    return g;
}

// ------------------------------------------------------------- kernels ---

namespace {

constexpr int kMaxStencil = 32;  // S = 2*off+1 <= 32  (errortol >= ~1e-21)

struct StencilArgs {
    double h[3];
    double eta[3];
    double xi;
    double cfac;   // folded into the x weights
    int N[3];
    int off, S;
    int z0, pruned, Zs;
    int layer;     // single layer: unit z weight at the centre (the real ones live in the k-space taps)
};

// Per point: nearest grid node (C round, halves away from zero), 1-D
// Gaussian weights along each axis, wrapped indices and z slot
// (monodisperse_ewald_electric_field.cu:716-746).
__global__ void k_stencil(const double* __restrict__ xyz, int n, StencilArgs a, int4* __restrict__ base,
                          double* __restrict__ w64, float* __restrict__ w32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int gw[3];
    for (int d = 0; d < 3; ++d) {
        const double p = xyz[d * n + i];
        const int g = static_cast<int>(round(p / a.h[d]));
        const double dd = g * a.h[d] - p;
        gw[d] = pmod(g, a.N[d]);
        const double c = (d == 0) ? a.cfac : 1.0;
        for (int o = 0; o < a.S; ++o) {
            const double gd = dd + (o - a.off) * a.h[d];
            const double w = (d == 2 && a.layer) ? (o == a.off ? 1.0 : 0.0)
                                                 : c * exp(-2.0 * a.xi * a.xi * gd * gd / a.eta[d]);
            w64[(size_t(i) * 3 + d) * a.S + o] = w;
            w32[(size_t(i) * 3 + d) * a.S + o] = static_cast<float>(w);
        }
    }
    const int slot = a.pruned ? pmod(gw[2] - a.z0, a.N[2]) : gw[2];
    base[i] = make_int4(gw[0], gw[1], slot, gw[2]);
}

// Gather spread: every voxel of this CTA's tile is written once with the sum
// of all particle contributions (no atomics).  grid[((x*Ny+y)*Zs+s)*B + b].
// Candidates come from the spatial bins that can reach the tile; for each
// (x, y) column of the tile the candidates whose x and y weights are both
// non-zero are listed once (in candidate order, so sums are deterministic),
// and each voxel then loops only over its column's list.
constexpr int kSpreadListCap = 64;
constexpr int kSpreadZMax = 16;   // largest z extent of a spread tile

template <typename R>
__global__ void __launch_bounds__(256) k_spread(const double2* __restrict__ X, int M, int N, int C,
                                                const int* __restrict__ quad_map,
                                                const int4* __restrict__ base, const R* __restrict__ w1,
                                                const int* __restrict__ bin_start, const int* __restrict__ bin_end,
                                                const int* __restrict__ sorted_idx, GridView g, int TX, int TY,
                                                int TZ, int nbx, int nby, int nzt, int cap, int bc,
                                                cplx<R>* __restrict__ grid) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int bx[8], by[8], bz[8], nbxs, nbys, nbzs;
    __shared__ int rstart[512], rlen[512], rpre[513], nranges;
    // blockIdx.z = z tile + nzt * (column chunk of bc columns)
    const int zt = blockIdx.z % nzt, chunk = blockIdx.z / nzt;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = zt * TZ;
    const int x1 = min(x0 + TX, g.Nx), y1 = min(y0 + TY, g.Ny), z1 = min(z0 + TZ, g.Zs);
    const int B = C * M;
    if (threadIdx.x == 0) {
        nbxs = reach_bins(x0 - g.off, x1 - 1 + g.off, g.Nx, TX, true, bx);
        nbys = reach_bins(y0 - g.off, y1 - 1 + g.off, g.Ny, TY, true, by);
        nbzs = reach_bins(z0 - g.off, z1 - 1 + g.off, g.Zs, TZ, !g.pruned, bz);
        int k = 0;
        rpre[0] = 0;
        for (int a = 0; a < nbzs; ++a)
            for (int b2 = 0; b2 < nbys; ++b2)
                for (int c = 0; c < nbxs; ++c) {
                    const int key = (bz[a] * nby + by[b2]) * nbx + bx[c];
                    const int s0 = bin_start[key];
                    if (s0 < 0 || k >= 512) continue;
                    rstart[k] = s0;
                    rlen[k] = bin_end[key] - s0;
                    rpre[k + 1] = rpre[k] + rlen[k];
                    ++k;
                }
        nranges = k;
    }
    __syncthreads();
    const int total = rpre[nranges];
    const int wlen = TX + TY + TZ;
    const int ncol = TX * TY;
    R* wT = reinterpret_cast<R*>(smem_raw);                                       // [cap][wlen]
    cplx<R>* pv = reinterpret_cast<cplx<R>*>(smem_raw + sizeof(R) * cap * wlen);   // [cap][bc]
    R* lw = reinterpret_cast<R*>(pv + size_t(cap) * bc);                           // [ncol][cap_l]
    int* lc = reinterpret_cast<int*>(lw + size_t(ncol) * kSpreadListCap);          // [ncol][cap_l]
    int* ln = lc + size_t(ncol) * kSpreadListCap;                                  // [ncol]
    int* cid = ln + ncol;                                                          // [cap]
    for (int r0 = 0; r0 < max(total, 1); r0 += cap) {
        const int nc = min(cap, total - r0);
        // candidate ids
        for (int t = threadIdx.x; t < nc; t += blockDim.x) {
            const int gidx = r0 + t;
            int k = 0;
            while (rpre[k + 1] <= gidx) ++k;
            cid[t] = sorted_idx[rstart[k] + gidx - rpre[k]];
        }
        __syncthreads();
        // per-candidate 1-D weights restricted to the tile (0 outside reach)
        for (int t = threadIdx.x; t < nc * wlen; t += blockDim.x) {
            const int c = t / wlen, l = t % wlen;
            const int i = cid[c];
            const int4 bs = base[i];
            R w = R(0);
            if (l < TX) {
                const int x = x0 + l;
                if (x < g.Nx) {
                    const int d = cyc_diff(x, bs.x, g.Nx);
                    if (d >= -g.off && d <= g.off) w = w1[(size_t(i) * 3 + 0) * g.S + d + g.off];
                }
            } else if (l < TX + TY) {
                const int y = y0 + l - TX;
                if (y < g.Ny) {
                    const int d = cyc_diff(y, bs.y, g.Ny);
                    if (d >= -g.off && d <= g.off) w = w1[(size_t(i) * 3 + 1) * g.S + d + g.off];
                }
            } else {
                const int s = z0 + l - TX - TY;
                if (s < g.Zs) {
                    const int d = g.pruned ? (s - bs.z) : cyc_diff(s, bs.z, g.Nz);
                    if (d >= -g.off && d <= g.off) w = w1[(size_t(i) * 3 + 2) * g.S + d + g.off];
                }
            }
            wT[c * wlen + l] = w;
        }
        __syncthreads();
        // contributor list per (x, y) column in candidate order, -1 = too
        // many (full loop): one warp per column, 32 candidates per ballot
        {
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
            for (int col = warp; col < ncol; col += nwarp) {
                const int lx = col / TY, ly = col % TY;
                int n = 0;
                for (int cb = 0; cb < nc; cb += 32) {
                    const int c = cb + lane;
                    const R wxy = c < nc ? wT[c * wlen + lx] * wT[c * wlen + TX + ly] : R(0);
                    const unsigned hit = __ballot_sync(0xffffffffu, wxy != R(0));
                    const int at = n + __popc(hit & ((1u << lane) - 1u));
                    if (wxy != R(0) && at < kSpreadListCap) {
                        lw[col * kSpreadListCap + at] = wxy;
                        lc[col * kSpreadListCap + at] = c;
                    }
                    n += __popc(hit);
                }
                if (lane == 0) ln[col] = n <= kSpreadListCap ? n : -1;
            }
        }
        {
            const int b0 = chunk * bc;
            const int nb = min(bc, B - b0);
            __syncthreads();
            for (int t = threadIdx.x; t < nc * nb; t += blockDim.x) {
                const int c = t / nb, bb = t % nb;
                const int i = cid[c];
                const int b = b0 + bb;
                const int comp = b / M;
                double2 v;
                if (comp < 3) {
                    v = X[size_t(3 * i) * M + b];
                } else {
                    const int q = quad_map ? quad_map[i] : -1;
                    v = (q >= 0) ? X[size_t(3 * N + 5 * q + comp - 3) * M + (b - comp * M)] : make_double2(0, 0);
                }
                pv[c * bc + bb] = to_r<R>(v);
            }
            __syncthreads();
            // thread = one (x, y) column of the tile x one grid column bb,
            // all TZ z slots in registers: a contributor's moment and x-y
            // weight are read once for the whole z run
            for (int t = threadIdx.x; t < ncol * nb; t += blockDim.x) {
                const int bb = t % nb, col = t / nb;
                const int lx = col / TY, ly = col % TY;
                const int x = x0 + lx, y = y0 + ly;
                if (x >= g.Nx || y >= g.Ny) continue;
                const int nl = ln[col];
                cplx<R> acc[kSpreadZMax];
#pragma unroll
                for (int lz = 0; lz < kSpreadZMax; ++lz) acc[lz] = mk<R>(0, 0);
                if (nl >= 0) {
                    const R* lwc = lw + col * kSpreadListCap;
                    const int* lcc = lc + col * kSpreadListCap;
                    for (int k = 0; k < nl; ++k) {
                        const int c = lcc[k];
                        const R wxy = lwc[k];
                        const cplx<R> pc = pv[c * bc + bb];
                        const R* wz = wT + c * wlen + TX + TY;
#pragma unroll
                        for (int lz = 0; lz < kSpreadZMax; ++lz)
                            if (lz < TZ) fma_rc(acc[lz], wxy * wz[lz], pc);
                    }
                } else {
                    for (int c = 0; c < nc; ++c) {
                        const R* wc = wT + c * wlen;
                        const R wxy = wc[lx] * wc[TX + ly];
                        const cplx<R> pc = pv[c * bc + bb];
#pragma unroll
                        for (int lz = 0; lz < kSpreadZMax; ++lz)
                            if (lz < TZ) fma_rc(acc[lz], wxy * wc[TX + TY + lz], pc);
                    }
                }
                const size_t o0 = ((size_t(x) * g.Ny + y) * g.Zs + z0) * B + b0 + bb;
#pragma unroll
                for (int lz = 0; lz < kSpreadZMax; ++lz) {
                    if (lz >= TZ || z0 + lz >= g.Zs) break;
                    const size_t o = o0 + size_t(lz) * B;
                    if (r0 == 0) grid[o] = acc[lz];
                    else grid[o] += acc[lz];
                }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Spread plan, built once per frame (positions are fixed during a solve).
// For every tile: the candidate particles whose stencil reaches it (in bin
// order, the order k_spread uses), their 1-D weights restricted to the tile,
// and every (x, y) column's contributor list, so that a spread launch only
// loads moments and accumulates.  pass 0 counts each tile's candidates (and
// the largest count); pass 1 writes the plan at capT entries per tile.
constexpr int kPlanCandMax = 256;   // candidates of one tile the plan kernel can hold

__global__ void __launch_bounds__(256) k_spread_plan(const int4* __restrict__ base, const double* __restrict__ w1,
                                                     const int* __restrict__ bin_start,
                                                     const int* __restrict__ bin_end,
                                                     const int* __restrict__ sorted_idx, GridView g, int TX, int TY,
                                                     int TZ, int nbx, int nby, int pass, int capT,
                                                     int* __restrict__ ncT, int* __restrict__ maxc,
                                                     int* __restrict__ overflow, int* __restrict__ cidT,
                                                     double* __restrict__ w64T, float* __restrict__ w32T,
                                                     double* __restrict__ lw64, float* __restrict__ lw32,
                                                     int* __restrict__ lcT, int* __restrict__ lnT) {
    __shared__ int bx[8], by[8], bz[8], nbxs, nbys, nbzs;
    __shared__ int rstart[512], rlen[512], rpre[513], nranges;
    __shared__ int cand[kPlanCandMax];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* wloc = reinterpret_cast<double*>(smem_raw);   // [kPlanCandMax][wlen]
    const int tile = blockIdx.x;
    const int tx = tile % nbx, ty = (tile / nbx) % nby, zt = tile / (nbx * nby);
    const int x0 = tx * TX, y0 = ty * TY, z0 = zt * TZ;
    const int x1 = min(x0 + TX, g.Nx), y1 = min(y0 + TY, g.Ny), z1 = min(z0 + TZ, g.Zs);
    if (threadIdx.x == 0) {
        nbxs = reach_bins(x0 - g.off, x1 - 1 + g.off, g.Nx, TX, true, bx);
        nbys = reach_bins(y0 - g.off, y1 - 1 + g.off, g.Ny, TY, true, by);
        nbzs = reach_bins(z0 - g.off, z1 - 1 + g.off, g.Zs, TZ, !g.pruned, bz);
        int k = 0;
        rpre[0] = 0;
        for (int a = 0; a < nbzs; ++a)
            for (int b2 = 0; b2 < nbys; ++b2)
                for (int c = 0; c < nbxs; ++c) {
                    const int key = (bz[a] * nby + by[b2]) * nbx + bx[c];
                    const int s0 = bin_start[key];
                    if (s0 < 0 || k >= 512) continue;
                    rstart[k] = s0;
                    rlen[k] = bin_end[key] - s0;
                    rpre[k + 1] = rpre[k] + rlen[k];
                    ++k;
                }
        nranges = k;
    }
    __syncthreads();
    const int total = rpre[nranges];
    if (total > kPlanCandMax) {
        if (threadIdx.x == 0) atomicOr(overflow, 1);
        return;
    }
    const int wlen = TX + TY + TZ;
    const int ncol = TX * TY;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int k = 0;
        while (rpre[k + 1] <= t) ++k;
        cand[t] = sorted_idx[rstart[k] + t - rpre[k]];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < total * wlen; t += blockDim.x) {
        const int c = t / wlen, l = t % wlen;
        const int i = cand[c];
        const int4 bs = base[i];
        double w = 0.0;
        if (l < TX) {
            const int x = x0 + l;
            if (x < g.Nx) {
                const int d = cyc_diff(x, bs.x, g.Nx);
                if (d >= -g.off && d <= g.off) w = w1[(size_t(i) * 3 + 0) * g.S + d + g.off];
            }
        } else if (l < TX + TY) {
            const int y = y0 + l - TX;
            if (y < g.Ny) {
                const int d = cyc_diff(y, bs.y, g.Ny);
                if (d >= -g.off && d <= g.off) w = w1[(size_t(i) * 3 + 1) * g.S + d + g.off];
            }
        } else {
            const int s = z0 + l - TX - TY;
            if (s < g.Zs) {
                const int d = g.pruned ? (s - bs.z) : cyc_diff(s, bs.z, g.Nz);
                if (d >= -g.off && d <= g.off) w = w1[(size_t(i) * 3 + 2) * g.S + d + g.off];
            }
        }
        wloc[c * wlen + l] = w;
    }
    __syncthreads();
    if (pass == 0) {
        if (threadIdx.x == 0) {
            ncT[tile] = total;
            atomicMax(maxc, total);
        }
        return;
    }
    const size_t trow = size_t(tile) * capT;
    for (int t = threadIdx.x; t < total; t += blockDim.x) cidT[trow + t] = cand[t];
    for (int t = threadIdx.x; t < total * wlen; t += blockDim.x) {
        w64T[trow * wlen + t] = wloc[t];
        w32T[trow * wlen + t] = static_cast<float>(wloc[t]);
    }
    // contributor list per (x, y) column in candidate order, -1 = too many.
    // A one-slot tile (TZ = Zs = 1) stores the x-y weight times the
    // candidate's z weight, the factor its spread kernel applies.
    const bool premul = TZ == 1 && g.Zs == 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int col = warp; col < ncol; col += nwarp) {
        const int lx = col / TY, ly = col % TY;
        const size_t lrow = (size_t(tile) * ncol + col) * kSpreadListCap;
        int n = 0;
        for (int cb = 0; cb < total; cb += 32) {
            const int c = cb + lane;
            const double wxy = c < total ? wloc[c * wlen + lx] * wloc[c * wlen + TX + ly] : 0.0;
            // the fp32 kernel multiplies the fp32 weights
            const float wxy32 = c < total ? static_cast<float>(wloc[c * wlen + lx]) *
                                                static_cast<float>(wloc[c * wlen + TX + ly])
                                          : 0.f;
            const unsigned hit = __ballot_sync(0xffffffffu, wxy != 0.0);
            const int at = n + __popc(hit & ((1u << lane) - 1u));
            if (wxy != 0.0 && at < kSpreadListCap) {
                const double wz = premul ? wloc[c * wlen + TX + TY] : 1.0;
                lw64[lrow + at] = premul ? wxy * wz : wxy;
                lw32[lrow + at] = premul ? wxy32 * static_cast<float>(wz) : wxy32;
                lcT[lrow + at] = c;
            }
            n += __popc(hit);
        }
        if (lane == 0) lnT[size_t(tile) * ncol + col] = n <= kSpreadListCap ? n : -1;
    }
}

// Spread with the per-frame plan: CTA = one tile x one chunk of bc grid
// columns; loads the tile's candidate moments, then thread = one (x, y)
// column x one grid column with the whole z run in registers.  The same
// contributors in the same order as k_spread.
template <typename R, int ZMAX>
__global__ void __launch_bounds__(256) k_spread_planned(const double2* __restrict__ X, int M, int N, int C,
                                                        const int* __restrict__ quad_map, GridView g, int TX,
                                                        int TY, int TZ, int nbx, int nby, int nzt, int capT, int bc,
                                                        const int* __restrict__ ncT, const int* __restrict__ cidT,
                                                        const R* __restrict__ wT, const R* __restrict__ lwT,
                                                        const int* __restrict__ lcT, const int* __restrict__ lnT,
                                                        cplx<R>* __restrict__ grid) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R>* pv = reinterpret_cast<cplx<R>*>(smem_raw);   // [capT][bc]
    const int zt = blockIdx.z % nzt, chunk = blockIdx.z / nzt;
    const int tile = (zt * nby + blockIdx.y) * nbx + blockIdx.x;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = zt * TZ;
    const int B = C * M;
    const int wlen = TX + TY + TZ;
    const int ncol = TX * TY;
    const int nc = ncT[tile];
    const size_t trow = size_t(tile) * capT;
    const int b0 = chunk * bc;
    const int nb = min(bc, B - b0);
    for (int t = threadIdx.x; t < nc * nb; t += blockDim.x) {
        const int c = t / nb, bb = t % nb;
        const int i = cidT[trow + c];
        const int b = b0 + bb;
        const int comp = b / M;
        double2 v;
        if (comp < 3) {
            v = X[size_t(3 * i) * M + b];
        } else {
            const int q = quad_map ? quad_map[i] : -1;
            v = (q >= 0) ? X[size_t(3 * N + 5 * q + comp - 3) * M + (b - comp * M)] : make_double2(0, 0);
        }
        pv[c * bc + bb] = to_r<R>(v);
    }
    __syncthreads();
    const R* wTt = wT + trow * wlen;
    for (int t = threadIdx.x; t < ncol * nb; t += blockDim.x) {
        const int bb = t % nb, col = t / nb;
        const int lx = col / TY, ly = col % TY;
        const int x = x0 + lx, y = y0 + ly;
        if (x >= g.Nx || y >= g.Ny) continue;
        const int nl = lnT[size_t(tile) * ncol + col];
        cplx<R> acc[ZMAX];
#pragma unroll
        for (int lz = 0; lz < ZMAX; ++lz) acc[lz] = mk<R>(0, 0);
        if (nl >= 0) {
            const size_t lrow = (size_t(tile) * ncol + col) * kSpreadListCap;
            for (int k = 0; k < nl; ++k) {
                const int c = lcT[lrow + k];
                const R wxy = lwT[lrow + k];
                const cplx<R> pc = pv[c * bc + bb];
                const R* wz = wTt + c * wlen + TX + TY;
#pragma unroll
                for (int lz = 0; lz < ZMAX; ++lz)
                    if (lz < TZ) fma_rc(acc[lz], wxy * wz[lz], pc);
            }
        } else {
            for (int c = 0; c < nc; ++c) {
                const R* wc = wTt + c * wlen;
                const R wxy = wc[lx] * wc[TX + ly];
                const cplx<R> pc = pv[c * bc + bb];
#pragma unroll
                for (int lz = 0; lz < ZMAX; ++lz)
                    if (lz < TZ) fma_rc(acc[lz], wxy * wc[TX + TY + lz], pc);
            }
        }
        const size_t o0 = ((size_t(x) * g.Ny + y) * g.Zs + z0) * B + b0 + bb;
#pragma unroll
        for (int lz = 0; lz < ZMAX; ++lz) {
            if (lz >= TZ || z0 + lz >= g.Zs) break;
            grid[o0 + size_t(lz) * B] = acc[lz];
        }
    }
}

// Spread with the per-frame plan for one-slot tiles (a single layer): the
// tile's candidate moments and every (x, y) column's contributor list
// (candidate, x-y weight times the candidate's z weight, premultiplied by
// the plan) are staged in shared memory first, a warp's loads for eight
// columns in flight together; then a group of gsz lanes per column (gsz =
// the chunk's grid columns rounded up to a power of two, at most 32), lanes
// over those grid columns, walks the list by broadcast reads: a
// contribution costs three shared loads and an FMA, and a group's stores are
// one contiguous row.  Same contributors in the same order as
// k_spread_planned.
template <typename R>
__global__ void __launch_bounds__(256) k_spread_planned_1z(const double2* __restrict__ X, int M, int N, int C,
                                                           const int* __restrict__ quad_map, GridView g, int TX,
                                                           int TY, int nbx, int nby, int capT, int bc,
                                                           const int* __restrict__ ncT, const int* __restrict__ cidT,
                                                           const R* __restrict__ wT, const R* __restrict__ lwT,
                                                           const int* __restrict__ lcT, const int* __restrict__ lnT,
                                                           cplx<R>* __restrict__ grid) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ncol = TX * TY;
    cplx<R>* pv = reinterpret_cast<cplx<R>*>(smem_raw);             // [capT][bc]
    R* lwS = reinterpret_cast<R*>(pv + size_t(capT) * bc);           // [ncol][kSpreadListCap]
    int* lcS = reinterpret_cast<int*>(lwS + size_t(ncol) * kSpreadListCap);
    int* lnS = lcS + size_t(ncol) * kSpreadListCap;                   // [ncol]
    const int chunk = blockIdx.z;
    const int tile = blockIdx.y * nbx + blockIdx.x;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int B = C * M;
    const int wlen = TX + TY + 1;
    const int nc = ncT[tile];
    const size_t trow = size_t(tile) * capT;
    const int b0 = chunk * bc;
    const int nb = min(bc, B - b0);
    const R* wTt = wT + trow * wlen;
    for (int t = threadIdx.x; t < nc * nb; t += blockDim.x) {
        const int c = t / nb, bb = t % nb;
        const int i = cidT[trow + c];
        const int b = b0 + bb;
        const int comp = b / M;
        double2 v;
        if (comp < 3) {
            v = X[size_t(3 * i) * M + b];
        } else {
            const int q = quad_map ? quad_map[i] : -1;
            v = (q >= 0) ? X[size_t(3 * N + 5 * q + comp - 3) * M + (b - comp * M)] : make_double2(0, 0);
        }
        pv[c * bc + bb] = to_r<R>(v);
    }
    for (int t = threadIdx.x; t < ncol; t += blockDim.x) lnS[t] = lnT[size_t(tile) * ncol + t];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    constexpr int kCPW = 8;   // columns whose list loads a warp issues together
    for (int col0 = warp; col0 < ncol; col0 += nwarp * kCPW) {
        for (int k0 = 0; k0 < kSpreadListCap; k0 += 32) {
            int cc[kCPW];
            R ww[kCPW];
#pragma unroll
            for (int u = 0; u < kCPW; ++u) {
                const int col = col0 + u * nwarp, k = k0 + lane;
                cc[u] = -1;
                if (col < ncol && k < lnS[col]) {
                    const size_t lrow = (size_t(tile) * ncol + col) * kSpreadListCap;
                    cc[u] = lcT[lrow + k];
                    ww[u] = lwT[lrow + k];
                }
            }
#pragma unroll
            for (int u = 0; u < kCPW; ++u) {
                if (cc[u] < 0) continue;
                const int col = col0 + u * nwarp, k = k0 + lane;
                lcS[col * kSpreadListCap + k] = cc[u];
                lwS[col * kSpreadListCap + k] = ww[u];
            }
        }
    }
    __syncthreads();
    const int gsz = nb > 16 ? 32 : nb > 8 ? 16 : nb > 4 ? 8 : 4;
    const int per = 32 / gsz, sub = lane / gsz, sl = lane % gsz;
    for (int col0 = warp * per; col0 < ncol; col0 += nwarp * per) {
        const int col = col0 + sub;
        if (col >= ncol) continue;
        const int lx = col / TY, ly = col % TY;
        const int x = x0 + lx, y = y0 + ly;
        if (x >= g.Nx || y >= g.Ny) continue;
        const int nl = lnS[col];
        const int* lc = lcS + col * kSpreadListCap;
        const R* lw = lwS + col * kSpreadListCap;
        for (int bb = sl; bb < nb; bb += gsz) {
            cplx<R> acc = mk<R>(0, 0);
            if (nl >= 0) {
                for (int k = 0; k < nl; ++k) fma_rc(acc, lw[k], pv[lc[k] * bc + bb]);
            } else {   // list overflowed: every candidate, in order
                for (int c = 0; c < nc; ++c) {
                    const R* wc = wTt + c * wlen;
                    fma_rc(acc, (wc[lx] * wc[TX + ly]) * wc[TX + TY], pv[c * bc + bb]);
                }
            }
            grid[(size_t(x) * g.Ny + y) * B + b0 + bb] = acc;
        }
    }
}

// Full layout: k-space Green tensor, dipoles only (scale_kernel,
// monodisperse_ewald_electric_field.cu:1406-1432) or joint dipole/quadrupole
// (scale_kernel_joint, :1434-1486).  One thread per (voxel, rhs).
template <typename R>
__device__ __forceinline__ void khat_at(int ix, int iy, int iz, int Nx, int Ny, int Nz, double Lx, double Ly,
                                        double Lz, R& kx, R& ky, R& kz, double bx = 0.0, double by = 0.0) {
    const double fx = (ix <= (Nx - 1) / 2) ? ix : ix - Nx;
    const double fy = (iy <= (Ny - 1) / 2) ? iy : iy - Ny;
    const double fz = (iz <= (Nz - 1) / 2) ? iz : iz - Nz;
    // Bloch wavevector (bx, by): the direction of k - b
    // (monodisperse_ewald_electric_field.cu:1329-1331)
    const double ax = fx * 2.0 * kPi / Lx - bx, ay = fy * 2.0 * kPi / Ly - by, az = fz * 2.0 * kPi / Lz;
    const double km = sqrt(ax * ax + ay * ay + az * az);
    if (km < 1e-12) { kx = ky = kz = R(0); return; }
    kx = R(ax / km); ky = R(ay / km); kz = R(az / km);
}

template <typename R, bool QUADS>
__global__ void k_scale(cplx<R>* __restrict__ grid, const R* __restrict__ sc, int Nx, int Ny, int Nz, double Lx,
                        double Ly, double Lz, int M, double bx, double by) {
    const size_t V = size_t(Nx) * Ny * Nz;
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= V * M) return;
    const size_t v = t / M;
    const int m = int(t % M);
    const int iz = int(v % Nz), iy = int((v / Nz) % Ny), ix = int(v / (size_t(Nz) * Ny));
    R kx, ky, kz;
    khat_at<R>(ix, iy, iz, Nx, Ny, Nz, Lx, Ly, Lz, kx, ky, kz, bx, by);
    constexpr int C = QUADS ? 8 : 3;
    cplx<R>* f = grid + v * (size_t(C) * M) + m;
    const cplx<R> f0 = f[0], f1 = f[size_t(M)], f2 = f[size_t(2) * M];
    cplx<R> dot = f0 * kx + f1 * ky + f2 * kz;
    if (!QUADS) {
        const R s = sc[v];
        const cplx<R> e = dot * s;
        f[0] = e * kx; f[size_t(M)] = e * ky; f[size_t(2) * M] = e * kz;
    } else {
        const R s = sc[4 * v + 0], sQ = sc[4 * v + 1], sGP = sc[4 * v + 2], sGQ = sc[4 * v + 3];
        const R qd[5] = {kx * kx - kz * kz, R(2) * kx * ky, R(2) * kx * kz, ky * ky - kz * kz, R(2) * ky * kz};
        const R third = R(1) / R(3);
        const R qf[5] = {kx * kx - third, kx * ky, kx * kz, ky * ky - third, ky * kz};
        cplx<R> gdot = mk<R>(0, 0);
        for (int c = 0; c < 5; ++c) gdot += f[size_t(3 + c) * M] * qd[c];
        // i*a*z = (-a z.y, a z.x)
        const cplx<R> eE = dot * s + mk<R>(-sQ * gdot.y, sQ * gdot.x);
        const cplx<R> gG = mk<R>(-sGP * dot.y, sGP * dot.x) + gdot * sGQ;
        f[0] = eE * kx; f[size_t(M)] = eE * ky; f[size_t(2) * M] = eE * kz;
        for (int c = 0; c < 5; ++c) f[size_t(3 + c) * M] = gG * qf[c];
    }
}

// Per-voxel scale coefficients (compute_scale_coefficients_kernel,
// monodisperse_ewald_electric_field.cu:1300-1404), float64.
// With a Bloch wavevector (bx, by): |k - b| in the Green function, the
// window deconvolution on the grid wavevector g itself
// (monodisperse_ewald_electric_field.cu:1329-1331).
__device__ void scale_coefs(int ix, int iy, int iz, int Nx, int Ny, int Nz, double Lx, double Ly, double Lz,
                            double xi, const double* eta, double V, double out[4], double bx = 0.0,
                            double by = 0.0) {
    const double fx = (ix <= (Nx - 1) / 2) ? ix : ix - Nx;
    const double fy = (iy <= (Ny - 1) / 2) ? iy : iy - Ny;
    const double fz = (iz <= (Nz - 1) / 2) ? iz : iz - Nz;
    const double gx = fx * 2.0 * kPi / Lx, gy = fy * 2.0 * kPi / Ly, gz = fz * 2.0 * kPi / Lz;
    const double qx = gx - bx, qy = gy - by;
    const double ks = qx * qx + qy * qy + gz * gz;
    const double km = sqrt(ks);
    if (km < 1e-12) { out[0] = out[1] = out[2] = out[3] = 0.0; return; }
    const double etaksq = ks - (gx * gx * eta[0] + gy * gy * eta[1] + gz * gz * eta[2]);
    const double term = sin(km) / km - cos(km);
    const double ex = exp(-etaksq / (4.0 * xi * xi));
    out[0] = (9.0 * term * term * ex / (ks * ks)) / V;
    const double j1 = term / km;
    const double j2 = (3.0 / ks - 1.0) * sin(km) / km - 3.0 * cos(km) / ks;
    const double e2 = ex / ks;
    out[1] = (-22.5 * j1 * j2 * e2) / V;
    out[2] = (45.0 * j1 * j2 * e2) / V;
    out[3] = (112.5 * j2 * j2 * e2) / V;
}

struct ScaleArgs {
    int Nx, Ny, Nz;
    double Lx, Ly, Lz, xi, eta[3];
    double bx = 0.0, by = 0.0;   // Bloch wavevector (full layout and column kernel)
};

__global__ void k_build_scale(ScaleArgs a, int quads, double* __restrict__ s64, float* __restrict__ s32) {
    const size_t V = size_t(a.Nx) * a.Ny * a.Nz;
    const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const int iz = int(v % a.Nz), iy = int((v / a.Nz) % a.Ny), ix = int(v / (size_t(a.Nz) * a.Ny));
    double o[4];
    scale_coefs(ix, iy, iz, a.Nx, a.Ny, a.Nz, a.Lx, a.Ly, a.Lz, a.xi, a.eta, double(V), o, a.bx, a.by);
    if (quads) {
        for (int c = 0; c < 4; ++c) { s64[4 * v + c] = o[c]; s32[4 * v + c] = float(o[c]); }
    } else {
        s64[v] = o[0];
        s32[v] = float(o[0]);
    }
}

// Pruned layout: Toeplitz kernel over the occupied planes for each (kx, ky)
// column, K_ab(d) = sum_kz exp(+2 pi i kz d / Nz) S(k) khat_a khat_b for the
// six symmetric ab pairs and d in [-(Z-1), Z-1]; for a single layer
// (Z = 1, w2 given) the z-weighted K_ab = sum_kz |W(kz)|^2 S khat_a khat_b.
// Computed in float64.
__global__ void k_build_column(ScaleArgs a, int Z, const double* __restrict__ w2, double2* __restrict__ K64,
                               float2* __restrict__ K32) {
    extern __shared__ double sh[];
    const int col = blockIdx.x;
    const int ix = col / a.Ny, iy = col % a.Ny;
    const int Nz = a.Nz;
    double* C6 = sh;                 // [Nz][6]
    double* tw = sh + 6 * Nz;        // [Nz][2] twiddles
    const double V = double(a.Nx) * a.Ny * a.Nz;
    for (int iz = threadIdx.x; iz < Nz; iz += blockDim.x) {
        double o[4];
        scale_coefs(ix, iy, iz, a.Nx, a.Ny, Nz, a.Lx, a.Ly, a.Lz, a.xi, a.eta, V, o, a.bx, a.by);
        double kx, ky, kz;
        khat_at<double>(ix, iy, iz, a.Nx, a.Ny, Nz, a.Lx, a.Ly, a.Lz, kx, ky, kz, a.bx, a.by);
        // single layer (Z = 1): weighted by |sum_o w_o exp(-2 pi i kz o / Nz)|^2
        const double s = w2 ? o[0] * w2[iz] : o[0];
        C6[iz * 6 + 0] = s * kx * kx; C6[iz * 6 + 1] = s * kx * ky; C6[iz * 6 + 2] = s * kx * kz;
        C6[iz * 6 + 3] = s * ky * ky; C6[iz * 6 + 4] = s * ky * kz; C6[iz * 6 + 5] = s * kz * kz;
        double sn, cs;
        sincospi(2.0 * iz / Nz, &sn, &cs);
        tw[2 * iz] = cs; tw[2 * iz + 1] = sn;
    }
    __syncthreads();
    const int nd = 2 * Z - 1;
    for (int t = threadIdx.x; t < 6 * nd; t += blockDim.x) {
        const int ab = t / nd, di = t % nd;
        const int d = di - (Z - 1);
        double re = 0.0, im = 0.0;
        for (int iz = 0; iz < Nz; ++iz) {
            const int k = pmod(iz * d, Nz);
            const double c = C6[iz * 6 + ab];
            re += c * tw[2 * k];
            im += c * tw[2 * k + 1];
        }
        const size_t o = (size_t(col) * 6 + ab) * nd + di;
        K64[o] = make_double2(re, im);
        K32[o] = make_float2(float(re), float(im));
    }
}

// Pruned layout, fused path: the three scalar Toeplitz kernels of each
// (kx, ky) column, t_n(d) = sum_kz exp(+2 pi i kz d / Nz) kz^n S(k) / |k|^2
// (kz the signed wavenumber, zero at k = 0), d in [-(Z-1), Z-1], so that
// K_ab(d) above is kx^2 t0, kx ky t0, kx t1, ky^2 t0, ky t1, t2 for
// ab = xx, xy, xz, yy, yz, zz.  Computed in float64.
__global__ void k_build_slab_taps(ScaleArgs a, int Z, double2* __restrict__ T64, float2* __restrict__ T32) {
    extern __shared__ double sh[];
    const int col = blockIdx.x;
    const int ix = col / a.Ny, iy = col % a.Ny;
    const int Nz = a.Nz;
    double* C3 = sh;                 // [Nz][3]: S/|k|^2 times kz^0, kz^1, kz^2
    double* tw = sh + 3 * Nz;        // [Nz][2] twiddles
    const double V = double(a.Nx) * a.Ny * a.Nz;
    for (int iz = threadIdx.x; iz < Nz; iz += blockDim.x) {
        double o[4];
        scale_coefs(ix, iy, iz, a.Nx, a.Ny, Nz, a.Lx, a.Ly, a.Lz, a.xi, a.eta, V, o);
        const double fx = (ix <= (a.Nx - 1) / 2) ? ix : ix - a.Nx;
        const double fy = (iy <= (a.Ny - 1) / 2) ? iy : iy - a.Ny;
        const double fz = (iz <= (Nz - 1) / 2) ? iz : iz - Nz;
        const double gx = fx * 2.0 * kPi / a.Lx, gy = fy * 2.0 * kPi / a.Ly, gz = fz * 2.0 * kPi / a.Lz;
        const double k2 = gx * gx + gy * gy + gz * gz;
        const double t = k2 < 1e-24 ? 0.0 : o[0] / k2;
        C3[iz * 3 + 0] = t;
        C3[iz * 3 + 1] = t * gz;
        C3[iz * 3 + 2] = t * gz * gz;
        double sn, cs;
        sincospi(2.0 * iz / Nz, &sn, &cs);
        tw[2 * iz] = cs; tw[2 * iz + 1] = sn;
    }
    __syncthreads();
    const int nd = 2 * Z - 1;
    for (int t = threadIdx.x; t < 3 * nd; t += blockDim.x) {
        const int k = t / nd, di = t % nd;
        const int d = di - (Z - 1);
        double re = 0.0, im = 0.0;
        for (int iz = 0; iz < Nz; ++iz) {
            const int e = pmod(iz * d, Nz);
            const double c = C3[iz * 3 + k];
            re += c * tw[2 * e];
            im += c * tw[2 * e + 1];
        }
        const size_t o = (size_t(col) * 3 + k) * nd + di;
        T64[o] = make_double2(re, im);
        T32[o] = make_float2(float(re), float(im));
    }
}

// Single layer: the taps of one z slot, tau_n = sum_{o,o'} w_o w_o' t_n(o - o')
// = sum_kz kz^n S(k) / |k|^2 |sum_o w_o exp(-2 pi i kz o / Nz)|^2 (real), with
// the layer's common z weights w_o; w2[kz] holds the squared modulus.
// Stored as the taps of a one-slot slab ([col][3][1]).  Float64, one thread
// per column, kz summed in order.
__global__ void k_layer_w2(const double* __restrict__ w, int S, int Nz, double* __restrict__ w2) {
    const int iz = blockIdx.x * blockDim.x + threadIdx.x;
    if (iz >= Nz) return;
    double re = 0.0, im = 0.0;
    for (int o = 0; o < S; ++o) {
        double sn, cs;
        sincospi(2.0 * double((long long)iz * o % Nz) / Nz, &sn, &cs);
        re += w[o] * cs;
        im -= w[o] * sn;
    }
    w2[iz] = re * re + im * im;
}

__global__ void k_build_layer_taps(ScaleArgs a, const double* __restrict__ w2, double2* __restrict__ T64,
                                   float2* __restrict__ T32) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= a.Nx * a.Ny) return;
    const int ix = col / a.Ny, iy = col % a.Ny;
    const int Nz = a.Nz;
    const double V = double(a.Nx) * a.Ny * a.Nz;
    const double fx = (ix <= (a.Nx - 1) / 2) ? ix : ix - a.Nx;
    const double fy = (iy <= (a.Ny - 1) / 2) ? iy : iy - a.Ny;
    const double gx = fx * 2.0 * kPi / a.Lx, gy = fy * 2.0 * kPi / a.Ly;
    double t0 = 0.0, t1 = 0.0, t2 = 0.0;
    for (int iz = 0; iz < Nz; ++iz) {
        double o[4];
        scale_coefs(ix, iy, iz, a.Nx, a.Ny, Nz, a.Lx, a.Ly, a.Lz, a.xi, a.eta, V, o);
        const double fz = (iz <= (Nz - 1) / 2) ? iz : iz - Nz;
        const double gz = fz * 2.0 * kPi / a.Lz;
        const double k2 = gx * gx + gy * gy + gz * gz;
        const double t = k2 < 1e-24 ? 0.0 : o[0] / k2 * w2[iz];
        t0 += t;
        t1 += t * gz;
        t2 += t * gz * gz;
    }
    const double tv[3] = {t0, t1, t2};
    for (int k = 0; k < 3; ++k) {
        T64[size_t(col) * 3 + k] = make_double2(tv[k], 0.0);
        T32[size_t(col) * 3 + k] = make_float2(float(tv[k]), 0.f);
    }
}

// Pruned layout: out[zo][c'][m] = sum_{zi,c} K_{c'c}(zo - zi) in[zi][c][m]
// on one (kx, ky) column per CTA, in place.  The column's Z x 3 inputs of a
// right-hand side sit in registers; for each source component c the 2Z-1
// Toeplitz coefficients K_{c'c}(.) are read once from shared memory and
// applied to all Z outputs (ZMAX bounds Z at compile time).
template <typename R, int ZMAX>
__global__ void k_column(cplx<R>* __restrict__ grid, const cplx<R>* __restrict__ K, int Z, int M) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int col = blockIdx.x;
    const int B = 3 * M;
    const int nd = 2 * Z - 1;
    cplx<R>* in = reinterpret_cast<cplx<R>*>(smem_raw);   // [Z][B]
    cplx<R>* kk = in + size_t(Z) * B;                       // [6][nd]
    cplx<R>* g = grid + size_t(col) * Z * B;
    for (int t = threadIdx.x; t < Z * B; t += blockDim.x) in[t] = g[t];
    for (int t = threadIdx.x; t < 6 * nd; t += blockDim.x) kk[t] = K[size_t(col) * 6 * nd + t];
    __syncthreads();
    const int pairidx[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    for (int t = threadIdx.x; t < B; t += blockDim.x) {
        const int cp = t / M, m = t % M;
        cplx<R> acc[ZMAX];
#pragma unroll
        for (int zo = 0; zo < ZMAX; ++zo) acc[zo] = mk<R>(0, 0);
        for (int c = 0; c < 3; ++c) {
            cplx<R> x[ZMAX];
#pragma unroll
            for (int zi = 0; zi < ZMAX; ++zi) x[zi] = zi < Z ? in[zi * B + c * M + m] : mk<R>(0, 0);
            const cplx<R>* kab = kk + pairidx[cp][c] * nd + (Z - 1);   // kab[d], d = zo - zi in [-(Z-1), Z-1]
#pragma unroll
            for (int d = -(ZMAX - 1); d <= ZMAX - 1; ++d) {
                if (d < -(Z - 1) || d > Z - 1) continue;
                const cplx<R> kv = kab[d];
#pragma unroll
                for (int zo = 0; zo < ZMAX; ++zo) {
                    const int zi = zo - d;
                    if (zi >= 0 && zi < ZMAX) {
                        // acc += kv * x, four FMAs
                        acc[zo].x = fma(kv.x, x[zi].x, acc[zo].x);
                        acc[zo].x = fma(-kv.y, x[zi].y, acc[zo].x);
                        acc[zo].y = fma(kv.x, x[zi].y, acc[zo].y);
                        acc[zo].y = fma(kv.y, x[zi].x, acc[zo].y);
                    }
                }
            }
        }
        for (int zo = 0; zo < Z; ++zo) g[zo * B + t] = acc[zo];
    }
}

// Contraction: field at each target from its Gaussian stencil for all B
// columns (contract_kernel, monodisperse_ewald_electric_field.cu:1488-1587).
// Writes Y rows (overwrites), or with `accumulate` adds to the dipole rows
// already in Y (the real-space part, computed concurrently) and, when jsc
// is given, scales the sum by the Jacobi factor 1/s of the target and
// column.  C = 3 (dipoles) or 8 (plus field gradient).  SZ > 0: the
// stencil's z run (g.Sz <= SZ) unrolled, so that its grid loads are in
// flight together; SZ = 0: any stencil length.  SXY > 0: the stencil width
// g.S == SXY at compile time, its y run unrolled as well.  Grid offsets of
// the stencil's x and y indices are precomputed once per target.
template <typename R, int SZ, int SXY>
__global__ void k_contract(const cplx<R>* __restrict__ grid, GridView g, int M, int C, int Nt,
                           const int4* __restrict__ base, const R* __restrict__ w1, double factor,
                           const int* __restrict__ quad_map, double2* __restrict__ Y, int negate,
                           const int* __restrict__ order, int accumulate, const double2* __restrict__ jsc) {
    __shared__ R w[3 * kMaxStencil];
    __shared__ int idx[3 * kMaxStencil];
    __shared__ long long offxy[2 * kMaxStencil];   // x then y stencil offsets into the grid (elements)
    // targets in spatial-bin order when given: CTAs that run together share
    // their stencils' voxels in L2
    const int j = order ? order[blockIdx.x] : blockIdx.x;
    const int B = C * M;
    const int4 bs = base[j];
    for (int t = threadIdx.x; t < 3 * g.S; t += blockDim.x) {
        const int d = t / g.S, o = t % g.S;
        w[t] = w1[(size_t(j) * 3 + d) * g.S + o];
        const int dd = o - g.off;
        idx[t] = (d == 0) ? pmod(bs.x + dd, g.Nx) : (d == 1) ? pmod(bs.y + dd, g.Ny)
                 : (g.pruned ? bs.z + dd : pmod(bs.z + dd, g.Nz));
        if (d == 0) offxy[o] = (long long)idx[t] * g.Ny * g.Zs * B;
        else if (d == 1) offxy[g.S + o] = (long long)idx[t] * g.Zs * B;
    }
    __syncthreads();
    // the z window on the stored grid: entries zb .. zb + Sz - 1 of the z
    // stencil (all of it, or the single layer's centre)
    const int zb = 2 * g.S + g.off - g.offz;
    const int q = (C > 3 && quad_map) ? quad_map[j] : -1;
    for (int b = threadIdx.x; b < B; b += blockDim.x) {
        const int comp = b / M;
        if (comp >= 3 && q < 0) continue;
        cplx<R> acc = mk<R>(0, 0);
        // the z weights and z offsets are the same for every (x, y) of the
        // stencil: keep them in registers
        R wz[SZ > 0 ? SZ : 1];
        int zo[SZ > 0 ? SZ : 1];   // < Zs * B
        if constexpr (SZ > 0) {
#pragma unroll
            for (int oz = 0; oz < SZ; ++oz) {
                wz[oz] = oz < g.Sz ? w[zb + oz] : R(0);
                zo[oz] = oz < g.Sz ? idx[zb + oz] * B + b : b;
            }
        }
        const int S = SXY > 0 ? SXY : g.S;
        // one stencil column (x, y): its z run from gp (the grid at (x, y), slot 0)
        auto column = [&](const cplx<R>* gp) {
            cplx<R> a2 = mk<R>(0, 0);
            if constexpr (SZ > 0) {
                cplx<R> v[SZ];
#pragma unroll
                for (int oz = 0; oz < SZ; ++oz)
                    if (oz < g.Sz) v[oz] = gp[zo[oz]];
#pragma unroll
                for (int oz = 0; oz < SZ; ++oz)
                    if (oz < g.Sz) fma_rc(a2, wz[oz], v[oz]);
            } else {
                for (int oz = 0; oz < g.Sz; ++oz) fma_rc(a2, w[zb + oz], gp[size_t(idx[zb + oz]) * B + b]);
            }
            return a2;
        };
        for (int ox = 0; ox < S; ++ox) {
            const R wx = w[ox];
            const cplx<R>* gx = grid + offxy[ox];
            if constexpr (SXY > 0) {
#pragma unroll
                for (int oy = 0; oy < SXY; ++oy) fma_rc(acc, wx * w[SXY + oy], column(gx + offxy[SXY + oy]));
            } else {
                for (int oy = 0; oy < S; ++oy) fma_rc(acc, wx * w[S + oy], column(gx + offxy[S + oy]));
            }
        }
        double2 v = to_d(acc);
        v.x *= factor; v.y *= factor;
        if (negate) { v.x = -v.x; v.y = -v.y; }
        const int m = b - comp * M;
        const size_t row = (comp < 3) ? size_t(3 * j + comp) : size_t(3 * Nt + 5 * q + comp - 3);
        if (accumulate && comp < 3) {
            v += Y[row * M + m];
            if (jsc) {
                const double2 sv = jsc[size_t(j) * M + m];
                const double den = sv.x * sv.x + sv.y * sv.y;
                if (den > 1e-30) v = v * make_double2(sv.x / den, -sv.y / den);
            }
        }
        Y[row * M + m] = v;
    }
}

// k_contract for one stored z slot (single layer) and few grid columns
// (B = 3M <= 16, dipoles only): a CTA holds 128 / gsz targets, gsz = B
// rounded up to a power of two lanes each, instead of one target per CTA
// with B of its 32 lanes busy.  Same arithmetic, in the same order, as
// k_contract<R, 1, SXY>.
constexpr int kContractSmallMaxT = 32;   // targets per CTA (gsz >= 4)

template <typename R, int SXY>
__global__ void __launch_bounds__(128) k_contract_small(const cplx<R>* __restrict__ grid, GridView g, int M, int Nt,
                                                        const int4* __restrict__ base, const R* __restrict__ w1,
                                                        double factor, double2* __restrict__ Y, int negate,
                                                        const int* __restrict__ order, int accumulate,
                                                        const double2* __restrict__ jsc, int gsz) {
    __shared__ R wxy[kContractSmallMaxT][2 * kMaxStencil];
    __shared__ long long offxy[kContractSmallMaxT][2 * kMaxStencil];
    __shared__ R wzs[kContractSmallMaxT];
    __shared__ int zos[kContractSmallMaxT];
    const int B = 3 * M;
    const int per = blockDim.x / gsz;
    const int slot = threadIdx.x / gsz, sl = threadIdx.x % gsz;
    const int jj = blockIdx.x * per + slot;
    const bool live = jj < Nt;
    const int j = live ? (order ? order[jj] : jj) : 0;
    if (live) {
        const int4 bs = base[j];
        const int zc = g.off - g.offz;   // the stored slot's entry of the z stencil
        for (int t = sl; t < 2 * g.S + 1; t += gsz) {
            if (t < 2 * g.S) {
                const int d = t / g.S, o = t % g.S;
                wxy[slot][t] = w1[(size_t(j) * 3 + d) * g.S + o];
                const int dd = o - g.off;
                if (d == 0) offxy[slot][t] = (long long)pmod(bs.x + dd, g.Nx) * g.Ny * g.Zs * B;
                else offxy[slot][t] = (long long)pmod(bs.y + dd, g.Ny) * g.Zs * B;
            } else {
                wzs[slot] = w1[(size_t(j) * 3 + 2) * g.S + zc];
                const int dz = zc - g.off;
                zos[slot] = g.pruned ? bs.z + dz : pmod(bs.z + dz, g.Nz);
            }
        }
    }
    __syncthreads();
    if (!live) return;
    const int S = SXY > 0 ? SXY : g.S;
    const R* w = wxy[slot];
    const long long* off = offxy[slot];
    const R wz = wzs[slot];
    for (int b = sl; b < B; b += gsz) {
        const int comp = b / M;
        const int zo = zos[slot] * B + b;
        cplx<R> acc = mk<R>(0, 0);
        for (int ox = 0; ox < S; ++ox) {
            const R wx = w[ox];
            const cplx<R>* gx = grid + off[ox];
            auto cell = [&](int oy) {
                cplx<R> a2 = mk<R>(0, 0);
                fma_rc(a2, wz, gx[off[S + oy] + zo]);
                fma_rc(acc, wx * w[S + oy], a2);
            };
            if constexpr (SXY > 0) {
#pragma unroll
                for (int oy = 0; oy < SXY; ++oy) cell(oy);
            } else {
                for (int oy = 0; oy < S; ++oy) cell(oy);
            }
        }
        double2 v = to_d(acc);
        v.x *= factor; v.y *= factor;
        if (negate) { v.x = -v.x; v.y = -v.y; }
        const int m = b - comp * M;
        const size_t row = size_t(3 * j + comp);
        if (accumulate) {
            v += Y[row * M + m];
            if (jsc) {
                const double2 sv = jsc[size_t(j) * M + m];
                const double den = sv.x * sv.x + sv.y * sv.y;
                if (den > 1e-30) v = v * make_double2(sv.x / den, -sv.y / den);
            }
        }
        Y[row * M + m] = v;
    }
}

// ------------------------------------------------------------ neighbours

struct CellArgs {
    double L[3];
    double cs[3];
    int nc[3];
};

__device__ __forceinline__ int cell_of(double p, double L, double cs, int nc) {
    const double w = p - L * floor(p / L);
    int c = int(floor(w / cs));
    return min(max(c, 0), nc - 1);
}

__global__ void k_cell_keys(const double* __restrict__ xyz, int n, CellArgs a, int* __restrict__ key,
                            int* __restrict__ idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int cx = cell_of(xyz[i], a.L[0], a.cs[0], a.nc[0]);
    const int cy = cell_of(xyz[n + i], a.L[1], a.cs[1], a.nc[1]);
    const int cz = cell_of(xyz[2 * n + i], a.L[2], a.cs[2], a.nc[2]);
    key[i] = (cz * a.nc[1] + cy) * a.nc[0] + cx;
    idx[i] = i;
}

// For each target: sources within rc (minimum image, d^2 <= rc^2 and then
// d < rc as in neighbor_list.cu:186-223 + the pair kernels' cut), visiting
// the distinct neighbouring cells.  pass 0 counts, pass 1 writes pair data.
// Warp per target: the lanes take a cell's candidates 32 at a time, in
// order, and a ballot places the accepted ones, so the pairs of a target
// come out in cell-list order (the order a single thread walking the cells
// would give).  pass 0 counts, pass 1 writes at off[j].
__global__ void k_pairs(const double* __restrict__ src, int ns, const double* __restrict__ tgt, int nt, CellArgs a,
                        const int* __restrict__ cstart, const int* __restrict__ cend,
                        const int* __restrict__ sidx, double rc, int solver_ax, int pass,
                        int* __restrict__ cnt, const int* __restrict__ off, int* __restrict__ psrc,
                        double* __restrict__ pgeo /*[P][4]: dx,dy,dz,d*/) {
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= nt) return;   // whole warps leave together
    const double xj = tgt[j], yj = tgt[nt + j], zj = tgt[2 * nt + j];
    const int c[3] = {cell_of(xj, a.L[0], a.cs[0], a.nc[0]), cell_of(yj, a.L[1], a.cs[1], a.nc[1]),
                      cell_of(zj, a.L[2], a.cs[2], a.nc[2])};
    int lst[3][3], nl[3];
    for (int d = 0; d < 3; ++d) {
        nl[d] = 0;
        for (int o = -1; o <= 1; ++o) {
            const int v = pmod(c[d] + o, a.nc[d]);
            bool seen = false;
            for (int k = 0; k < nl[d]; ++k) seen |= lst[d][k] == v;
            if (!seen) lst[d][nl[d]++] = v;
        }
    }
    int count = 0;   // the same in every lane
    const int base = pass ? off[j] : 0;
    const double rc2 = rc * rc;
    for (int a2 = 0; a2 < nl[2]; ++a2)
        for (int a1 = 0; a1 < nl[1]; ++a1)
            for (int a0 = 0; a0 < nl[0]; ++a0) {
                const int key = (lst[2][a2] * a.nc[1] + lst[1][a1]) * a.nc[0] + lst[0][a0];
                const int s0 = cstart[key];
                if (s0 < 0) continue;
                const int s1 = cend[key];
                for (int k0 = s0; k0 < s1; k0 += 32) {
                    const int k = k0 + lane;
                    bool keep = false;
                    int i = 0;
                    double dx = 0, dy = 0, dz = 0, d = 0;
                    if (k < s1) {
                        i = sidx[k];
                        if (!(solver_ax && i == j)) {
                            dx = src[i] - xj;
                            dy = src[ns + i] - yj;
                            dz = src[2 * ns + i] - zj;
                            dx -= a.L[0] * round(dx / a.L[0]);
                            dy -= a.L[1] * round(dy / a.L[1]);
                            dz -= a.L[2] * round(dz / a.L[2]);
                            const double d2 = dx * dx + dy * dy + dz * dz;
                            if (d2 <= rc2) {
                                d = sqrt(d2);
                                keep = d < rc;
                            }
                        }
                    }
                    const unsigned hit = __ballot_sync(0xffffffffu, keep);
                    if (pass && keep) {
                        const int o = base + count + __popc(hit & ((1u << lane) - 1u));
                        psrc[o] = i;
                        pgeo[4 * size_t(o) + 0] = dx;
                        pgeo[4 * size_t(o) + 1] = dy;
                        pgeo[4 * size_t(o) + 2] = dz;
                        pgeo[4 * size_t(o) + 3] = d;
                    }
                    count += __popc(hit);
                }
            }
    if (!pass && lane == 0) cnt[j] = count;
}

__device__ double table_at(double r, const double* __restrict__ rt, const double* __restrict__ y) {
    constexpr int n = kTableSize;
    if (r <= 0.0) return y[0];
    if (r >= rt[n - 1]) return y[n - 1];
    if (r < 1.0) return y[0] * (1.0 - r) + y[1] * r;
    const size_t k = 1 + static_cast<size_t>((r - 1.0) / kTableDr);
    if (k >= size_t(n - 1)) return y[n - 1];
    const double t = (r - rt[k]) / (rt[k + 1] - rt[k]);
    return y[k] * (1.0 - t) + y[k + 1] * t;
}

// Pair coefficients (real_space_precalcs_kernel_joint,
// monodisperse_ewald_electric_field.cu:877-958): delta = r / max(d, 1) and
// the table values at max(d, 1).  Layout per pair: T64[8] = {dx,dy,dz,perp,
// para,0,0,0}; Q[8] = {Q1,Q2,Q3,G1,G2,G3,G4,0}.
__global__ void k_pair_coefs(const double* __restrict__ pgeo, long long np, const double* __restrict__ rt,
                             const double* __restrict__ tf, int quads, double* __restrict__ T64,
                             float* __restrict__ T32, double* __restrict__ Q) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const double d = pgeo[4 * p + 3];
    const double de = d < 1.0 ? 1.0 : d;
    const double dx = pgeo[4 * p + 0] / de, dy = pgeo[4 * p + 1] / de, dz = pgeo[4 * p + 2] / de;
    const double perp = table_at(de, rt, tf + T_FD1 * kTableSize);
    const double para = table_at(de, rt, tf + T_FD2 * kTableSize);
    double* t = T64 + 8 * p;
    t[0] = dx; t[1] = dy; t[2] = dz; t[3] = perp; t[4] = para; t[5] = t[6] = t[7] = 0.0;
    float* f = T32 + 8 * p;
    f[0] = float(dx); f[1] = float(dy); f[2] = float(dz); f[3] = float(perp); f[4] = float(para);
    f[5] = f[6] = f[7] = 0.f;
    if (quads) {
        double* qq = Q + 8 * p;
        for (int k = 0; k < 7; ++k) qq[k] = table_at(de, rt, tf + (T_FQ1 + k) * kTableSize);
        qq[7] = 0.0;
    }
}

// Bloch phase of every pair, exp(i phi) with phi = -(bx r_x + by r_y), r =
// source - target (minimum image) (monodisperse_ewald_electric_field.cu:
// 1749-1756).
__global__ void k_pair_phase(const double* __restrict__ pgeo, long long np, double bx, double by,
                             double2* __restrict__ P64, float2* __restrict__ P32) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    double sn, cs;
    sincos(-(bx * pgeo[4 * p + 0] + by * pgeo[4 * p + 1]), &sn, &cs);
    P64[p] = make_double2(cs, sn);
    P32[p] = make_float2(float(cs), float(sn));
}

// ------------------------------------------------------------ real space

// Gather by target (warp per target, lanes over right-hand sides) of the
// real-space pair sum, plus self term, optional Jacobi scaling and the
// INTERACTION_FIELD sign (monodisperse_ewald_electric_field.cu:1589-1869,
// 2395-2404).  If add_recip, Y already holds the reciprocal part.
struct RealArgs {
    int M, N, Nt, Nq;
    double selfo, self_grad;
    int solver_ax, jacobi, add_recip, quads;
    int pairs_plus;   // pairs enter with +1 in INTERACTION_FIELD too (polydisperse, :780-826)
    // polydisperse quadrupole self term 2.5 s / a^2 + 0.5 g(a) per target
    // (real_space_self_kernel_polydisperse_joint, :1148-1195); null: a = 1,
    // g = self_grad (monodisperse)
    const double* qa2;
    const double* qg2;
};

// Dipole pairs of one target, kPairBatch pairs at a time: the source
// indices, pair coefficients and moments of a batch are all loaded before
// any is used, so the pair loop waits on one memory latency per batch
// rather than two per pair.  Accumulation order is the pair order.
constexpr int kPairBatch = 4;

// pairs p0, p0 + stride, p0 + 2 stride, ... below p1 (stride 1: all of
// them in order)
// ph (may be null): the pairs' Bloch phases, each pair's term multiplied
// by its phase.
template <typename R>
__device__ __forceinline__ void real_dipole_pairs(const double2* __restrict__ X, int M, int m, int p0, int p1,
                                                  int stride, const int* __restrict__ src,
                                                  const R* __restrict__ T, const cplx<R>* __restrict__ ph,
                                                  cplx<R>& e0, cplx<R>& e1, cplx<R>& e2) {
    for (int p = p0; p < p1; p += kPairBatch * stride) {
        int ii[kPairBatch];
        R dx[kPairBatch], dy[kPairBatch], dz[kPairBatch], pe[kPairBatch], pa[kPairBatch];
        cplx<R> px[kPairBatch], py[kPairBatch], pz[kPairBatch], pf[kPairBatch];
#pragma unroll
        for (int u = 0; u < kPairBatch; ++u) ii[u] = (p + u * stride < p1) ? src[p + u * stride] : -1;
#pragma unroll
        for (int u = 0; u < kPairBatch; ++u) {
            if (ii[u] >= 0) {
                const R* t = T + 8 * size_t(p + u * stride);
                dx[u] = t[0]; dy[u] = t[1]; dz[u] = t[2]; pe[u] = t[3]; pa[u] = t[4];
                if (ph) pf[u] = ph[p + u * stride];
                const double2* xi = X + size_t(3 * ii[u]) * M + m;
                px[u] = to_r<R>(xi[0]);
                py[u] = to_r<R>(xi[size_t(M)]);
                pz[u] = to_r<R>(xi[size_t(2) * M]);
            }
        }
#pragma unroll
        for (int u = 0; u < kPairBatch; ++u) {
            if (ii[u] >= 0) {
                const cplx<R> rp = px[u] * dx[u] + py[u] * dy[u] + pz[u] * dz[u];
                const cplx<R> k = rp * (pa[u] - pe[u]);
                if (ph) {
                    e0 += (px[u] * pe[u] + k * dx[u]) * pf[u];
                    e1 += (py[u] * pe[u] + k * dy[u]) * pf[u];
                    e2 += (pz[u] * pe[u] + k * dz[u]) * pf[u];
                } else {
                    e0 += px[u] * pe[u] + k * dx[u];
                    e1 += py[u] * pe[u] + k * dy[u];
                    e2 += pz[u] * pe[u] + k * dz[u];
                }
            }
        }
    }
}

template <typename R, bool QUADS>
__global__ void __launch_bounds__(128) k_real(const double2* __restrict__ X, double2* __restrict__ Y, RealArgs a,
                                              const int* __restrict__ off, const int* __restrict__ src,
                                              const R* __restrict__ T, const double* __restrict__ Qt,
                                              const int* __restrict__ quad_map,
                                              const double2* __restrict__ sc, const double* __restrict__ selfv,
                                              const cplx<R>* __restrict__ ph) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= a.Nt) return;
    const int j = warp;
    const int p0 = off[j], p1 = off[j + 1];
    const int M = a.M;
    const double sign = (a.solver_ax || a.pairs_plus) ? 1.0 : -1.0;
    const double selfc = selfv ? selfv[j] : a.selfo;  // polydisperse: self value of the particle's radius class
    const int qt = (QUADS && quad_map && j < a.N) ? quad_map[j] : -1;
    // fewer than 32 columns (dipoles only): the warp splits into 32 / gsz
    // groups of gsz lanes (gsz = M rounded up to a power of two); group g
    // takes pairs p0 + g, p0 + g + 32/gsz, ... and the groups' sums meet in a
    // fixed shuffle tree
    const int gsz = (!QUADS && M < 32) ? (M <= 1 ? 1 : M <= 2 ? 2 : M <= 4 ? 4 : M <= 8 ? 8 : 16) : 32;
    const int ng = 32 / gsz, grp = lane / gsz;
    for (int m0 = 0; m0 < M; m0 += gsz) {
        const int m = m0 + lane % gsz;
        cplx<R> e0 = mk<R>(0, 0), e1 = e0, e2 = e0;
        double2 G[5] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0),
                        make_double2(0, 0)};
        if constexpr (!QUADS) {
            if (m < M) real_dipole_pairs<R>(X, M, m, p0 + grp, p1, ng, src, T, ph, e0, e1, e2);
            for (int o = gsz; o < 32; o <<= 1) {
                e0.x += __shfl_xor_sync(0xffffffffu, e0.x, o);
                e0.y += __shfl_xor_sync(0xffffffffu, e0.y, o);
                e1.x += __shfl_xor_sync(0xffffffffu, e1.x, o);
                e1.y += __shfl_xor_sync(0xffffffffu, e1.y, o);
                e2.x += __shfl_xor_sync(0xffffffffu, e2.x, o);
                e2.y += __shfl_xor_sync(0xffffffffu, e2.y, o);
            }
        }
        if (m >= M || grp != 0) continue;
        for (int p = p0; QUADS && p < p1; ++p) {
            const int i = src[p];
            const R* t = T + 8 * size_t(p);
            const R dx = t[0], dy = t[1], dz = t[2], perp = t[3], para = t[4];
            const cplx<R> px = to_r<R>(X[size_t(3 * i) * M + m]);
            const cplx<R> py = to_r<R>(X[size_t(3 * i + 1) * M + m]);
            const cplx<R> pz = to_r<R>(X[size_t(3 * i + 2) * M + m]);
            const cplx<R> rp = px * dx + py * dy + pz * dz;
            const cplx<R> k = rp * (para - perp);
            e0 += px * perp + k * dx;
            e1 += py * perp + k * dy;
            e2 += pz * perp + k * dz;
            {
                // quadrupole couplings in float64 (reference :1758-1866)
                const double* qc = Qt + 8 * size_t(p);
                const double Q1 = qc[0], Q2 = qc[1], Q3 = qc[2];
                const double ddx = dx, ddy = dy, ddz = dz;
                const int qs = quad_map[i];
                double2 q[5] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0),
                                make_double2(0, 0)};
                if (qs >= 0)
                    for (int c = 0; c < 5; ++c) q[c] = X[size_t(3 * a.N + 5 * qs + c) * M + m];
                const double2 Qr0 = q[0] * ddx + q[1] * ddy + q[2] * ddz;
                const double2 Qr1 = q[1] * ddx + q[3] * ddy + q[4] * ddz;
                const double2 Qr2 = q[2] * ddx + q[4] * ddy - (q[0] + q[3]) * ddz;
                if (qs >= 0) {
                    const double rr0 = ddx * ddx - ddz * ddz, rr1 = 2 * ddx * ddy, rr2 = 2 * ddx * ddz,
                                 rr3 = ddy * ddy - ddz * ddz, rr4 = 2 * ddy * ddz;
                    const double2 Qrr = q[0] * rr0 + q[1] * rr1 + q[2] * rr2 + q[3] * rr3 + q[4] * rr4;
                    const double2 eq0 = (Qrr * (Q1 * ddx) + Qr0 * (2.0 * Q2)) * 0.5;
                    const double2 eq1 = (Qrr * (Q1 * ddy) + Qr1 * (2.0 * Q2)) * 0.5;
                    const double2 eq2 = (Qrr * (Q1 * ddz) + Qr2 * (2.0 * Q2)) * 0.5;
                    e0 -= to_r<R>(eq0); e1 -= to_r<R>(eq1); e2 -= to_r<R>(eq2);
                }
                if (qt >= 0) {
                    const double rs[5] = {ddx * ddx, ddx * ddy, ddx * ddz, ddy * ddy, ddy * ddz};
                    const double I5[5] = {1, 0, 0, 1, 0};
                    const double2 dpx = to_d(px), dpy = to_d(py), dpz = to_d(pz);
                    const double2 drp = dpx * ddx + dpy * ddy + dpz * ddz;
                    const double2 Pr[5] = {dpx * (2.0 * ddx), dpx * ddy + dpy * ddx, dpx * ddz + dpz * ddx,
                                           dpy * (2.0 * ddy), dpy * ddz + dpz * ddy};
                    for (int c = 0; c < 5; ++c) G[c] += (drp * (Q1 * rs[c] + (Q2 + Q3) * I5[c]) + Pr[c] * Q2) * sign;
                    if (qs >= 0) {
                        const double G1 = qc[3], G2 = qc[4], G3 = qc[5], G4 = qc[6];
                        const double2 Qrr2 = Qr0 * ddx + Qr1 * ddy + Qr2 * ddz;
                        const double2 QQ[5] = {Qr0 * (2.0 * ddx), Qr0 * ddy + Qr1 * ddx, Qr0 * ddz + Qr2 * ddx,
                                               Qr1 * (2.0 * ddy), Qr1 * ddz + Qr2 * ddy};
                        for (int c = 0; c < 5; ++c)
                            G[c] += ((Qrr2 * (G1 * I5[c] + G3 * I5[c] + G4 * rs[c]) + q[c] * G2 + QQ[c] * (2.0 * G3)) *
                                     0.5) * sign;
                    }
                }
            }
        }
        double2 out[3] = {to_d(e0) * sign, to_d(e1) * sign, to_d(e2) * sign};
        double2 inv = make_double2(1.0, 0.0);
        double2 s = make_double2(0.0, 0.0);
        if (a.solver_ax && sc) s = sc[size_t(j) * M + m];
        if (a.jacobi && sc) {
            const double den = s.x * s.x + s.y * s.y;
            inv = den > 1e-30 ? make_double2(s.x / den, -s.y / den) : make_double2(1.0, 0.0);
        }
        for (int c = 0; c < 3; ++c) {
            const size_t o = size_t(3 * j + c) * M + m;
            double2 v = out[c];
            if (a.add_recip) {
                const double2 r = Y[o];
                v = a.solver_ax ? v + r : (r + v) * -1.0;  // INTERACTION_FIELD: -(recip + sign*pairs)
            }
            if (a.solver_ax) {
                const double2 pj = X[o];
                v += make_double2(s.x + selfc, s.y) * pj;
            }
            if (a.jacobi) v = v * inv;
            Y[o] = v;
        }
        if (qt >= 0) {
            for (int c = 0; c < 5; ++c) {
                const size_t o = size_t(3 * a.Nt + 5 * qt + c) * M + m;
                double2 v = G[c];
                if (a.add_recip) {
                    const double2 r = Y[o];
                    v = a.solver_ax ? v + r : (r + v) * -1.0;
                }
                if (a.solver_ax) {
                    const double2 qv = X[size_t(3 * a.N + 5 * qt + c) * M + m];
                    const double qa2 = a.qa2 ? a.qa2[j] : 1.0;
                    const double qg2 = a.qg2 ? a.qg2[j] : a.self_grad;
                    v += make_double2(2.5 * s.x / qa2 + 0.5 * qg2, 2.5 * s.y / qa2) * qv;
                }
                if (a.jacobi) v = v * inv;
                Y[o] = v;
            }
        }
    }
}

// -------------------------------------------------------------- direct ---

// Open-boundary all-pairs field (direct_field_kernel,
// direct_electric_field.cu:42-324).  Thread per target, blockIdx.y = rhs,
// source tiles staged in shared memory.
template <typename R>
__global__ void __launch_bounds__(128) k_direct(const double2* __restrict__ X, double2* __restrict__ Y, int M, int N,
                                                int Nt, const double* __restrict__ src,
                                                const double* __restrict__ tgt, const double* __restrict__ rad,
                                                const int* __restrict__ quad_map, int quads,
                                                const double2* __restrict__ sc, int solver_ax, int jacobi) {
    constexpr int TILE = 128;
    __shared__ R sx[TILE], sy[TILE], sz[TILE], sr[TILE];
    __shared__ cplx<R> sp[TILE][3];
    __shared__ cplx<R> sq[TILE][5];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    const R inv4pi = R(1.0 / (4.0 * kPi));
    const R k4 = inv4pi * (solver_ax ? R(-1) : R(1));
    const R jx = j < Nt ? R(tgt[j]) : R(0), jy = j < Nt ? R(tgt[Nt + j]) : R(0),
            jz = j < Nt ? R(tgt[2 * Nt + j]) : R(0);
    const int qt = (quads && j < N && j < Nt) ? quad_map[j] : -1;
    cplx<R> E[3] = {mk<R>(0, 0), mk<R>(0, 0), mk<R>(0, 0)};
    cplx<R> G[5] = {mk<R>(0, 0), mk<R>(0, 0), mk<R>(0, 0), mk<R>(0, 0), mk<R>(0, 0)};
    const R eps_orig = sizeof(R) == 4 ? R(1e-6) : R(1e-9);
    const R eps_sing = sizeof(R) == 4 ? R(1e-12) : R(1e-18);
    for (int t0 = 0; t0 < N; t0 += TILE) {
        const int s = t0 + threadIdx.x;
        if (s < N) {
            sx[threadIdx.x] = R(src[s]); sy[threadIdx.x] = R(src[N + s]); sz[threadIdx.x] = R(src[2 * N + s]);
            sr[threadIdx.x] = rad ? R(rad[s]) : R(0);
            for (int c = 0; c < 3; ++c) sp[threadIdx.x][c] = to_r<R>(X[size_t(3 * s + c) * M + m]);
            const int qs = quads ? quad_map[s] : -1;
            for (int c = 0; c < 5; ++c)
                sq[threadIdx.x][c] = qs >= 0 ? to_r<R>(X[size_t(3 * N + 5 * qs + c) * M + m]) : mk<R>(0, 0);
        }
        __syncthreads();
        if (j < Nt) {
            const int te = min(TILE, N - t0);
            for (int k = 0; k < te; ++k) {
                const int i = t0 + k;
                if (solver_ax && i == j) continue;
                R rx = sx[k] - jx, ry = sy[k] - jy, rz = sz[k] - jz;
                R r2 = rx * rx + ry * ry + rz * rz;
                const R md2 = sr[k] * sr[k];
                const R ro = sqrt(r2);
                if (r2 < md2) {
                    if (ro > eps_orig) {
                        const R scl = sqrt(md2 / r2);
                        rx *= scl; ry *= scl; rz *= scl;
                    }
                    r2 = md2;
                }
                if (r2 < eps_sing) continue;
                const R r = sqrt(r2);
                const R ir = R(1) / r, ir2 = R(1) / r2;
                const R ir3 = ir2 * ir, ir4 = ir3 * ir, ir5 = ir4 * ir;
                const R ux = rx * ir, uy = ry * ir, uz = rz * ir;
                const cplx<R> px = sp[k][0], py = sp[k][1], pz = sp[k][2];
                const cplx<R> pr = px * ux + py * uy + pz * uz;
                const R df = k4 * ir3;
                E[0] += (pr * (R(3) * ux) - px) * df;
                E[1] += (pr * (R(3) * uy) - py) * df;
                E[2] += (pr * (R(3) * uz) - pz) * df;
                if (quads) {
                    const cplx<R> q0 = sq[k][0] * R(-1), q1 = sq[k][1] * R(-2), q2 = sq[k][2] * R(-2),
                                  q3 = sq[k][3] * R(-1), q4 = sq[k][4] * R(-2);
                    const cplx<R> qzz = (q0 + q3) * R(-1);
                    const cplx<R> Qx = q0 * ux + q1 * uy + q2 * uz;
                    const cplx<R> Qy = q1 * ux + q3 * uy + q4 * uz;
                    const cplx<R> Qz = q2 * ux + q4 * uy + qzz * uz;
                    const cplx<R> Qrr = Qx * ux + Qy * uy + Qz * uz;
                    const R qf = R(3) * k4 * ir4;
                    E[0] += (Qrr * (R(2.5) * ux) - Qx) * qf;
                    E[1] += (Qrr * (R(2.5) * uy) - Qy) * qf;
                    E[2] += (Qrr * (R(2.5) * uz) - Qz) * qf;
                    if (qt >= 0) {
                        const R rs[5] = {ux * ux, ux * uy, ux * uz, uy * uy, uy * uz};
                        const cplx<R> Gd[5] = {pr * (R(-5) * rs[0] + R(1)) + px * (R(2) * ux),
                                               pr * (R(-5) * rs[1]) + (px * uy + py * ux),
                                               pr * (R(-5) * rs[2]) + (px * uz + pz * ux),
                                               pr * (R(-5) * rs[3] + R(1)) + py * (R(2) * uy),
                                               pr * (R(-5) * rs[4]) + (py * uz + pz * uy)};
                        const R gdf = R(-3) * k4 * ir4;
                        const cplx<R> QQ[5] = {Qx * (R(2) * ux), Qx * uy + Qy * ux, Qx * uz + Qz * ux,
                                               Qy * (R(2) * uy), Qy * uz + Qz * uy};
                        const cplx<R> qp[5] = {q0, q1, q2, q3, q4};
                        const R dg[5] = {R(1), R(0), R(0), R(1), R(0)};
                        const R f = -k4 * ir5;
                        for (int c = 0; c < 5; ++c) {
                            const cplx<R> gq = qp[c] * R(-1.5) + Qrr * (R(52.5) * rs[c] - R(7.5) * dg[c]) -
                                               QQ[c] * R(15);
                            G[c] += Gd[c] * gdf + gq * f;
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    if (j >= Nt) return;
    double2 inv = make_double2(1.0, 0.0);
    double2 s = make_double2(0.0, 0.0);
    if (solver_ax && sc) s = sc[size_t(j) * M + m];
    if (jacobi && sc) {
        const double den = s.x * s.x + s.y * s.y;
        inv = den > 1e-30 ? make_double2(s.x / den, -s.y / den) : make_double2(1.0, 0.0);
    }
    const double rj = (solver_ax && rad) ? rad[j] : 1.0;
    const double corr = (1.0 / (4.0 * kPi)) / (rj * rj * rj);
    for (int c = 0; c < 3; ++c) {
        const size_t o = size_t(3 * j + c) * M + m;
        double2 v = to_d(E[c]);
        if (solver_ax) v += make_double2(s.x + corr, s.y) * X[o];
        if (jacobi) v = v * inv;
        Y[o] = v;
    }
    if (qt >= 0) {
        const double cq = 3.0 * corr / (rj * rj);
        const double fs = 2.5 / (rj * rj);
        for (int c = 0; c < 5; ++c) {
            const size_t o = size_t(3 * Nt + 5 * qt + c) * M + m;
            double2 v = to_d(G[c]);
            if (solver_ax) v += make_double2(fs * s.x + cq, fs * s.y) * X[size_t(3 * N + 5 * qt + c) * M + m];
            if (jacobi) v = v * inv;
            Y[o] = v;
        }
    }
}

inline int nblk(long long n, int b) { return int((n + b - 1) / b); }

}  // namespace

// ------------------------------------------------------------ host side --

Field::Field(const FieldSpec& spec) : spec_(spec) {
    if (spec_.kind == FIELD_MONO) {
        geom_ = make_ewald_geom(spec_.box, spec_.errortol, spec_.xi, spec_.grid, spec_.support);
        if (2 * geom_.off + 1 > kMaxStencil) throw std::runtime_error("Ewald stencil wider than supported (errortol too small)");
        // a spread tile reaches at most 8 bins per axis (the spread kernels'
        // bin lists) and holds at most 128 (x, y) columns
        for (int d = 0; d < 2; ++d) {
            const int t = spec_.tile[d];
            if (t != 0 && (t < 1 || (t + 2 * geom_.off + t - 1) / t + 1 > 8))
                throw std::invalid_argument("spread tile " + std::to_string(t) + " too small for stencil half width " +
                                            std::to_string(geom_.off));
        }
        if (spec_.tile[0] * spec_.tile[1] > 128 || (spec_.tile[0] == 0 ? 8 : spec_.tile[0]) *
                                                           (spec_.tile[1] == 0 ? 8 : spec_.tile[1]) > 128)
            throw std::invalid_argument("a spread tile holds at most 128 columns");
        tables_ = build_mono_tables(spec_.xi);
        tab_r_.ensure(sizeof(double) * kTableSize);
        tab_f_.ensure(sizeof(double) * kTableSize * T_COUNT);
        MPM_CUDA(cudaMemcpy(tab_r_.p, tables_.r.data(), sizeof(double) * kTableSize, cudaMemcpyHostToDevice));
        for (int f = 0; f < T_COUNT; ++f)
            MPM_CUDA(cudaMemcpy(tab_f_.as<double>() + size_t(f) * kTableSize, tables_.f[f].data(),
                                sizeof(double) * kTableSize, cudaMemcpyHostToDevice));
    } else if (spec_.kind == FIELD_POLY) {
        poly_init();
    } else if (spec_.kind != FIELD_DIRECT) {
        throw std::runtime_error("unsupported field kind");
    }
}

Field::~Field() {
    for (auto& p : plans_) cufftDestroy(p.h);
    if (ev_fork_) cudaEventDestroy(ev_fork_);
    if (ev_join_) cudaEventDestroy(ev_join_);
    if (aux_) cudaStreamDestroy(aux_);
}

FieldStats Field::stats() const {
    FieldStats s;
    s.pruned = gv_.pruned;
    s.z_slots = gv_.Zs;
    s.num_pairs = num_pairs_;
    for (int d = 0; d < 3; ++d) s.grid[d] = geom_.ng[d];
    s.stencil = gv_.S;
    s.slab_fused = (spec_.kind == FIELD_MONO && use_slab()) ? 1 : 0;
    s.single_layer = (spec_.kind == FIELD_MONO && gv_.layer) ? 1 : 0;
    return s;
}

void Field::set_positions(const double* x, const double* y, const double* z, int n, cudaStream_t s) {
    if (n <= 0) throw std::invalid_argument("set_positions: empty coordinate set");
    const bool resized = (n != N_);
    N_ = n;
    if (resized || quad_map_.p == nullptr) {
        // quadrupole bookkeeping (base_electric_field.cu:193-220)
        std::vector<int> qidx;
        if (spec_.quads) {
            if (spec_.quad_idxs.empty()) {
                qidx.resize(N_);
                std::iota(qidx.begin(), qidx.end(), 0);
            } else {
                qidx = spec_.quad_idxs;
            }
        }
        Nq_ = int(qidx.size());
        std::vector<int> qmap(N_, -1);
        for (int q = 0; q < Nq_; ++q)
            if (qidx[q] >= 0 && qidx[q] < N_) qmap[qidx[q]] = q;
        quad_map_.ensure(sizeof(int) * N_);
        MPM_CUDA(cudaMemcpy(quad_map_.p, qmap.data(), sizeof(int) * N_, cudaMemcpyHostToDevice));
        if (Nq_) {
            quad_idx_.ensure(sizeof(int) * Nq_);
            MPM_CUDA(cudaMemcpy(quad_idx_.p, qidx.data(), sizeof(int) * Nq_, cudaMemcpyHostToDevice));
        }
        if (spec_.kind == FIELD_POLY && int(spec_.radius.size()) != N_)
            throw std::invalid_argument("Polydisperse field: radius size must match num_particles.");
        if (spec_.kind == FIELD_DIRECT) {
            std::vector<double> rad = spec_.radius;
            if (rad.empty()) rad.assign(N_, 0.0);
            if (int(rad.size()) != N_) throw std::invalid_argument("Direct field: radius size must match num_particles.");
            radius_.ensure(sizeof(double) * N_);
            MPM_CUDA(cudaMemcpy(radius_.p, rad.data(), sizeof(double) * N_, cudaMemcpyHostToDevice));
        }
    }
    sources_.n = n;
    sources_.xyz.ensure(sizeof(double) * 3 * n);
    MPM_CUDA(cudaMemcpyAsync(sources_.xyz.as<double>(), x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    MPM_CUDA(cudaMemcpyAsync(sources_.xyz.as<double>() + n, y, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    MPM_CUDA(cudaMemcpyAsync(sources_.xyz.as<double>() + 2 * n, z, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    if (spec_.kind == FIELD_MONO) {
        // occupied z planes are decided on the host from the same rounding rule
        std::vector<double> zz(z, z + n);
        host_z_.assign(zz.begin(), zz.end());
    }
    precalc_dirty_ = true;
    precalc(s);
}

void Field::set_field_points(const double* x, const double* y, const double* z, int n, cudaStream_t s) {
    if (spec_.solver_ax) throw std::runtime_error("Cannot update field coordinates when SOLVER_AX mode is active.");
    targets_.n = n;
    targets_.xyz.ensure(sizeof(double) * 3 * std::max(n, 1));
    MPM_CUDA(cudaMemcpyAsync(targets_.xyz.as<double>(), x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    MPM_CUDA(cudaMemcpyAsync(targets_.xyz.as<double>() + n, y, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    MPM_CUDA(cudaMemcpyAsync(targets_.xyz.as<double>() + 2 * n, z, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    precalc_dirty_ = true;
    if (N_ > 0) precalc(s);
}

void Field::choose_layout(cudaStream_t) {
    const int Nz = geom_.ng[2];
    gv_.Nx = geom_.ng[0];
    gv_.Ny = geom_.ng[1];
    gv_.Nz = Nz;
    gv_.off = geom_.off;
    gv_.S = 2 * geom_.off + 1;
    gv_.Sz = gv_.S;
    gv_.offz = gv_.off;
    gv_.layer = 0;
    gv_.pruned = 0;
    gv_.z0 = 0;
    gv_.Zs = Nz;
    // Pruned slab layout only for the dipole matvec with targets == sources.
    if (!spec_.solver_ax || Nq_ > 0) return;
    // A single layer: every particle has the same nearest z node and the
    // same offset from it (a planar monolayer), so every z stencil is the
    // same weight vector w_o.  The grid then keeps one z slot and the
    // k-space step carries sum_{o,o'} w_o w_o' K(o - o') (the same
    // discretisation, z summed first).
    if (!host_z_.empty()) {
        const double hz = geom_.h[2];
        const long g0 = std::lround(host_z_[0] / hz);
        const double d0 = double(g0) * hz - host_z_[0];
        bool same = true;
        for (double zv : host_z_) {
            const long g = std::lround(zv / hz);
            if (pmod(int(g), Nz) != pmod(int(g0), Nz) || double(g) * hz - zv != d0) {
                same = false;
                break;
            }
        }
        if (same) {
            gv_.pruned = 1;
            gv_.layer = 1;
            gv_.Zs = 1;
            gv_.z0 = pmod(int(g0), Nz);
            gv_.Sz = 1;
            gv_.offz = 0;
            layer_w_.resize(gv_.S);
            for (int o = 0; o < gv_.S; ++o) {
                const double gd = d0 + (o - gv_.off) * hz;
                layer_w_[o] = std::exp(-2.0 * spec_.xi * spec_.xi * gd * gd / geom_.eta[2]);
            }
            if (pmod(int(g0), Nz) != layer_key_g_ || d0 != layer_key_d_) layer_taps_ = layer_colK_ = false;
            layer_key_g_ = pmod(int(g0), Nz);
            layer_key_d_ = d0;
            return;
        }
    }
    std::vector<char> occ(Nz, 0);
    for (double zv : host_z_) {
        const long g = std::lround(zv / geom_.h[2]);  // C round, halves away from zero
        for (int o = -geom_.off; o <= geom_.off; ++o) occ[pmod(int(g + o), Nz)] = 1;
    }
    // smallest cyclic interval covering all occupied planes = complement of
    // the largest run of empty planes
    int best_len = 0, best_start = 0;
    int run = 0, run_start = 0;
    for (int k = 0; k < 2 * Nz; ++k) {
        if (!occ[k % Nz]) {
            if (run == 0) run_start = k;
            ++run;
            if (run > best_len && run <= Nz) { best_len = run; best_start = run_start; }
        } else {
            run = 0;
        }
    }
    const int Z = Nz - best_len;
    if (best_len == 0 || Z > 24 || 4 * Z > Nz) return;
    gv_.pruned = 1;
    gv_.Zs = Z;
    gv_.z0 = (best_start + best_len) % Nz;
}

// The spread plan (see k_spread_plan).  Left out (plan_cap_ = 0, spread
// builds its lists in every launch) when a tile has more candidates than the
// plan kernel holds or the plan would take more than 512 MB.
void Field::build_spread_plan(cudaStream_t s) {
    plan_cap_ = 0;
    const PointSet& ps = sources_;
    const int TX = ps.tile[0], TY = ps.tile[1], TZ = ps.tile[2];
    const int wlen = TX + TY + TZ;
    const int ntile = ps.nb[0] * ps.nb[1] * ps.nb[2];
    const int ncol = TX * TY;
    if (TZ > kSpreadZMax || ntile < 1) return;
    const size_t shm = sizeof(double) * kPlanCandMax * wlen;
    set_smem_limit(k_spread_plan, shm);
    plan_nc_.ensure(sizeof(int) * ntile);
    plan_cnt_.ensure(sizeof(int) * 2);
    MPM_CUDA(cudaMemsetAsync(plan_cnt_.p, 0, sizeof(int) * 2, s));
    int* cnt = plan_cnt_.as<int>();
    auto run = [&](int pass, int cap) {
        k_spread_plan<<<ntile, 256, shm, s>>>(ps.base.as<int4>(), ps.w64.as<double>(), ps.bin_start.as<int>(),
                                              ps.bin_end.as<int>(), ps.idx_sorted.as<int>(), gv_, TX, TY, TZ,
                                              ps.nb[0], ps.nb[1], pass, cap, plan_nc_.as<int>(), cnt, cnt + 1,
                                              plan_cid_.as<int>(), plan_w64_.as<double>(), plan_w32_.as<float>(),
                                              plan_lw64_.as<double>(), plan_lw32_.as<float>(), plan_lc_.as<int>(),
                                              plan_ln_.as<int>());
        MPM_LAUNCH();
    };
    run(0, 0);
    int h[2] = {0, 0};
    MPM_CUDA(cudaMemcpyAsync(h, plan_cnt_.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    if (h[1]) return;
    const int cap = std::max(1, h[0]);
    const size_t lists = size_t(ntile) * ncol * kSpreadListCap;
    const size_t bytes = size_t(ntile) * cap * (sizeof(int) + wlen * (sizeof(double) + sizeof(float))) +
                         lists * (sizeof(double) + sizeof(float) + sizeof(int)) + sizeof(int) * ntile * ncol;
    if (bytes > (size_t(512) << 20)) return;
    plan_cid_.ensure(sizeof(int) * ntile * cap);
    plan_w64_.ensure(sizeof(double) * ntile * cap * wlen);
    plan_w32_.ensure(sizeof(float) * ntile * cap * wlen);
    plan_lw64_.ensure(sizeof(double) * lists);
    plan_lw32_.ensure(sizeof(float) * lists);
    plan_lc_.ensure(sizeof(int) * lists);
    plan_ln_.ensure(sizeof(int) * size_t(ntile) * ncol);
    run(1, cap);
    plan_cap_ = cap;
}

void Field::build_stencil(PointSet& ps, cudaStream_t s, bool bins) {
    const int n = ps.n;
    const int S = gv_.S;
    ps.base.ensure(sizeof(int4) * n);
    ps.w64.ensure(sizeof(double) * size_t(n) * 3 * S);
    ps.w32.ensure(sizeof(float) * size_t(n) * 3 * S);
    StencilArgs a;
    for (int d = 0; d < 3; ++d) { a.h[d] = geom_.h[d]; a.eta[d] = geom_.eta[d]; a.N[d] = geom_.ng[d]; }
    a.xi = spec_.xi;
    a.cfac = geom_.spread_const;
    a.off = geom_.off;
    a.S = S;
    a.z0 = gv_.z0;
    a.pruned = gv_.pruned;
    a.Zs = gv_.Zs;
    a.layer = gv_.layer;
    k_stencil<<<nblk(n, 128), 128, 0, s>>>(ps.xyz.as<double>(), n, a, ps.base.as<int4>(), ps.w64.as<double>(),
                                            ps.w32.as<float>());
    MPM_LAUNCH();
    if (!bins) return;
    ps.tile[0] = spec_.tile[0] > 0 ? spec_.tile[0] : 8;
    ps.tile[1] = spec_.tile[1] > 0 ? spec_.tile[1] : 8;
    ps.tile[2] = (gv_.pruned && gv_.Zs <= 16) ? gv_.Zs : 8;
    ps.nb[0] = (gv_.Nx + ps.tile[0] - 1) / ps.tile[0];
    ps.nb[1] = (gv_.Ny + ps.tile[1] - 1) / ps.tile[1];
    ps.nb[2] = (gv_.Zs + ps.tile[2] - 1) / ps.tile[2];
    const int nbins = ps.nb[0] * ps.nb[1] * ps.nb[2];
    ps.bin_key.ensure(sizeof(int) * n);
    ps.bin_key_sorted.ensure(sizeof(int) * n);
    ps.idx.ensure(sizeof(int) * n);
    ps.idx_sorted.ensure(sizeof(int) * n);
    ps.bin_start.ensure(sizeof(int) * nbins);
    ps.bin_end.ensure(sizeof(int) * nbins);
    k_bin_keys<<<nblk(n, 128), 128, 0, s>>>(ps.base.as<int4>(), n, ps.tile[0], ps.tile[1], ps.tile[2], ps.nb[0],
                                            ps.nb[1], ps.bin_key.as<int>(), ps.idx.as<int>());
    MPM_LAUNCH();
    size_t tmp = 0;
    int bits = 1;
    while ((1 << bits) < nbins) ++bits;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, ps.bin_key.as<int>(), ps.bin_key_sorted.as<int>(),
                                    ps.idx.as<int>(), ps.idx_sorted.as<int>(), n, 0, bits, s);
    ps.cub_tmp.ensure(tmp);
    MPM_CUDA(cub::DeviceRadixSort::SortPairs(ps.cub_tmp.p, tmp, ps.bin_key.as<int>(), ps.bin_key_sorted.as<int>(),
                                             ps.idx.as<int>(), ps.idx_sorted.as<int>(), n, 0, bits, s));
    k_fill_int<<<nblk(nbins, 256), 256, 0, s>>>(ps.bin_start.as<int>(), nbins, -1);
    MPM_LAUNCH();
    k_fill_int<<<nblk(nbins, 256), 256, 0, s>>>(ps.bin_end.as<int>(), nbins, -1);
    MPM_LAUNCH();
    k_bin_bounds<<<nblk(n, 256), 256, 0, s>>>(ps.bin_key_sorted.as<int>(), n, ps.bin_start.as<int>(),
                                              ps.bin_end.as<int>());
    MPM_LAUNCH();
}

void Field::build_pairs(cudaStream_t s) {
    const PointSet& tg = spec_.solver_ax ? sources_ : targets_;
    const int ns = sources_.n, nt = tg.n;
    const double rc = geom_.rc;
    CellArgs a;
    for (int d = 0; d < 3; ++d) {
        a.L[d] = spec_.box[d];
        a.nc[d] = std::max(1, int(std::floor(spec_.box[d] / rc)));
        a.cs[d] = spec_.box[d] / a.nc[d];
    }
    const int ncell = a.nc[0] * a.nc[1] * a.nc[2];
    cell_key_.ensure(sizeof(int) * ns);
    cell_idx_.ensure(sizeof(int) * ns);
    cell_key_s_.ensure(sizeof(int) * ns);
    cell_idx_s_.ensure(sizeof(int) * ns);
    cell_start_.ensure(sizeof(int) * ncell);
    cell_end_.ensure(sizeof(int) * ncell);
    k_cell_keys<<<nblk(ns, 128), 128, 0, s>>>(sources_.xyz.as<double>(), ns, a, cell_key_.as<int>(),
                                               cell_idx_.as<int>());
    MPM_LAUNCH();
    int bits = 1;
    while ((1 << bits) < ncell) ++bits;
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, cell_key_.as<int>(), cell_key_s_.as<int>(), cell_idx_.as<int>(),
                                    cell_idx_s_.as<int>(), ns, 0, bits, s);
    cub_tmp_.ensure(tmp);
    MPM_CUDA(cub::DeviceRadixSort::SortPairs(cub_tmp_.p, tmp, cell_key_.as<int>(), cell_key_s_.as<int>(),
                                             cell_idx_.as<int>(), cell_idx_s_.as<int>(), ns, 0, bits, s));
    k_fill_int<<<nblk(ncell, 256), 256, 0, s>>>(cell_start_.as<int>(), ncell, -1);
    MPM_LAUNCH();
    k_fill_int<<<nblk(ncell, 256), 256, 0, s>>>(cell_end_.as<int>(), ncell, -1);
    MPM_LAUNCH();
    k_bin_bounds<<<nblk(ns, 256), 256, 0, s>>>(cell_key_s_.as<int>(), ns, cell_start_.as<int>(),
                                               cell_end_.as<int>());
    MPM_LAUNCH();
    pair_cnt_.ensure(sizeof(int) * (nt + 1));
    pair_off_.ensure(sizeof(int) * (nt + 1));
    MPM_CUDA(cudaMemsetAsync(pair_cnt_.p, 0, sizeof(int) * (nt + 1), s));
    k_pairs<<<nblk((long long)nt * 32, 128), 128, 0, s>>>(sources_.xyz.as<double>(), ns, tg.xyz.as<double>(), nt, a,
                                           cell_start_.as<int>(), cell_end_.as<int>(), cell_idx_s_.as<int>(), rc,
                                           spec_.solver_ax ? 1 : 0, 0, pair_cnt_.as<int>(), nullptr, nullptr,
                                           nullptr);
    MPM_LAUNCH();
    size_t need = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, pair_cnt_.as<int>(), pair_off_.as<int>(), nt + 1, s);
    cub_tmp_.ensure(need);
    MPM_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp_.p, need, pair_cnt_.as<int>(), pair_off_.as<int>(), nt + 1, s));
    int total = 0;
    MPM_CUDA(cudaMemcpyAsync(&total, pair_off_.as<int>() + nt, sizeof(int), cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    num_pairs_ = total;
    const size_t np = std::max<long long>(1, num_pairs_);
    pair_src_.ensure(sizeof(int) * np);
    DevBuf& geo = pair_geo_;
    geo.ensure(sizeof(double) * 4 * np);
    k_pairs<<<nblk((long long)nt * 32, 128), 128, 0, s>>>(sources_.xyz.as<double>(), ns, tg.xyz.as<double>(), nt, a,
                                           cell_start_.as<int>(), cell_end_.as<int>(), cell_idx_s_.as<int>(), rc,
                                           spec_.solver_ax ? 1 : 0, 1, nullptr, pair_off_.as<int>(),
                                           pair_src_.as<int>(), geo.as<double>());
    MPM_LAUNCH();
    pair_T64_.ensure(sizeof(double) * 8 * np);
    pair_T32_.ensure(sizeof(float) * 8 * np);
    if (Nq_) pair_Q_.ensure(sizeof(double) * 8 * np);
    if (bloch_on()) build_pair_phases(s);
    if (num_pairs_ > 0 && spec_.kind == FIELD_MONO) {  // polydisperse: poly_pair_coefs
        k_pair_coefs<<<nblk(num_pairs_, 256), 256, 0, s>>>(geo.as<double>(), num_pairs_, tab_r_.as<double>(),
                                                            tab_f_.as<double>(), Nq_ > 0, pair_T64_.as<double>(),
                                                            pair_T32_.as<float>(), pair_Q_.as<double>());
        MPM_LAUNCH();
    }
}

void Field::build_pair_phases(cudaStream_t s) {
    const size_t np = std::max<long long>(1, num_pairs_);
    pair_ph64_.ensure(sizeof(double2) * np);
    pair_ph32_.ensure(sizeof(float2) * np);
    if (num_pairs_ <= 0) return;
    k_pair_phase<<<nblk(num_pairs_, 256), 256, 0, s>>>(pair_geo_.as<double>(), num_pairs_, spec_.bloch[0],
                                                        spec_.bloch[1], pair_ph64_.as<double2>(),
                                                        pair_ph32_.as<float2>());
    MPM_LAUNCH();
}

void Field::set_bloch(double bx, double by) {
    if (spec_.kind == FIELD_DIRECT && (bx != 0.0 || by != 0.0))
        throw std::invalid_argument("a Bloch wavevector needs a periodic (Ewald) field");
    if ((bx != 0.0 || by != 0.0) && spec_.quads)
        throw std::invalid_argument("a Bloch wavevector is supported for dipoles only");
    if (bx == spec_.bloch[0] && by == spec_.bloch[1]) return;
    spec_.bloch[0] = bx;
    spec_.bloch[1] = by;
    // every k-space table and the pair phases follow the wavevector
    scale_built_ = 0;
    colK_Z_ = -1;
    slab_Z_ = -1;
    layer_colK_ = layer_taps_ = false;
    if (spec_.kind == FIELD_POLY) poly_build_scale();
    // the tables and pair phases are per-frame state: rebuilt now (applies
    // use what the last set_positions / set_bloch built)
    precalc_dirty_ = true;
    if (N_ > 0) {
        precalc(nullptr);
        MPM_CUDA(cudaStreamSynchronize(nullptr));
    }
}

void Field::build_scale(cudaStream_t s) {
    const size_t V = size_t(geom_.ng[0]) * geom_.ng[1] * geom_.ng[2];
    const int per = Nq_ ? 4 : 1;
    scale64_.ensure(sizeof(double) * V * per);
    scale32_.ensure(sizeof(float) * V * per);
    ScaleArgs a;
    a.Nx = geom_.ng[0]; a.Ny = geom_.ng[1]; a.Nz = geom_.ng[2];
    a.Lx = spec_.box[0]; a.Ly = spec_.box[1]; a.Lz = spec_.box[2];
    a.xi = spec_.xi;
    for (int d = 0; d < 3; ++d) a.eta[d] = geom_.eta[d];
    a.bx = spec_.bloch[0];
    a.by = spec_.bloch[1];
    k_build_scale<<<nblk((long long)V, 256), 256, 0, s>>>(a, Nq_ ? 1 : 0, scale64_.as<double>(), scale32_.as<float>());
    MPM_LAUNCH();
    scale_built_ = per;
}

void Field::build_column_kernel(cudaStream_t s) {
    const int Z = gv_.Zs;
    const int ncol = gv_.Nx * gv_.Ny;
    const int nd = 2 * Z - 1;
    colK64_.ensure(sizeof(double2) * size_t(ncol) * 6 * nd);
    colK32_.ensure(sizeof(float2) * size_t(ncol) * 6 * nd);
    ScaleArgs a;
    a.Nx = gv_.Nx; a.Ny = gv_.Ny; a.Nz = gv_.Nz;
    a.Lx = spec_.box[0]; a.Ly = spec_.box[1]; a.Lz = spec_.box[2];
    a.xi = spec_.xi;
    for (int d = 0; d < 3; ++d) a.eta[d] = geom_.eta[d];
    a.bx = spec_.bloch[0];
    a.by = spec_.bloch[1];
    const size_t shm = sizeof(double) * 8 * gv_.Nz;
    if (shm > 48 * 1024)
        set_smem_limit(k_build_column, shm);
    const double* w2 = nullptr;
    if (gv_.layer) {
        layer_wd_.ensure(sizeof(double) * (gv_.S + gv_.Nz));
        double* wd = layer_wd_.as<double>();
        MPM_CUDA(cudaMemcpyAsync(wd, layer_w_.data(), sizeof(double) * gv_.S, cudaMemcpyHostToDevice, s));
        k_layer_w2<<<nblk(gv_.Nz, 128), 128, 0, s>>>(wd, gv_.S, gv_.Nz, wd + gv_.S);
        MPM_LAUNCH();
        w2 = wd + gv_.S;
    }
    k_build_column<<<ncol, 128, shm, s>>>(a, Z, w2, colK64_.as<double2>(), colK32_.as<float2>());
    MPM_LAUNCH();
    if (gv_.layer) {
        MPM_CUDA(cudaStreamSynchronize(s));   // layer_w_ is read by the copy above
        layer_colK_ = true;
        colK_Z_ = -1;
    } else {
        layer_colK_ = false;
        colK_Z_ = Z;
    }
}

bool Field::use_slab() const {
    // the fused pass's taps assume the grid wavevectors themselves (no Bloch
    // shift); with one the pruned layout takes the column kernel
    return gv_.pruned && own_fft_ && ffty_.slab_ok(gv_.Zs, true) && ffty_.slab_ok(gv_.Zs, false) && !bloch_on();
}

void Field::build_slab_taps(cudaStream_t s) {
    const int Z = gv_.Zs;
    const int ncol = gv_.Nx * gv_.Ny;
    const int nd = 2 * Z - 1;
    slabT64_.ensure(sizeof(double2) * size_t(ncol) * 3 * nd);
    slabT32_.ensure(sizeof(float2) * size_t(ncol) * 3 * nd);
    ScaleArgs a;
    a.Nx = gv_.Nx; a.Ny = gv_.Ny; a.Nz = gv_.Nz;
    a.Lx = spec_.box[0]; a.Ly = spec_.box[1]; a.Lz = spec_.box[2];
    a.xi = spec_.xi;
    for (int d = 0; d < 3; ++d) a.eta[d] = geom_.eta[d];
    if (gv_.layer) {
        // |sum_o w_o exp(-2 pi i kz o / Nz)|^2 per kz, then the taps
        layer_wd_.ensure(sizeof(double) * (gv_.S + gv_.Nz));
        double* wd = layer_wd_.as<double>();
        MPM_CUDA(cudaMemcpyAsync(wd, layer_w_.data(), sizeof(double) * gv_.S, cudaMemcpyHostToDevice, s));
        k_layer_w2<<<nblk(gv_.Nz, 128), 128, 0, s>>>(wd, gv_.S, gv_.Nz, wd + gv_.S);
        MPM_LAUNCH();
        k_build_layer_taps<<<nblk(ncol, 128), 128, 0, s>>>(a, wd + gv_.S, slabT64_.as<double2>(),
                                                           slabT32_.as<float2>());
        MPM_LAUNCH();
        MPM_CUDA(cudaStreamSynchronize(s));   // layer_w_ is read by the copy above
        layer_taps_ = true;
        slab_Z_ = -1;
        return;
    }
    layer_taps_ = false;
    const size_t shm = sizeof(double) * 5 * gv_.Nz;
    if (shm > 48 * 1024)
        set_smem_limit(k_build_slab_taps, shm);
    k_build_slab_taps<<<ncol, 128, shm, s>>>(a, Z, slabT64_.as<double2>(), slabT32_.as<float2>());
    MPM_LAUNCH();
    slab_Z_ = Z;
}

void Field::precalc(cudaStream_t s) {
    if (!precalc_dirty_) return;
    StageScope scope(ST_PRECALC, s);
    if (spec_.kind == FIELD_MONO) {
        choose_layout(s);
        own_fft_ = AxisFFT::fits(gv_.Nx, true) && AxisFFT::fits(gv_.Ny, true) && AxisFFT::fits(gv_.Nz, true);
        if (own_fft_) {
            fftx_.init(gv_.Nx);
            ffty_.init(gv_.Ny);
            if (!gv_.pruned) fftz_.init(gv_.Nz);
        }
        build_stencil(sources_, s, true);
        build_spread_plan(s);
        if (!spec_.solver_ax) build_stencil(targets_, s, false);  // SOLVER_AX: targets share the source stencil
        build_pairs(s);
        if (use_slab()) {
            if (gv_.layer ? !layer_taps_ : slab_Z_ != gv_.Zs) build_slab_taps(s);
        } else if (gv_.pruned) {
            if (gv_.layer ? !layer_colK_ : colK_Z_ != gv_.Zs) build_column_kernel(s);
        } else if (scale_built_ != (Nq_ ? 4 : 1)) {
            build_scale(s);
        }
    } else if (spec_.kind == FIELD_POLY) {
        poly_precalc(s);
    }
    precalc_dirty_ = false;
    ++adj_frame_;
}

cufftHandle Field::plan_for(int B, bool fp32) {
    for (auto& p : plans_)
        if (p.M == B && p.fp32 == fp32 && p.pruned == gv_.pruned && p.Zs == gv_.Zs) return p.h;
    cufftHandle h;
    if (cufftCreate(&h) != CUFFT_SUCCESS) throw std::runtime_error("cuFFT plan creation failed");
    cufftResult r;
    size_t ws = 0;
    if (gv_.pruned) {
        int n[2] = {gv_.Nx, gv_.Ny};
        const int stride = gv_.Zs * B;
        r = cufftMakePlanMany(h, 2, n, n, stride, 1, n, stride, 1, fp32 ? CUFFT_C2C : CUFFT_Z2Z, stride, &ws);
    } else {
        int n[3] = {gv_.Nx, gv_.Ny, gv_.Nz};
        r = cufftMakePlanMany(h, 3, n, n, B, 1, n, B, 1, fp32 ? CUFFT_C2C : CUFFT_Z2Z, B, &ws);
    }
    if (r != CUFFT_SUCCESS) {
        cufftDestroy(h);
        throw std::runtime_error("cuFFT plan creation failed with code: " + std::to_string(int(r)));
    }
    plans_.push_back({B, fp32, gv_.pruned, gv_.Zs, h});
    return h;
}

// 3-D (full layout) or x-y (pruned layout) transform of the [x][y][slot][b]
// grid: in-house batched line transforms, cuFFT when a line is too long.
template <typename R>
void Field::transform(cplx<R>* grid, int B, bool inverse, cudaStream_t s) {
    if (own_fft_) {
        const size_t Bi = size_t(gv_.Zs) * B;
        if (!gv_.pruned) fftz_.run<R>(grid, size_t(B), B, size_t(gv_.Nz) * B, gv_.Nx * gv_.Ny, inverse, s);
        ffty_.run<R>(grid, Bi, int(Bi), size_t(gv_.Ny) * Bi, gv_.Nx, inverse, s);
        fftx_.run<R>(grid, size_t(gv_.Ny) * Bi, int(Bi), Bi, gv_.Ny, inverse, s);
        return;
    }
    cufftHandle plan = plan_for(B, sizeof(R) == 4);
    cufftSetStream(plan, s);
    cufftResult fr;
    const int dir = inverse ? CUFFT_INVERSE : CUFFT_FORWARD;
    if (sizeof(R) == 4)
        fr = cufftExecC2C(plan, reinterpret_cast<cufftComplex*>(grid), reinterpret_cast<cufftComplex*>(grid), dir);
    else
        fr = cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(grid), reinterpret_cast<cufftDoubleComplex*>(grid), dir);
    if (fr != CUFFT_SUCCESS) throw std::runtime_error("cuFFT execution failed with code: " + std::to_string(int(fr)));
}

template void Field::transform<float>(cplx<float>*, int, bool, cudaStream_t);
template void Field::transform<double>(cplx<double>*, int, bool, cudaStream_t);

template <typename R>
void Field::recip(const double2* X, double2* Y, int M, cudaStream_t s, const RealOverlap* ov) {
    grid_.ensure(grid_bytes(M, sizeof(R) == 8));
    if (spec_.kind == FIELD_POLY) poly_recip_on<R>(X, Y, M, grid_.as<cplx<R>>(), s);
    else recip_on<R>(X, Y, M, grid_.as<cplx<R>>(), s, ov);
}

size_t Field::grid_bytes(int M, bool fp64) const {
    const int C = spec_.kind == FIELD_POLY ? (Nq_ ? 6 : 1) : (Nq_ ? 8 : 3);
    return (fp64 ? sizeof(double2) : sizeof(float2)) * size_t(gv_.Nx) * gv_.Ny * gv_.Zs * size_t(C) * M;
}

// Reciprocal-space part on a caller-provided grid of grid_bytes(M) bytes.
template <typename R>
void Field::recip_on(const double2* X, double2* Y, int M, cplx<R>* grid, cudaStream_t s, const RealOverlap* ov) {
    const int C = Nq_ ? 8 : 3;
    const int B = C * M;
    // spread
    const PointSet& ps = sources_;
    const int TX = ps.tile[0], TY = ps.tile[1], TZ = ps.tile[2];
    const int bc = sizeof(R) == 4 ? 32 : 16;
    const int cap = 96;
    const size_t ncol = size_t(TX) * TY;
    const size_t shm = sizeof(R) * cap * (TX + TY + TZ) + sizeof(cplx<R>) * cap * bc +
                       (sizeof(R) + sizeof(int)) * ncol * kSpreadListCap + sizeof(int) * (ncol + cap);
    set_smem_limit(k_spread<R>, shm);
    const int nchunk = (B + bc - 1) / bc;
    dim3 grd(ps.nb[0], ps.nb[1], ps.nb[2] * nchunk);  // one CTA per tile and column chunk
    const R* w1 = sizeof(R) == 4 ? reinterpret_cast<const R*>(ps.w32.p) : reinterpret_cast<const R*>(ps.w64.p);
    Profiler::get().begin(ST_SPREAD, s);
    if (plan_cap_ > 0) {
        const size_t pshm = sizeof(cplx<R>) * size_t(plan_cap_) * bc;
        const bool f32 = sizeof(R) == 4;
        const R* wT = f32 ? reinterpret_cast<const R*>(plan_w32_.p) : reinterpret_cast<const R*>(plan_w64_.p);
        const R* lw = f32 ? reinterpret_cast<const R*>(plan_lw32_.p) : reinterpret_cast<const R*>(plan_lw64_.p);
        auto go = [&](auto kern) {
            set_smem_limit(kern, pshm);
            kern<<<grd, 256, pshm, s>>>(X, M, N_, C, quad_map_.as<int>(), gv_, TX, TY, TZ, ps.nb[0], ps.nb[1],
                                        ps.nb[2], plan_cap_, bc, plan_nc_.as<int>(), plan_cid_.as<int>(), wT, lw,
                                        plan_lc_.as<int>(), plan_ln_.as<int>(), grid);
        };
        // the tile's z run in registers: as many accumulators as it needs
        if (TZ == 1 && gv_.Zs == 1) {
            const size_t lshm = pshm + (sizeof(R) + sizeof(int)) * ncol * kSpreadListCap + sizeof(int) * ncol;
            set_smem_limit(k_spread_planned_1z<R>, lshm);
            k_spread_planned_1z<R><<<grd, 256, lshm, s>>>(X, M, N_, C, quad_map_.as<int>(), gv_, TX, TY, ps.nb[0],
                                                          ps.nb[1], plan_cap_, bc, plan_nc_.as<int>(),
                                                          plan_cid_.as<int>(), wT, lw, plan_lc_.as<int>(),
                                                          plan_ln_.as<int>(), grid);
        }
        else if (TZ <= 9) go(k_spread_planned<R, 9>);
        else go(k_spread_planned<R, kSpreadZMax>);
    } else {
        k_spread<R><<<grd, 256, shm, s>>>(X, M, N_, C, quad_map_.as<int>(), ps.base.as<int4>(), w1,
                                          ps.bin_start.as<int>(), ps.bin_end.as<int>(), ps.idx_sorted.as<int>(),
                                          gv_, TX, TY, TZ, ps.nb[0], ps.nb[1], ps.nb[2], cap, bc, grid);
    }
    MPM_LAUNCH();
    Profiler::get().end(ST_SPREAD, s);
    if (use_slab()) {
        // x forward; y forward, slab Green tensor and y inverse in one pass;
        // x inverse (the axis transforms commute)
        const size_t Bi = size_t(gv_.Zs) * B;
        const cplx<R>* taps = sizeof(R) == 4 ? reinterpret_cast<const cplx<R>*>(slabT32_.p)
                                             : reinterpret_cast<const cplx<R>*>(slabT64_.p);
        Profiler::get().begin(ST_FFT_FWD, s);
        fftx_.run<R>(grid, size_t(gv_.Ny) * Bi, int(Bi), Bi, gv_.Ny, false, s);
        Profiler::get().end(ST_FFT_FWD, s);
        Profiler::get().begin(ST_KSPACE, s);
        if (!(gv_.layer ? layer_taps_ : slab_Z_ == gv_.Zs) || !taps)
            throw std::runtime_error("slab taps not built for the current layout");
        ffty_.run_slab<R>(grid, gv_.Nx, gv_.Zs, M, taps, 2.0 * kPi / spec_.box[0], 2.0 * kPi / spec_.box[1], s);
        Profiler::get().end(ST_KSPACE, s);
        Profiler::get().begin(ST_FFT_INV, s);
        fftx_.run<R>(grid, size_t(gv_.Ny) * Bi, int(Bi), Bi, gv_.Ny, true, s);
        Profiler::get().end(ST_FFT_INV, s);
    } else {
        // forward transform
        Profiler::get().begin(ST_FFT_FWD, s);
        transform<R>(grid, B, false, s);
        Profiler::get().end(ST_FFT_FWD, s);
        Profiler::get().begin(ST_KSPACE, s);
        // k-space Green tensor
        if (gv_.pruned) {
            const int Z = gv_.Zs;
            const int nd = 2 * Z - 1;
            const size_t shm2 = sizeof(cplx<R>) * (size_t(Z) * B + 6 * nd);
            const int thr = std::min(1024, ((B + 31) / 32) * 32);
            const cplx<R>* K = sizeof(R) == 4 ? reinterpret_cast<const cplx<R>*>(colK32_.p)
                                              : reinterpret_cast<const cplx<R>*>(colK64_.p);
            if (!(gv_.layer ? layer_colK_ : colK_Z_ == gv_.Zs) || !K)
                throw std::runtime_error("column kernel not built for the current layout");
            auto go = [&](auto kern) {
                set_smem_limit(kern, shm2);
                kern<<<gv_.Nx * gv_.Ny, thr, shm2, s>>>(grid, K, Z, M);
            };
            if (Z <= 9) go(k_column<R, 9>);
            else if (Z <= 16) go(k_column<R, 16>);
            else go(k_column<R, 24>);
            MPM_LAUNCH();
        } else {
            const size_t V = size_t(gv_.Nx) * gv_.Ny * gv_.Zs;
            const R* sc = sizeof(R) == 4 ? reinterpret_cast<const R*>(scale32_.p) : reinterpret_cast<const R*>(scale64_.p);
            if (scale_built_ != (Nq_ ? 4 : 1) || !sc) throw std::runtime_error("k-space scale not built");
            if (Nq_)
                k_scale<R, true><<<nblk((long long)(V * M), 256), 256, 0, s>>>(grid, sc, gv_.Nx, gv_.Ny, gv_.Nz, spec_.box[0],
                                                                               spec_.box[1], spec_.box[2], M, spec_.bloch[0], spec_.bloch[1]);
            else
                k_scale<R, false><<<nblk((long long)(V * M), 256), 256, 0, s>>>(grid, sc, gv_.Nx, gv_.Ny, gv_.Nz, spec_.box[0],
                                                                                spec_.box[1], spec_.box[2], M, spec_.bloch[0], spec_.bloch[1]);
            MPM_LAUNCH();
        }
        Profiler::get().end(ST_KSPACE, s);
        Profiler::get().begin(ST_FFT_INV, s);
        transform<R>(grid, B, true, s);
        Profiler::get().end(ST_FFT_INV, s);
    }
    StageScope scope(ST_CONTRACT, s);
    // contract
    const PointSet& tg = spec_.solver_ax ? sources_ : targets_;
    const int nt = tg.n;
    const double factor = geom_.h[0] * geom_.h[1] * geom_.h[2];
    const R* tw = sizeof(R) == 4 ? reinterpret_cast<const R*>(tg.w32.p) : reinterpret_cast<const R*>(tg.w64.p);
    const int thr = std::min(256, ((B + 31) / 32) * 32);
    if (ov) MPM_CUDA(cudaStreamWaitEvent(s, ov->join, 0));   // the real-space part is in Y
    auto contract = [&](auto kern) {
        kern<<<nt, thr, 0, s>>>(grid, gv_, M, C, nt, tg.base.as<int4>(), tw, factor,
                                spec_.solver_ax ? quad_map_.as<int>() : nullptr, Y, 0,
                                spec_.solver_ax ? sources_.idx_sorted.as<int>() : nullptr, ov ? 1 : 0,
                                ov ? ov->jacobi_sc : nullptr);
    };
    if (gv_.Sz == 1 && C == 3 && B <= 16) {
        const int gsz = B <= 4 ? 4 : B <= 8 ? 8 : 16;
        const int per = 128 / gsz;
        auto small = [&](auto kern) {
            kern<<<nblk(nt, per), 128, 0, s>>>(grid, gv_, M, nt, tg.base.as<int4>(), tw, factor, Y, 0,
                                               spec_.solver_ax ? sources_.idx_sorted.as<int>() : nullptr,
                                               ov ? 1 : 0, ov ? ov->jacobi_sc : nullptr, gsz);
        };
        if (gv_.S == 9) small(k_contract_small<R, 9>);
        else small(k_contract_small<R, 0>);
    } else if (gv_.Sz == 1) {
        if (gv_.S == 9) contract(k_contract<R, 1, 9>);
        else contract(k_contract<R, 1, 0>);
    } else if (gv_.Sz <= 9) {
        if (gv_.S == 9) contract(k_contract<R, 9, 9>);
        else contract(k_contract<R, 9, 0>);
    } else if (gv_.Sz <= 13) {
        contract(k_contract<R, 13, 0>);
    } else {
        contract(k_contract<R, 0, 0>);
    }
    MPM_LAUNCH();
}

void Field::real_part(const double2* X, double2* Y, int M, const double2* sc, bool jacobi, bool fp32, bool add_recip,
                      cudaStream_t s) {
    RealArgs a;
    a.M = M;
    a.N = N_;
    a.Nt = num_targets();
    a.Nq = Nq_;
    a.selfo = tables_.selfo;
    a.self_grad = tables_.self_grad;
    a.solver_ax = spec_.solver_ax ? 1 : 0;
    a.jacobi = jacobi ? 1 : 0;
    a.add_recip = add_recip ? 1 : 0;
    a.quads = Nq_ > 0 ? 1 : 0;
    a.pairs_plus = spec_.kind == FIELD_POLY ? 1 : 0;
    a.qa2 = (spec_.kind == FIELD_POLY && Nq_) ? pqa2_.as<double>() : nullptr;
    a.qg2 = (spec_.kind == FIELD_POLY && Nq_) ? pqg2_.as<double>() : nullptr;
    const double* selfv = spec_.kind == FIELD_POLY ? pself_.as<double>() : nullptr;
    const int warps = a.Nt;
    const int thr = 128;
    const int blocks = nblk((long long)warps * 32, thr);
    StageScope scope(ST_REAL, s);
    const bool ph = bloch_on();
    if (ph && num_pairs_ > 0 && pair_ph64_.bytes < sizeof(double2) * size_t(num_pairs_))
        throw std::runtime_error("Bloch pair phases not built for the current pairs");
    auto go = [&](auto kern, const auto* T, const auto* P) {
        kern<<<blocks, thr, 0, s>>>(X, Y, a, pair_off_.as<int>(), pair_src_.as<int>(), T, pair_Q_.as<double>(),
                                    quad_map_.as<int>(), sc, selfv, P);
    };
    if (fp32) {
        const float2* P = ph ? pair_ph32_.as<float2>() : nullptr;
        if (a.quads) go(k_real<float, true>, pair_T32_.as<float>(), P);
        else go(k_real<float, false>, pair_T32_.as<float>(), P);
    } else {
        const double2* P = ph ? pair_ph64_.as<double2>() : nullptr;
        if (a.quads) go(k_real<double, true>, pair_T64_.as<double>(), P);
        else go(k_real<double, false>, pair_T64_.as<double>(), P);
    }
    MPM_LAUNCH();
}

void Field::direct(const double2* X, double2* Y, int M, const double2* sc, bool jacobi, bool fp32, cudaStream_t s) {
    const int nt = num_targets();
    const double* tg = spec_.solver_ax ? sources_.xyz.as<double>() : targets_.xyz.as<double>();
    dim3 grd(nblk(nt, 128), M);
    StageScope scope(ST_DIRECT, s);
    if (fp32)
        k_direct<float><<<grd, 128, 0, s>>>(X, Y, M, N_, nt, sources_.xyz.as<double>(), tg, radius_.as<double>(),
                                            quad_map_.as<int>(), Nq_ > 0, sc, spec_.solver_ax, jacobi);
    else
        k_direct<double><<<grd, 128, 0, s>>>(X, Y, M, N_, nt, sources_.xyz.as<double>(), tg, radius_.as<double>(),
                                             quad_map_.as<int>(), Nq_ > 0, sc, spec_.solver_ax, jacobi);
    MPM_LAUNCH();
}

void Field::apply(const double2* X, double2* Y, int M, const double2* sc, bool jacobi, bool recip_fp32,
                  bool real_fp32, cudaStream_t s) {
    if (N_ == 0) throw std::runtime_error("Field::apply before set_positions");
    if (!spec_.solver_ax && targets_.n == 0) throw std::runtime_error("Field::apply without field points");
    if (spec_.kind == FIELD_DIRECT) {
        direct(X, Y, M, sc, jacobi, recip_fp32, s);
        return;
    }
    if (spec_.kind == FIELD_MONO && spec_.solver_ax && Nq_ == 0) {
        // the real-space sum runs on a second stream while the reciprocal
        // chain (spread, transforms, k-space step) runs on s; it writes the
        // pairs and self terms into Y, and the contraction, after waiting
        // for it, adds the reciprocal part and applies the Jacobi scaling
        if (!aux_) {
            MPM_CUDA(cudaStreamCreateWithFlags(&aux_, cudaStreamNonBlocking));
            MPM_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
            MPM_CUDA(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
        }
        MPM_CUDA(cudaEventRecord(ev_fork_, s));
        MPM_CUDA(cudaStreamWaitEvent(aux_, ev_fork_, 0));
        real_part(X, Y, M, sc, false, real_fp32, false, aux_);
        MPM_CUDA(cudaEventRecord(ev_join_, aux_));
        const RealOverlap ov{ev_join_, jacobi ? sc : nullptr};
        if (recip_fp32) recip<float>(X, Y, M, s, &ov);
        else recip<double>(X, Y, M, s, &ov);
        return;
    }
    if (recip_fp32) recip<float>(X, Y, M, s);
    else recip<double>(X, Y, M, s);
    real_part(X, Y, M, sc, jacobi, real_fp32, true, s);
}

void Field::apply_scratch(const double2* X, double2* Y, int M, const double2* sc, bool jacobi, bool recip_fp32,
                          bool real_fp32, void* scratch, size_t scratch_bytes, cudaStream_t s) {
    if (N_ == 0) throw std::runtime_error("Field::apply before set_positions");
    if (!spec_.solver_ax && targets_.n == 0) throw std::runtime_error("Field::apply without field points");
    if (spec_.kind == FIELD_DIRECT) {
        direct(X, Y, M, sc, jacobi, recip_fp32, s);
        return;
    }
    if (!own_fft_) throw std::runtime_error("grid lines too long for the in-house transform; scratch apply unavailable");
    const size_t need = grid_bytes(M, !recip_fp32);
    if (need > scratch_bytes)
        throw std::invalid_argument("reciprocal grid needs " + std::to_string(need) + " bytes of scratch, " +
                                    std::to_string(scratch_bytes) + " available");
    if (spec_.kind == FIELD_POLY) {
        if (recip_fp32) poly_recip_on<float>(X, Y, M, static_cast<float2*>(scratch), s);
        else poly_recip_on<double>(X, Y, M, static_cast<double2*>(scratch), s);
    } else {
        if (recip_fp32) recip_on<float>(X, Y, M, static_cast<float2*>(scratch), s);
        else recip_on<double>(X, Y, M, static_cast<double2*>(scratch), s);
    }
    real_part(X, Y, M, sc, jacobi, real_fp32, true, s);
}

void Field::apply_part(const double2* X, double2* Y, int M, const double2* sc, bool recip_fp32, bool real_fp32,
                       int part, cudaStream_t s) {
    if (spec_.kind == FIELD_DIRECT) throw std::runtime_error("apply_part needs an Ewald field");
    if (part == 0) {  // reciprocal only (no self, no sign change)
        if (recip_fp32) recip<float>(X, Y, M, s);
        else recip<double>(X, Y, M, s);
    } else {          // real space + self only
        real_part(X, Y, M, sc, false, real_fp32, false, s);
    }
}

}  // namespace mpm
