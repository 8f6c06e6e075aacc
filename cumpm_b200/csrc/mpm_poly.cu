// Polydisperse spectral-Ewald dipole field (FIELD_POLY).
//
// Same operator as the reference's Polydisperse_Ewald_Electric_Field
// (electric_field/polydisperse_ewald_electric_field.cu) for dipoles:
//   spread   rho(v) = sum_i w_i(v) . p_i          (:189-263, :443-562)
//   FFT      forward, unnormalised                 (:2553-2690)
//   scale    rho^(k) *= exp(-(1-eta) k^2/4xi^2) / (k^2 V), 0 at k = 0 (:565-651)
//   FFT      inverse, unnormalised
//   contract E_j = h^3 sum_v w_j(v) phi(v)          (:265-350, :653-693)
//   real     self (s_i + self(a_i, a_i)) p_i and pairs T(r; a_i, a_j) p_i
//            within rc from per-radius-pair tables   (:352-441, :695-826)
// where w_i(v) is the 3-vector smoothed-sphere weight of particle i at the
// grid node v (radial profile times direction), P^3 nodes per particle.
//
// B200 layout and choices:
//  * The grid is scalar per right-hand side: [x][y][z][M] complex, so every
//    voxel's M columns are one coalesced vector.
//  * Spreading is a gather over 8^3 voxel tiles from spatial bins of the
//    stencil origins (no atomics, deterministic, every voxel written once).
//  * Contraction is one CTA per target, its warps splitting the P^3 nodes,
//    lanes over right-hand sides, a fixed-order reduction at the end.
//  * The reference tabulates the pair functions on r = 0, 1, 1.001, ... for
//    every pair of radius classes and interpolates linearly.  Here each
//    pair's value is that same interpolation, but the two table nodes it
//    reads are evaluated on the fly, so no table is stored: a continuous
//    radius distribution (one class per particle) costs nothing extra.
#include "mpm_bins.cuh"
#include "mpm_field.h"
#include "mpm_poly.cuh"
#include "mpm_profile.h"

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <set>

namespace mpm {

// ------------------------------------------------------------ parameters

PolyGeom make_poly_geom(const double box[3], double errortol, double xi, const std::vector<double>& radii,
                        const int* grid, int support) {
    if (radii.empty()) throw std::invalid_argument("polydisperse field needs one radius per particle");
    PolyGeom g;
    // radius classes: a radius joins an existing class within 1e-5, classes
    // are sorted, each particle takes the first sorted class within 1e-5
    std::set<double> seen;
    for (double r : radii) {
        bool found = false;
        for (auto it = seen.lower_bound(r - 1e-5); it != seen.end() && *it <= r + 1e-5; ++it)
            if (std::abs(*it - r) < 1e-5) { found = true; break; }
        if (!found) seen.insert(r);
    }
    g.unique.assign(seen.begin(), seen.end());
    g.cls.resize(radii.size());
    for (size_t i = 0; i < radii.size(); ++i) {
        const double r = radii[i];
        auto it = std::lower_bound(g.unique.begin(), g.unique.end(), r - 1e-5);
        while (it != g.unique.end() && !(std::abs(*it - r) < 1e-5)) ++it;
        if (it == g.unique.end()) throw std::runtime_error("radius class lookup failed");
        g.cls[i] = int(it - g.unique.begin());
    }
    double rc = std::sqrt(-std::log(errortol)) / xi;
    const double rc_min = 2.0 * g.unique.back();
    if (rc < rc_min) rc = rc_min;
    if (rc > box[0] / 2.0 || rc > box[1] / 2.0 || rc > box[2] / 2.0)
        throw std::runtime_error("Real space cutoff (" + std::to_string(rc) + ") larger than half the box length.");
    g.rc = rc;
    const double kcut = 2.0 * xi * xi * rc;
    for (int d = 0; d < 3; ++d) {
        g.ng[d] = static_cast<int>(std::ceil(1.0 + box[d] * kcut / kPi));
        if (grid && grid[d] > 0) g.ng[d] = grid[d];
        g.h[d] = box[d] / g.ng[d];
    }
    const double mean_h = (g.h[0] + g.h[1] + g.h[2]) / 3.0;
    g.P = static_cast<int>(std::ceil(2.0 / mean_h - 2.0 * std::log(errortol) / kPi));
    if (support > 0) g.P = support;
    g.eta = g.P * std::pow(mean_h * xi, 2.0) / kPi;
    g.off_min = -static_cast<int>(std::floor((g.P - 1) / 2.0));
    const double rc_val = rc < 1.001 ? 1.001 : rc;
    g.table_n = static_cast<int>(std::ceil((rc_val - 1.0) / 0.001)) + 1;
    return g;
}

// --------------------------------------------------------------- kernels

namespace {

inline int nblk(long long n, int b) { return int((n + b - 1) / b); }

struct PolyArgs {
    double h[3];
    int N[3];
    int P, off_min;
    double eta, xi;
};

// One thread per (point, support node): the smoothed-sphere weight vector
// (spread_precalcs_kernel_polydisperse, :189-263; the contraction weights of
// :265-350 are the same function).  Node order o = (ox*P + oy)*P + oz.
// base[i] = wrapped first node of the point's P^3 box (x, y, z, z).
__global__ void k_poly_weights(const double* __restrict__ xyz, int n, const double* __restrict__ rad, PolyArgs a,
                               int4* __restrict__ base, double* __restrict__ w64, float* __restrict__ w32) {
    const int P3 = a.P * a.P * a.P;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * P3) return;
    const int i = int(t / P3), o = int(t - (long long)i * P3);
    const int oo[3] = {o / (a.P * a.P), (o / a.P) % a.P, o % a.P};
    double gd[3];
    int g[3];
    for (int d = 0; d < 3; ++d) {
        const double p = xyz[size_t(d) * n + i];
        g[d] = static_cast<int>(round(p / a.h[d]));
        const double d0 = g[d] * a.h[d] - p;
        gd[d] = d0 + double(a.off_min + oo[d]) * a.h[d];
    }
    if (o == 0)
        base[i] = make_int4(pmod(g[0] + a.off_min, a.N[0]), pmod(g[1] + a.off_min, a.N[1]),
                            pmod(g[2] + a.off_min, a.N[2]), pmod(g[2] + a.off_min, a.N[2]));
    const double dist = sqrt(gd[0] * gd[0] + gd[1] * gd[1] + gd[2] * gd[2]);
    const double ai = rad[i];
    const double x2 = a.xi * a.xi;
    double w[3];
    if (dist >= 1e-6) {
        const double k = 3.0 / (8.0 * sqrt(2.0) * pow(kPi, 1.5) * pow(ai, 3.0) * sqrt(a.eta) * a.xi * dist * dist);
        const double tp = (a.eta + 4.0 * ai * x2 * dist) * exp(-2.0 * pow(dist + ai, 2) * x2 / a.eta);
        const double tm = (a.eta - 4.0 * ai * x2 * dist) * exp(-2.0 * pow(dist - ai, 2) * x2 / a.eta);
        const double cs = k * (tp - tm);
        for (int d = 0; d < 3; ++d) w[d] = cs * (gd[d] / dist);
    } else {
        const double kn = 8.0 * sqrt(2.0) * pow(a.xi, 5.0) * exp(-2.0 * ai * x2 / a.eta) /
                          (pow(kPi, 1.5) * pow(a.eta, 2.5));
        for (int d = 0; d < 3; ++d) w[d] = kn * gd[d];
    }
    for (int d = 0; d < 3; ++d) {
        w64[size_t(t) * 3 + d] = w[d];
        w32[size_t(t) * 3 + d] = static_cast<float>(w[d]);
    }
}

struct PolyTile {
    int N[3];
    int P;
    int T;        // tile edge (voxels)
    int nb[3];    // bins per dimension
    int cap;      // candidate capacity of the shared list
};

// Candidate particles of tile (bx, by, bz): those binned (by stencil origin)
// in the bins that can hold an origin within P-1 voxels below the tile.
__device__ int poly_tile_bins(const PolyTile& t, int bx, int by, int bz, int (&bxs)[8], int (&bys)[8], int (&bzs)[8],
                              int nbv[3]) {
    nbv[0] = reach_bins(bx * t.T - t.P + 1, bx * t.T + t.T - 1, t.N[0], t.T, true, bxs);
    nbv[1] = reach_bins(by * t.T - t.P + 1, by * t.T + t.T - 1, t.N[1], t.T, true, bys);
    nbv[2] = reach_bins(bz * t.T - t.P + 1, bz * t.T + t.T - 1, t.N[2], t.T, true, bzs);
    return nbv[0] * nbv[1] * nbv[2];
}

// Candidate lists of the spread tiles, built once per frame: pass 0 counts
// (and keeps the largest count), pass 1 writes each tile's list in bin
// order at its CSR offset.
__global__ void k_poly_cands(PolyTile t, const int* __restrict__ bin_start, const int* __restrict__ bin_end,
                             const int* __restrict__ idx_sorted, int pass, int* __restrict__ cnt,
                             int* __restrict__ maxc, const int* __restrict__ off, int* __restrict__ list) {
    const int tile = blockIdx.x * blockDim.x + threadIdx.x;
    const int ntile = t.nb[0] * t.nb[1] * t.nb[2];
    if (tile >= ntile) return;
    const int bx = tile % t.nb[0], by = (tile / t.nb[0]) % t.nb[1], bz = tile / (t.nb[0] * t.nb[1]);
    int xs[8], ys[8], zs[8], nbv[3];
    poly_tile_bins(t, bx, by, bz, xs, ys, zs, nbv);
    int c = 0;
    int* out = pass ? list + off[tile] : nullptr;
    for (int k = 0; k < nbv[2]; ++k)
        for (int j = 0; j < nbv[1]; ++j)
            for (int i = 0; i < nbv[0]; ++i) {
                const int b = (zs[k] * t.nb[1] + ys[j]) * t.nb[0] + xs[i];
                if (bin_start[b] < 0) continue;
                if (pass)
                    for (int q = bin_start[b]; q < bin_end[b]; ++q) out[c++] = idx_sorted[q];
                else
                    c += bin_end[b] - bin_start[b];
            }
    if (!pass) {
        cnt[tile] = c;
        atomicMax(maxc, c);
    }
}

// Covered runs of every tile candidate, built once per frame (thread per
// tile, candidates in list order).  The support index along an axis is
// k = (t0 + u - origin) mod N and a tile offset u is covered when k < P;
// within a covered run k grows by one per voxel (P < N, so a wrap would pass
// N-1 >= P, which is not covered): at most two runs per axis.  Run word:
// u | len << 4 | k << 8; word 6 holds the run counts (2 bits per axis).
// Candidates that miss the tile along an axis are dropped, the others keep
// their order (so each voxel's sum keeps its order): cnt[tile] of them at the
// tile's CSR offset in clist / 8 words each in cruns.
__global__ void k_poly_runs(PolyTile t, const int4* __restrict__ base, const int* __restrict__ off,
                            const int* __restrict__ list, int* __restrict__ cnt, int* __restrict__ clist,
                            int* __restrict__ cruns) {
    const int tile = blockIdx.x * blockDim.x + threadIdx.x;
    const int ntile = t.nb[0] * t.nb[1] * t.nb[2];
    if (tile >= ntile) return;
    const int bx = tile % t.nb[0], by = (tile / t.nb[0]) % t.nb[1], bz = tile / (t.nb[0] * t.nb[1]);
    const int t0[3] = {bx * 8, by * 8, bz * 8};
    const int c0 = off[tile], c1 = off[tile + 1];
    int kept = 0;
    for (int c = c0; c < c1; ++c) {
        const int i = list[c];
        const int4 o = base[i];
        const int org[3] = {o.x, o.y, o.z};
        int w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        bool all = true;
        for (int d = 0; d < 3; ++d) {
            int nr = 0, open = 0, r0 = 0, r1 = 0;
            int k = pmod(t0[d] - org[d], t.N[d]);
            for (int u = 0; u < 8; ++u) {
                const int cov = (t0[d] + u < t.N[d]) && k < t.P;
                if (cov && open) {
                    if (nr == 1) r0 += 1 << 4; else r1 += 1 << 4;
                } else if (cov && nr < 2) {
                    const int word = u | (1 << 4) | (k << 8);
                    if (nr == 0) r0 = word; else r1 = word;
                    ++nr;
                    open = 1;
                } else {
                    open = 0;
                }
                k = k + 1 == t.N[d] ? 0 : k + 1;
            }
            w[2 * d] = r0;
            w[2 * d + 1] = r1;
            w[6] |= nr << (2 * d);
            all = all && nr > 0;
        }
        if (!all) continue;
        clist[c0 + kept] = i;
        for (int q = 0; q < 8; ++q) cruns[size_t(c0 + kept) * 8 + q] = w[q];
        ++kept;
    }
    cnt[tile] = kept;
}

// Spread onto one 8^3 voxel tile x CM consecutive columns per CTA.  The
// tile's accumulators live in shared memory; the tile's candidate particles
// are added one after another in candidate order, all threads sharing the
// (covered voxel, column) pairs of the current particle, with a barrier
// between particles.  So every voxel's sum has a fixed order, there are no
// atomics, and every voxel of the grid is written exactly once.
// grid[((x*Ny+y)*Nz+z)*M + m].
template <typename R, int CM>
__global__ void __launch_bounds__(256) k_poly_spread(const double2* __restrict__ X, int M, const R* __restrict__ w,
                                                     const int* __restrict__ toff, const int* __restrict__ tcnt,
                                                     const int* __restrict__ clist, const int* __restrict__ cruns,
                                                     PolyTile t, cplx<R>* __restrict__ grid) {
    extern __shared__ __align__(16) unsigned char shraw[];
    cplx<R>* acc = reinterpret_cast<cplx<R>*>(shraw);              // [512][CM] tile accumulators
    cplx<R>* pm = acc + 512 * CM;                                 // [cap][3][CM] candidate moments
    int* runs = reinterpret_cast<int*>(pm + size_t(t.cap) * 3 * CM);  // [cap][8] covered runs
    int* cand = runs + 8 * t.cap;                                 // [cap] particle index
    // the column blocks of one tile are adjacent in launch order, so the
    // candidates' weights are read from DRAM once and then hit in L2
    const int ncb = (M + CM - 1) / CM;
    const int tile = blockIdx.x / ncb;
    const int m0 = (blockIdx.x - tile * ncb) * CM;
    const int bx = tile % t.nb[0], by = (tile / t.nb[0]) % t.nb[1], bz = tile / (t.nb[0] * t.nb[1]);
    const int t0[3] = {bx * 8, by * 8, bz * 8};
    const int c0 = toff[tile];
    const int nc = min(tcnt[tile], t.cap);
    const int P = t.P, P3 = P * P * P;
    // the tile's covering candidates and their runs (k_poly_runs)
    for (int c = threadIdx.x; c < nc; c += blockDim.x) cand[c] = clist[c0 + c];
    for (int q = threadIdx.x; q < nc * 8; q += blockDim.x) runs[q] = cruns[size_t(c0) * 8 + q];
    for (int k = threadIdx.x; k < nc * 3 * CM; k += blockDim.x) {
        const int cm = k % CM, comp = (k / CM) % 3, c = k / (3 * CM);
        const int m = m0 + cm;
        pm[k] = m < M ? to_r<R>(X[size_t(3 * clist[c0 + c] + comp) * M + m]) : mk<R>(0, 0);
    }
    for (int k = threadIdx.x; k < 512 * CM; k += blockDim.x) acc[k] = mk<R>(0, 0);
    __syncthreads();
    const int cm = threadIdx.x % CM;            // this thread's column
    const int slot = threadIdx.x / CM;          // and voxel slot
    constexpr int NSLOT = 256 / CM;
    for (int c = 0; c < nc; ++c) {
        const int* rr = runs + c * 8;
        const int nrs = rr[6];
        // a candidate that misses the tile along some axis adds nothing (the
        // branch is uniform across the CTA, so its barrier goes too)
        if (!(nrs & 3) || !(nrs & 12) || !(nrs & 48)) continue;
        const cplx<R> p0 = pm[(c * 3 + 0) * CM + cm], p1 = pm[(c * 3 + 1) * CM + cm], p2 = pm[(c * 3 + 2) * CM + cm];
        const R* wi = w + size_t(cand[c]) * P3 * 3;
        for (int ax = 0; ax < (nrs & 3); ++ax)
            for (int ay = 0; ay < ((nrs >> 2) & 3); ++ay)
                for (int az = 0; az < ((nrs >> 4) & 3); ++az) {
                    const int qx = rr[ax], qy = rr[2 + ay], qz = rr[4 + az];
                    const int lx = (qx >> 4) & 15, ly = (qy >> 4) & 15, lz = (qz >> 4) & 15;
                    // slot = one (x, y) row of the covered box; its z run is
                    // contiguous in both the accumulators and the weights
                    for (int r = slot; r < lx * ly; r += NSLOT) {
                        const int ix = r / ly, iy = r - ix * ly;
                        const int ux = (qx & 15) + ix, uy = (qy & 15) + iy;
                        const int kx = (qx >> 8) + ix, ky = (qy >> 8) + iy;
                        const R* wp = wi + ((kx * P + ky) * P + (qz >> 8)) * 3;
                        cplx<R>* ap = acc + ((ux * 8 + uy) * 8 + (qz & 15)) * CM + cm;
                        for (int iz = 0; iz < lz; ++iz, wp += 3, ap += CM)
                            *ap += p0 * wp[0] + p1 * wp[1] + p2 * wp[2];
                    }
                }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < 512 * CM; k += blockDim.x) {
        const int kc = k % CM, v = k / CM;
        const int x = t0[0] + (v >> 6), y = t0[1] + ((v >> 3) & 7), z = t0[2] + (v & 7);
        const int m = m0 + kc;
        if (m < M && x < t.N[0] && y < t.N[1] && z < t.N[2])
            grid[((size_t(x) * t.N[1] + y) * t.N[2] + z) * M + m] = acc[k];
    }
}

// (bx, by): Bloch wavevector, the scale taken at k - b
__global__ void k_poly_build_scale(int Nx, int Ny, int Nz, double Lx, double Ly, double Lz, double xi, double eta,
                                   double bx, double by, double* __restrict__ s64, float* __restrict__ s32) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long V = (long long)Nx * Ny * Nz;
    if (t >= V) return;
    const int ix = int(t / ((long long)Ny * Nz)), iy = int((t / Nz) % Ny), iz = int(t % Nz);
    const double fx = ix <= (Nx - 1) / 2 ? ix : ix - Nx;
    const double fy = iy <= (Ny - 1) / 2 ? iy : iy - Ny;
    const double fz = iz <= (Nz - 1) / 2 ? iz : iz - Nz;
    const double kx = fx * 2.0 * kPi / Lx - bx, ky = fy * 2.0 * kPi / Ly - by, kz = fz * 2.0 * kPi / Lz;
    const double k2 = kx * kx + ky * ky + kz * kz;
    double v = 0.0;
    if (!(k2 < 1e-12)) v = (exp(-(1.0 - eta) * k2 / (4.0 * xi * xi)) / k2) * (1.0 / double(V));
    s64[t] = v;
    s32[t] = static_cast<float>(v);
}

template <typename R>
__global__ void k_poly_scale(cplx<R>* __restrict__ grid, const R* __restrict__ sc, long long n, int M) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    grid[t] = grid[t] * sc[t / M];
}

// Contraction.  CTA = one target x one block of up to 32*MC columns; its
// CW warps take every CW-th support node (unrolled so several grid loads are
// in flight), lanes over columns, then a fixed-order sum over the warps.
// Y rows 3j+c, already scaled by h^3.
template <typename R, int MC>
__global__ void __launch_bounds__(256) k_poly_contract(const cplx<R>* __restrict__ grid, int M,
                                                       const int4* __restrict__ base, const R* __restrict__ w, int P,
                                                       int Nx, int Ny, int Nz, double factor,
                                                       double2* __restrict__ Y) {
    constexpr int CW = 8;
    __shared__ cplx<R> red[CW][3][32];
    const int j = blockIdx.x;
    const int m0 = blockIdx.y * 32 * MC;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int P3 = P * P * P;
    const int4 o = base[j];
    cplx<R> acc[3][MC];
#pragma unroll
    for (int q = 0; q < MC; ++q) acc[0][q] = acc[1][q] = acc[2][q] = mk<R>(0, 0);
    // warp = (x, y) rows of the support (P < N, so a coordinate wraps at
    // most once); each row's z run is contiguous in the weights and, up to
    // one wrap, in the grid
    for (int r = warp; r < P * P; r += CW) {
        const int kx = r / P, ky = r - kx * P;
        int x = o.x + kx, y = o.y + ky;
        if (x >= Nx) x -= Nx;
        if (y >= Ny) y -= Ny;
        const size_t rowbase = (size_t(x) * Ny + y) * Nz;
        const R* wp = w + (size_t(j) * P3 + size_t(r) * P) * 3;
        int z = o.z;
#pragma unroll 4
        for (int kz = 0; kz < P; ++kz) {
            const size_t vo = (rowbase + z) * M;
            const R w0 = wp[3 * kz], w1 = wp[3 * kz + 1], w2 = wp[3 * kz + 2];
#pragma unroll
            for (int q = 0; q < MC; ++q) {
                const int m = m0 + q * 32 + lane;
                if (m < M) {
                    const cplx<R> g = grid[vo + m];
                    acc[0][q] += g * w0;
                    acc[1][q] += g * w1;
                    acc[2][q] += g * w2;
                }
            }
            z = z + 1 == Nz ? 0 : z + 1;
        }
    }
#pragma unroll
    for (int q = 0; q < MC; ++q) {
        for (int c = 0; c < 3; ++c) red[warp][c][lane] = acc[c][q];
        __syncthreads();
        if (warp == 0) {
            const int m = m0 + q * 32 + lane;
            if (m < M) {
                for (int c = 0; c < 3; ++c) {
                    cplx<R> s = red[0][c][lane];
                    for (int q2 = 1; q2 < CW; ++q2) s += red[q2][c][lane];
                    const double2 d = to_d(s);
                    Y[size_t(3 * j + c) * M + m] = make_double2(d.x * factor, d.y * factor);
                }
            }
        }
        __syncthreads();
    }
}

// Per pair: delta = r / max(d, 1e-6) and the pair-table values of the two
// radius classes at max(d, 1e-6) (real_space_precalcs_kernel_polydisperse,
// :352-441).  Thread per target; a target index past the particles takes
// class 0 (:407).  Same layout as the monodisperse pair coefficients.
__global__ void k_poly_pair_coefs(const double* __restrict__ pgeo, const int* __restrict__ off,
                                  const int* __restrict__ src, int nt, int N, const int* __restrict__ cls,
                                  const double* __restrict__ rad, double xi, int table_n, double* __restrict__ T64,
                                  float* __restrict__ T32) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nt) return;
    const int cj = j < N ? cls[j] : 0;
    for (int p = off[j]; p < off[j + 1]; ++p) {
        const int ci = cls[src[p]];
        const double a = rad[min(ci, cj)], b = rad[max(ci, cj)];
        const double d = pgeo[4 * size_t(p) + 3];
        const double de = d < 1e-6 ? 1e-6 : d;
        const double dx = pgeo[4 * size_t(p)] / de, dy = pgeo[4 * size_t(p) + 1] / de, dz = pgeo[4 * size_t(p) + 2] / de;
        double perp, para;
        poly::table_lookup(de, a, b, xi, table_n, perp, para);
        double* t = T64 + 8 * size_t(p);
        t[0] = dx; t[1] = dy; t[2] = dz; t[3] = perp; t[4] = para; t[5] = t[6] = t[7] = 0.0;
        float* f = T32 + 8 * size_t(p);
        f[0] = float(dx); f[1] = float(dy); f[2] = float(dz); f[3] = float(perp); f[4] = float(para);
        f[5] = f[6] = f[7] = 0.f;
    }
}

// Reference table lookup with n nodes 0, 1, 1.001, ...
// (interpolate_table_gpu_polydisperse, :161-187).
__device__ double poly_table_at(double r, const double* __restrict__ rt, const double* __restrict__ y, int n) {
    if (r <= 0.0) return y[0];
    if (r >= rt[n - 1]) return y[n - 1];
    if (r < 1.0) return y[0] * (1.0 - r) + y[1] * r;
    const size_t k = 1 + static_cast<size_t>((r - 1.0) / kTableDr);
    if (k >= size_t(n - 1)) return y[n - 1];
    const double t = (r - rt[k]) / (rt[k + 1] - rt[k]);
    return y[k] * (1.0 - t) + y[k + 1] * t;
}

// Quadrupole pair coefficients: the seven radius-1 quadrupole tables at
// max(d, 1e-6) (real_space_precalcs_kernel_polydisperse, :421-429).  Same
// per-pair layout as the monodisperse Q[8] = {Q1,Q2,Q3,G1,G2,G3,G4,0}.
__global__ void k_poly_pair_quad(const double* __restrict__ pgeo, long long np, const double* __restrict__ qtab,
                                 int qn, double* __restrict__ Q) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const double d = pgeo[4 * p + 3];
    const double de = d < 1e-6 ? 1e-6 : d;
    double* qq = Q + 8 * p;
    for (int k = 0; k < 7; ++k) qq[k] = poly_table_at(de, qtab, qtab + size_t(k + 1) * qn, qn);
    qq[7] = 0.0;
}

// Point-Gaussian weight of the quadrupole grids per (point, support node):
// c exp(-2 xi^2 |g|^2) with c = (2 xi^2/pi)^1.5 h^3
// (spread_precalcs_kernel_point / contract_precalcs_kernel_point, :828-922;
// the constant from :2145).  Node order as k_poly_weights.
__global__ void k_poly_point_weights(const double* __restrict__ xyz, int n, PolyArgs a, double c,
                                     double* __restrict__ w64, float* __restrict__ w32) {
    const int P3 = a.P * a.P * a.P;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * P3) return;
    const int i = int(t / P3), o = int(t - (long long)i * P3);
    const int oo[3] = {o / (a.P * a.P), (o / a.P) % a.P, o % a.P};
    double d2 = 0.0;
    for (int d = 0; d < 3; ++d) {
        const double p = xyz[size_t(d) * n + i];
        const int g = static_cast<int>(round(p / a.h[d]));
        const double gd = (g * a.h[d] - p) + double(a.off_min + oo[d]) * a.h[d];
        d2 += gd * gd;
    }
    const double w = c * exp(-2.0 * a.xi * a.xi * d2);
    w64[t] = w;
    w32[t] = static_cast<float>(w);
}

// Quadrupole grids, five planes gq[c][V][M]: quadrupole q adds Q_qc w_o on
// the support of particle q (spread_quadrupoles_kernel_polydisperse,
// :964-1087, indexes the particle stencils by q, which is particle
// quad_idxs[q] only when every particle carries a quadrupole).  Thread per
// (quadrupole, node), atomics: the quadrupole grids are zeroed first.
template <typename R>
__global__ void k_poly_quad_spread(const double2* __restrict__ X, int M, int N, int Nq,
                                   const int4* __restrict__ base, const R* __restrict__ w, int P, int Nx, int Ny,
                                   int Nz, cplx<R>* __restrict__ gq) {
    const int P3 = P * P * P;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)Nq * P3) return;
    const int q = int(t / P3), o = int(t - (long long)q * P3);
    if (q >= N) return;   // more quadrupoles than particle stencils: nothing to spread on
    const int4 b = base[q];
    // P < N along every axis, so a coordinate wraps at most once
    int x = b.x + o / (P * P), y = b.y + (o / P) % P, z = b.z + o % P;
    if (x >= Nx) x -= Nx;
    if (y >= Ny) y -= Ny;
    if (z >= Nz) z -= Nz;
    const size_t V = size_t(Nx) * Ny * Nz;
    const size_t v = (size_t(x) * Ny + y) * Nz + z;
    const R wo = w[size_t(q) * P3 + o];
    for (int c = 0; c < 5; ++c)
        for (int m = 0; m < M; ++m) {
            const cplx<R> qv = to_r<R>(X[size_t(3 * N + 5 * q + c) * M + m]) * wo;
            R* dst = reinterpret_cast<R*>(gq + (size_t(c) * V + v) * M + m);
            atomicAdd(dst, qv.x);
            atomicAdd(dst + 1, qv.y);
        }
}

// Joint k-space step of the dipole grid phi and the quadrupole grids G_c
// (compute_scale_coefficients_polydisperse_kernel, :565-638, and
// scale_kernel_joint_polydisperse, :925-962).  With e = exp(-(1-eta) k^2 /
// 4 xi^2) / V and gdot = sum_c qd_c G_c:
//   phi <- (e/k^2) phi - (e/2) gdot,   G_c <- qf_c (-e phi + (e k^2/2) gdot),
// all zero at k = 0; the coefficients are rounded to R as stored there.
template <typename R>
__global__ void k_poly_quad_scale(cplx<R>* __restrict__ grid, cplx<R>* __restrict__ gq, int M, int Nx, int Ny,
                                  int Nz, double Lx, double Ly, double Lz, double xi, double eta) {
    const long long V = (long long)Nx * Ny * Nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= V) return;
    const int ix = int(t / ((long long)Ny * Nz)), iy = int((t / Nz) % Ny), iz = int(t % Nz);
    const double fx = ix <= (Nx - 1) / 2 ? ix : ix - Nx;
    const double fy = iy <= (Ny - 1) / 2 ? iy : iy - Ny;
    const double fz = iz <= (Nz - 1) / 2 ? iz : iz - Nz;
    const double kx = fx * 2.0 * kPi / Lx, ky = fy * 2.0 * kPi / Ly, kz = fz * 2.0 * kPi / Lz;
    const double k2 = kx * kx + ky * ky + kz * kz;
    double sc = 0.0, sQ = 0.0, sGP = 0.0, sGQ = 0.0;
    double qf[5] = {0, 0, 0, 0, 0}, qd[5] = {0, 0, 0, 0, 0};
    if (!(k2 < 1e-12)) {
        const double e = exp(-(1.0 - eta) * k2 / (4.0 * xi * xi));
        const double inv = 1.0 / double(V);
        sc = (e / k2) * inv;
        sQ = (-0.5 * e) * inv;
        sGP = e * inv;
        sGQ = (-0.5 * e * k2) * inv;
        const double km = sqrt(k2);
        const double h0 = kx / km, h1 = ky / km, h2 = kz / km;
        qf[0] = h0 * h0 - 1.0 / 3.0; qf[1] = h0 * h1; qf[2] = h0 * h2; qf[3] = h1 * h1 - 1.0 / 3.0; qf[4] = h1 * h2;
        qd[0] = h0 * h0 - h2 * h2; qd[1] = 2.0 * h0 * h1; qd[2] = 2.0 * h0 * h2; qd[3] = h1 * h1 - h2 * h2;
        qd[4] = 2.0 * h1 * h2;
    }
    const R rsc = R(sc), rsQ = R(sQ), rsGP = R(sGP), rsGQ = R(sGQ);
    for (int m = 0; m < M; ++m) {
        const cplx<R> e = grid[size_t(t) * M + m];
        cplx<R> gd = mk<R>(0, 0);
        for (int c = 0; c < 5; ++c) gd += gq[(size_t(c) * V + t) * M + m] * R(qd[c]);
        grid[size_t(t) * M + m] = e * rsc + gd * rsQ;
        const cplx<R> G = e * (-rsGP) - gd * rsGQ;
        for (int c = 0; c < 5; ++c) gq[(size_t(c) * V + t) * M + m] = G * R(qf[c]);
    }
}

// G at the quadrupole particles: the sum over the support of particle
// quad_idxs[q] of w_o G_c (contract_kernel_G_polydisperse and
// copy_G_to_E_kernel_polydisperse, :1090-1146; no h^3 factor, the point
// weights carry it).  CTA per quadrupole, threads over the support nodes,
// fixed-order tree sum per column.  Y rows 3*Nt + 5q + c; rows of a
// quadrupole whose particle index is out of range are zero.
template <typename R>
__global__ void __launch_bounds__(128) k_poly_quad_contract(const cplx<R>* __restrict__ gq, int M,
                                                            const int4* __restrict__ base, const R* __restrict__ w,
                                                            int P, int Nx, int Ny, int Nz,
                                                            const int* __restrict__ qidx, int Nt,
                                                            double2* __restrict__ Y) {
    __shared__ double2 red[5][128];
    const int q = blockIdx.x;
    const int i = qidx[q];
    if (i < 0 || i >= Nt) {   // uniform across the CTA
        for (int k = threadIdx.x; k < 5 * M; k += blockDim.x)
            Y[size_t(3 * Nt + 5 * q + k / M) * M + (k % M)] = make_double2(0.0, 0.0);
        return;
    }
    const int P3 = P * P * P;
    const size_t V = size_t(Nx) * Ny * Nz;
    const int4 b = base[i];
    for (int m = 0; m < M; ++m) {
        double2 acc[5];
        for (int c = 0; c < 5; ++c) acc[c] = make_double2(0.0, 0.0);
        for (int o = threadIdx.x; o < P3; o += blockDim.x) {
            int x = b.x + o / (P * P), y = b.y + (o / P) % P, z = b.z + o % P;
            if (x >= Nx) x -= Nx;
            if (y >= Ny) y -= Ny;
            if (z >= Nz) z -= Nz;
            const size_t v = (size_t(x) * Ny + y) * Nz + z;
            const R wo = w[size_t(i) * P3 + o];
            for (int c = 0; c < 5; ++c) acc[c] += to_d(gq[(size_t(c) * V + v) * M + m] * wo);
        }
        for (int c = 0; c < 5; ++c) red[c][threadIdx.x] = acc[c];
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h)
                for (int c = 0; c < 5; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x < 5) Y[size_t(3 * Nt + 5 * q + threadIdx.x) * M + m] = red[threadIdx.x][0];
        __syncthreads();
    }
}

}  // namespace

// ------------------------------------------------------------------ host

void Field::poly_init() {
    if (spec_.quads && !spec_.solver_ax)
        throw std::runtime_error("polydisperse quadrupoles are computed at the particles (SOLVER_AX) only");
    pgeom_ = make_poly_geom(spec_.box, spec_.errortol, spec_.xi, spec_.radius, spec_.grid, spec_.support);
    geom_ = EwaldGeom{};
    geom_.rc = pgeom_.rc;
    for (int d = 0; d < 3; ++d) {
        geom_.ng[d] = pgeom_.ng[d];
        geom_.h[d] = pgeom_.h[d];
    }
    const int n = int(spec_.radius.size());
    const int nu = int(pgeom_.unique.size());
    std::vector<double> selfv(n);
    std::vector<double> cself(nu);
    for (int k = 0; k < nu; ++k) cself[k] = poly::self_value(pgeom_.unique[k], pgeom_.unique[k], spec_.xi);
    for (int i = 0; i < n; ++i) selfv[i] = cself[pgeom_.cls[i]];
    pcls_.ensure(sizeof(int) * n);
    prad_.ensure(sizeof(double) * nu);
    pself_.ensure(sizeof(double) * n);
    radius_.ensure(sizeof(double) * n);
    MPM_CUDA(cudaMemcpy(pcls_.p, pgeom_.cls.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    MPM_CUDA(cudaMemcpy(prad_.p, pgeom_.unique.data(), sizeof(double) * nu, cudaMemcpyHostToDevice));
    MPM_CUDA(cudaMemcpy(pself_.p, selfv.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    MPM_CUDA(cudaMemcpy(radius_.p, spec_.radius.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    if (spec_.quads) {
        const int qn = pgeom_.table_n;
        const auto QT = build_poly_quad_tables(spec_.xi, qn);
        pqtab_.ensure(sizeof(double) * 8 * size_t(qn));
        MPM_CUDA(cudaMemcpy(pqtab_.p, QT.r.data(), sizeof(double) * qn, cudaMemcpyHostToDevice));
        for (int f = 0; f < PQ_COUNT; ++f)
            MPM_CUDA(cudaMemcpy(pqtab_.as<double>() + size_t(f + 1) * qn, QT.f[f].data(), sizeof(double) * qn,
                                cudaMemcpyHostToDevice));
        // a from the particle, the self value from its radius class (:1171-1177)
        std::vector<double> a2(n), g2(n);
        for (int i = 0; i < n; ++i) {
            a2[i] = spec_.radius[i] * spec_.radius[i];
            g2[i] = poly_quad_self_value(pgeom_.unique[pgeom_.cls[i]], spec_.xi);
        }
        pqa2_.ensure(sizeof(double) * n);
        pqg2_.ensure(sizeof(double) * n);
        MPM_CUDA(cudaMemcpy(pqa2_.p, a2.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        MPM_CUDA(cudaMemcpy(pqg2_.p, g2.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    }
    gv_.Nx = pgeom_.ng[0];
    gv_.Ny = pgeom_.ng[1];
    gv_.Nz = pgeom_.ng[2];
    gv_.Zs = gv_.Nz;
    gv_.z0 = 0;
    gv_.pruned = 0;
    gv_.off = 0;
    gv_.S = pgeom_.P;
    gv_.Sz = gv_.S;
    gv_.offz = 0;
    gv_.layer = 0;
    if (gv_.Nx < 16 || gv_.Ny < 16 || gv_.Nz < 16 || pgeom_.P >= std::min(gv_.Nx, std::min(gv_.Ny, gv_.Nz)))
        throw std::runtime_error("polydisperse grid shorter than 16 points or than the support along an axis");
    poly_build_scale();
    own_fft_ = AxisFFT::fits(gv_.Nx, true) && AxisFFT::fits(gv_.Ny, true) && AxisFFT::fits(gv_.Nz, true);
    if (own_fft_) {
        fftx_.init(gv_.Nx);
        ffty_.init(gv_.Ny);
        fftz_.init(gv_.Nz);
    }
}

void Field::poly_build_scale() {
    const size_t V = size_t(gv_.Nx) * gv_.Ny * gv_.Nz;
    scale64_.ensure(sizeof(double) * V);
    scale32_.ensure(sizeof(float) * V);
    k_poly_build_scale<<<nblk((long long)V, 256), 256>>>(gv_.Nx, gv_.Ny, gv_.Nz, spec_.box[0], spec_.box[1],
                                                         spec_.box[2], spec_.xi, pgeom_.eta, spec_.bloch[0],
                                                         spec_.bloch[1], scale64_.as<double>(), scale32_.as<float>());
    MPM_LAUNCH();
    MPM_CUDA(cudaDeviceSynchronize());
}

void Field::poly_weights(PointSet& ps, const double* radius_dev, cudaStream_t s, bool bins) {
    const int n = ps.n;
    const int P3 = pgeom_.P * pgeom_.P * pgeom_.P;
    ps.base.ensure(sizeof(int4) * n);
    ps.w64.ensure(sizeof(double) * size_t(n) * P3 * 3);
    ps.w32.ensure(sizeof(float) * size_t(n) * P3 * 3);
    PolyArgs a;
    for (int d = 0; d < 3; ++d) { a.h[d] = pgeom_.h[d]; a.N[d] = pgeom_.ng[d]; }
    a.P = pgeom_.P;
    a.off_min = pgeom_.off_min;
    a.eta = pgeom_.eta;
    a.xi = spec_.xi;
    k_poly_weights<<<nblk((long long)n * P3, 256), 256, 0, s>>>(ps.xyz.as<double>(), n, radius_dev, a,
                                                                 ps.base.as<int4>(), ps.w64.as<double>(),
                                                                 ps.w32.as<float>());
    MPM_LAUNCH();
    if (!bins) return;
    for (int d = 0; d < 3; ++d) {
        ps.tile[d] = 8;
        ps.nb[d] = (pgeom_.ng[d] + 7) / 8;
    }
    const int nbins = ps.nb[0] * ps.nb[1] * ps.nb[2];
    ps.bin_key.ensure(sizeof(int) * n);
    ps.bin_key_sorted.ensure(sizeof(int) * n);
    ps.idx.ensure(sizeof(int) * n);
    ps.idx_sorted.ensure(sizeof(int) * n);
    ps.bin_start.ensure(sizeof(int) * nbins);
    ps.bin_end.ensure(sizeof(int) * nbins);
    k_bin_keys<<<nblk(n, 128), 128, 0, s>>>(ps.base.as<int4>(), n, 8, 8, 8, ps.nb[0], ps.nb[1],
                                            ps.bin_key.as<int>(), ps.idx.as<int>());
    MPM_LAUNCH();
    size_t tmp = 0;
    int bits = 1;
    while ((1 << bits) < nbins) ++bits;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, ps.bin_key.as<int>(), ps.bin_key_sorted.as<int>(),
                                    ps.idx.as<int>(), ps.idx_sorted.as<int>(), n, 0, bits, s);
    ps.cub_tmp.ensure(tmp + sizeof(int));
    MPM_CUDA(cub::DeviceRadixSort::SortPairs(ps.cub_tmp.p, tmp, ps.bin_key.as<int>(), ps.bin_key_sorted.as<int>(),
                                             ps.idx.as<int>(), ps.idx_sorted.as<int>(), n, 0, bits, s));
    k_fill_int<<<nblk(nbins, 256), 256, 0, s>>>(ps.bin_start.as<int>(), nbins, -1);
    MPM_LAUNCH();
    k_fill_int<<<nblk(nbins, 256), 256, 0, s>>>(ps.bin_end.as<int>(), nbins, -1);
    MPM_LAUNCH();
    k_bin_bounds<<<nblk(n, 256), 256, 0, s>>>(ps.bin_key_sorted.as<int>(), n, ps.bin_start.as<int>(),
                                              ps.bin_end.as<int>());
    MPM_LAUNCH();
    // candidate list of every spread tile (CSR) and the largest one
    PolyTile t;
    for (int d = 0; d < 3; ++d) { t.N[d] = pgeom_.ng[d]; t.nb[d] = ps.nb[d]; }
    t.P = pgeom_.P;
    t.T = 8;
    t.cap = 0;
    ptmax_.ensure(sizeof(int));
    DevBuf& cnt = ps.bin_key;  // reuse: nbins + 1 ints needed
    cnt.ensure(sizeof(int) * std::max(n, nbins + 1));
    ptoff_.ensure(sizeof(int) * (nbins + 1));
    MPM_CUDA(cudaMemsetAsync(ptmax_.p, 0, sizeof(int), s));
    MPM_CUDA(cudaMemsetAsync(cnt.as<int>() + nbins, 0, sizeof(int), s));
    k_poly_cands<<<nblk(nbins, 128), 128, 0, s>>>(t, ps.bin_start.as<int>(), ps.bin_end.as<int>(), nullptr, 0,
                                                  cnt.as<int>(), ptmax_.as<int>(), nullptr, nullptr);
    MPM_LAUNCH();
    size_t need = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, cnt.as<int>(), ptoff_.as<int>(), nbins + 1, s);
    ps.cub_tmp.ensure(need);
    MPM_CUDA(cub::DeviceScan::ExclusiveSum(ps.cub_tmp.p, need, cnt.as<int>(), ptoff_.as<int>(), nbins + 1, s));
    int hv[2] = {0, 0};
    MPM_CUDA(cudaMemcpyAsync(&hv[0], ptmax_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaMemcpyAsync(&hv[1], ptoff_.as<int>() + nbins, sizeof(int), cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    const int h = hv[0];
    ptlist_.ensure(sizeof(int) * std::max(1, hv[1]));
    k_poly_cands<<<nblk(nbins, 128), 128, 0, s>>>(t, ps.bin_start.as<int>(), ps.bin_end.as<int>(),
                                                  ps.idx_sorted.as<int>(), 1, nullptr, nullptr, ptoff_.as<int>(),
                                                  ptlist_.as<int>());
    MPM_LAUNCH();
    ptcnt_.ensure(sizeof(int) * std::max(1, nbins));
    ptclist_.ensure(sizeof(int) * std::max(1, hv[1]));
    ptruns_.ensure(sizeof(int) * 8 * size_t(std::max(1, hv[1])));
    k_poly_runs<<<nblk(nbins, 128), 128, 0, s>>>(t, ps.base.as<int4>(), ptoff_.as<int>(), ptlist_.as<int>(),
                                                 ptcnt_.as<int>(), ptclist_.as<int>(), ptruns_.as<int>());
    MPM_LAUNCH();
    pcand_cap_ = std::max(1, h);
    const size_t shm = 65536 + (3 * 128 + 9 * sizeof(int)) * size_t(pcand_cap_);
    if (shm > 200 * 1024 || pgeom_.P > 255)
        throw std::runtime_error("polydisperse spread: " + std::to_string(h) +
                                 " particles reach one 8^3 voxel tile, more than the shared candidate list holds");
}

void Field::poly_pair_coefs(cudaStream_t s) {
    const int nt = spec_.solver_ax ? N_ : targets_.n;
    if (num_pairs_ <= 0) return;
    k_poly_pair_coefs<<<nblk(nt, 128), 128, 0, s>>>(pair_geo_.as<double>(), pair_off_.as<int>(), pair_src_.as<int>(),
                                                    nt, N_, pcls_.as<int>(), prad_.as<double>(), spec_.xi,
                                                    pgeom_.table_n, pair_T64_.as<double>(), pair_T32_.as<float>());
    MPM_LAUNCH();
    if (Nq_) {
        k_poly_pair_quad<<<nblk(num_pairs_, 256), 256, 0, s>>>(pair_geo_.as<double>(), num_pairs_,
                                                               pqtab_.as<double>(), pgeom_.table_n,
                                                               pair_Q_.as<double>());
        MPM_LAUNCH();
    }
}

void Field::poly_precalc(cudaStream_t s) {
    poly_weights(sources_, radius_.as<double>(), s, true);
    if (Nq_) {
        // point weights of the quadrupole grids (targets are the particles)
        const int P3 = pgeom_.P * pgeom_.P * pgeom_.P;
        pqw64_.ensure(sizeof(double) * size_t(N_) * P3);
        pqw32_.ensure(sizeof(float) * size_t(N_) * P3);
        PolyArgs a;
        for (int d = 0; d < 3; ++d) { a.h[d] = pgeom_.h[d]; a.N[d] = pgeom_.ng[d]; }
        a.P = pgeom_.P;
        a.off_min = pgeom_.off_min;
        a.eta = pgeom_.eta;
        a.xi = spec_.xi;
        const double c = std::pow(2.0 * spec_.xi * spec_.xi / kPi, 1.5) * pgeom_.h[0] * pgeom_.h[1] * pgeom_.h[2];
        k_poly_point_weights<<<nblk((long long)N_ * P3, 256), 256, 0, s>>>(sources_.xyz.as<double>(), N_, a, c,
                                                                           pqw64_.as<double>(), pqw32_.as<float>());
        MPM_LAUNCH();
    }
    if (!spec_.solver_ax) {
        // field points past the particles take the first particle's radius (:297)
        const int nt = targets_.n;
        std::vector<double> tr(nt);
        for (int j = 0; j < nt; ++j) tr[j] = spec_.radius[j < N_ ? j : 0];
        ptrad_.ensure(sizeof(double) * std::max(1, nt));
        MPM_CUDA(cudaMemcpyAsync(ptrad_.p, tr.data(), sizeof(double) * nt, cudaMemcpyHostToDevice, s));
        poly_weights(targets_, ptrad_.as<double>(), s, false);
        MPM_CUDA(cudaStreamSynchronize(s));  // tr is a host temporary
    }
    build_pairs(s);
    poly_pair_coefs(s);
}

template <typename R>
void Field::poly_recip_on(const double2* X, double2* Y, int M, cplx<R>* grid, cudaStream_t s) {
    constexpr int MC = sizeof(R) == 4 ? 4 : 2;   // contraction column chunks of 32 per CTA
    const int nmb = (M + 32 * MC - 1) / (32 * MC);
    constexpr int CM = sizeof(R) == 4 ? 16 : 8;   // spread columns per CTA (64 KB of accumulators)
    const PointSet& ps = sources_;
    PolyTile t;
    for (int d = 0; d < 3; ++d) { t.N[d] = pgeom_.ng[d]; t.nb[d] = ps.nb[d]; }
    t.P = pgeom_.P;
    t.T = 8;
    t.cap = pcand_cap_;
    const size_t shm = sizeof(cplx<R>) * (512 + 3 * size_t(t.cap)) * CM + sizeof(int) * 9 * t.cap;
    set_smem_limit(k_poly_spread<R, CM>, shm);
    const R* w1 = sizeof(R) == 4 ? reinterpret_cast<const R*>(ps.w32.p) : reinterpret_cast<const R*>(ps.w64.p);
    const int ntile = ps.nb[0] * ps.nb[1] * ps.nb[2];
    {
        StageScope sc(ST_SPREAD, s);
        k_poly_spread<R, CM><<<ntile * ((M + CM - 1) / CM), 256, shm, s>>>(
            X, M, w1, ptoff_.as<int>(), ptcnt_.as<int>(), ptclist_.as<int>(), ptruns_.as<int>(), t, grid);
        MPM_LAUNCH();
    }
    const R* scl = sizeof(R) == 4 ? reinterpret_cast<const R*>(scale32_.p) : reinterpret_cast<const R*>(scale64_.p);
    const size_t V = size_t(gv_.Nx) * gv_.Ny * gv_.Nz;
    // quadrupole grids [5][V][M] after phi (grid_bytes holds six grids then)
    cplx<R>* gq = Nq_ ? grid + V * M : nullptr;
    const R* qw = sizeof(R) == 4 ? reinterpret_cast<const R*>(pqw32_.p) : reinterpret_cast<const R*>(pqw64_.p);
    if (Nq_) {
        // the quadrupole grids couple with phi in k space, so the forward,
        // joint scale and inverse run as separate passes over six grids
        const int P3 = pgeom_.P * pgeom_.P * pgeom_.P;
        {
            StageScope sc(ST_SPREAD, s);
            MPM_CUDA(cudaMemsetAsync(gq, 0, sizeof(cplx<R>) * 5 * V * M, s));
            k_poly_quad_spread<R><<<nblk((long long)Nq_ * P3, 128), 128, 0, s>>>(
                X, M, N_, Nq_, ps.base.as<int4>(), qw, pgeom_.P, gv_.Nx, gv_.Ny, gv_.Nz, gq);
            MPM_LAUNCH();
        }
        {
            StageScope sc(ST_FFT_FWD, s);
            for (int c = 0; c < 6; ++c) transform<R>(c == 0 ? grid : gq + size_t(c - 1) * V * M, M, false, s);
        }
        {
            StageScope sc(ST_KSPACE, s);
            k_poly_quad_scale<R><<<nblk((long long)V, 128), 128, 0, s>>>(grid, gq, M, gv_.Nx, gv_.Ny, gv_.Nz,
                                                                          spec_.box[0], spec_.box[1], spec_.box[2],
                                                                          spec_.xi, pgeom_.eta);
            MPM_LAUNCH();
        }
        {
            StageScope sc(ST_FFT_INV, s);
            for (int c = 0; c < 6; ++c) transform<R>(c == 0 ? grid : gq + size_t(c - 1) * V * M, M, true, s);
        }
    } else if (own_fft_) {
        // z and y forward; x forward, scale and x inverse in one pass over
        // the x lines; y and z inverse (the 1-D transforms commute)
        const size_t Bi = size_t(gv_.Nz) * M;
        {
            StageScope sc(ST_FFT_FWD, s);
            fftz_.run<R>(grid, size_t(M), M, size_t(gv_.Nz) * M, gv_.Nx * gv_.Ny, false, s);
            ffty_.run<R>(grid, Bi, int(Bi), size_t(gv_.Ny) * Bi, gv_.Nx, false, s);
        }
        {
            StageScope sc(ST_KSPACE, s);
            fftx_.run_scaled<R>(grid, size_t(gv_.Ny) * Bi, int(Bi), Bi, gv_.Ny, scl, gv_.Nz, M, s);
        }
        {
            StageScope sc(ST_FFT_INV, s);
            ffty_.run<R>(grid, Bi, int(Bi), size_t(gv_.Ny) * Bi, gv_.Nx, true, s);
            fftz_.run<R>(grid, size_t(M), M, size_t(gv_.Nz) * M, gv_.Nx * gv_.Ny, true, s);
        }
    } else {
        {
            StageScope sc(ST_FFT_FWD, s);
            transform<R>(grid, M, false, s);
        }
        {
            StageScope sc(ST_KSPACE, s);
            const long long n = (long long)gv_.Nx * gv_.Ny * gv_.Nz * M;
            k_poly_scale<R><<<nblk(n, 256), 256, 0, s>>>(grid, scl, n, M);
            MPM_LAUNCH();
        }
        {
            StageScope sc(ST_FFT_INV, s);
            transform<R>(grid, M, true, s);
        }
    }
    if (!Y) return;  // potential only (grid holds phi = IFFT(S FFT(rho)))
    StageScope sc(ST_CONTRACT, s);
    const PointSet& tg = spec_.solver_ax ? sources_ : targets_;
    const R* tw = sizeof(R) == 4 ? reinterpret_cast<const R*>(tg.w32.p) : reinterpret_cast<const R*>(tg.w64.p);
    const double factor = pgeom_.h[0] * pgeom_.h[1] * pgeom_.h[2];
    k_poly_contract<R, MC><<<dim3(tg.n, nmb), 256, 0, s>>>(grid, M, tg.base.as<int4>(), tw, pgeom_.P, gv_.Nx, gv_.Ny,
                                                          gv_.Nz, factor, Y);
    MPM_LAUNCH();
    if (Nq_) {
        k_poly_quad_contract<R><<<Nq_, 128, 0, s>>>(gq, M, tg.base.as<int4>(), qw, pgeom_.P, gv_.Nx, gv_.Ny, gv_.Nz,
                                                   quad_idx_.as<int>(), tg.n, Y);
        MPM_LAUNCH();
    }
}

template void Field::poly_recip_on<float>(const double2*, double2*, int, cplx<float>*, cudaStream_t);
template void Field::poly_recip_on<double>(const double2*, double2*, int, cplx<double>*, cudaStream_t);

}  // namespace mpm
