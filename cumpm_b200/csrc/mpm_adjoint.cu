// Gradients of the field operator's bilinear form (the adjoint's
// "derivative interaction tensor").
//
// For M column pairs (lam_m, p_m) this computes, summed over m,
//     gx[k] = d/dx_k  sum_m lam_m^T G p_m,     ga[k] = d/da_k  sum_m lam_m^T G p_m
// for G = the polydisperse spectral-Ewald operator (reciprocal part, pair
// sum, self value) or the open-boundary direct sum, in SOLVER_AX mode and
// without the caller's self coefficients.  With p the forward solution and
// lam the adjoint solution (A is complex-symmetric, so the adjoint solve
// reuses A), dL/dtheta = -Im(sum lam^T dA/dtheta p).
//
// Polydisperse (polydisperse_ewald_electric_field.cu): with rho_q = spread(q)
// and phi_q = IFFT(S FFT(rho_q)),
//     lam^T G_recip p = h^3 sum_v rho_lam(v) phi_p(v)
// (S is real and even, so the k-space operator is symmetric), hence
//     d/dx_k = h^3 sum_v (dW_k(v)/dx_k)^T [lam_k phi_p(v) + p_k phi_lam(v)]
// and likewise for a_k, where W_k(v) = F(|g|, a_k) g, g = node - x_k, is the
// smoothed-sphere weight (:189-263).  Both potentials come from one spread /
// FFT pass over the stacked columns [p | lam].  The pair sum differentiates
// the reference's linear table lookup (:170-187): the d-derivative is the
// slope of the interpolating segment, the radius derivative interpolates
// central differences of the node values.  Each particle gathers its own
// derivative over its neighbour list (no atomics); the list is symmetric, so
//     d/dx_k = -sum_j [grad f(r_jk; lam_k, p_j) + grad f(r_jk; lam_j, p_k)]
// with r_jk = x_j - x_k and f(r; l, q) = l^T T(r) q.
#include "mpm_field.h"
#include "mpm_poly.cuh"
#include "mpm_profile.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace mpm {

namespace {

inline int nblk(long long n, int b) { return int((n + b - 1) / b); }

constexpr int kGradCols = 64;   // columns per CTA in the reciprocal gradient

// out[row][m] = p[row][m], out[row][M + m] = lam[row][m]
__global__ void k_stack2(const double2* __restrict__ p, const double2* __restrict__ lam, double2* __restrict__ out,
                         int rows, int M) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)rows * 2 * M) return;
    const int row = int(t / (2 * M)), c = int(t - (long long)row * 2 * M);
    out[t] = c < M ? p[size_t(row) * M + c] : lam[size_t(row) * M + c - M];
}

struct GradArgs {
    double h[3];
    int N[3];
    int P, off_min;
    double eta, xi;
};

// CTA = (particle k, block of kGradCols columns), 4 warps.  Nodes are taken
// 128 at a time: each thread evaluates the weight derivatives of one node
// into shared memory, then the warps sweep the nodes with lanes over columns.
// partial[(blk * n + k) * 4 + e] = sum over the block's columns (e < 3: x_e,
// e = 3: radius), without the h^3 factor.
__global__ void __launch_bounds__(128) k_poly_grad_recip(const double* __restrict__ xyz, int n,
                                                         const double* __restrict__ rad, GradArgs a,
                                                         const double2* __restrict__ grid, const double2* __restrict__ p,
                                                         const double2* __restrict__ lam, int M,
                                                         double2* __restrict__ partial) {
    __shared__ double dw[128][12];   // dW_c/dx_e at [3c+e], dW_c/da at [9+c]
    __shared__ long long vox[128];
    __shared__ double2 red[4][4];
    const int k = blockIdx.x;
    const int blk = blockIdx.y;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int P = a.P, P3 = P * P * P;
    const double ak = rad[k];
    int g0[3];
    double d0[3];
    for (int d = 0; d < 3; ++d) {
        const double x = xyz[size_t(d) * n + k];
        g0[d] = static_cast<int>(round(x / a.h[d]));
        d0[d] = g0[d] * a.h[d] - x;
    }
    const double x2 = a.xi * a.xi;
    const double C = 3.0 / (8.0 * sqrt(2.0) * pow(kPi, 1.5) * sqrt(a.eta) * a.xi);
    // this lane's two columns and the particle's moments there
    const int mA = blk * kGradCols + lane, mB = mA + 32;
    double2 lk[2][3], pk[2][3];
    for (int q = 0; q < 2; ++q) {
        const int m = q ? mB : mA;
        for (int c = 0; c < 3; ++c) {
            lk[q][c] = m < M ? lam[size_t(3 * k + c) * M + m] : make_double2(0, 0);
            pk[q][c] = m < M ? p[size_t(3 * k + c) * M + m] : make_double2(0, 0);
        }
    }
    double2 acc[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    for (int base = 0; base < P3; base += 128) {
        const int o = base + threadIdx.x;
        if (o < P3) {
            const int oo[3] = {o / (P * P), (o / P) % P, o % P};
            double g[3];
            int gw[3];
            for (int d = 0; d < 3; ++d) {
                g[d] = d0[d] + double(a.off_min + oo[d]) * a.h[d];
                gw[d] = pmod(g0[d] + a.off_min + oo[d], a.N[d]);
            }
            const double dist = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
            double F, Fd, Fa;
            if (dist >= 1e-6) {
                const double ep = exp(-2.0 * (dist + ak) * (dist + ak) * x2 / a.eta);
                const double em = exp(-2.0 * (dist - ak) * (dist - ak) * x2 / a.eta);
                const double tp = (a.eta + 4.0 * ak * x2 * dist) * ep, tm = (a.eta - 4.0 * ak * x2 * dist) * em;
                const double tpd = 4.0 * ak * x2 * ep + (a.eta + 4.0 * ak * x2 * dist) * (-4.0 * (dist + ak) * x2 / a.eta) * ep;
                const double tmd = -4.0 * ak * x2 * em + (a.eta - 4.0 * ak * x2 * dist) * (-4.0 * (dist - ak) * x2 / a.eta) * em;
                const double tpa = 4.0 * x2 * dist * ep + (a.eta + 4.0 * ak * x2 * dist) * (-4.0 * (dist + ak) * x2 / a.eta) * ep;
                const double tma = -4.0 * x2 * dist * em + (a.eta - 4.0 * ak * x2 * dist) * (4.0 * (dist - ak) * x2 / a.eta) * em;
                const double a3 = ak * ak * ak, d3 = dist * dist * dist;
                F = C / (a3 * d3) * (tp - tm);
                Fd = C / a3 * ((tpd - tmd) / d3 - 3.0 * (tp - tm) / (d3 * dist));
                Fa = C / d3 * (-3.0 / (a3 * ak) * (tp - tm) + (tpa - tma) / a3);
            } else {
                F = 8.0 * sqrt(2.0) * pow(a.xi, 5.0) * exp(-2.0 * ak * x2 / a.eta) / (pow(kPi, 1.5) * pow(a.eta, 2.5));
                Fd = 0.0;
                Fa = F * (-2.0 * x2 / a.eta);
            }
            const double fd = dist >= 1e-6 ? Fd / dist : 0.0;
            for (int c = 0; c < 3; ++c) {
                for (int e = 0; e < 3; ++e) dw[threadIdx.x][3 * c + e] = -((c == e ? F : 0.0) + fd * g[c] * g[e]);
                dw[threadIdx.x][9 + c] = Fa * g[c];
            }
            vox[threadIdx.x] = ((long long)gw[0] * a.N[1] + gw[1]) * a.N[2] + gw[2];
        }
        __syncthreads();
        const int cnt = min(128, P3 - base);
        for (int t = warp; t < cnt; t += 4) {
            const double* D = dw[t];
            const double2* gv = grid + vox[t] * 2 * M;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int m = q ? mB : mA;
                if (m >= M) continue;
                const double2 fp = gv[m], fl = gv[M + m];
                double2 tc[3];
                for (int c = 0; c < 3; ++c) tc[c] = lk[q][c] * fp + pk[q][c] * fl;
                for (int e = 0; e < 3; ++e)
                    acc[e] += tc[0] * D[e] + tc[1] * D[3 + e] + tc[2] * D[6 + e];
                acc[3] += tc[0] * D[9] + tc[1] * D[10] + tc[2] * D[11];
            }
        }
        __syncthreads();
    }
    // lanes, then warps, in a fixed order
    for (int e = 0; e < 4; ++e) {
        for (int off = 16; off > 0; off >>= 1) {
            acc[e].x += __shfl_xor_sync(0xffffffffu, acc[e].x, off);
            acc[e].y += __shfl_xor_sync(0xffffffffu, acc[e].y, off);
        }
    }
    if (lane == 0)
        for (int e = 0; e < 4; ++e) red[warp][e] = acc[e];
    __syncthreads();
    if (threadIdx.x < 4) {
        const int e = threadIdx.x;
        partial[(size_t(blk) * n + k) * 4 + e] = red[0][e] + red[1][e] + red[2][e] + red[3][e];
    }
}

// gx[k] = h3 * sum_blk partial, ga[k] = h3 * sum_blk partial (fixed order)
__global__ void k_grad_reduce(const double2* __restrict__ partial, int nblkc, int n, double h3,
                              double2* __restrict__ gx, double2* __restrict__ ga) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * 4) return;
    const int k = t / 4, e = t % 4;
    double2 s = make_double2(0, 0);
    for (int b = 0; b < nblkc; ++b) s += partial[(size_t(b) * n + k) * 4 + e];
    s = s * h3;
    if (e < 3) gx[3 * k + e] = s;
    else ga[k] = s;
}

// Per pair (CSR by target j, source i): the d-slope of the perp/para lookup
// and their derivatives in the target's radius a_j.  dT[4p..4p+3] =
// {perp_d, para_d, perp_aj, para_aj}.
__device__ void lookup_pair(double d, double a, double b, double xi, int tn, double& pe, double& pa) {
    poly::table_lookup(d, a, b, xi, tn, pe, pa);
}

__global__ void k_poly_pair_dT(const double* __restrict__ pgeo, const int* __restrict__ off,
                               const int* __restrict__ src, int nt, const int* __restrict__ cls,
                               const double* __restrict__ crad, double xi, int table_n, double* __restrict__ dT) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nt) return;
    const double aj = crad[cls[j]];
    for (int p = off[j]; p < off[j + 1]; ++p) {
        const double ai = crad[cls[src[p]]];
        const double d = pgeo[4 * size_t(p) + 3];
        const double de = d < 1e-6 ? 1e-6 : d;
        const double lo = fmin(ai, aj), hi = fmax(ai, aj);
        // slope of the interpolating segment
        const double last = poly::node(table_n - 1);
        double sp = 0.0, sq = 0.0;
        if (de < last) {
            const int kk = de < 1.0 ? 0 : 1 + static_cast<int>((de - 1.0) / poly::kTableDr);
            if (kk < table_n - 1) {
                const double r0 = poly::node(kk), r1 = poly::node(kk + 1);
                double y0a, y0b, y1a, y1b;
                if (kk == 0) y0a = y0b = poly::self_value(lo, hi, xi);
                else poly::pair_functions(r0, lo, hi, xi, y0a, y0b);
                poly::pair_functions(r1, lo, hi, xi, y1a, y1b);
                const double w = kk == 0 ? 1.0 : (r1 - r0);
                sp = (y1a - y0a) / w;
                sq = (y1b - y0b) / w;
            }
        }
        // derivative in a_j: a_j fills the 'a' slot when it is the smaller
        // radius (either slot when equal: the functions are symmetric there)
        const bool jlo = aj <= ai;
        const double h = 1e-5 * aj;
        double pp, qp, pm, qm;
        if (jlo) {
            if (aj + h <= ai) lookup_pair(de, aj + h, ai, xi, table_n, pp, qp);
            else lookup_pair(de, ai, aj + h, xi, table_n, pp, qp);
            lookup_pair(de, aj - h, ai, xi, table_n, pm, qm);
        } else {
            lookup_pair(de, ai, aj + h, xi, table_n, pp, qp);
            if (ai <= aj - h) lookup_pair(de, ai, aj - h, xi, table_n, pm, qm);
            else lookup_pair(de, aj - h, ai, xi, table_n, pm, qm);
        }
        double* o = dT + 4 * size_t(p);
        o[0] = sp;
        o[1] = sq;
        o[2] = (pp - pm) / (2 * h);
        o[3] = (qp - qm) / (2 * h);
    }
}

__device__ __forceinline__ double2 dot3(const double2 (&a)[3], const double2 (&b)[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ double2 dot3r(const double2 (&a)[3], const double (&u)[3]) {
    return a[0] * u[0] + a[1] * u[1] + a[2] * u[2];
}

// grad_r of f(r; l, q) = l^T [perp (I - u u^T) + para u u^T] q at r = d u
__device__ __forceinline__ void pair_grad(const double2 (&l)[3], const double2 (&q)[3], const double (&u)[3],
                                          double de, double perp, double para, double sp, double sq,
                                          double2 (&out)[3]) {
    const double2 lp = dot3(l, q), lu = dot3r(l, u), qu = dot3r(q, u);
    const double2 luqu = lu * qu;
    for (int e = 0; e < 3; ++e) {
        const double2 t1 = lp * (sp * u[e]) + luqu * ((sq - sp) * u[e]);
        const double2 t2 = ((l[e] - lu * u[e]) * qu + lu * (q[e] - qu * u[e])) * ((para - perp) / de);
        out[e] = t1 + t2;
    }
}

// Warp per target k, lanes over columns: pair and self-value contributions,
// added to gx[k], ga[k].
__global__ void __launch_bounds__(128) k_poly_grad_pairs(const double* __restrict__ pgeo, const int* __restrict__ off,
                                                         const int* __restrict__ src, const double* __restrict__ T64,
                                                         const double* __restrict__ dT,
                                                         const double* __restrict__ self_d, int n,
                                                         const double2* __restrict__ p, const double2* __restrict__ lam,
                                                         int M, double2* __restrict__ gx, double2* __restrict__ ga) {
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (k >= n) return;
    double2 ax[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    double2 aa = make_double2(0, 0);
    for (int m = lane; m < M; m += 32) {
        double2 lk[3], pk[3];
        for (int c = 0; c < 3; ++c) {
            lk[c] = lam[size_t(3 * k + c) * M + m];
            pk[c] = p[size_t(3 * k + c) * M + m];
        }
        aa += dot3(lk, pk) * self_d[k];
        for (int q = off[k]; q < off[k + 1]; ++q) {
            const int j = src[q];
            const double* t = T64 + 8 * size_t(q);
            const double u[3] = {t[0], t[1], t[2]};
            const double perp = t[3], para = t[4];
            const double d = pgeo[4 * size_t(q) + 3];
            const double de = d < 1e-6 ? 1e-6 : d;
            const double* D = dT + 4 * size_t(q);
            double2 lj[3], pj[3];
            for (int c = 0; c < 3; ++c) {
                lj[c] = lam[size_t(3 * j + c) * M + m];
                pj[c] = p[size_t(3 * j + c) * M + m];
            }
            double2 g1[3], g2[3];
            pair_grad(lk, pj, u, de, perp, para, D[0], D[1], g1);
            pair_grad(lj, pk, u, de, perp, para, D[0], D[1], g2);
            for (int e = 0; e < 3; ++e) ax[e] -= g1[e] + g2[e];
            const double2 lu1 = dot3r(lk, u) * dot3r(pj, u), lu2 = dot3r(lj, u) * dot3r(pk, u);
            aa += (dot3(lk, pj) - lu1) * D[2] + lu1 * D[3];
            aa += (dot3(lj, pk) - lu2) * D[2] + lu2 * D[3];
        }
    }
    for (int off2 = 16; off2 > 0; off2 >>= 1) {
        for (int e = 0; e < 3; ++e) {
            ax[e].x += __shfl_xor_sync(0xffffffffu, ax[e].x, off2);
            ax[e].y += __shfl_xor_sync(0xffffffffu, ax[e].y, off2);
        }
        aa.x += __shfl_xor_sync(0xffffffffu, aa.x, off2);
        aa.y += __shfl_xor_sync(0xffffffffu, aa.y, off2);
    }
    if (lane == 0) {
        for (int e = 0; e < 3; ++e) gx[3 * k + e] += ax[e];
        ga[k] += aa;
    }
}

// Open-boundary sum (direct_electric_field.cu:148-309, SOLVER_AX):
// f(r; l, q) = -(1/4 pi) [3 (l.u)(q.u) - l.q] / d^3 over all pairs, self
// value 1/(4 pi a^3).  Warp per target k, lanes over columns.  Spheres are
// taken as non-overlapping (d >= a).
__global__ void __launch_bounds__(128) k_direct_grad(const double* __restrict__ xyz, const double* __restrict__ rad,
                                                     int n, const double2* __restrict__ p,
                                                     const double2* __restrict__ lam, int M,
                                                     double2* __restrict__ gx, double2* __restrict__ ga) {
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (k >= n) return;
    const double kf = -1.0 / (4.0 * kPi);
    const double xk[3] = {xyz[k], xyz[n + k], xyz[2 * n + k]};
    double2 ax[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    double2 aa = make_double2(0, 0);
    const double ak = rad[k];
    for (int m = lane; m < M; m += 32) {
        double2 lk[3], pk[3];
        for (int c = 0; c < 3; ++c) {
            lk[c] = lam[size_t(3 * k + c) * M + m];
            pk[c] = p[size_t(3 * k + c) * M + m];
        }
        aa += dot3(lk, pk) * (-3.0 / (4.0 * kPi * ak * ak * ak * ak));
        for (int j = 0; j < n; ++j) {
            if (j == k) continue;
            double r[3];
            for (int d = 0; d < 3; ++d) r[d] = xyz[size_t(d) * n + j] - xk[d];
            const double dd = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            const double u[3] = {r[0] / dd, r[1] / dd, r[2] / dd};
            double2 lj[3], pj[3];
            for (int c = 0; c < 3; ++c) {
                lj[c] = lam[size_t(3 * j + c) * M + m];
                pj[c] = p[size_t(3 * j + c) * M + m];
            }
            const double d4 = dd * dd * dd * dd;
            for (int s = 0; s < 2; ++s) {
                const double2(&l)[3] = s ? lj : lk;
                const double2(&q)[3] = s ? pk : pj;
                const double2 lp = dot3(l, q), lu = dot3r(l, u), qu = dot3r(q, u);
                const double2 f0 = lu * qu * 3.0 - lp;
                for (int e = 0; e < 3; ++e) {
                    const double2 g = (f0 * (-3.0 * u[e]) + ((l[e] - lu * u[e]) * qu + lu * (q[e] - qu * u[e])) * 3.0) *
                                      (kf / d4);
                    ax[e] -= g;
                }
            }
        }
    }
    for (int off2 = 16; off2 > 0; off2 >>= 1) {
        for (int e = 0; e < 3; ++e) {
            ax[e].x += __shfl_xor_sync(0xffffffffu, ax[e].x, off2);
            ax[e].y += __shfl_xor_sync(0xffffffffu, ax[e].y, off2);
        }
        aa.x += __shfl_xor_sync(0xffffffffu, aa.x, off2);
        aa.y += __shfl_xor_sync(0xffffffffu, aa.y, off2);
    }
    if (lane == 0) {
        for (int e = 0; e < 3; ++e) gx[3 * k + e] = ax[e];
        ga[k] = aa;
    }
}

}  // namespace

void Field::grad_bilinear(const double2* lam, const double2* p, int M, double2* gx, double2* ga, cudaStream_t s) {
    if (N_ == 0) throw std::runtime_error("gradient before set_positions");
    if (!spec_.solver_ax) throw std::runtime_error("gradients need the SOLVER_AX operator");
    if (Nq_ > 0) throw std::runtime_error("gradients are available for dipoles only");
    if (bloch_on()) throw std::runtime_error("gradients are available without a Bloch wavevector only");
    if (M < 1) throw std::invalid_argument("M must be >= 1");
    if (spec_.kind == FIELD_DIRECT) {
        if (int(spec_.radius.size()) != N_) throw std::runtime_error("direct gradient needs one radius per particle");
        k_direct_grad<<<nblk((long long)N_ * 32, 128), 128, 0, s>>>(sources_.xyz.as<double>(), radius_.as<double>(),
                                                                    N_, p, lam, M, gx, ga);
        MPM_LAUNCH();
        return;
    }
    if (spec_.kind != FIELD_POLY)
        throw std::runtime_error("gradients need the polydisperse (or direct) field; equal radii work as polydisperse");
    // potentials phi_p, phi_lam of the stacked columns [p | lam], fp64
    const int rows = rows_in();
    adj_x_.ensure(sizeof(double2) * size_t(rows) * 2 * M);
    k_stack2<<<nblk((long long)rows * 2 * M, 256), 256, 0, s>>>(p, lam, adj_x_.as<double2>(), rows, M);
    MPM_LAUNCH();
    adj_grid_.ensure(grid_bytes(2 * M, true));
    poly_recip_on<double>(adj_x_.as<double2>(), nullptr, 2 * M, adj_grid_.as<double2>(), s);
    // reciprocal part
    GradArgs a;
    for (int d = 0; d < 3; ++d) { a.h[d] = pgeom_.h[d]; a.N[d] = pgeom_.ng[d]; }
    a.P = pgeom_.P;
    a.off_min = pgeom_.off_min;
    a.eta = pgeom_.eta;
    a.xi = spec_.xi;
    const int nb = (M + kGradCols - 1) / kGradCols;
    DevBuf& part = adj_part_;
    part.ensure(sizeof(double2) * size_t(nb) * N_ * 4);
    k_poly_grad_recip<<<dim3(N_, nb), 128, 0, s>>>(sources_.xyz.as<double>(), N_, radius_.as<double>(), a,
                                                    adj_grid_.as<double2>(), p, lam, M, part.as<double2>());
    MPM_LAUNCH();
    const double h3 = pgeom_.h[0] * pgeom_.h[1] * pgeom_.h[2];
    k_grad_reduce<<<nblk(N_ * 4, 128), 128, 0, s>>>(part.as<double2>(), nb, N_, h3, gx, ga);
    MPM_LAUNCH();
    // per-frame pair derivatives and self-value derivatives
    if (pair_dT_frame_ != adj_frame_) {
        const size_t np = size_t(std::max<long long>(1, num_pairs_));
        pair_dT_.ensure(sizeof(double) * 4 * np);
        if (num_pairs_ > 0) {
            k_poly_pair_dT<<<nblk(N_, 128), 128, 0, s>>>(pair_geo_.as<double>(), pair_off_.as<int>(),
                                                         pair_src_.as<int>(), N_, pcls_.as<int>(), prad_.as<double>(),
                                                         spec_.xi, pgeom_.table_n, pair_dT_.as<double>());
            MPM_LAUNCH();
        }
        std::vector<double> sd(N_);
        for (int i = 0; i < N_; ++i) {
            const double r = pgeom_.unique[pgeom_.cls[i]], h = 1e-5 * r;
            sd[i] = (poly::self_value(r + h, r + h, spec_.xi) - poly::self_value(r - h, r - h, spec_.xi)) / (2 * h);
        }
        pself_d_.ensure(sizeof(double) * N_);
        MPM_CUDA(cudaMemcpyAsync(pself_d_.p, sd.data(), sizeof(double) * N_, cudaMemcpyHostToDevice, s));
        MPM_CUDA(cudaStreamSynchronize(s));  // sd is a host temporary
        pair_dT_frame_ = adj_frame_;
    }
    k_poly_grad_pairs<<<nblk((long long)N_ * 32, 128), 128, 0, s>>>(
        pair_geo_.as<double>(), pair_off_.as<int>(), pair_src_.as<int>(), pair_T64_.as<double>(),
        pair_dT_.as<double>(), pself_d_.as<double>(), N_, p, lam, M, gx, ga);
    MPM_LAUNCH();
}

}  // namespace mpm
