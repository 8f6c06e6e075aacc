// Batched device Krylov solvers (see mpm_krylov.h).
#include "mpm_krylov.h"
#include "mpm_profile.h"

#include <algorithm>
#include <cmath>

namespace mpm {

namespace {

inline int nblk(long long n, int b) { return int((n + b - 1) / b); }

// ----------------------------------------------------------- reductions --

// out[i][m] = sum_row op(V_i[row][m]) * w[row][m], op = conj or identity.
// Stage 1 writes per-CTA partials; stage 2 sums them.  shift >= 0 (the
// GMRES step, w = V_{nvec-1} = A V_shift): the sums are taken with
// u = w - V_shift in place of w, and the last vector's entry is |u|^2.
__global__ void __launch_bounds__(256) k_dots1(const double2* __restrict__ V, size_t vstride, int nvec,
                                               const double2* __restrict__ w, int rows, int M, int conj,
                                               double2* __restrict__ partial, int shift) {
    __shared__ double2 red[8][8][32];
    const int m = blockIdx.y * 32 + threadIdx.x;
    const int i0 = blockIdx.z * 8;
    double2 acc[8];
    for (int k = 0; k < 8; ++k) acc[k] = make_double2(0, 0);
    const int nv = min(8, nvec - i0);
    if (m < M) {
#pragma unroll 4
        for (int row = blockIdx.x * 8 + threadIdx.y; row < rows; row += gridDim.x * 8) {
            double2 wv = w[size_t(row) * M + m];
            if (shift >= 0) wv -= V[size_t(shift) * vstride + size_t(row) * M + m];
            for (int k = 0; k < nv; ++k) {
                const double2 v = (shift >= 0 && i0 + k == nvec - 1) ? wv
                                                                       : V[size_t(i0 + k) * vstride + size_t(row) * M + m];
                if (conj) acc[k] += conjmul(v, wv);
                else acc[k] += v * wv;
            }
        }
    }
    for (int k = 0; k < 8; ++k) red[k][threadIdx.y][threadIdx.x] = acc[k];
    __syncthreads();
    if (threadIdx.y < nv && m < M) {
        double2 s = make_double2(0, 0);
        for (int r = 0; r < 8; ++r) s += red[threadIdx.y][r][threadIdx.x];
        partial[(size_t(blockIdx.x) * nvec + i0 + threadIdx.y) * M + m] = s;
    }
}

// k_dots1 + k_dots2 for few columns (M < 16): threads run over the flat
// [row][M] elements, (256 / M) * M of them per CTA, so that each thread
// keeps one column m for the whole grid-stride loop (the stride is a
// multiple of M); the CTA's per-column sums are taken over the threads of
// that column in a fixed order and written as k_dots1's partials.  The last
// CTA of each vector group to finish (a counter per group, no waiting) then
// reduces the partials exactly as k_dots2 does (lanes over CTAs, fixed
// shuffle tree) into out, and resets its counter.
__global__ void __launch_bounds__(256) k_dots1s(const double2* __restrict__ V, size_t vstride, int nvec,
                                                const double2* __restrict__ w, int rows, int M, int conj,
                                                double2* __restrict__ partial, int shift,
                                                double2* __restrict__ out, unsigned int* __restrict__ done) {
    __shared__ double2 red[8][256];
    const int L = (256 / M) * M;
    const int j = threadIdx.x;
    const int i0 = blockIdx.z * 8;
    const int nv = min(8, nvec - i0);
    const size_t n = size_t(rows) * M;
    double2 acc[8];
    for (int k = 0; k < 8; ++k) acc[k] = make_double2(0, 0);
    if (j < L) {
        for (size_t t = size_t(blockIdx.x) * L + j; t < n; t += size_t(gridDim.x) * L) {
            double2 wv = w[t];
            if (shift >= 0) wv -= V[size_t(shift) * vstride + t];
            // a fixed trip count, so that the group's loads issue together
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                if (k >= nv) break;
                const double2 v = (shift >= 0 && i0 + k == nvec - 1) ? wv : V[size_t(i0 + k) * vstride + t];
                if (conj) acc[k] += conjmul(v, wv);
                else acc[k] += v * wv;
            }
        }
    }
    for (int k = 0; k < 8; ++k) red[k][j] = acc[k];
    __syncthreads();
    if (j < nv * M) {
        const int k = j / M, m = j % M;
        double2 sum = make_double2(0, 0);
        for (int q = m; q < L; q += M) sum += red[k][q];
        partial[(size_t(blockIdx.x) * nvec + i0 + k) * M + m] = sum;
    }
    __threadfence();
    __syncthreads();
    __shared__ int last;
    if (j == 0) last = atomicAdd(&done[blockIdx.z], 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int lane = j & 31, warp = j >> 5;
    for (int o = warp; o < nv * M; o += 8) {
        const int t = (i0 + o / M) * M + o % M;
        double2 sum = make_double2(0, 0);
        for (int b = lane; b < int(gridDim.x); b += 32) sum += __ldcg(&partial[size_t(b) * nvec * M + t]);
        for (int off = 16; off > 0; off >>= 1) {
            sum.x += __shfl_xor_sync(0xffffffffu, sum.x, off);
            sum.y += __shfl_xor_sync(0xffffffffu, sum.y, off);
        }
        if (lane == 0) out[t] = sum;
    }
    if (j == 0) done[blockIdx.z] = 0u;
}

// one warp per output: lanes stride over the per-CTA partials, then a fixed
// shuffle tree (deterministic order)
__global__ void k_dots2(const double2* __restrict__ partial, int gx, int nvec, int M, double2* __restrict__ out) {
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= nvec * M) return;
    double2 s = make_double2(0, 0);
    for (int b = lane; b < gx; b += 32) s += partial[size_t(b) * nvec * M + t];
    for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
    }
    if (lane == 0) out[t] = s;
}

__global__ void k_sqrt_re(const double2* __restrict__ in, int M, double* __restrict__ out) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < M) out[m] = sqrt(fmax(in[m].x, 0.0));
}

// w[row][m] += sgn * sum_{i < n_m} V_i[row][m] h[i][m]
__global__ void k_vupdate(double2* __restrict__ w, const double2* __restrict__ V, size_t vstride, int nvec,
                          const double2* __restrict__ h, int rows, int M, double sgn, const int* __restrict__ nper) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(rows) * M) return;
    const int m = int(t % M);
    const int n = nper ? nper[m] : nvec;
    double2 acc = make_double2(0, 0);
    for (int i = 0; i < n; ++i) acc += V[size_t(i) * vstride + t] * h[size_t(i) * M + m];
    w[t] += acc * sgn;
}

// out = a - b
__global__ void k_sub(const double2* __restrict__ a, const double2* __restrict__ b, double2* __restrict__ out,
                      size_t n) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n) out[t] = a[t] - b[t];
}

// out = diag(self)^-1 in  over the unknown layout (jacobi_precond_kernel,
// numerical_solver.cu:250-285: per particle 1/s, quads use their particle).
__global__ void k_jacobi(const double2* __restrict__ in, double2* __restrict__ out, int N, int Nq, int M,
                         const int* __restrict__ quad_idx, const double2* __restrict__ sc) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t rows = size_t(3 * N + 5 * Nq);
    if (t >= rows * M) return;
    const int row = int(t / M), m = int(t % M);
    int p;
    if (row < 3 * N) p = row / 3;
    else {
        p = quad_idx[(row - 3 * N) / 5];
        if (p < 0 || p >= N) p = 0;
    }
    const double2 s = sc[size_t(p) * M + m];
    const double den = s.x * s.x + s.y * s.y;
    const double2 inv = den > 1e-30 ? make_double2(s.x / den, -s.y / den) : make_double2(1.0, 0.0);
    out[t] = in[t] * inv;
}

// ------------------------------------------------------------ GMRES state --

struct GState {
    int active;      // still solving (outer)
    int cyc;         // in the current Arnoldi cycle
    int kcount;      // Arnoldi columns of the current cycle
    int iters;       // total Arnoldi steps
    int converged;
    int reorth;      // this Arnoldi step: 0 one projection, 1 second pass pending, 2 second pass done
    int pad[2];
};

__device__ __forceinline__ double col_tol(double tol, const double* tolv, int m) { return tolv ? tolv[m] : tol; }

// start of a restart cycle: residual norm test and V_0 = r / |r|.
// flag[0] counts the cycling columns, flag[1 + m] is column m's cycle flag.
__global__ void k_gm_begin(GState* __restrict__ st, const double* __restrict__ rn, const double* __restrict__ bn,
                           double tol, const double* __restrict__ tolv, int maxiter, int restart,
                           double2* __restrict__ g, int M, int* __restrict__ flag) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    GState s = st[m];
    s.cyc = 0;
    s.kcount = 0;
    if (s.active) {
        if (rn[m] < col_tol(tol, tolv, m) * bn[m]) {
            s.active = 0;
            s.converged = 1;
        } else if (s.iters >= maxiter) {
            s.active = 0;
        } else {
            s.cyc = 1;
            g[size_t(m) * (restart + 1)] = make_double2(rn[m], 0.0);
            for (int i = 1; i <= restart; ++i) g[size_t(m) * (restart + 1) + i] = make_double2(0, 0);
            atomicAdd(flag, 1);
        }
    }
    flag[1 + m] = s.cyc;
    st[m] = s;
}

// V_dst[row][m] = src[row][m] / nrm[m] for cycling RHS (0 otherwise)
__global__ void k_normalize(const double2* __restrict__ src, double2* __restrict__ dst,
                            const double* __restrict__ nrm, const GState* __restrict__ st, size_t n, int M) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int m = int(t % M);
    const double d = nrm[m];
    dst[t] = (st[m].cyc && d > 0.0) ? src[t] * (1.0 / d) : make_double2(0, 0);
}

// ------------------------------------------------- Arnoldi step kernels --
//
// The operator writes A V_k straight into V_{k+1}, so one pass of k_dots1 over
// the k+2 vectors V_0..V_{k+1} gives h_i = V_i^H u (i <= k) and |u|^2 (i =
// k+1) for u = w - V_k (then h_k(w) = h_k(u) + 1; u has the same projection
// remainder w' as w).  Classical Gram-Schmidt with selective
// re-orthogonalisation: after the projection |w'|^2 = |u|^2 - |h(u)|^2
// (Pythagoras, V orthonormal); a column whose norm dropped below 0.7 |u|
// (|w'|^2 <= 0.49 |u|^2, where that difference loses digits and
// orthogonality may suffer) takes a second projection (Kahan and Parlett's
// "twice is enough" test); the others are finished after one.  The Givens rotation of a column uses the final h and
// |w'|; k_arn_update projects and normalises V_{k+1} in place.

// Givens update of Hessenberg column k of one right-hand side (the previous
// rotations, a new rotation, the residual estimate; gmres_solver.cu:120-184)
__device__ void gm_givens(GState& s, const double2* __restrict__ h, double wn, double2* __restrict__ Hm,
                          double2* __restrict__ gm, double* __restrict__ csm, double2* __restrict__ snm, int k,
                          int ld, int M, int m, int restart, double tolm, double bnm, int maxiter) {
    double2* col = Hm + size_t(k) * ld;
    // the previous rotations applied down the column, the running entry in
    // a register (the column's inputs and the rotations are independent loads)
    double2 carry = h[m];
#pragma unroll 4
    for (int i = 0; i < k; ++i) {
        const double2 h2 = h[size_t(i + 1) * M + m];
        const double c = csm[i];
        const double2 sv = snm[i];
        const double2 cs_ = make_double2(sv.x, -sv.y);
        col[i] = carry * c + cs_ * h2;
        carry = (sv * carry) * -1.0 + h2 * c;
    }
    const double2 h1 = carry, h2 = make_double2(wn, 0.0);
    double c = 1.0;
    double2 sv = make_double2(0, 0);
    if (h2.x != 0.0 || h2.y != 0.0) {
        const double a1 = hypot(h1.x, h1.y);
        if (a1 == 0.0) {
            c = 0.0;
            sv = make_double2(1.0, 0.0);
        } else {
            const double a2 = hypot(h2.x, h2.y);
            const double sc = a1 + a2;
            const double n1 = a1 / sc, n2 = a2 / sc;
            const double hh = sc * sqrt(n1 * n1 + n2 * n2);
            c = a1 / hh;
            // (conj(h1)/|h1|) * (h2/hh)
            const double2 u = make_double2(h1.x / a1, -h1.y / a1);
            sv = u * make_double2(h2.x / hh, h2.y / hh);
        }
    }
    csm[k] = c;
    snm[k] = sv;
    const double2 scj = make_double2(sv.x, -sv.y);
    col[k] = h1 * c + scj * h2;
    col[k + 1] = make_double2(0, 0);
    const double2 g1 = gm[k], g2 = gm[k + 1];
    gm[k] = g1 * c + scj * g2;
    gm[k + 1] = (sv * g1) * -1.0 + g2 * c;
    s.iters += 1;
    const double resid = hypot(gm[k + 1].x, gm[k + 1].y);
    if (resid < tolm * bnm || k + 1 >= restart || s.iters >= maxiter) {
        s.cyc = 0;
        s.kcount = k + 1;
    }
}

// givens = 0 (the seeds of a shifted solve): |w'| and the normalisation
// only; the Givens updates are the members' (shift_givens_body).  always2:
// every column takes the second projection (CGS2); else only those that
// fail the 0.7 test.
// pass 1: hh = [V_0..V_k, w]^H w.  Columns whose projection keeps |w'| >
// 0.7 |w| get |w'| by Pythagoras and their Givens update now; the others are
// marked for a second pass.  pass 2 (marked columns, hh2 = [V_0..V_k, w']^H w'
// after the first projection): h += h2, |w''| likewise, Givens.  Thread per
// column; one CTA: flag[0] = columns still cycling, flag[1 + m] = column m
// cycling, flag[1 + M] = columns marked for the second pass.
__device__ __forceinline__ void arn_finish_body(GState* __restrict__ st, double2* __restrict__ h,
                                                const double2* __restrict__ h2, int pass, int givens, int always2,
                                                double* __restrict__ nu_out, double* __restrict__ inv_nu,
                                                double2* __restrict__ H, double2* __restrict__ g,
                                                double* __restrict__ cs, double2* __restrict__ sn, int k, int restart,
                                                int M, const double* __restrict__ bn, double tol,
                                                const double* __restrict__ tolv, int maxiter,
                                                int* __restrict__ flag) {
    __shared__ int ncyc, nreo;
    if (threadIdx.x == 0) ncyc = nreo = 0;
    __syncthreads();
    const int ld = restart + 1;
    int c_cyc = 0, c_reo = 0;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        GState s = st[m];
        if (pass == 1) s.reorth = 0;
        bool go = s.cyc && (pass == 1 || s.reorth == 1);
        if (go) {
            double wn2, hs = 0.0;
            if (pass == 1) {
                // h holds V^H u and |u|^2 for u = w - V_k: h_k(w) = h_k(u) + 1
                wn2 = h[size_t(k + 1) * M + m].x;
                for (int i = 0; i <= k; ++i) {
                    const double2 v = h[size_t(i) * M + m];
                    hs += v.x * v.x + v.y * v.y;
                }
                h[size_t(k) * M + m].x += 1.0;
            } else {
                wn2 = h2[size_t(k + 1) * M + m].x;
                for (int i = 0; i <= k; ++i) {
                    const double2 v = h2[size_t(i) * M + m];
                    hs += v.x * v.x + v.y * v.y;
                    h[size_t(i) * M + m] += v;
                }
            }
            const double nu2 = wn2 - hs;
            if (pass == 1 && (always2 || !(nu2 > 0.49 * wn2))) {
                s.reorth = 1;   // second projection before the Givens update
            } else {
                const double nu = sqrt(fmax(nu2, 0.0));
                inv_nu[m] = nu > 0.0 ? 1.0 / nu : 0.0;
                if (nu_out) nu_out[m] = nu;
                if (givens)
                    gm_givens(s, h, nu, H + size_t(m) * ld * restart, g + size_t(m) * ld, cs + size_t(m) * restart,
                              sn + size_t(m) * restart, k, ld, M, m, restart, col_tol(tol, tolv, m), bn[m],
                              maxiter);
                if (pass == 2) s.reorth = 2;
            }
            st[m] = s;
        }
        c_cyc += s.cyc;
        c_reo += s.reorth == 1;
        flag[1 + m] = s.cyc;
    }
    if (c_cyc) atomicAdd(&ncyc, c_cyc);
    if (c_reo) atomicAdd(&nreo, c_reo);
    __syncthreads();
    if (threadIdx.x == 0) {
        flag[0] = ncyc;
        flag[1 + M] = nreo;
    }
}

__global__ void __launch_bounds__(1024) k_arn_finish(GState* __restrict__ st, double2* __restrict__ h,
                                                     const double2* __restrict__ h2, int pass, int givens, int always2,
                                                     double* __restrict__ nu_out,
                                                     double* __restrict__ inv_nu, double2* __restrict__ H,
                                                     double2* __restrict__ g, double* __restrict__ cs,
                                                     double2* __restrict__ sn, int k, int restart, int M,
                                                     const double* __restrict__ bn, double tol,
                                                     const double* __restrict__ tolv, int maxiter,
                                                     int* __restrict__ flag) {
    arn_finish_body(st, h, h2, pass, givens, always2, nu_out, inv_nu, H, g, cs, sn, k, restart, M, bn, tol, tolv,
                    maxiter, flag);
}

// V_{k+1} -= sum_{i <= k} V_i h_i for the columns of this pass (pass 1: the
// columns still cycling; pass 2: those whose second projection was just
// finished), then scaled by 1/|w'| unless a second pass is pending; the
// other columns of V_{k+1} (ended cycles, unused) are zeroed in pass 1.
__global__ void k_arn_update(double2* __restrict__ V, size_t vstride, int k, const double2* __restrict__ h,
                             const GState* __restrict__ st, const double* __restrict__ inv_nu, int rows, int M,
                             int pass) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(rows) * M) return;
    const int m = int(t % M);
    const GState s = st[m];
    double2* w = V + size_t(k + 1) * vstride + t;
    const bool mine = pass == 1 ? s.cyc != 0 : s.reorth == 2;
    if (!mine) {
        if (pass == 1) *w = make_double2(0, 0);
        return;
    }
    // four independent partial sums, so that a thread has four loads of V
    // in flight (the sum's order is fixed)
    double2 a0 = make_double2(0, 0), a1 = a0, a2 = a0, a3 = a0;
    int i = 0;
    for (; i + 3 <= k; i += 4) {
        a0 += V[size_t(i) * vstride + t] * h[size_t(i) * M + m];
        a1 += V[size_t(i + 1) * vstride + t] * h[size_t(i + 1) * M + m];
        a2 += V[size_t(i + 2) * vstride + t] * h[size_t(i + 2) * M + m];
        a3 += V[size_t(i + 3) * vstride + t] * h[size_t(i + 3) * M + m];
    }
    for (; i <= k; ++i) a0 += V[size_t(i) * vstride + t] * h[size_t(i) * M + m];
    const double2 acc = (a0 + a1) + (a2 + a3);
    double2 v = *w - acc;
    if (s.reorth != 1) v = v * inv_nu[m];
    *w = v;
}

// ---------------------------------------------------------- shifted solve --
//
// Columns m whose self coefficients are one particle profile c times a
// scalar, sc[:, m] = f_m c, have operators A_m = G + f_m diag(c) (G the
// interactions and the self value common to all columns); scaled by
// diag(c)^-1 they are the shifted family A0 + (f_m - 1) I with A0 = diag(c)^-1
// G + I, the operator apply gives with self coefficients c and Jacobi
// scaling.  Columns with the same right-hand side share one Krylov space of
// A0: one seed column per distinct right-hand side is iterated, and every
// member m of a seed's group runs its own Givens QR on the seed's Hessenberg
// column with sigma_m = f_m - 1 added to the diagonal (GMRES for shifted
// systems with x0 = 0, whose residuals stay collinear).

// f_m = sc[0][m] / sc[0][0]; bad[m] = 1 unless sc[i][m] = f_m sc[i][0] for
// every particle i (relative 1e-12)
__global__ void k_shift_ratio(const double2* __restrict__ sc, int N, int M, double2* __restrict__ f,
                              int* __restrict__ bad) {
    const int m = blockIdx.x;
    const double2 a = sc[m], c0 = sc[0];
    const double den = c0.x * c0.x + c0.y * c0.y;
    const double2 fm = den > 0.0 ? make_double2((a.x * c0.x + a.y * c0.y) / den, (a.y * c0.x - a.x * c0.y) / den)
                                 : make_double2(0, 0);
    int miss = den > 0.0 ? 0 : 1;
    for (int i = threadIdx.x; i < N && !miss; i += blockDim.x) {
        const double2 v = sc[size_t(i) * M + m], r = sc[size_t(i) * M] * fm;
        const double dx = v.x - r.x, dy = v.y - r.y;
        if (dx * dx + dy * dy > 1e-24 * (v.x * v.x + v.y * v.y) || (v.x == 0.0 && v.y == 0.0)) miss = 1;
    }
    miss = __syncthreads_or(miss);
    if (threadIdx.x == 0) {
        f[m] = fm;
        bad[m] = miss;
    }
}

// eq[m][m2] = 1 if right-hand-side columns m and m2 < m are equal
__global__ void k_col_equal(const double2* __restrict__ b, int rows, int M, int* __restrict__ eq) {
    const int m = blockIdx.x, m2 = blockIdx.y;
    if (m2 >= m) return;
    int diff = 0;
    for (int r = threadIdx.x; r < rows && !diff; r += blockDim.x) {
        const double2 u = b[size_t(r) * M + m], v = b[size_t(r) * M + m2];
        if (u.x != v.x || u.y != v.y) diff = 1;
    }
    diff = __syncthreads_or(diff);
    if (threadIdx.x == 0) eq[size_t(m) * M + m2] = !diff;
}

// member m of seed grp[m]: Hessenberg column k of the seed plus sigma_m on
// the diagonal, then its Givens update (gm_givens).  pass 1 takes the members
// of seeds finished after one projection, pass 2 those of seeds whose second
// projection just finished (reorth 2); members of a seed still waiting for
// its second projection keep it cycling.  A seed cycles while any member
// does (written back to its state).  One CTA: flag[0] = seeds cycling,
// flag[1 + g] = seed g cycling.
__device__ __forceinline__ void shift_givens_body(GState* __restrict__ mst, GState* __restrict__ sst,
                                                  const double2* __restrict__ hs, const double* __restrict__ nu,
                                                  const double2* __restrict__ sigma, const int* __restrict__ grp,
                                                  int G, int pass, double2* __restrict__ hm, double2* __restrict__ H,
                                                  double2* __restrict__ g, double* __restrict__ cs,
                                                  double2* __restrict__ sn, int k, int restart, int M,
                                                  const double* __restrict__ bs, const double* __restrict__ tolv,
                                                  int maxiter, int* __restrict__ seed_cyc, int* __restrict__ flag) {
    __shared__ int n;
    if (threadIdx.x == 0) n = 0;
    for (int t = threadIdx.x; t < G; t += blockDim.x) seed_cyc[t] = 0;
    __syncthreads();
    const int ld = restart + 1;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        GState s = mst[m];
        if (!s.cyc) continue;
        const int gi = grp[m];
        const int sr = sst[gi].reorth;
        if (sr == 1) {              // second projection pending
            atomicOr(&seed_cyc[gi], 1);
            continue;
        }
        if (sr == (pass == 1 ? 0 : 2)) {
            for (int i = 0; i <= k; ++i) hm[size_t(i) * M + m] = hs[size_t(i) * G + gi];
            hm[size_t(k) * M + m] += sigma[m];
            gm_givens(s, hm, nu[gi], H + size_t(m) * ld * restart, g + size_t(m) * ld, cs + size_t(m) * restart,
                      sn + size_t(m) * restart, k, ld, M, m, restart, tolv[m], bs[gi], maxiter);
            mst[m] = s;
        }
        if (s.cyc) atomicOr(&seed_cyc[gi], 1);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < G; t += blockDim.x) {
        flag[1 + t] = seed_cyc[t];
        sst[t].cyc = seed_cyc[t];
        if (seed_cyc[t]) atomicAdd(&n, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) flag[0] = n;
}

// The seeds' second projection (k_arn_finish pass 2, no Givens) and the
// members' Givens updates (shift_givens_body, pass 2) in one CTA: the members
// read only the seeds' Hessenberg column and norm, which the first part
// writes, so the seeds' normalisation of V_{k+1} can follow.
__global__ void __launch_bounds__(1024) k_seed_finish_givens(GState* __restrict__ sst, double2* __restrict__ h,
                                                             const double2* __restrict__ h2,
                                                             double* __restrict__ nu, double* __restrict__ inv_nu,
                                                             int k, int restart, int G, const double* __restrict__ bs,
                                                             double tol, int maxiter, GState* __restrict__ mst,
                                                             const double2* __restrict__ sigma,
                                                             const int* __restrict__ grp, double2* __restrict__ hm,
                                                             double2* __restrict__ H, double2* __restrict__ g,
                                                             double* __restrict__ cs, double2* __restrict__ sn, int M,
                                                             const double* __restrict__ tolv,
                                                             int* __restrict__ seed_cyc, int* __restrict__ flag) {
    arn_finish_body(sst, h, h2, 2, 0, 1, nu, inv_nu, nullptr, nullptr, nullptr, nullptr, k, restart, G, bs, tol,
                    nullptr, maxiter, flag);
    __syncthreads();
    shift_givens_body(mst, sst, h, nu, sigma, grp, G, 2, hm, H, g, cs, sn, k, restart, M, bs, tolv, maxiter,
                      seed_cyc, flag);
}

// member states: active and cycling from the start, x0 = 0; g_m = (beta, 0..);
// members already converged (skip[m], may be null) take no part
__global__ void k_shift_init(GState* __restrict__ mst, const int* __restrict__ grp, const double* __restrict__ bs,
                             const int* __restrict__ skip, double2* __restrict__ g, int restart, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    GState s{};
    const double beta = (skip && skip[m]) ? 0.0 : bs[grp[m]];
    s.active = beta > 0.0;
    s.cyc = s.active;
    s.converged = !s.active;
    mst[m] = s;
    g[size_t(m) * (restart + 1)] = make_double2(beta, 0.0);
    for (int i = 1; i <= restart; ++i) g[size_t(m) * (restart + 1) + i] = make_double2(0, 0);
}

// x[row][m] = sum_{i < kper[m]} V_i[row][grp[m]] y[i][m] (columns skipped
// as converged keep their x)
__global__ void k_shift_x(double2* __restrict__ x, const double2* __restrict__ V, size_t vstride, int G,
                          const double2* __restrict__ y, const int* __restrict__ grp, const int* __restrict__ kper,
                          const int* __restrict__ skip, int rows, int M) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(rows) * M) return;
    const size_t row = t / M;
    const int m = int(t - row * M);
    if (skip && skip[m]) return;
    const int gi = grp[m];
    double2 acc = make_double2(0, 0);
    for (int i = 0; i < kper[m]; ++i) acc += V[size_t(i) * vstride + row * G + gi] * y[size_t(i) * M + m];
    x[t] = acc;
}

// back substitution H y = g, y stored [i][m]
__global__ void k_gm_backsub(const GState* __restrict__ st, const double2* __restrict__ H,
                             const double2* __restrict__ g, double2* __restrict__ y, int restart, int M,
                             int* __restrict__ kper) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const int k = st[m].kcount;
    kper[m] = k;
    const int ld = restart + 1;
    const double2* Hm = H + size_t(m) * ld * restart;
    const double2* gm = g + size_t(m) * ld;
    for (int i = k - 1; i >= 0; --i) {
        double2 v = gm[i];
        for (int j = i + 1; j < k; ++j) v -= Hm[size_t(j) * ld + i] * y[size_t(j) * M + m];
        const double2 d = Hm[size_t(i) * ld + i];
        const double den = d.x * d.x + d.y * d.y;
        y[size_t(i) * M + m] = make_double2((v.x * d.x + v.y * d.y) / den, (v.y * d.x - v.x * d.y) / den);
    }
}

// seeds: cycling from the start unless their right-hand side is zero
__global__ void k_seed_init(GState* __restrict__ st, const double* __restrict__ bn, int G) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= G) return;
    GState s{};
    s.active = s.cyc = bn[m] > 0.0;
    st[m] = s;
}

__global__ void k_zero_rhs_cols(double2* __restrict__ x, const double* __restrict__ bn, size_t n, int M) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) return;
    if (bn[t % M] == 0.0) x[t] = make_double2(0, 0);
}

__global__ void k_gm_init(GState* __restrict__ st, const double* __restrict__ bn, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    GState s{};
    s.active = bn[m] > 0.0 ? 1 : 0;
    s.converged = bn[m] > 0.0 ? 0 : 1;
    st[m] = s;
}

// --------------------------------------------------------- BiCGSTAB state --

struct BState {
    double2 rho, alpha, omega, beta;
    int active, converged, iters, pad;
};

__global__ void k_bi_init(BState* __restrict__ st, const double* __restrict__ bn, const double* __restrict__ rn,
                          double tol, const double* __restrict__ tolv, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    BState s{};
    s.rho = s.alpha = s.omega = make_double2(1.0, 0.0);
    s.beta = make_double2(0, 0);
    s.active = 1;
    if (bn[m] == 0.0) { s.active = 0; s.converged = 1; }
    else if (rn[m] < col_tol(tol, tolv, m) * bn[m]) { s.active = 0; s.converged = 1; }
    st[m] = s;
}

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    const double den = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / den, (a.y * b.x - a.x * b.y) / den);
}
__device__ __forceinline__ double cabs_(double2 a) { return hypot(a.x, a.y); }

// step A: rho_new test and beta (bicgstab_solver.cu:153-169)
__global__ void k_bi_a(BState* __restrict__ st, const double2* __restrict__ rho_new, int it, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    BState s = st[m];
    if (!s.active) return;
    const double2 rn = rho_new[m];
    if (cabs_(rn) < 1e-16) { s.active = 0; st[m] = s; return; }
    s.beta = it > 0 ? cdiv(rn, s.rho) * cdiv(s.alpha, s.omega) : make_double2(0, 0);
    s.rho = rn;
    s.iters += 1;
    st[m] = s;
}

// p = r + beta (p - omega v)  (it > 0), p unchanged at it == 0
__global__ void k_bi_p(double2* __restrict__ p, const double2* __restrict__ v, const double2* __restrict__ r,
                       const BState* __restrict__ st, int it, size_t n, int M) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n || it == 0) return;
    const BState& s = st[t % M];
    if (!s.active) return;
    p[t] = (p[t] - s.omega * v[t]) * s.beta + r[t];
}

// step B: alpha = rho / (r0 . v)
__global__ void k_bi_b(BState* __restrict__ st, const double2* __restrict__ rv, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    BState s = st[m];
    if (!s.active) return;
    if (cabs_(rv[m]) < 1e-16) { s.active = 0; st[m] = s; return; }
    s.alpha = cdiv(s.rho, rv[m]);
    st[m] = s;
}

// s = r - alpha v
__global__ void k_bi_s(double2* __restrict__ sv, const double2* __restrict__ r, const double2* __restrict__ v,
                       const BState* __restrict__ st, size_t n, int M) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const BState& s = st[t % M];
    if (!s.active) return;
    sv[t] = r[t] - s.alpha * v[t];
}

// step C: |s| < tol |b| => x += alpha p and stop (mode 1)
__global__ void k_bi_c(BState* __restrict__ st, const double* __restrict__ sn, const double* __restrict__ bn,
                       double tol, const double* __restrict__ tolv, int* __restrict__ mode, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    BState s = st[m];
    mode[m] = 0;
    if (!s.active) return;
    if (sn[m] < col_tol(tol, tolv, m) * bn[m]) {
        mode[m] = 1;
        s.active = 0;
        s.converged = 1;
        st[m] = s;
    }
}

__global__ void k_bi_xfinal(double2* __restrict__ x, const double2* __restrict__ p, const BState* __restrict__ st,
                            const int* __restrict__ mode, size_t n, int M) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int m = int(t % M);
    if (mode[m] == 1) x[t] += st[m].alpha * p[t];
}

// step D: omega = (t, s) / (t, t)
__global__ void k_bi_d(BState* __restrict__ st, const double2* __restrict__ ts, const double2* __restrict__ tt, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    BState s = st[m];
    if (!s.active) return;
    if (cabs_(tt[m]) < 1e-16) { s.active = 0; st[m] = s; return; }
    s.omega = ts[m] * (1.0 / tt[m].x);
    st[m] = s;
}

// x += alpha p + omega s ; r = s - omega t
__global__ void k_bi_xr(double2* __restrict__ x, double2* __restrict__ r, const double2* __restrict__ p,
                        const double2* __restrict__ sv, const double2* __restrict__ tv,
                        const BState* __restrict__ st, size_t n, int M) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const BState& s = st[t % M];
    if (!s.active) return;
    x[t] += s.alpha * p[t] + s.omega * sv[t];
    r[t] = sv[t] - s.omega * tv[t];
}

// step E: |r| < tol |b| or omega ~ 0 => stop; count still active
__global__ void k_bi_e(BState* __restrict__ st, const double* __restrict__ rn, const double* __restrict__ bn,
                       double tol, const double* __restrict__ tolv, int maxiter, int* __restrict__ flag, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    BState s = st[m];
    if (s.active) {
        if (rn[m] < col_tol(tol, tolv, m) * bn[m]) { s.active = 0; s.converged = 1; }
        else if (cabs_(s.omega) < 1e-16) s.active = 0;
        else if (s.iters >= maxiter) s.active = 0;
        if (s.active) atomicAdd(flag, 1);
        st[m] = s;
    }
    flag[1 + m] = s.active;
}

__global__ void k_bi_count(const BState* __restrict__ st, int* __restrict__ flag, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    flag[1 + m] = st[m].active;
    if (st[m].active) atomicAdd(flag, 1);
}

// refinement bookkeeping: a column stays converged once its true residual
// met the target (later rounds leave its x and its stale residual alone)
__global__ void k_conv_update(const double* __restrict__ rn, const double* __restrict__ bn, double tol,
                              int* __restrict__ conv, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < M && !conv[m] && rn[m] <= tol * bn[m]) conv[m] = 1;
}

// zero the correction right-hand side of converged columns
__global__ void k_mask_conv(double2* __restrict__ r, const int* __restrict__ conv, size_t n, int M) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) return;
    if (conv[t % M]) r[t] = make_double2(0, 0);
}

// columns with sel[m] set take the fp64 residual (r, its norm) in place of
// the fp32 screen's
__global__ void k_take_cols(double2* __restrict__ r, const double2* __restrict__ r64, double* __restrict__ rn,
                            const double* __restrict__ rn64, const int* __restrict__ sel, size_t n, int M) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int m = int(t % M);
    if (!sel[m]) return;
    r[t] = r64[t];
    if (t < size_t(M)) rn[t] = rn64[t];
}

__global__ void k_axpy1(double2* __restrict__ x, const double2* __restrict__ d, size_t n) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < n) x[t] += d[t];
}

// dst[row][j] = src[row][idx[j]]  (compact batch of the listed columns)
__global__ void k_gather_cols(const double2* __restrict__ src, int M, double2* __restrict__ dst, int Ma,
                              const int* __restrict__ idx, int rows) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(rows) * Ma) return;
    const size_t row = t / Ma;
    const int j = int(t - row * Ma);
    dst[t] = src[row * M + idx[j]];
}

// dst[row][idx[j]] = src[row][j]
__global__ void k_scatter_cols(const double2* __restrict__ src, int Ma, double2* __restrict__ dst, int M,
                               const int* __restrict__ idx, int rows) {
    const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= size_t(rows) * Ma) return;
    const size_t row = t / Ma;
    const int j = int(t - row * Ma);
    dst[row * M + idx[j]] = src[t];
}

// inner tolerance of column m: stop once its residual is below 0.5 tol |b_m|,
// i.e. relative to its own right-hand side |r_m|: 0.5 tol |b_m| / |r_m|,
// but ask no inner solve for a reduction below `floor` (fp32 rounding of
// the operator limits what one inner solve can reach) nor above 0.5.
__global__ void k_inner_tol(const double* __restrict__ rn, const double* __restrict__ bn, double tol, double floor,
                            double* __restrict__ tolv, int M) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    double t = rn[m] > 0.0 ? 0.5 * tol * bn[m] / rn[m] : 0.5;
    tolv[m] = fmin(0.5, fmax(floor, t));
}

}  // namespace

// ------------------------------------------------------------ host side --

BatchSolver::BatchSolver() {
    MPM_CUDA(cudaMallocHost(&flag_, sizeof(int)));
    flag_cap_ = 1;
}
BatchSolver::~BatchSolver() {
    if (flag_) cudaFreeHost(flag_);
    if (hidx_) cudaFreeHost(hidx_);
}

int BatchSolver::read_flags(const int* dflag, int M, cudaStream_t s) {
    if (M + 1 > flag_cap_) {
        MPM_CUDA(cudaStreamSynchronize(s));
        if (flag_) MPM_CUDA(cudaFreeHost(flag_));
        flag_ = nullptr;
        MPM_CUDA(cudaMallocHost(&flag_, sizeof(int) * (M + 1)));
        flag_cap_ = M + 1;
    }
    MPM_CUDA(cudaMemcpyAsync(flag_, dflag, sizeof(int) * (M + 1), cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    return *flag_;
}

int BatchSolver::apply_cols(Field& F, const double2* X, double2* Y, int M, const double2* sc, bool jacobi,
                            bool r32, bool re32, const int* active, bool compact, cudaStream_t s) {
    if (!compact || !active) {
        F.apply(X, Y, M, sc, jacobi, r32, re32, s);
        return M;
    }
    std::vector<int> cols;
    cols.reserve(M);
    for (int m = 0; m < M; ++m)
        if (active[m]) cols.push_back(m);
    const int Ma = int(cols.size());
    if (Ma == 0) return 0;
    if (Ma == M) {
        F.apply(X, Y, M, sc, jacobi, r32, re32, s);
        return M;
    }
    const int rin = F.rows_in(), rout = F.rows_out(), N = F.num_particles();
    if (cols != cur_cols_) {
        StageScope scope(ST_KRYLOV, s);
        if (Ma > hidx_cap_) {
            MPM_CUDA(cudaStreamSynchronize(s));
            if (hidx_) MPM_CUDA(cudaFreeHost(hidx_));
            hidx_ = nullptr;
            MPM_CUDA(cudaMallocHost(&hidx_, sizeof(int) * M));
            hidx_cap_ = M;
        }
        // the previous upload from hidx_ has completed: every change of the
        // column set follows a flag read, which synchronises the stream
        std::copy(cols.begin(), cols.end(), hidx_);
        cidx_.ensure(sizeof(int) * M);
        MPM_CUDA(cudaMemcpyAsync(cidx_.p, hidx_, sizeof(int) * Ma, cudaMemcpyHostToDevice, s));
        if (sc) {
            scc_.ensure(sizeof(double2) * size_t(N) * M);
            k_gather_cols<<<nblk((long long)N * Ma, 256), 256, 0, s>>>(sc, M, scc_.as<double2>(), Ma,
                                                                        cidx_.as<int>(), N);
            MPM_LAUNCH();
        }
        cur_cols_ = cols;
    }
    xc_.ensure(sizeof(double2) * size_t(rin) * M);
    yc_.ensure(sizeof(double2) * size_t(rout) * M);
    {
        StageScope scope(ST_KRYLOV, s);
        k_gather_cols<<<nblk((long long)rin * Ma, 256), 256, 0, s>>>(X, M, xc_.as<double2>(), Ma, cidx_.as<int>(),
                                                                     rin);
        MPM_LAUNCH();
    }
    F.apply(xc_.as<double2>(), yc_.as<double2>(), Ma, sc ? scc_.as<double2>() : nullptr, jacobi, r32, re32, s);
    {
        StageScope scope(ST_KRYLOV, s);
        k_scatter_cols<<<nblk((long long)rout * Ma, 256), 256, 0, s>>>(yc_.as<double2>(), Ma, Y, M,
                                                                       cidx_.as<int>(), rout);
        MPM_LAUNCH();
    }
    return Ma;
}

void BatchSolver::dots(const double2* V, size_t vstride, int nvec, const double2* w, int rows, int M, int conj,
                       double2* out, cudaStream_t s, int shift) {
    StageScope scope(ST_KRYLOV, s);
    // four CTAs per SM: the sums are latency-bound, not bandwidth-bound
    if (M < 16) {
        const long long L = (256 / M) * M;
        const int gx = int(std::max(1LL, std::min(592LL, (1LL * rows * M + L - 1) / L)));
        const int nz = (nvec + 7) / 8;
        partial_.ensure(sizeof(double2) * size_t(gx) * nvec * M);
        if (!dots_done_.p || dots_done_.bytes < sizeof(unsigned int) * size_t(nz)) {
            dots_done_.ensure(sizeof(unsigned int) * std::max<size_t>(size_t(nz), 64));
            MPM_CUDA(cudaMemsetAsync(dots_done_.p, 0, dots_done_.bytes, s));
        }
        k_dots1s<<<dim3(gx, 1, nz), 256, 0, s>>>(V, vstride, nvec, w, rows, M, conj, partial_.as<double2>(), shift,
                                                 out, dots_done_.as<unsigned int>());
        MPM_LAUNCH();
        return;
    }
    const int gx = std::max(1, std::min(592, (rows + 7) / 8));
    partial_.ensure(sizeof(double2) * size_t(gx) * nvec * M);
    dim3 grd(gx, (M + 31) / 32, (nvec + 7) / 8);
    k_dots1<<<grd, dim3(32, 8), 0, s>>>(V, vstride, nvec, w, rows, M, conj, partial_.as<double2>(), shift);
    MPM_LAUNCH();
    k_dots2<<<nblk((long long)nvec * M * 32, 256), 256, 0, s>>>(partial_.as<double2>(), gx, nvec, M, out);
    MPM_LAUNCH();
}

void BatchSolver::norms(const double2* w, int rows, int M, double* out, cudaStream_t s) {
    h2_.ensure(sizeof(double2) * M);
    dots(w, 0, 1, w, rows, M, 1, h2_.as<double2>(), s);
    k_sqrt_re<<<nblk(M, 128), 128, 0, s>>>(h2_.as<double2>(), M, out);
    MPM_LAUNCH();
}

void BatchSolver::true_residual(Field& F, const double2* b, const double2* x, int M, const double2* sc,
                                std::vector<double>& out, cudaStream_t s) {
    const int rows = F.rows_in();
    const size_t n = size_t(rows) * M;
    w_.ensure(sizeof(double2) * n);
    rr_.ensure(sizeof(double2) * n);
    rnorm_.ensure(sizeof(double) * M * 2);
    F.apply(x, w_.as<double2>(), M, sc, false, false, false, s);
    k_sub<<<nblk((long long)n, 256), 256, 0, s>>>(b, w_.as<double2>(), rr_.as<double2>(), n);
    MPM_LAUNCH();
    norms(rr_.as<double2>(), rows, M, rnorm_.as<double>(), s);
    norms(b, rows, M, rnorm_.as<double>() + M, s);
    std::vector<double> h(2 * M);
    MPM_CUDA(cudaMemcpyAsync(h.data(), rnorm_.p, sizeof(double) * 2 * M, cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    out.resize(M);
    for (int m = 0; m < M; ++m) out[m] = h[M + m] > 0 ? h[m] / h[M + m] : 0.0;
}

void BatchSolver::gmres(Field& F, const double2* b, double2* x, int M, const double2* sc, const SolveOptions& opt,
                        SolveStats& st, bool r32, bool re32, cudaStream_t s, bool x_zero, const double* tolv,
                        bool precond_rel) {
    const int rows = F.rows_in();
    const size_t n = size_t(rows) * M;
    const int restart = std::max(1, std::min(rows, opt.restart));
    V_.ensure(sizeof(double2) * n * (restart + 1));
    H_.ensure(sizeof(double2) * size_t(M) * (restart + 1) * restart);
    g_.ensure(sizeof(double2) * size_t(M) * (restart + 1));
    cs_.ensure(sizeof(double) * size_t(M) * restart);
    sn_.ensure(sizeof(double2) * size_t(M) * restart);
    y_.ensure(sizeof(double2) * size_t(M) * restart);
    h_.ensure(sizeof(double2) * size_t(M) * (restart + 1));
    h2_.ensure(sizeof(double2) * size_t(M) * (restart + 1));
    bnorm_.ensure(sizeof(double) * M);
    rnorm_.ensure(sizeof(double) * M * 2);
    state_.ensure(sizeof(GState) * M + sizeof(int) * M);
    w_.ensure(sizeof(double2) * n);
    r_.ensure(sizeof(double2) * n);
    bj_.ensure(sizeof(double2) * n);
    flagdev_.ensure(sizeof(int) * (M + 2));   // count, M column flags, second-pass count
    cur_cols_.clear();  // self coefficients may differ from the previous call
    double2* V = V_.as<double2>();
    GState* gs = state_.as<GState>();
    int* kper = reinterpret_cast<int*>(gs + M);
    int* dflag = flagdev_.as<int>();
    const int mb = nblk(M, 128);
    const int vb = nblk((long long)n, 256);

    norms(b, rows, M, bnorm_.as<double>(), s);
    k_gm_init<<<mb, 128, 0, s>>>(gs, bnorm_.as<double>(), M);
    MPM_LAUNCH();
    k_zero_rhs_cols<<<vb, 256, 0, s>>>(x, bnorm_.as<double>(), n, M);
    MPM_LAUNCH();
    const double2* bj = b;
    if (opt.jacobi) {
        k_jacobi<<<vb, 256, 0, s>>>(b, bj_.as<double2>(), F.num_particles(), F.num_quads(), M, F.quad_idx_dev(), sc);
        MPM_LAUNCH();
        bj = bj_.as<double2>();
        if (precond_rel) norms(bj, rows, M, bnorm_.as<double>(), s);
    }
    // columns cycling at the start of the current cycle (empty: all)
    std::vector<int> begin_cols;
    bool first = true;
    while (true) {
        // r = D^-1 (b - A x), for the columns that cycled last time
        if (first && x_zero) {
            MPM_CUDA(cudaMemcpyAsync(r_.p, bj, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
        } else {
            st.column_matvecs += apply_cols(F, x, w_.as<double2>(), M, sc, opt.jacobi, r32, re32,
                                            begin_cols.empty() ? nullptr : begin_cols.data(), opt.compact, s);
            st.matvecs++;
            k_sub<<<vb, 256, 0, s>>>(bj, w_.as<double2>(), r_.as<double2>(), n);
            MPM_LAUNCH();
        }
        first = false;
        norms(r_.as<double2>(), rows, M, rnorm_.as<double>(), s);
        MPM_CUDA(cudaMemsetAsync(dflag, 0, sizeof(int), s));
        k_gm_begin<<<mb, 128, 0, s>>>(gs, rnorm_.as<double>(), bnorm_.as<double>(), opt.tol, tolv, opt.maxiter,
                                      restart, g_.as<double2>(), M, dflag);
        MPM_LAUNCH();
        k_normalize<<<vb, 256, 0, s>>>(r_.as<double2>(), V, rnorm_.as<double>(), gs, n, M);
        MPM_LAUNCH();
        if (read_flags(dflag, M, s) == 0) break;
        begin_cols.assign(flag_ + 1, flag_ + 1 + M);
        std::vector<int> cyc = begin_cols;
        for (int k = 0; k < restart; ++k) {
            double2* Vk = V + size_t(k) * n;
            double2* w = V + size_t(k + 1) * n;   // A V_k lands in V_{k+1}, projected and normalised in place
            st.column_matvecs += apply_cols(F, Vk, w, M, sc, opt.jacobi, r32, re32, cyc.data(), opt.compact, s);
            st.matvecs++;
            const int fthr = std::min(1024, ((M + 31) / 32) * 32);
            auto finish = [&](int pass) {
                k_arn_finish<<<1, fthr, 0, s>>>(gs, h_.as<double2>(), h2_.as<double2>(), pass, 1, 1, nullptr,
                                                rnorm_.as<double>(), H_.as<double2>(), g_.as<double2>(), cs_.as<double>(),
                                                sn_.as<double2>(), k, restart, M, bnorm_.as<double>(), opt.tol, tolv,
                                                opt.maxiter, dflag);
                MPM_LAUNCH();
            };
            auto update = [&](const double2* hv, int pass) {
                k_arn_update<<<vb, 256, 0, s>>>(V, n, k, hv, gs, rnorm_.as<double>(), rows, M, pass);
                MPM_LAUNCH();
            };
            // CGS2: [V_0..V_k, u]^H u with u = w - V_k (the preconditioned
            // operator is close to the identity, so w is mostly V_k: the
            // first projection then works on the part that is not), w -= V h;
            // then [V_0..V_k, w']^H w', w' -= V h2, normalised; one flag read
            dots(V, n, k + 2, w, rows, M, 1, h_.as<double2>(), s, k);
            {
                StageScope sc1(ST_KRYLOV, s);
                finish(1);
                update(h_.as<double2>(), 1);
            }
            dots(V, n, k + 2, w, rows, M, 1, h2_.as<double2>(), s);
            {
                StageScope sc2(ST_KRYLOV, s);
                finish(2);
                update(h2_.as<double2>(), 2);
            }
            st.reorth_steps++;
            // the count and the M column flags
            const int left = read_flags(dflag, M, s);
            if (left == 0) break;
            cyc.assign(flag_ + 1, flag_ + 1 + M);
        }
        k_gm_backsub<<<mb, 128, 0, s>>>(gs, H_.as<double2>(), g_.as<double2>(), y_.as<double2>(), restart, M, kper);
        MPM_LAUNCH();
        k_vupdate<<<vb, 256, 0, s>>>(x, V, n, restart, y_.as<double2>(), rows, M, 1.0, kper);
        MPM_LAUNCH();
    }
    std::vector<GState> h(M);
    MPM_CUDA(cudaMemcpyAsync(h.data(), gs, sizeof(GState) * M, cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    st.iters.resize(M);
    st.converged.resize(M);
    for (int m = 0; m < M; ++m) {
        st.iters[m] += h[m].iters;
        st.converged[m] = h[m].converged;
    }
}

bool BatchSolver::detect_shifts(const double2* b, const double2* sc, int rows, int N, int M, cudaStream_t s,
                                std::vector<int>& grp, std::vector<double2>& f) {
    if (M < 2 || M > 1024 || !sc) return false;
    shf_.ensure(sizeof(double2) * M);
    shflag_.ensure(sizeof(int) * (size_t(M) + size_t(M) * M));
    int* bad = shflag_.as<int>();
    int* eq = bad + M;
    MPM_CUDA(cudaMemsetAsync(eq, 0, sizeof(int) * size_t(M) * M, s));
    k_shift_ratio<<<M, 256, 0, s>>>(sc, N, M, shf_.as<double2>(), bad);
    MPM_LAUNCH();
    k_col_equal<<<dim3(M, M), 256, 0, s>>>(b, rows, M, eq);
    MPM_LAUNCH();
    std::vector<int> h(size_t(M) + size_t(M) * M);
    f.resize(M);
    MPM_CUDA(cudaMemcpyAsync(h.data(), bad, sizeof(int) * h.size(), cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaMemcpyAsync(f.data(), shf_.p, sizeof(double2) * M, cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    for (int m = 0; m < M; ++m)
        if (h[m]) return false;
    grp.assign(M, -1);
    int G = 0;
    for (int m = 0; m < M; ++m) {
        for (int m2 = 0; m2 < m && grp[m] < 0; ++m2)
            if (h[M + size_t(m) * M + m2]) grp[m] = grp[m2];
        if (grp[m] < 0) grp[m] = G++;
    }
    return G < M;   // no shared right-hand side: nothing to gain
}

void BatchSolver::gmres_shifted(Field& F, const double2* b, double2* x, int M, const double2* sc,
                                const SolveOptions& opt, SolveStats& st, bool r32, bool re32, cudaStream_t s,
                                const double* tolv, const std::vector<int>& grp, const std::vector<double2>& f,
                                const int* skip, const int* live) {
    const int rows = F.rows_in(), N = F.num_particles();
    const int G = 1 + *std::max_element(grp.begin(), grp.end());
    const int restart = std::max(1, std::min(rows, opt.restart));
    const size_t ns = size_t(rows) * G;
    std::vector<int> seed(G, -1), zeros(G, 0);
    for (int m = 0; m < M; ++m)
        if (seed[grp[m]] < 0) seed[grp[m]] = m;
    std::vector<double2> sigma(M);
    for (int m = 0; m < M; ++m) sigma[m] = make_double2(f[m].x - 1.0, f[m].y);
    // device copies: member -> seed, seed columns, zero indices (ints), then
    // sigma (double2) at a 16-byte aligned offset
    const size_t sig_off = (sizeof(int) * (size_t(M) + 2 * G) + 15) & ~size_t(15);
    shmeta_.ensure(sig_off + sizeof(double2) * M);
    int* dgrp = shmeta_.as<int>();
    int* dseed = dgrp + M;
    int* dzero = dseed + G;
    double2* dsig = reinterpret_cast<double2*>(shmeta_.as<char>() + sig_off);
    MPM_CUDA(cudaMemcpyAsync(dgrp, grp.data(), sizeof(int) * M, cudaMemcpyHostToDevice, s));
    MPM_CUDA(cudaMemcpyAsync(dseed, seed.data(), sizeof(int) * G, cudaMemcpyHostToDevice, s));
    MPM_CUDA(cudaMemcpyAsync(dzero, zeros.data(), sizeof(int) * G, cudaMemcpyHostToDevice, s));
    MPM_CUDA(cudaMemcpyAsync(dsig, sigma.data(), sizeof(double2) * M, cudaMemcpyHostToDevice, s));
    // seed operator: self coefficients c = sc[:, 0] for every seed, Jacobi
    // scaling: A0 = diag(c)^-1 G + I; seed right-hand sides diag(c)^-1 b
    shsc_.ensure(sizeof(double2) * size_t(N) * G);
    shb_.ensure(sizeof(double2) * ns * 2);
    double2* scs = shsc_.as<double2>();
    double2* sb = shb_.as<double2>();
    double2* sbj = sb + ns;
    k_gather_cols<<<nblk((long long)N * G, 256), 256, 0, s>>>(sc, M, scs, G, dzero, N);
    MPM_LAUNCH();
    k_gather_cols<<<nblk((long long)ns, 256), 256, 0, s>>>(b, M, sb, G, dseed, rows);
    MPM_LAUNCH();
    k_jacobi<<<nblk((long long)ns, 256), 256, 0, s>>>(sb, sbj, N, F.num_quads(), G, F.quad_idx_dev(), scs);
    MPM_LAUNCH();
    V_.ensure(sizeof(double2) * ns * (restart + 1));
    H_.ensure(sizeof(double2) * size_t(M) * (restart + 1) * restart);
    g_.ensure(sizeof(double2) * size_t(M) * (restart + 1));
    cs_.ensure(sizeof(double) * size_t(M) * restart);
    sn_.ensure(sizeof(double2) * size_t(M) * restart);
    y_.ensure(sizeof(double2) * size_t(M) * restart);
    h_.ensure(sizeof(double2) * size_t(G) * (restart + 1));
    h2_.ensure(sizeof(double2) * size_t(G) * (restart + 1));
    hm_.ensure(sizeof(double2) * size_t(M) * (restart + 1));
    state_.ensure(sizeof(GState) * M + sizeof(int) * M);
    // seed states, seed cycling flags, then |b~| and |w'| per seed (8-byte aligned)
    const size_t bs_off = (sizeof(GState) * G + sizeof(int) * G + 7) & ~size_t(7);
    shst_.ensure(bs_off + 2 * sizeof(double) * G);
    rnorm_.ensure(sizeof(double) * std::max(M, G) * 2);
    flagdev_.ensure(sizeof(int) * (G + 2));
    cur_cols_.clear();
    double2* V = V_.as<double2>();
    GState* mst = state_.as<GState>();
    int* kper = reinterpret_cast<int*>(mst + M);
    GState* sst = shst_.as<GState>();
    int* scyc = reinterpret_cast<int*>(sst + G);
    double* bs = reinterpret_cast<double*>(shst_.as<char>() + bs_off);
    double* nu = bs + G;
    int* dflag = flagdev_.as<int>();
    norms(sbj, rows, G, bs, s);
    k_seed_init<<<nblk(G, 128), 128, 0, s>>>(sst, bs, G);
    MPM_LAUNCH();
    k_shift_init<<<nblk(M, 128), 128, 0, s>>>(mst, dgrp, bs, skip, g_.as<double2>(), restart, M);
    MPM_LAUNCH();
    k_normalize<<<nblk((long long)ns, 256), 256, 0, s>>>(sbj, V, bs, sst, ns, G);
    MPM_LAUNCH();
    std::vector<double> hbs(G);
    MPM_CUDA(cudaMemcpyAsync(hbs.data(), bs, sizeof(double) * G, cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    std::vector<int> cyc(G);
    std::vector<int> used(G, live ? 0 : 1);
    for (int m = 0; m < M && live; ++m) used[grp[m]] |= live[m] != 0;
    for (int gi = 0; gi < G; ++gi) cyc[gi] = hbs[gi] > 0.0 && used[gi];
    const int vb = nblk((long long)ns, 256);
    const int fthr = std::min(1024, ((std::max(M, G) + 31) / 32) * 32);
    for (int k = 0; k < restart; ++k) {
        if (std::count(cyc.begin(), cyc.end(), 1) == 0) break;
        double2* Vk = V + size_t(k) * ns;
        double2* w = V + size_t(k + 1) * ns;
        st.column_matvecs += apply_cols(F, Vk, w, G, scs, true, r32, re32, cyc.data(), opt.compact, s);
        st.matvecs++;
        auto seed_pass = [&](int pass, const double2* hv) {
            // (every seed takes both projections: the members' Givens updates
            // follow the second, in the same one-CTA kernel)
            StageScope sc1(ST_KRYLOV, s);
            if (pass == 1) {
                k_arn_finish<<<1, fthr, 0, s>>>(sst, h_.as<double2>(), h2_.as<double2>(), pass, 0, 1, nu,
                                                rnorm_.as<double>(), nullptr, nullptr, nullptr, nullptr, k, restart,
                                                G, bs, opt.tol, nullptr, opt.maxiter, dflag);
            } else {
                k_seed_finish_givens<<<1, fthr, 0, s>>>(sst, h_.as<double2>(), h2_.as<double2>(), nu,
                                                        rnorm_.as<double>(), k, restart, G, bs, opt.tol,
                                                        opt.maxiter, mst, dsig, dgrp, hm_.as<double2>(),
                                                        H_.as<double2>(), g_.as<double2>(), cs_.as<double>(),
                                                        sn_.as<double2>(), M, tolv, scyc, dflag);
            }
            MPM_LAUNCH();
            k_arn_update<<<vb, 256, 0, s>>>(V, ns, k, hv, sst, rnorm_.as<double>(), rows, G, pass);
            MPM_LAUNCH();
        };
        dots(V, ns, k + 2, w, rows, G, 1, h_.as<double2>(), s, k);
        seed_pass(1, h_.as<double2>());
        dots(V, ns, k + 2, w, rows, G, 1, h2_.as<double2>(), s);
        seed_pass(2, h2_.as<double2>());
        st.reorth_steps++;
        const int left = read_flags(dflag, G, s);
        if (left == 0) break;
        cyc.assign(flag_ + 1, flag_ + 1 + G);
    }
    k_gm_backsub<<<nblk(M, 128), 128, 0, s>>>(mst, H_.as<double2>(), g_.as<double2>(), y_.as<double2>(), restart, M,
                                              kper);
    MPM_LAUNCH();
    k_shift_x<<<nblk((long long)rows * M, 256), 256, 0, s>>>(x, V, ns, G, y_.as<double2>(), dgrp, kper, skip, rows,
                                                             M);
    MPM_LAUNCH();
    std::vector<GState> h(M);
    MPM_CUDA(cudaMemcpyAsync(h.data(), mst, sizeof(GState) * M, cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    st.iters.resize(M);
    st.converged.resize(M);
    for (int m = 0; m < M; ++m) {
        st.iters[m] += h[m].iters;
        st.converged[m] = h[m].converged;
    }
    st.shift_seeds = G;
}

void BatchSolver::bicgstab(Field& F, const double2* b, double2* x, int M, const double2* sc, const SolveOptions& opt,
                           SolveStats& st, bool r32, bool re32, cudaStream_t s, bool x_zero, const double* tolv,
                        bool precond_rel) {
    const int rows = F.rows_in();
    const size_t n = size_t(rows) * M;
    for (DevBuf* d : {&r0_, &p_, &v_, &s_, &t_, &r_, &w_, &bj_}) d->ensure(sizeof(double2) * n);
    bnorm_.ensure(sizeof(double) * M);
    rnorm_.ensure(sizeof(double) * M * 2);
    scal_.ensure(sizeof(BState) * M + sizeof(int) * M);
    h_.ensure(sizeof(double2) * M * 2);
    flagdev_.ensure(sizeof(int) * (M + 1));
    cur_cols_.clear();
    BState* bs = scal_.as<BState>();
    int* mode = reinterpret_cast<int*>(bs + M);
    int* dflag = flagdev_.as<int>();
    double2* hv = h_.as<double2>();
    const int mb = nblk(M, 128);
    const int vb = nblk((long long)n, 256);

    norms(b, rows, M, bnorm_.as<double>(), s);
    k_zero_rhs_cols<<<vb, 256, 0, s>>>(x, bnorm_.as<double>(), n, M);
    MPM_LAUNCH();
    const double2* bj = b;
    if (opt.jacobi) {
        k_jacobi<<<vb, 256, 0, s>>>(b, bj_.as<double2>(), F.num_particles(), F.num_quads(), M, F.quad_idx_dev(), sc);
        MPM_LAUNCH();
        bj = bj_.as<double2>();
        if (precond_rel) norms(bj, rows, M, bnorm_.as<double>(), s);
    }
    double2* r = r_.as<double2>();
    if (x_zero) {
        MPM_CUDA(cudaMemcpyAsync(r, bj, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
    } else {
        F.apply(x, w_.as<double2>(), M, sc, opt.jacobi, r32, re32, s);
        st.matvecs++;
        st.column_matvecs += M;
        k_sub<<<vb, 256, 0, s>>>(bj, w_.as<double2>(), r, n);
        MPM_LAUNCH();
    }
    norms(r, rows, M, rnorm_.as<double>(), s);
    k_bi_init<<<mb, 128, 0, s>>>(bs, bnorm_.as<double>(), rnorm_.as<double>(), opt.tol, tolv, M);
    MPM_LAUNCH();
    MPM_CUDA(cudaMemcpyAsync(r0_.p, r, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
    MPM_CUDA(cudaMemcpyAsync(p_.p, r, sizeof(double2) * n, cudaMemcpyDeviceToDevice, s));
    MPM_CUDA(cudaMemsetAsync(v_.p, 0, sizeof(double2) * n, s));
    MPM_CUDA(cudaMemsetAsync(dflag, 0, sizeof(int), s));
    k_bi_count<<<mb, 128, 0, s>>>(bs, dflag, M);
    MPM_LAUNCH();
    if (read_flags(dflag, M, s) > 0) {
        std::vector<int> act(flag_ + 1, flag_ + 1 + M);
        for (int it = 0; it < opt.maxiter; ++it) {
            dots(r0_.as<double2>(), 0, 1, r, rows, M, 0, hv, s);
            k_bi_a<<<mb, 128, 0, s>>>(bs, hv, it, M);
            MPM_LAUNCH();
            k_bi_p<<<vb, 256, 0, s>>>(p_.as<double2>(), v_.as<double2>(), r, bs, it, n, M);
            MPM_LAUNCH();
            st.column_matvecs += apply_cols(F, p_.as<double2>(), v_.as<double2>(), M, sc, opt.jacobi, r32, re32,
                                            act.data(), opt.compact, s);
            st.matvecs++;
            dots(r0_.as<double2>(), 0, 1, v_.as<double2>(), rows, M, 0, hv, s);
            k_bi_b<<<mb, 128, 0, s>>>(bs, hv, M);
            MPM_LAUNCH();
            k_bi_s<<<vb, 256, 0, s>>>(s_.as<double2>(), r, v_.as<double2>(), bs, n, M);
            MPM_LAUNCH();
            norms(s_.as<double2>(), rows, M, rnorm_.as<double>(), s);
            k_bi_c<<<mb, 128, 0, s>>>(bs, rnorm_.as<double>(), bnorm_.as<double>(), opt.tol, tolv, mode, M);
            MPM_LAUNCH();
            k_bi_xfinal<<<vb, 256, 0, s>>>(x, p_.as<double2>(), bs, mode, n, M);
            MPM_LAUNCH();
            st.column_matvecs += apply_cols(F, s_.as<double2>(), t_.as<double2>(), M, sc, opt.jacobi, r32, re32,
                                            act.data(), opt.compact, s);
            st.matvecs++;
            dots(t_.as<double2>(), 0, 1, s_.as<double2>(), rows, M, 1, hv, s);
            dots(t_.as<double2>(), 0, 1, t_.as<double2>(), rows, M, 1, hv + M, s);
            k_bi_d<<<mb, 128, 0, s>>>(bs, hv, hv + M, M);
            MPM_LAUNCH();
            k_bi_xr<<<vb, 256, 0, s>>>(x, r, p_.as<double2>(), s_.as<double2>(), t_.as<double2>(), bs, n, M);
            MPM_LAUNCH();
            norms(r, rows, M, rnorm_.as<double>(), s);
            MPM_CUDA(cudaMemsetAsync(dflag, 0, sizeof(int), s));
            k_bi_e<<<mb, 128, 0, s>>>(bs, rnorm_.as<double>(), bnorm_.as<double>(), opt.tol, tolv, opt.maxiter, dflag,
                                      M);
            MPM_LAUNCH();
            if (read_flags(dflag, M, s) == 0) break;
            act.assign(flag_ + 1, flag_ + 1 + M);
        }
    }
    std::vector<BState> h(M);
    MPM_CUDA(cudaMemcpyAsync(h.data(), bs, sizeof(BState) * M, cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    st.iters.resize(M);
    st.converged.resize(M);
    for (int m = 0; m < M; ++m) {
        st.iters[m] += h[m].iters;
        st.converged[m] = h[m].converged;
    }
}

void BatchSolver::solve(Field& F, const double2* b, double2* x, int M, const double2* sc, const SolveOptions& opt,
                        SolveStats& st, cudaStream_t s) {
    st.iters.assign(M, 0);
    st.converged.assign(M, 0);
    st.matvecs = 0;
    st.column_matvecs = 0;
    st.refine_steps = 0;
    st.reorth_steps = 0;
    st.shift_seeds = 0;
    st.fp64_matvecs = 0;
    if (!opt.refine) {
        if (opt.method == SOLVER_BICGSTAB) bicgstab(F, b, x, M, sc, opt, st, opt.recip_fp32, opt.real_fp32, s);
        else gmres(F, b, x, M, sc, opt, st, opt.recip_fp32, opt.real_fp32, s);
        return;
    }
    // Mixed-precision iterative refinement: fp64 true residual outside,
    // fp32 operator inside.
    const int rows = F.rows_in();
    const size_t n = size_t(rows) * M;
    xr_.ensure(sizeof(double2) * n);
    d_.ensure(sizeof(double2) * n);
    bn2_.ensure(sizeof(double) * M);
    rn2_.ensure(sizeof(double) * M);
    convd_.ensure(sizeof(int) * M);
    double* bn2 = bn2_.as<double>();
    double* rn2 = rn2_.as<double>();
    int* convd = convd_.as<int>();
    const int vb = nblk((long long)n, 256);
    norms(b, rows, M, bn2, s);
    MPM_CUDA(cudaMemsetAsync(convd, 0, sizeof(int) * M, s));
    SolveOptions in = opt;
    in.refine = false;
    const double floor = opt.inner_tol > 0.0 ? opt.inner_tol : 1e-4;
    in.tol = 0.5;
    tolv_.ensure(sizeof(double) * M);
    std::vector<int> conv(M, 0), act(M, 1);
    st.rel_resid.assign(M, 0.0);
    cur_cols_.clear();
    // Shifted structure (one particle profile of self coefficients, shared
    // right-hand sides: a frequency sweep of one material): the first
    // correction is solved from x = 0 for all columns at once on the seeds'
    // Krylov spaces; later corrections are per column.
    std::vector<int> grp;
    std::vector<double2> fsh;
    // (quadrupole rows carry 2.5 s / a^2 + 0.5 g on the diagonal, which is
    // not a multiple of s: no shifted family with quadrupoles)
    const bool shifted = opt.shifted && opt.method == SOLVER_GMRES && F.num_quads() == 0 &&
                         detect_shifts(b, sc, rows, F.num_particles(), M, s, grp, fsh);
    bool reset = false;   // x replaced by the shifted solve from zero: every column active again
    std::vector<double> hb(M), hr(M);
    for (int step = 0; step < opt.max_refine; ++step) {
        // true residual of the columns not yet converged (a converged
        // column's x no longer changes).  The initial guess is screened with
        // the fp32 operator first: a column whose fp32 residual is above
        // 4 tol is not converged whatever the fp32 operator's error (about
        // 1e-7 relative), so only the columns below that take the fp64
        // residual; every later check is fp64 for all unconverged columns.
        const bool screen = step == 0 && !reset && opt.tol < 0.25;
        st.column_matvecs += apply_cols(F, x, xr_.as<double2>(), M, sc, false, screen, screen,
                                        step == 0 || reset ? nullptr : act.data(), opt.compact, s);
        reset = false;
        st.matvecs++;
        if (!screen) st.fp64_matvecs++;
        k_sub<<<vb, 256, 0, s>>>(b, xr_.as<double2>(), xr_.as<double2>(), n);
        MPM_LAUNCH();
        norms(xr_.as<double2>(), rows, M, rn2, s);
        if (screen) {
            MPM_CUDA(cudaMemcpyAsync(hb.data(), bn2, sizeof(double) * M, cudaMemcpyDeviceToHost, s));
            MPM_CUDA(cudaMemcpyAsync(hr.data(), rn2, sizeof(double) * M, cudaMemcpyDeviceToHost, s));
            MPM_CUDA(cudaStreamSynchronize(s));
            std::vector<int> near(M, 0);
            int nnear = 0;
            for (int m = 0; m < M; ++m) {
                near[m] = hr[m] <= 4.0 * opt.tol * hb[m];
                nnear += near[m];
            }
            if (nnear) {
                // fp64 residual of those columns into d_, swapped in
                st.column_matvecs += apply_cols(F, x, d_.as<double2>(), M, sc, false, false, false, near.data(),
                                                opt.compact, s);
                st.matvecs++;
                st.fp64_matvecs++;
                k_sub<<<vb, 256, 0, s>>>(b, d_.as<double2>(), d_.as<double2>(), n);
                MPM_LAUNCH();
                sel_.ensure(sizeof(int) * M);
                rn64_.ensure(sizeof(double) * M);
                norms(d_.as<double2>(), rows, M, rn64_.as<double>(), s);
                MPM_CUDA(cudaMemcpyAsync(sel_.p, near.data(), sizeof(int) * M, cudaMemcpyHostToDevice, s));
                k_take_cols<<<vb, 256, 0, s>>>(xr_.as<double2>(), d_.as<double2>(), rn2, rn64_.as<double>(),
                                               sel_.as<int>(), n, M);
                MPM_LAUNCH();
            }
        }
        k_conv_update<<<nblk(M, 128), 128, 0, s>>>(rn2, bn2, opt.tol, convd, M);
        MPM_LAUNCH();
        MPM_CUDA(cudaMemcpyAsync(hb.data(), bn2, sizeof(double) * M, cudaMemcpyDeviceToHost, s));
        MPM_CUDA(cudaMemcpyAsync(hr.data(), rn2, sizeof(double) * M, cudaMemcpyDeviceToHost, s));
        MPM_CUDA(cudaStreamSynchronize(s));
        int left = 0;
        for (int m = 0; m < M; ++m) {
            if (!act[m]) continue;  // converged in an earlier round
            st.rel_resid[m] = hb[m] > 0 ? hr[m] / hb[m] : 0.0;
            conv[m] = hr[m] <= opt.tol * hb[m];
            act[m] = !conv[m];
            left += act[m];
        }
        if (!left) break;
        double best = 1e300;
        int live_seeds = 0;
        if (shifted) {
            std::vector<char> seen(M, 0);
            for (int m = 0; m < M; ++m)
                if (act[m] && !seen[grp[m]]) {
                    seen[grp[m]] = 1;
                    ++live_seeds;
                }
        }
        for (int m = 0; m < M; ++m)
            if (act[m]) best = std::min(best, st.rel_resid[m]);
        if (step == 0 && shifted && (best >= 0.05 || left >= 8 * live_seeds)) {
            // a poor initial guess (every unconverged column's residual at
            // least 5% of |b|), or at least eight unconverged columns per
            // seed (the seeds' Krylov spaces cost a small part of per-column
            // solves even from x = 0): those columns start again from x = 0
            // and their first correction is solved on the seeds' Krylov
            // spaces; converged columns (a warm start) keep their x.  The
            // target is the outer one (half of it, no inner floor): the
            // seeds' GMRES works in fp64 on the fp32 operator, so its
            // residual estimate keeps falling below the fp32 operator error,
            // and a first correction this tight usually leaves nothing for
            // the per-column corrections but the fp64 check
            k_inner_tol<<<nblk(M, 128), 128, 0, s>>>(bn2, bn2, opt.tol, 0.0, tolv_.as<double>(), M);
            MPM_LAUNCH();
            SolveStats inner;
            inner.iters.assign(M, 0);
            gmres_shifted(F, b, x, M, sc, in, inner, true, true, s, tolv_.as<double>(), grp, fsh, convd,
                          act.data());
            for (int m = 0; m < M; ++m) st.iters[m] += inner.iters[m];
            st.matvecs += inner.matvecs;
            st.column_matvecs += inner.column_matvecs;
            st.reorth_steps += inner.reorth_steps;
            st.shift_seeds = inner.shift_seeds;
            st.refine_steps++;
            reset = true;
            continue;
        }
        k_mask_conv<<<vb, 256, 0, s>>>(xr_.as<double2>(), convd, n, M);
        MPM_LAUNCH();
        MPM_CUDA(cudaMemsetAsync(d_.p, 0, sizeof(double2) * n, s));
        k_inner_tol<<<nblk(M, 128), 128, 0, s>>>(rn2, bn2, opt.tol, floor, tolv_.as<double>(), M);
        MPM_LAUNCH();
        const double* tolv = tolv_.as<double>();
        SolveStats inner;
        inner.iters.assign(M, 0);
        if (opt.method == SOLVER_BICGSTAB)
            bicgstab(F, xr_.as<double2>(), d_.as<double2>(), M, sc, in, inner, true, true, s, true, tolv, true);
        else
            gmres(F, xr_.as<double2>(), d_.as<double2>(), M, sc, in, inner, true, true, s, true, tolv, true);
        k_axpy1<<<vb, 256, 0, s>>>(x, d_.as<double2>(), n);
        MPM_LAUNCH();
        for (int m = 0; m < M; ++m) st.iters[m] += inner.iters[m];
        st.matvecs += inner.matvecs;
        st.column_matvecs += inner.column_matvecs;
        st.reorth_steps += inner.reorth_steps;
        st.refine_steps++;
    }
    for (int m = 0; m < M; ++m) st.converged[m] = conv[m];
}

}  // namespace mpm
