// Batched in-place 1-D DFT along a strided axis (see mpm_fft.h).
#include "mpm_fft.h"
#include "mpm_fft_consts.cuh"

#include <algorithm>
#include <type_traits>
#include <utility>
#include <cmath>
#include <vector>

namespace mpm {

namespace {

constexpr int kFftThreads = 256;
constexpr size_t kFftSmemBudget = 110 * 1024;   // two CTAs per SM (228 KB per SM)
constexpr size_t kFftSmemMax = 220 * 1024;

// Stockham autosort, mixed radix.  With Ns = product of the radices already
// applied and L = Ns * r, butterfly j (j < n/r, k1 = j mod Ns) reads
// x_q = in[j + q n/r] * W_L^(q k1) (q < r; q k1 < L, no reduction needed)
// and writes out[(j/Ns) L + p Ns + k1] = sum_q x_q W_r^(p q), W = exp(-+2 pi i/.).
// Outputs come in conjugate pairs (p, r - p) since W_r^((r-p) q) is the
// conjugate of W_r^(p q).  Each CTA owns CW adjacent columns of one line;
// thread = (row lane, column), CW a power of two.

// small radices: the r twiddled inputs live in registers
template <typename R, int CW, int MAXR>
__device__ __forceinline__ void pass_reg(const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                                         const cplx<R>* __restrict__ T, const int2* __restrict__ jt, int n, int r,
                                         int L) {
    constexpr int ROWS = kFftThreads / CW;
    const int c = threadIdx.x & (CW - 1);
    const int lane = threadIdx.x / CW;
    const int nr = n / r;
    const int stepL = n / L;
    const int stepR = nr;
    const int H = r / 2 + 1;
    const int Ns = L / r;
    for (int j = lane; j < nr; j += ROWS) {
        const int2 kb = jt[j];  // (k1, output base)
        cplx<R> x[MAXR];
#pragma unroll
        for (int q = 0; q < MAXR; ++q) {
            if (q < r) {
                const cplx<R> v = in[(j + q * nr) * CW + c];
                const cplx<R> w = T[q * kb.x * stepL];
                x[q] = mk<R>(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
            }
        }
        for (int h = 0; h < H; ++h) {
            R s1 = R(0), s2 = R(0), s3 = R(0), s4 = R(0);
            int ep = 0;
#pragma unroll
            for (int q = 0; q < MAXR; ++q) {
                if (q < r) {
                    const cplx<R> w = T[ep * stepR];
                    s1 = fma(x[q].x, w.x, s1);
                    s2 = fma(x[q].y, w.y, s2);
                    s3 = fma(x[q].x, w.y, s3);
                    s4 = fma(x[q].y, w.x, s4);
                    ep += h;
                    if (ep >= r) ep -= r;
                }
            }
            out[(kb.y + h * Ns) * CW + c] = mk<R>(s1 - s2, s3 + s4);
            if (h > 0 && 2 * h != r) out[(kb.y + (r - h) * Ns) * CW + c] = mk<R>(s1 + s2, s4 - s3);
        }
    }
}

// -i v (forward rotation) or +i v (inverse)
template <typename R, bool INV>
__device__ __forceinline__ cplx<R> rot(cplx<R> v) {
    return INV ? mk<R>(-v.y, v.x) : mk<R>(v.y, -v.x);
}

template <typename R, bool INV, int RAD>
__device__ __forceinline__ void dft_small(cplx<R> (&x)[RAD]);

// W_N^j = exp(-2 pi i j / N) (conjugated for INV) from the constant tables
template <typename R, bool INV, int N>
__device__ __forceinline__ cplx<R> wconst(int j) {
    cplx<R> w;
    static_assert(N == 7 || (N >= 9 && N <= 16), "no constant table for this radix");
    if constexpr (sizeof(R) == 8) {
        if constexpr (N == 7) w = kW7d[j];
        else if constexpr (N == 9) w = kW9d[j];
        else if constexpr (N == 10) w = kW10d[j];
        else if constexpr (N == 11) w = kW11d[j];
        else if constexpr (N == 12) w = kW12d[j];
        else if constexpr (N == 13) w = kW13d[j];
        else if constexpr (N == 14) w = kW14d[j];
        else if constexpr (N == 15) w = kW15d[j];
        else w = kW16d[j];
    } else {
        if constexpr (N == 7) w = kW7f[j];
        else if constexpr (N == 9) w = kW9f[j];
        else if constexpr (N == 10) w = kW10f[j];
        else if constexpr (N == 11) w = kW11f[j];
        else if constexpr (N == 12) w = kW12f[j];
        else if constexpr (N == 13) w = kW13f[j];
        else if constexpr (N == 14) w = kW14f[j];
        else if constexpr (N == 15) w = kW15f[j];
        else w = kW16f[j];
    }
    if (INV) w.y = -w.y;
    return w;
}

// Composite DFT of A*B points in registers (Cooley-Tukey, decimation in
// time): input m = B m1 + m2, output k = k1 + A k2,
//   y_k = sum_m2 W_B^(m2 k2) [ W_N^(m2 k1) sum_m1 x_(B m1 + m2) W_A^(m1 k1) ].
template <typename R, bool INV, int A, int B>
__device__ __forceinline__ void dft_ct(cplx<R> (&x)[A * B]) {
    constexpr int N = A * B;
    cplx<R> z[B][A];
#pragma unroll
    for (int m2 = 0; m2 < B; ++m2) {
        cplx<R> t[A];
#pragma unroll
        for (int m1 = 0; m1 < A; ++m1) t[m1] = x[B * m1 + m2];
        dft_small<R, INV, A>(t);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) z[m2][k1] = m2 * k1 == 0 ? t[k1] : t[k1] * wconst<R, INV, N>(m2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
        cplx<R> t[B];
#pragma unroll
        for (int m2 = 0; m2 < B; ++m2) t[m2] = z[m2][k1];
        dft_small<R, INV, B>(t);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) x[k1 + A * k2] = t[k2];
    }
}

// Odd prime P in registers: with a_q = x_q + x_(P-q), b_q = x_q - x_(P-q),
// y_p = x_0 + sum_q a_q cos(2 pi p q / P) -+ i sum_q b_q sin(2 pi p q / P)
// and y_(P-p) the same with the sine term negated.
template <typename R, bool INV, int P>
__device__ __forceinline__ void dft_odd(cplx<R> (&x)[P]) {
    constexpr int H = (P - 1) / 2;
    cplx<R> a[H], b[H];
#pragma unroll
    for (int q = 1; q <= H; ++q) {
        a[q - 1] = x[q] + x[P - q];
        b[q - 1] = x[q] - x[P - q];
    }
    cplx<R> y0 = x[0];
#pragma unroll
    for (int q = 0; q < H; ++q) y0 += a[q];
#pragma unroll
    for (int p = 1; p <= H; ++p) {
        cplx<R> t = x[0], u = mk<R>(R(0), R(0));
#pragma unroll
        for (int q = 1; q <= H; ++q) {
            const cplx<R> w = wconst<R, false, P>((p * q) % P);   // (cos, -sin)
            t = t + a[q - 1] * w.x;
            u = u + b[q - 1] * (-w.y);
        }
        // -i u (forward) or +i u (inverse)
        const cplx<R> ru = rot<R, INV>(u);
        x[p] = t + ru;
        x[P - p] = t - ru;
    }
    x[0] = y0;
}

// In-register DFT of RAD points, y_p = sum_q x_q W^(p q), W = exp(-+2 pi i/RAD),
// written out for 2, 3, 4, 5, 6, 8, tabulated primes 7, 11, 13 and composed
// 9, 10, 12, 14, 15, 16.
template <typename R, bool INV, int RAD>
__device__ __forceinline__ void dft_small(cplx<R> (&x)[RAD]) {
    if constexpr (RAD == 1) {
    } else if constexpr (RAD == 7) {
        dft_odd<R, INV, 7>(x);
    } else if constexpr (RAD == 9) {
        dft_ct<R, INV, 3, 3>(x);
    } else if constexpr (RAD == 10) {
        dft_ct<R, INV, 2, 5>(x);
    } else if constexpr (RAD == 11) {
        dft_odd<R, INV, 11>(x);
    } else if constexpr (RAD == 12) {
        dft_ct<R, INV, 4, 3>(x);
    } else if constexpr (RAD == 13) {
        dft_odd<R, INV, 13>(x);
    } else if constexpr (RAD == 14) {
        dft_ct<R, INV, 2, 7>(x);
    } else if constexpr (RAD == 15) {
        dft_ct<R, INV, 3, 5>(x);
    } else if constexpr (RAD == 16) {
        dft_ct<R, INV, 4, 4>(x);
    } else if constexpr (RAD == 2) {
        const cplx<R> a = x[0], b = x[1];
        x[0] = a + b;
        x[1] = a - b;
    } else if constexpr (RAD == 3) {
        const R h = R(0.86602540378443864676);   // sin(2 pi / 3)
        const cplx<R> s = x[1] + x[2];
        const cplx<R> t = x[0] - s * R(0.5);
        const cplx<R> d = (x[1] - x[2]) * h;
        x[0] = x[0] + s;
        x[1] = t + rot<R, INV>(d);
        x[2] = t - rot<R, INV>(d);
    } else if constexpr (RAD == 4) {
        const cplx<R> a = x[0] + x[2], b = x[0] - x[2], c = x[1] + x[3], d = rot<R, INV>(x[1] - x[3]);
        x[0] = a + c;
        x[2] = a - c;
        x[1] = b + d;
        x[3] = b - d;
    } else if constexpr (RAD == 5) {
        const R c1 = R(0.30901699437494742410), c2 = R(-0.80901699437494742410);
        const R s1 = R(0.95105651629515357212), s2 = R(0.58778525229247312917);
        const cplx<R> a1 = x[1] + x[4], b1 = x[1] - x[4], a2 = x[2] + x[3], b2 = x[2] - x[3];
        const cplx<R> t1 = x[0] + a1 * c1 + a2 * c2, t2 = x[0] + a1 * c2 + a2 * c1;
        const cplx<R> u1 = rot<R, INV>(b1 * s1 + b2 * s2), u2 = rot<R, INV>(b1 * s2 - b2 * s1);
        x[0] = x[0] + a1 + a2;
        x[1] = t1 + u1;
        x[4] = t1 - u1;
        x[2] = t2 + u2;
        x[3] = t2 - u2;
    } else if constexpr (RAD == 6) {
        // even / odd halves as two 3-point DFTs, then W6^p between them
        cplx<R> e[3] = {x[0], x[2], x[4]}, o[3] = {x[1], x[3], x[5]};
        dft_small<R, INV, 3>(e);
        dft_small<R, INV, 3>(o);
        const R h = R(0.86602540378443864676);
        const cplx<R> w1 = mk<R>(R(0.5), INV ? h : -h), w2 = mk<R>(R(-0.5), INV ? h : -h);
        const cplx<R> o1 = o[1] * w1, o2 = o[2] * w2;
        x[0] = e[0] + o[0];
        x[3] = e[0] - o[0];
        x[1] = e[1] + o1;
        x[4] = e[1] - o1;
        x[2] = e[2] + o2;
        x[5] = e[2] - o2;
    } else if constexpr (RAD == 8) {
        const R q = R(0.70710678118654752440);
        cplx<R> u[4], v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            u[k] = x[k] + x[k + 4];
            v[k] = x[k] - x[k + 4];
        }
        // v_k *= W8^k
        v[1] = (v[1] + rot<R, INV>(v[1])) * q;
        v[2] = rot<R, INV>(v[2]);
        v[3] = (rot<R, INV>(v[3]) - v[3]) * q;
        dft_small<R, INV, 4>(u);
        dft_small<R, INV, 4>(v);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            x[2 * k] = u[k];
            x[2 * k + 1] = v[k];
        }
    }
}

// fixed small radix: twiddled inputs in registers, butterfly written out
template <typename R, int CW, bool INV, int RAD>
__device__ __forceinline__ void pass_fixed(const cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                                           const cplx<R>* __restrict__ T, const int2* __restrict__ jt, int n, int L) {
    constexpr int ROWS = kFftThreads / CW;
    const int c = threadIdx.x & (CW - 1);
    const int lane = threadIdx.x / CW;
    const int nr = n / RAD;
    const int stepL = n / L;
    const int Ns = L / RAD;
    for (int j = lane; j < nr; j += ROWS) {
        const int2 kb = jt[j];  // (k1, output base)
        cplx<R> x[RAD];
#pragma unroll
        for (int q = 0; q < RAD; ++q) x[q] = in[(j + q * nr) * CW + c];
        if (Ns > 1) {
#pragma unroll
            for (int q = 1; q < RAD; ++q) {
                const cplx<R> w = T[q * kb.x * stepL];
                x[q] = mk<R>(x[q].x * w.x - x[q].y * w.y, x[q].x * w.y + x[q].y * w.x);
            }
        }
        dft_small<R, INV, RAD>(x);
#pragma unroll
        for (int p = 0; p < RAD; ++p) out[(kb.y + p * Ns) * CW + c] = x[p];
    }
}

// large radices (always odd primes here): twiddle the inputs in place, then
// stream them from shared memory.  With a_q = x_q + x_{r-q}, b_q = x_q - x_{r-q}
// (q = 1..(r-1)/2) and W_r^(p q) = (wr, wi):
//   y_p     = x_0 + sum_q (a.x wr - wi b.y, a.y wr + wi b.x)
//   y_{r-p} = x_0 + sum_q (a.x wr + wi b.y, a.y wr - wi b.x)
// i.e. r-1 FMAs per output; each thread accumulates PC output pairs.  The
// W_r^(p q) of a thread's PC outputs are PC consecutive entries of row q of
// the precomputed table `pt` (ld per row), staged in shared memory.
template <typename R, bool INV, int CW>
__device__ __forceinline__ void pass_stream(cplx<R>* __restrict__ in, cplx<R>* __restrict__ out,
                                            const cplx<R>* __restrict__ T, const int2* __restrict__ jt, int n, int r,
                                            int L, const cplx<R>* __restrict__ pt, int ld) {
    constexpr int ROWS = kFftThreads / CW;
    constexpr int PC = 8;
    const int c = threadIdx.x & (CW - 1);
    const int lane = threadIdx.x / CW;
    const int nr = n / r;
    const int Ns = L / r;
    const int stepL = n / L;
    const int stepR = nr;
    const int half = (r - 1) / 2;
    const int nchunk = (half + PC - 1) / PC;
    if (Ns > 1) {
        for (int q = 1; q < r; ++q)
            for (int j = lane; j < nr; j += ROWS) {
                const cplx<R> w = T[q * jt[j].x * stepL];
                const cplx<R> v = in[(j + q * nr) * CW + c];
                in[(j + q * nr) * CW + c] = mk<R>(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
            }
        __syncthreads();
    }
    for (int u = lane; u < nr * nchunk; u += ROWS) {
        const int oc = u / nr;
        const int j = u - oc * nr;
        const int base = jt[j].y;
        const int p0 = 1 + oc * PC;
        const cplx<R> x0 = in[j * CW + c];
        R px[PC], py[PC], qx[PC], qy[PC];
#pragma unroll
        for (int k = 0; k < PC; ++k) px[k] = py[k] = qx[k] = qy[k] = R(0);
        R sx = R(0), sy = R(0);
        const cplx<R>* prow = pt ? pt + (p0 - 1) : nullptr;
        int ep[PC];
#pragma unroll
        for (int k = 0; k < PC; ++k) ep[k] = 0;
        for (int q = 1; q <= half; ++q) {
            const cplx<R> xa = in[(j + q * nr) * CW + c];
            const cplx<R> xb = in[(j + (r - q) * nr) * CW + c];
            const R ax = xa.x + xb.x, ay = xa.y + xb.y, bx = xa.x - xb.x, by = xa.y - xb.y;
            sx += ax;
            sy += ay;
            cplx<R> wk[PC];
            if (!prow) {
                // W_r^(p q) from the line's twiddles, p q reduced mod r incrementally
#pragma unroll
                for (int k = 0; k < PC; ++k) {
                    ep[k] += p0 + k;
                    if (ep[k] >= r) ep[k] -= r;
                    const cplx<R> w = T[ep[k] * stepR];
                    wk[k] = mk<R>(w.x, INV ? -w.y : w.y);   // T is already conjugated for INV
                }
            } else if constexpr (sizeof(R) == 4) {
                const float4* p4 = reinterpret_cast<const float4*>(prow);
#pragma unroll
                for (int k = 0; k < PC / 2; ++k) {
                    const float4 v = p4[k];
                    wk[2 * k] = mk<R>(v.x, v.y);
                    wk[2 * k + 1] = mk<R>(v.z, v.w);
                }
            } else {
#pragma unroll
                for (int k = 0; k < PC; ++k) wk[k] = prow[k];
            }
            if (prow) prow += ld;
#pragma unroll
            for (int k = 0; k < PC; ++k) {
                const R wy = INV ? -wk[k].y : wk[k].y;
                px[k] = fma(ax, wk[k].x, px[k]);
                py[k] = fma(ay, wk[k].x, py[k]);
                qx[k] = fma(bx, wy, qx[k]);
                qy[k] = fma(by, wy, qy[k]);
            }
        }
        if (oc == 0) out[base * CW + c] = mk<R>(x0.x + sx, x0.y + sy);
#pragma unroll
        for (int k = 0; k < PC; ++k) {
            const int p = p0 + k;
            if (p <= half) {
                out[(base + p * Ns) * CW + c] = mk<R>(x0.x + px[k] - qy[k], x0.y + py[k] + qx[k]);
                out[(base + (r - p) * Ns) * CW + c] = mk<R>(x0.x + px[k] + qy[k], x0.y + py[k] - qx[k]);
            }
        }
    }
}

// global -> shared copy of one element without a register round trip, so a
// thread's whole share of the line is in flight at once (src_bytes = 0 fills
// the element with zeros and reads nothing)
template <typename R>
__device__ __forceinline__ void copy_async(cplx<R>* dst, const cplx<R>* src, bool live) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    const int bytes = live ? int(sizeof(cplx<R>)) : 0;
    if constexpr (sizeof(cplx<R>) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void copy_async_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// All radix passes of one line held in shared memory (ping-pong between
// `in` and `out`); returns the buffer that holds the result.  T holds the
// line's twiddles, conjugated for INV.
template <typename R, bool INV, int CW, int MAXR, bool STREAM>
__device__ __forceinline__ cplx<R>* line_passes(cplx<R>* in, cplx<R>* out, const cplx<R>* T, int2* jt,
                                                const FftFactors& f, const cplx<R>* PT) {
    const int n = f.n;
    int Ns = 1;
    for (int ps = 0; ps < f.nf; ++ps) {
        const int r = f.r[ps];
        const int nr = n / r;
        const int L = Ns * r;
        __syncthreads();  // previous pass complete; jt free
        for (int j = threadIdx.x; j < nr; j += kFftThreads) {
            const int k1 = j % Ns;
            jt[j] = make_int2(k1, (j / Ns) * L + k1);
        }
        __syncthreads();
        if (r == 2) pass_fixed<R, CW, INV, 2>(in, out, T, jt, n, L);
        else if (r == 3) pass_fixed<R, CW, INV, 3>(in, out, T, jt, n, L);
        else if (r == 4) pass_fixed<R, CW, INV, 4>(in, out, T, jt, n, L);
        else if (r == 5) pass_fixed<R, CW, INV, 5>(in, out, T, jt, n, L);
        else if (r == 6) pass_fixed<R, CW, INV, 6>(in, out, T, jt, n, L);
        else if (r == 8) pass_fixed<R, CW, INV, 8>(in, out, T, jt, n, L);
        else if (r <= 8) pass_reg<R, CW, 8>(in, out, T, jt, n, r, L);
        else if (MAXR > 8 && r <= MAXR) pass_reg<R, CW, (MAXR > 8 ? MAXR : 8)>(in, out, T, jt, n, r, L);
        else if (STREAM)
            pass_stream<R, INV, CW>(in, out, T, jt, n, r, L, f.pt_total ? PT + f.pt_off[ps] : nullptr, f.pt_ld[ps]);
        cplx<R>* tmp = in;
        in = out;
        out = tmp;
        Ns = L;
    }
    __syncthreads();
    return in;
}

// Diagonal k-space factor of the fused transform: element e of line o,
// column c is multiplied by sc[(e * nouter + o) * sz + c / sb].
template <typename R>
struct LineScale {
    const R* sc = nullptr;
    int nouter = 0, sz = 1, sb = 1;
};

// One CTA = CW adjacent columns of one line.  KSCALE: forward transform,
// k-space scale, inverse transform in one round trip of the line (INV is
// then unused); else a single transform in the direction INV.
template <typename R, bool INV, int CW, int MAXR, bool STREAM, bool KSCALE>
__global__ void __launch_bounds__(kFftThreads) k_fft_axis(cplx<R>* __restrict__ data, FftFactors f,
                                                          const cplx<R>* __restrict__ tw, size_t es, int ncols,
                                                          size_t os, const cplx<R>* __restrict__ ptw,
                                                          int ngroups, LineScale<R> ks) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int ROWS = kFftThreads / CW;
    constexpr bool FWD_INV = KSCALE ? false : INV;
    const int n = f.n;
    cplx<R>* A = reinterpret_cast<cplx<R>*>(smem_raw);
    cplx<R>* Bv = A + size_t(n) * CW;
    cplx<R>* T = Bv + size_t(n) * CW;
    int2* jt = reinterpret_cast<int2*>(T + n);
    // streamed-pass twiddle tables after jt, at a 16-byte aligned offset
    const size_t pt_off_bytes =
        ((size_t(2 * n * CW + n) * sizeof(cplx<R>) + 8 * size_t(n)) + 15) & ~size_t(15);
    cplx<R>* PT = reinterpret_cast<cplx<R>*>(smem_raw + pt_off_bytes);
    const int c = threadIdx.x & (CW - 1);
    const int lane = threadIdx.x / CW;
    // column groups of one line are adjacent in launch order
    const int o = blockIdx.x / ngroups;
    const int c0 = (blockIdx.x - o * ngroups) * CW;
    const bool live = c0 + c < ncols;
    cplx<R>* line = data + size_t(o) * os + c0 + c;
    // dead columns copy nothing; their source address is only a placeholder
    const cplx<R>* src = live ? line : data;
    const size_t ses = live ? es : 0;
    for (int e = lane; e < n; e += ROWS) copy_async<R>(A + e * CW + c, src + size_t(e) * ses, live);
    if (STREAM)
        for (int t = threadIdx.x; t < f.pt_total; t += kFftThreads) PT[t] = ptw[t];
    for (int t = threadIdx.x; t < n; t += kFftThreads) {
        cplx<R> w = tw[t];
        if (FWD_INV) w.y = -w.y;
        T[t] = w;
    }
    copy_async_wait();
    cplx<R>* res = line_passes<R, FWD_INV, CW, MAXR, STREAM>(A, Bv, T, jt, f, PT);
    if constexpr (KSCALE) {
        // each thread scales the elements it loaded; the inverse twiddles
        // replace the forward ones (line_passes ends with a barrier)
        if (live) {
            const R* sc = ks.sc + size_t(o) * ks.sz + (c0 + c) / ks.sb;
            const size_t sstep = size_t(ks.nouter) * ks.sz;
            for (int e = lane; e < n; e += ROWS) res[e * CW + c] = res[e * CW + c] * sc[size_t(e) * sstep];
        }
        for (int t = threadIdx.x; t < n; t += kFftThreads) T[t].y = -T[t].y;
        res = line_passes<R, true, CW, MAXR, STREAM>(res, res == A ? Bv : A, T, jt, f, PT);
    }
    if (live)
        for (int e = lane; e < n; e += ROWS) line[size_t(e) * es] = res[e * CW + c];
}

// ---------------------------------------------------------------------------
// Two-pass line transform for n = r1 * r2 with both factors in-register
// radices (<= 16).  Thread (lane, c) of a CTA of CW columns runs one
// butterfly per pass, so a line makes a single round trip through shared
// memory: pass 1 (radix r1, no twiddles) reads its r1 inputs straight from
// global memory (all loads in flight together) and writes shared; pass 2
// (radix r2, twiddles W_n^(q j)) reads shared and writes global.  Stockham
// indexing as above: pass 1 butterfly j < r2 reads x[j + q r2], writes
// S[j r1 + p]; pass 2 butterfly j < r1 reads S[j + q r1], writes y[p r1 + j].
//
// KSCALE (mode 2): after the forward pass 2 a thread holds y[p r1 + j],
// p < r2, which are exactly the inputs of butterfly j of an inverse
// transform whose first radix is r2; it scales them, runs that butterfly in
// registers and writes S[j r2 + p]; the inverse radix-r1 pass (butterfly
// j < r2 reads S[j + q r2] W_n^(-q j), writes x[p r2 + j]) ends in global
// memory.  Forward, scale and inverse thus cost one global round trip and
// two shared ones.

constexpr int kFft2MaxThreads = 384;

template <int CLS, typename Fn>
__device__ __forceinline__ void radix_dispatch(int r, Fn&& fn) {
    switch (r) {
        case 1: fn(std::integral_constant<int, 1>{}); break;
        case 2: fn(std::integral_constant<int, 2>{}); break;
        case 3: fn(std::integral_constant<int, 3>{}); break;
        case 4: fn(std::integral_constant<int, 4>{}); break;
        case 5: fn(std::integral_constant<int, 5>{}); break;
        case 6: fn(std::integral_constant<int, 6>{}); break;
        case 7: fn(std::integral_constant<int, 7>{}); break;
        case 8: fn(std::integral_constant<int, 8>{}); break;
        default:
            // register classes: radices up to CLS only (8, 12 or 16)
            if constexpr (CLS > 8) {
                switch (r) {
                    case 9: fn(std::integral_constant<int, 9>{}); break;
                    case 10: fn(std::integral_constant<int, 10>{}); break;
                    case 11: fn(std::integral_constant<int, 11>{}); break;
                    case 12: fn(std::integral_constant<int, 12>{}); break;
                    default: break;
                }
            }
            if constexpr (CLS > 12) {
                switch (r) {
                    case 13: fn(std::integral_constant<int, 13>{}); break;
                    case 14: fn(std::integral_constant<int, 14>{}); break;
                    case 15: fn(std::integral_constant<int, 15>{}); break;
                    case 16: fn(std::integral_constant<int, 16>{}); break;
                    default: break;
                }
            }
            break;
    }
}

template <typename R, int CW, int MODE, int CLS>
__global__ void __launch_bounds__(kFft2MaxThreads) k_fft2(cplx<R>* __restrict__ data, const cplx<R>* __restrict__ tw,
                                                          int r1, int r2, size_t es, int ncols, size_t os,
                                                          int ngroups, LineScale<R> ks) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr bool INV = MODE == 1;
    const int n = r1 * r2;
    cplx<R>* S = reinterpret_cast<cplx<R>*>(smem_raw);
    cplx<R>* T = S + size_t(n) * CW;
    // column groups of one line are adjacent in launch order, so the DRAM
    // lines their row pieces share are fetched once
    const int o = blockIdx.x / ngroups;
    const int g = blockIdx.x - o * ngroups;
    const int c = threadIdx.x & (CW - 1);
    const int lane = threadIdx.x / CW;
    const int c0 = g * CW;
    const bool live = c0 + c < ncols;
    cplx<R>* line = data + size_t(o) * os + c0 + c;
    for (int t = threadIdx.x; t < n; t += blockDim.x) T[t] = tw[t];
    // pass 1: radix r1, butterfly lane < r2, global -> shared
    radix_dispatch<CLS>(r1, [&](auto rc) {
        constexpr int RAD = decltype(rc)::value;
        if (lane < r2) {
            cplx<R> x[RAD];
#pragma unroll
            for (int q = 0; q < RAD; ++q) x[q] = live ? line[size_t(lane + q * r2) * es] : mk<R>(R(0), R(0));
            dft_small<R, INV, RAD>(x);
#pragma unroll
            for (int p = 0; p < RAD; ++p) S[(lane * RAD + p) * CW + c] = x[p];
        }
    });
    __syncthreads();
    // pass 2: radix r2, butterfly lane < r1, shared -> global (or on to the
    // scale and the first inverse butterfly)
    radix_dispatch<CLS>(r2, [&](auto rc) {
        constexpr int RAD = decltype(rc)::value;
        const bool act = lane < r1;
        cplx<R> x[RAD];
        if (act) {
            x[0] = S[lane * CW + c];
#pragma unroll
            for (int q = 1; q < RAD; ++q) {
                cplx<R> w = T[q * lane];
                if (INV) w.y = -w.y;
                x[q] = S[(lane + q * r1) * CW + c] * w;
            }
            dft_small<R, INV, RAD>(x);
        }
        if constexpr (MODE == 2) {
            if (act) {
                if (live) {
                    const R* sc = ks.sc + size_t(o) * ks.sz + (c0 + c) / ks.sb;
                    const size_t sstep = size_t(ks.nouter) * ks.sz;
#pragma unroll
                    for (int p = 0; p < RAD; ++p) x[p] = x[p] * sc[size_t(p * r1 + lane) * sstep];
                }
                dft_small<R, true, RAD>(x);
            }
            __syncthreads();   // every read of S above is done
            if (act) {
#pragma unroll
                for (int p = 0; p < RAD; ++p) S[(lane * RAD + p) * CW + c] = x[p];
            }
        } else {
            if (act && live) {
#pragma unroll
                for (int p = 0; p < RAD; ++p) line[size_t(p * r1 + lane) * es] = x[p];
            }
        }
    });
    if constexpr (MODE == 2) {
        __syncthreads();
        // inverse radix-r1 pass, butterfly lane < r2: shared -> global
        radix_dispatch<CLS>(r1, [&](auto rc) {
            constexpr int RAD = decltype(rc)::value;
            if (lane < r2) {
                cplx<R> x[RAD];
                x[0] = S[lane * CW + c];
#pragma unroll
                for (int q = 1; q < RAD; ++q) {
                    cplx<R> w = T[q * lane];
                    w.y = -w.y;
                    x[q] = S[(lane + q * r2) * CW + c] * w;
                }
                dft_small<R, true, RAD>(x);
                if (live) {
#pragma unroll
                    for (int p = 0; p < RAD; ++p) line[size_t(p * r2 + lane) * es] = x[p];
                }
            }
        });
    }
}

// radices the two-pass kernels have in-register butterflies for
bool fft2_radix(int r) { return r >= 1 && r <= 16; }

// the kernel instantiation (largest radix compiled in) for a largest radix r
int register_class(int r) { return r <= 8 ? 8 : (r <= 12 ? 12 : 16); }

// (r1, r2) with r1 * r2 = n, both in-register radices, max(r1, r2) smallest
// (0, 0) when n has no such split
std::pair<int, int> fft2_split(int n) {
    std::pair<int, int> best(0, 0);
    for (int a = 1; a <= 16 && a <= n; ++a) {
        if (n % a) continue;
        const int b = n / a;
        if (!fft2_radix(a) || !fft2_radix(b) || a < b) continue;
        if (!best.first || a < best.first) best = {a, b};
    }
    return best;
}

size_t fft2_smem(int n, int cw, size_t elem) { return (size_t(n) * cw + n) * elem; }

template <typename R, int MODE, int CW>
void launch2_cw(int cls, int nblocks, int nthreads, size_t shm, cudaStream_t s, cplx<R>* data, const cplx<R>* tw,
                int r1, int r2, size_t es, int ncols, size_t os, int ngroups, const LineScale<R>& ks) {
    auto go = [&](auto kern) {
        set_smem_limit(kern, shm);
        kern<<<nblocks, nthreads, shm, s>>>(data, tw, r1, r2, es, ncols, os, ngroups, ks);
    };
    if (cls == 8) go(k_fft2<R, CW, MODE, 8>);
    else if (cls == 12) go(k_fft2<R, CW, MODE, 12>);
    else go(k_fft2<R, CW, MODE, 16>);
}

// ---------------------------------------------------------------------------
// The z-slab k-space step fused with the y transforms (AxisFFT::run_slab).
//
// One CTA owns one kx plane and MC right-hand sides: the tile
// S[y][col], col = (z * 3 + c) * MC + mi, NCOL = Zs * 3 * MC columns of
// n = Ny points, lives in shared memory for the whole step, with a second
// tile of the same size for the transforms.  The y transforms are the
// two-pass (r1, r2) split of k_fft2 between the two tiles (pass 1 S -> S2,
// pass 2 S2 -> S), so a pass needs one barrier, not one per group of
// columns.  Between the transforms thread (ky, mi) reads the 3 x Zs values
// of its (kx, ky, mi) column and writes the Green-tensor product back in
// place (four Toeplitz products of Zs x Zs); no other thread touches them.

// right-hand sides per CTA: two tiles of n x Zs x 3 x MC within ~70 KB
template <typename R> __host__ __device__ constexpr int slab_mc(bool one_slot) {
    return one_slot ? (sizeof(R) == 8 ? 4 : 8) : (sizeof(R) == 8 ? 1 : 2);
}
constexpr int kSlabThreads = 128;

struct SlabArgs {
    int Nx, Zs, M, nchunk;
    double kxu, kyu;
};

// one radix pass over all NCOL columns, src -> dst, thread task t =
// (butterfly j, column col), col fastest.  Pass 1 (radix r1, butterfly
// j < r2) reads src[j + q r2] and writes dst[j r1 + p]; pass 2 (radix r2,
// butterfly j < r1) reads src[j + q r1] W_n^(q j) and writes dst[p r1 + j].
template <typename R, bool INV, int RAD, bool PASS2>
__device__ __forceinline__ void slab_pass(const cplx<R>* __restrict__ src, cplx<R>* __restrict__ dst,
                                          const cplx<R>* __restrict__ T, int n, int NCOL) {
    const int nb = n / RAD;   // butterflies per column
    for (int t = threadIdx.x; t < nb * NCOL; t += kSlabThreads) {
        const int j = t / NCOL, col = t - j * NCOL;
        cplx<R> x[RAD];
        if constexpr (!PASS2) {
#pragma unroll
            for (int q = 0; q < RAD; ++q) x[q] = src[(j + q * nb) * NCOL + col];
        } else {
            x[0] = src[j * NCOL + col];
#pragma unroll
            for (int q = 1; q < RAD; ++q) {
                cplx<R> w = T[q * j];
                if (INV) w.y = -w.y;
                x[q] = src[(j + q * nb) * NCOL + col] * w;
            }
        }
        dft_small<R, INV, RAD>(x);
        if constexpr (!PASS2) {
#pragma unroll
            for (int p = 0; p < RAD; ++p) dst[(j * RAD + p) * NCOL + col] = x[p];
        } else {
#pragma unroll
            for (int p = 0; p < RAD; ++p) dst[(p * nb + j) * NCOL + col] = x[p];
        }
    }
    __syncthreads();
}

// y transform of every column of S (result back in S; S2 is scratch)
template <typename R, bool INV, int CLS>
__device__ __forceinline__ void slab_ytransform(cplx<R>* S, cplx<R>* S2, const cplx<R>* T, int r1, int r2,
                                                int NCOL) {
    const int n = r1 * r2;
    radix_dispatch<CLS>(r1, [&](auto rc) { slab_pass<R, INV, decltype(rc)::value, false>(S, S2, T, n, NCOL); });
    radix_dispatch<CLS>(r2, [&](auto rc) { slab_pass<R, INV, decltype(rc)::value, true>(S2, S, T, n, NCOL); });
}

template <typename R, int MC, int ZMAX, int CLS>
__global__ void __launch_bounds__(kSlabThreads) k_slab(cplx<R>* __restrict__ data, const cplx<R>* __restrict__ tw,
                                                       const cplx<R>* __restrict__ taps, int r1, int r2,
                                                       SlabArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = r1 * r2;
    const int Zs = a.Zs, M = a.M, B = 3 * M;
    const int NCOL = Zs * 3 * MC;
    cplx<R>* S = reinterpret_cast<cplx<R>*>(smem_raw);
    cplx<R>* S2 = S + size_t(n) * NCOL;
    cplx<R>* T = S2 + size_t(n) * NCOL;
    // the right-hand-side chunks of one kx plane are adjacent in launch order
    const int ix = blockIdx.x / a.nchunk;
    const int m0 = (blockIdx.x - ix * a.nchunk) * MC;
    const int mc = min(MC, M - m0);
    cplx<R>* g = data + size_t(ix) * n * Zs * B;
    const int tot = n * NCOL;
    // tile element t = ((y Zs + z) 3 + c) MC + mi  <-  g[(y Zs + z) B + c M + m0 + mi]
    for (int t = threadIdx.x; t < tot; t += kSlabThreads) {
        const int mi = t % MC;
        const int r = t / MC;
        const bool live = mi < mc;
        const cplx<R>* src = live ? g + size_t(r / 3) * B + (r % 3) * M + m0 + mi : data;
        copy_async<R>(S + t, src, live);
    }
    for (int t = threadIdx.x; t < n; t += kSlabThreads) T[t] = tw[t];
    copy_async_wait();
    __syncthreads();
    slab_ytransform<R, false, CLS>(S, S2, T, r1, r2, NCOL);
    // Green tensor per (ky, mi), in place: a = kx E_x + ky E_y,
    // u = t0 * a + t1 * E_z  ->  E_x = kx u, E_y = ky u;  E_z = t1 * a + t2 * E_z
    const double fx = (ix <= (a.Nx - 1) / 2) ? ix : ix - a.Nx;
    const R kx = R(fx * a.kxu);
    const int nd = 2 * Zs - 1;
    for (int t = threadIdx.x; t < n * MC; t += kSlabThreads) {
        const int ky_i = t / MC;
        const int mi = t - ky_i * MC;
        const double fy = (ky_i <= (n - 1) / 2) ? ky_i : ky_i - n;
        const R ky = R(fy * a.kyu);
        cplx<R>* b = S + size_t(ky_i) * NCOL + mi;
        cplx<R> av[ZMAX], zv[ZMAX];
#pragma unroll
        for (int z = 0; z < ZMAX; ++z) {
            if (z < Zs) {
                const cplx<R> ex = b[(z * 3 + 0) * MC], ey = b[(z * 3 + 1) * MC];
                av[z] = ex * kx + ey * ky;
                zv[z] = b[(z * 3 + 2) * MC];
            } else {
                av[z] = mk<R>(R(0), R(0));
                zv[z] = mk<R>(R(0), R(0));
            }
        }
        const cplx<R>* tp = taps + (size_t(ix) * n + ky_i) * 3 * nd + (Zs - 1);   // tp[k nd + d]
#pragma unroll
        for (int part = 0; part < 2; ++part) {
            const cplx<R>* ta = tp + part * nd;         // t0 | t1 on a
            const cplx<R>* tb = tp + (part + 1) * nd;   // t1 | t2 on E_z
            cplx<R> acc[ZMAX];
#pragma unroll
            for (int zo = 0; zo < ZMAX; ++zo) acc[zo] = mk<R>(R(0), R(0));
#pragma unroll
            for (int d = -(ZMAX - 1); d <= ZMAX - 1; ++d) {
                if (d < -(Zs - 1) || d > Zs - 1) continue;
                const cplx<R> ka = ta[d], kb = tb[d];
#pragma unroll
                for (int zo = 0; zo < ZMAX; ++zo) {
                    const int zi = zo - d;
                    if (zi >= 0 && zi < ZMAX) {
                        acc[zo].x = fma(ka.x, av[zi].x, acc[zo].x);
                        acc[zo].x = fma(-ka.y, av[zi].y, acc[zo].x);
                        acc[zo].y = fma(ka.x, av[zi].y, acc[zo].y);
                        acc[zo].y = fma(ka.y, av[zi].x, acc[zo].y);
                        acc[zo].x = fma(kb.x, zv[zi].x, acc[zo].x);
                        acc[zo].x = fma(-kb.y, zv[zi].y, acc[zo].x);
                        acc[zo].y = fma(kb.x, zv[zi].y, acc[zo].y);
                        acc[zo].y = fma(kb.y, zv[zi].x, acc[zo].y);
                    }
                }
            }
#pragma unroll
            for (int zo = 0; zo < ZMAX; ++zo) {
                if (zo < Zs) {
                    if (part == 0) {
                        b[(zo * 3 + 0) * MC] = acc[zo] * kx;
                        b[(zo * 3 + 1) * MC] = acc[zo] * ky;
                    } else {
                        b[(zo * 3 + 2) * MC] = acc[zo];
                    }
                }
            }
        }
    }
    __syncthreads();
    slab_ytransform<R, true, CLS>(S, S2, T, r1, r2, NCOL);
    for (int t = threadIdx.x; t < tot; t += kSlabThreads) {
        const int mi = t % MC;
        if (mi < mc) {
            const int r = t / MC;
            g[size_t(r / 3) * B + (r % 3) * M + m0 + mi] = S[t];
        }
    }
}

// ---------------------------------------------------------------------------
// Two-pass line transform for n = r1 * p, r1 an in-register radix and p an
// odd prime above 16 (the monolayer x axis: 366 = 6 * 61).  Pass 1 (radix
// r1, butterfly j1 < p) reads x[j1 + q p] straight from global memory and
// stores S[j1 r1 + p1] already multiplied by pass 2's twiddle W_n^(j1 p1)
// (pass 2 butterfly j reads S[j + q r1], i.e. j1 = q, p1 = j).  Pass 2 (radix
// p, butterfly j < r1) streams its inputs from shared memory as the general
// kernel's prime pass does (a_q = x_q + x_(p-q), b_q = x_q - x_(p-q), PC
// output pairs per work item, W_p^(p' q) from the table PT in shared memory)
// and writes y[p' r1 + j] straight to global memory.  One CTA = CW columns
// of one line; L = blockDim.x / CW lanes loop over pass 1's p butterflies and
// pass 2's r1 * ceil(((p-1)/2) / PC) work items.

// fp64 work items carry half the output pairs, so that their accumulators
// leave room for three CTAs per SM
template <typename R>
__host__ __device__ constexpr int fft2p_pc() { return sizeof(R) == 8 ? 4 : 8; }

template <typename R, int CW, bool INV, int CLS>
__global__ void __launch_bounds__(kFft2MaxThreads) k_fft2p(cplx<R>* __restrict__ data, const cplx<R>* __restrict__ tw,
                                                           const cplx<R>* __restrict__ ptw, int pt_total, int pt_ld,
                                                           int r1, int p, size_t es, int ncols, size_t os,
                                                           int ngroups) {
    constexpr int PC = fft2p_pc<R>();   // output pairs per work item
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = r1 * p;
    const int L = blockDim.x / CW;
    cplx<R>* S = reinterpret_cast<cplx<R>*>(smem_raw);   // [n][CW]
    cplx<R>* PT = S + size_t(n) * CW;                      // [pt_total], 16-byte aligned (CW >= 2)
    cplx<R>* T = PT + pt_total;                            // [n]
    const int o = blockIdx.x / ngroups;
    const int g = blockIdx.x - o * ngroups;
    const int c = threadIdx.x & (CW - 1);
    const int lane = threadIdx.x / CW;
    const int c0 = g * CW;
    const bool live = c0 + c < ncols;
    cplx<R>* line = data + size_t(o) * os + c0 + c;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        cplx<R> w = tw[t];
        if (INV) w.y = -w.y;
        T[t] = w;
    }
    for (int t = threadIdx.x; t < pt_total; t += blockDim.x) PT[t] = ptw[t];
    __syncthreads();
    // pass 1: radix r1, global -> shared with pass 2's twiddles applied
    radix_dispatch<CLS>(r1, [&](auto rc) {
        constexpr int RAD = decltype(rc)::value;
#pragma unroll 2
        for (int j1 = lane; j1 < p; j1 += L) {
            cplx<R> x[RAD];
#pragma unroll
            for (int q = 0; q < RAD; ++q) x[q] = live ? line[size_t(j1 + q * p) * es] : mk<R>(R(0), R(0));
            dft_small<R, INV, RAD>(x);
            S[(j1 * RAD) * CW + c] = x[0];
#pragma unroll
            for (int p1 = 1; p1 < RAD; ++p1) S[(j1 * RAD + p1) * CW + c] = x[p1] * T[j1 * p1];
        }
    });
    __syncthreads();
    // pass 2: radix p streamed from shared memory, outputs to global memory
    const int half = (p - 1) / 2;
    const int nchunk = (half + PC - 1) / PC;
    for (int u = lane; u < r1 * nchunk; u += L) {
        const int ch = u / r1;
        const int j = u - ch * r1;
        const int p0 = 1 + ch * PC;
        const cplx<R> x0 = S[j * CW + c];
        R px[PC], py[PC], qx[PC], qy[PC];
#pragma unroll
        for (int k = 0; k < PC; ++k) px[k] = py[k] = qx[k] = qy[k] = R(0);
        R sx = R(0), sy = R(0);
        const cplx<R>* prow = PT + (p0 - 1);
        for (int q = 1; q <= half; ++q, prow += pt_ld) {
            const cplx<R> xa = S[(j + q * r1) * CW + c];
            const cplx<R> xb = S[(j + (p - q) * r1) * CW + c];
            const R ax = xa.x + xb.x, ay = xa.y + xb.y, bx = xa.x - xb.x, by = xa.y - xb.y;
            sx += ax;
            sy += ay;
            cplx<R> wk[PC];
            if constexpr (sizeof(R) == 4) {
                const float4* p4 = reinterpret_cast<const float4*>(prow);
#pragma unroll
                for (int k = 0; k < PC / 2; ++k) {
                    const float4 v = p4[k];
                    wk[2 * k] = mk<R>(v.x, v.y);
                    wk[2 * k + 1] = mk<R>(v.z, v.w);
                }
            } else {
#pragma unroll
                for (int k = 0; k < PC; ++k) wk[k] = prow[k];
            }
#pragma unroll
            for (int k = 0; k < PC; ++k) {
                const R wy = INV ? -wk[k].y : wk[k].y;
                px[k] = fma(ax, wk[k].x, px[k]);
                py[k] = fma(ay, wk[k].x, py[k]);
                qx[k] = fma(bx, wy, qx[k]);
                qy[k] = fma(by, wy, qy[k]);
            }
        }
        if (!live) continue;
        if (ch == 0) line[size_t(j) * es] = mk<R>(x0.x + sx, x0.y + sy);
#pragma unroll
        for (int k = 0; k < PC; ++k) {
            const int pp = p0 + k;
            if (pp <= half) {
                line[size_t(pp * r1 + j) * es] = mk<R>(x0.x + px[k] - qy[k], x0.y + py[k] + qx[k]);
                line[size_t((p - pp) * r1 + j) * es] = mk<R>(x0.x + px[k] + qy[k], x0.y + py[k] - qx[k]);
            }
        }
    }
}

// W_r^(p q) table of a streamed prime pass: rows q = 1..(r-1)/2, columns
// p = 1..(r-1)/2 padded to a multiple of 8 with zeros, plus 8 spare entries
// so that a padded row can always be read whole.  Appended to `out`; returns
// the row length.
int append_prime_table(int r, std::vector<double2>& out) {
    const int half = (r - 1) / 2;
    const int ld = (half + 7) / 8 * 8;
    for (int q = 1; q <= half; ++q)
        for (int c = 0; c < ld; ++c) {
            const int p = c + 1;
            if (p > half) {
                out.push_back(make_double2(0.0, 0.0));
                continue;
            }
            const double a = -2.0 * kPi * double((long long)p * q % r) / double(r);
            out.push_back(make_double2(std::cos(a), std::sin(a)));
        }
    for (int c = 0; c < 8; ++c) out.push_back(make_double2(0.0, 0.0));
    return ld;
}

bool is_prime(int m) {
    if (m < 2) return false;
    for (int d = 2; d * d <= m; ++d)
        if (m % d == 0) return false;
    return true;
}

// (r1, p) with n = r1 * p, p the largest prime factor, p > 16, r1 an
// in-register radix; (0, 0) otherwise
std::pair<int, int> fft2p_split(int n) {
    int p = 1, m = n;
    for (int d = 2; d * d <= m; ++d)
        while (m % d == 0) {
            p = std::max(p, d);
            m /= d;
        }
    if (m > 1) p = std::max(p, m);
    if (p <= 16 || !is_prime(p) || !fft2_radix(n / p)) return {0, 0};
    return {n / p, p};
}

size_t fft2p_smem(int n, int cw, size_t elem, int pt_total) { return (size_t(n) * cw + pt_total + n) * elem; }

template <typename R, bool INV, int CW>
void launch2p_cw(int cls, int nblocks, int nthreads, size_t shm, cudaStream_t s, cplx<R>* data, const cplx<R>* tw,
                 const cplx<R>* ptw, int pt_total, int pt_ld, int r1, int p, size_t es, int ncols, size_t os,
                 int ngroups) {
    auto go = [&](auto kern) {
        set_smem_limit(kern, shm);
        kern<<<nblocks, nthreads, shm, s>>>(data, tw, ptw, pt_total, pt_ld, r1, p, es, ncols, os, ngroups);
    };
    if (cls == 8) go(k_fft2p<R, CW, INV, 8>);
    else go(k_fft2p<R, CW, INV, 16>);
}

// ---------------------------------------------------------------------------
// Two-pass line transform n = r1 * p with the prime pass done by Rader's
// algorithm: with g a primitive root mod p, a_q = x[g^-q], b_s = W_p^(g^s),
//   y[0] = x[0] + sum_q a_q,   y[g^m] = x[0] + (a (*) b)_m   (cyclic, length N = p-1)
// and the cyclic convolution is IDFT_N(DFT_N(a) . Bh) with Bh = DFT_N(b) / N
// precomputed.  N = A * B with both in-register radices, so DFT_N is one
// Cooley-Tukey step through shared memory: R1 (thread per (j, q2)) an A-point
// DFT over q1 of a[B q1 + q2] and the twiddles W_N^(q2 k1); R2 (thread per
// (j, k1)) the B-point DFT over q2, the product with Bh, the B-point inverse
// DFT and the twiddles W_N^(-m1 k1) in registers; R4 (thread per (j, m1)) the
// A-point inverse DFT giving c[m1 + B m2], written to global memory at row
// g^(m1 + B m2).  About a quarter of the direct prime pass's arithmetic.
// Pass 1 is k_fft2p's (radix r1 from global memory, pass-2 twiddles fused).
template <typename R, int CW, bool INV, int CLS>
__global__ void __launch_bounds__(kFft2MaxThreads) k_fft2r(cplx<R>* __restrict__ data, const cplx<R>* __restrict__ tw,
                                                           const cplx<R>* __restrict__ rtab,
                                                           const int* __restrict__ rperm, int r1, int p, int A,
                                                           int B, size_t es, int ncols, size_t os, int ngroups) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = r1 * p;
    const int N = p - 1;
    const int L = blockDim.x / CW;
    cplx<R>* S = reinterpret_cast<cplx<R>*>(smem_raw);   // [n][CW] pass-1 output
    cplx<R>* Tt = S + size_t(n) * CW;                      // [r1 * N][CW] Rader work rows
    cplx<R>* T = Tt + size_t(r1) * N * CW;                 // [n] line twiddles
    cplx<R>* WN = T + n;                                   // [N] W_N^t
    cplx<R>* Bh = WN + N;                                  // [N] this direction's Bh
    int* pin = reinterpret_cast<int*>(Bh + N);             // [N] g^-q
    int* pout = pin + N;                                   // [N] g^m
    const int o = blockIdx.x / ngroups;
    const int g = blockIdx.x - o * ngroups;
    const int c = threadIdx.x & (CW - 1);
    const int lane = threadIdx.x / CW;
    const int c0 = g * CW;
    const bool live = c0 + c < ncols;
    cplx<R>* line = data + size_t(o) * os + c0 + c;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        cplx<R> w = tw[t];
        if (INV) w.y = -w.y;
        T[t] = w;
    }
    for (int t = threadIdx.x; t < N; t += blockDim.x) {
        WN[t] = rtab[t];
        Bh[t] = rtab[(INV ? 2 : 1) * N + t];
        pin[t] = rperm[t];
        pout[t] = rperm[N + t];
    }
    __syncthreads();
    // pass 1: radix r1, global -> shared with pass 2's twiddles applied
    radix_dispatch<CLS>(r1, [&](auto rc) {
        constexpr int RAD = decltype(rc)::value;
#pragma unroll 2
        for (int j1 = lane; j1 < p; j1 += L) {
            cplx<R> x[RAD];
#pragma unroll
            for (int q = 0; q < RAD; ++q) x[q] = live ? line[size_t(j1 + q * p) * es] : mk<R>(R(0), R(0));
            dft_small<R, INV, RAD>(x);
            S[(j1 * RAD) * CW + c] = x[0];
#pragma unroll
            for (int p1 = 1; p1 < RAD; ++p1) S[(j1 * RAD + p1) * CW + c] = x[p1] * T[j1 * p1];
        }
    });
    __syncthreads();
    // R1: A-point DFTs over q1 of a[B q1 + q2], twiddled by W_N^(q2 k1)
    radix_dispatch<CLS>(A, [&](auto rc) {
        constexpr int RA = decltype(rc)::value;
        for (int u = lane; u < r1 * B; u += L) {
            const int q2 = u / r1;
            const int j = u - q2 * r1;
            cplx<R> z[RA];
#pragma unroll
            for (int q1 = 0; q1 < RA; ++q1) z[q1] = S[(j + pin[B * q1 + q2] * r1) * CW + c];
            dft_small<R, false, RA>(z);
            cplx<R>* trow = Tt + (size_t(j) * N + q2 * RA) * CW + c;
            trow[0] = z[0];
#pragma unroll
            for (int k1 = 1; k1 < RA; ++k1) trow[k1 * CW] = q2 ? z[k1] * WN[q2 * k1] : z[k1];
        }
    });
    __syncthreads();
    // R2: B-point DFT over q2 (-> DFT_N(a) at k1 + A k2), times Bh, B-point
    // inverse DFT over k2, twiddles W_N^(-m1 k1); the thread rewrites the
    // same Tt slots it read
    radix_dispatch<CLS>(B, [&](auto rc) {
        constexpr int RB = decltype(rc)::value;
        for (int u = lane; u < r1 * A; u += L) {
            const int k1 = u / r1;
            const int j = u - k1 * r1;
            cplx<R>* tcol = Tt + (size_t(j) * N + k1) * CW + c;
            cplx<R> v[RB];
#pragma unroll
            for (int q2 = 0; q2 < RB; ++q2) v[q2] = tcol[q2 * A * CW];
            dft_small<R, false, RB>(v);
            if (k1 == 0 && live) {
                const cplx<R> x0 = S[j * CW + c];
                line[size_t(j) * es] = x0 + v[0];   // y[0] = x[0] + sum a
            }
#pragma unroll
            for (int k2 = 0; k2 < RB; ++k2) v[k2] = v[k2] * Bh[k1 + A * k2];
            dft_small<R, true, RB>(v);
            tcol[0] = v[0];
#pragma unroll
            for (int m1 = 1; m1 < RB; ++m1) {
                cplx<R> w = WN[m1 * k1];
                w.y = -w.y;
                tcol[m1 * A * CW] = k1 ? v[m1] * w : v[m1];
            }
        }
    });
    __syncthreads();
    // R4: A-point inverse DFT over k1 -> c[m1 + B m2]; y[g^m] = x[0] + c[m]
    radix_dispatch<CLS>(A, [&](auto rc) {
        constexpr int RA = decltype(rc)::value;
        for (int u = lane; u < r1 * B; u += L) {
            const int m1 = u / r1;
            const int j = u - m1 * r1;
            const cplx<R>* trow = Tt + (size_t(j) * N + m1 * RA) * CW + c;
            cplx<R> d[RA];
#pragma unroll
            for (int k1 = 0; k1 < RA; ++k1) d[k1] = trow[k1 * CW];
            dft_small<R, true, RA>(d);
            if (!live) continue;
            const cplx<R> x0 = S[j * CW + c];
#pragma unroll
            for (int m2 = 0; m2 < RA; ++m2) line[size_t(pout[m1 + B * m2] * r1 + j) * es] = x0 + d[m2];
        }
    });
}

size_t fft2r_smem(int n, int r1, int N, int cw, size_t elem) {
    return (size_t(n) * cw + size_t(r1) * N * cw + n + 2 * size_t(N)) * elem + 2 * sizeof(int) * N;
}

template <typename R, bool INV, int CW>
void launch2r_cw(int cls, int nblocks, int nthreads, size_t shm, cudaStream_t s, cplx<R>* data, const cplx<R>* tw,
                 const cplx<R>* rtab, const int* rperm, int r1, int p, int A, int B, size_t es, int ncols, size_t os,
                 int ngroups) {
    auto go = [&](auto kern) {
        set_smem_limit(kern, shm);
        kern<<<nblocks, nthreads, shm, s>>>(data, tw, rtab, rperm, r1, p, A, B, es, ncols, os, ngroups);
    };
    if (cls == 8) go(k_fft2r<R, CW, INV, 8>);
    else if (cls == 12) go(k_fft2r<R, CW, INV, 12>);
    else go(k_fft2r<R, CW, INV, 16>);
}

// smallest primitive root of the prime p
int primitive_root(int p) {
    std::vector<int> f;
    int m = p - 1;
    for (int d = 2; d * d <= m; ++d)
        if (m % d == 0) {
            f.push_back(d);
            while (m % d == 0) m /= d;
        }
    if (m > 1) f.push_back(m);
    for (int g = 2; g < p; ++g) {
        bool ok = true;
        for (int q : f) {
            long long e = (p - 1) / q, r = 1, b = g;
            while (e) {
                if (e & 1) r = r * b % p;
                b = b * b % p;
                e >>= 1;
            }
            if (r == 1) { ok = false; break; }
        }
        if (ok) return g;
    }
    return 0;
}

size_t fft_smem(int n, int cw, size_t elem, int pt_total) {
    const size_t pt_off_bytes = (((2 * size_t(n) * cw + n) * elem + 8 * size_t(n)) + 15) & ~size_t(15);
    return pt_off_bytes + size_t(pt_total) * elem;
}

int pick_cw(int n, size_t elem, int ncols, int pt_total) {
    int cw = 32;
    while (cw > 1 && fft_smem(n, cw, elem, pt_total) > kFftSmemBudget) cw /= 2;
    while (cw > 1 && cw / 2 >= ncols) cw /= 2;
    return cw;
}

template <typename R, bool INV, bool KSCALE, int CW>
void launch_cw(int cls, bool stream, int nouter, size_t shm, cudaStream_t s, cplx<R>* data, const FftFactors& f,
               const cplx<R>* tw, size_t es, int ncols, size_t os, const cplx<R>* ptw, const LineScale<R>& ks) {
    const int ngroups = (ncols + CW - 1) / CW;
    auto go = [&](auto kern) {
        set_smem_limit(kern, shm);
        kern<<<nouter * ngroups, kFftThreads, shm, s>>>(data, f, tw, es, ncols, os, ptw, ngroups, ks);
    };
    if (stream) {
        if (cls == 8) go(k_fft_axis<R, INV, CW, 8, true, KSCALE>);
        else go(k_fft_axis<R, INV, CW, 16, true, KSCALE>);
    } else {
        if (cls == 8) go(k_fft_axis<R, INV, CW, 8, false, KSCALE>);
        else go(k_fft_axis<R, INV, CW, 16, false, KSCALE>);
    }
}

template <typename R, bool INV, bool KSCALE>
void launch(int cw, int cls, bool stream, int grd, size_t shm, cudaStream_t s, cplx<R>* data, const FftFactors& f,
            const cplx<R>* tw, size_t es, int ncols, size_t os, const cplx<R>* ptw, const LineScale<R>& ks) {
    switch (cw) {
        case 32: launch_cw<R, INV, KSCALE, 32>(cls, stream, grd, shm, s, data, f, tw, es, ncols, os, ptw, ks); break;
        case 16: launch_cw<R, INV, KSCALE, 16>(cls, stream, grd, shm, s, data, f, tw, es, ncols, os, ptw, ks); break;
        case 8: launch_cw<R, INV, KSCALE, 8>(cls, stream, grd, shm, s, data, f, tw, es, ncols, os, ptw, ks); break;
        case 4: launch_cw<R, INV, KSCALE, 4>(cls, stream, grd, shm, s, data, f, tw, es, ncols, os, ptw, ks); break;
        case 2: launch_cw<R, INV, KSCALE, 2>(cls, stream, grd, shm, s, data, f, tw, es, ncols, os, ptw, ks); break;
        default: launch_cw<R, INV, KSCALE, 1>(cls, stream, grd, shm, s, data, f, tw, es, ncols, os, ptw, ks); break;
    }
}

}  // namespace

bool AxisFFT::fits(int n, bool fp64) {
    const size_t elem = fp64 ? sizeof(double2) : sizeof(float2);
    return (3 * size_t(n)) * elem + 8 * size_t(n) + 16 <= kFftSmemMax;
}

void AxisFFT::init(int n) {
    if (n == f_.n && tw64_.p) return;
    f_ = FftFactors{};
    f_.n = n;
    // prime factors, small ones merged while the product stays <= 8
    std::vector<int> pf;
    int m = n;
    for (int p = 2; p * p <= m; ++p)
        while (m % p == 0) { pf.push_back(p); m /= p; }
    if (m > 1) pf.push_back(m);
    std::sort(pf.begin(), pf.end());
    std::vector<int> rs;
    for (int x : pf) {
        if (!rs.empty() && rs.back() * x <= 8) rs.back() *= x;
        else rs.push_back(x);
    }
    if (int(rs.size()) > kFftMaxFactors) throw std::runtime_error("FFT length has too many factors");
    f_.nf = int(rs.size());
    for (int i = 0; i < f_.nf; ++i) f_.r[i] = rs[i];
    std::pair<int, int> sp = fft2_split(n);
    kind_ = sp.first ? 1 : 0;
    if (!kind_) {
        sp = fft2p_split(n);
        kind_ = sp.first ? 2 : 0;
    }
    r1_ = sp.first;
    r2_ = sp.second;
    std::vector<double2> t64(n);
    std::vector<float2> t32(n);
    for (int t = 0; t < n; ++t) {
        const double a = -2.0 * kPi * double(t) / double(n);
        t64[t] = make_double2(std::cos(a), std::sin(a));
        t32[t] = make_float2(float(t64[t].x), float(t64[t].y));
    }
    tw64_.ensure(sizeof(double2) * n);
    tw32_.ensure(sizeof(float2) * n);
    MPM_CUDA(cudaMemcpy(tw64_.p, t64.data(), sizeof(double2) * n, cudaMemcpyHostToDevice));
    MPM_CUDA(cudaMemcpy(tw32_.p, t32.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
    // W_r^(p q) tables of the general kernel's streamed (r > 16) passes
    std::vector<double2> p64;
    for (int i = 0; i < f_.nf; ++i) {
        if (f_.r[i] <= 16) continue;
        f_.pt_off[i] = int(p64.size());
        f_.pt_ld[i] = append_prime_table(f_.r[i], p64);
    }
    f_.pt_total = int(p64.size());
    upload_table(p64, pt64_, pt32_);
    // Rader tables when p - 1 splits into two in-register radices and the
    // kernel's shared memory fits at its narrowest tile (4 fp64 columns)
    ra_ = rb_ = 0;
    if (kind_ == 2) {
        const int pr = r2_, N = pr - 1;
        const std::pair<int, int> ab = fft2_split(N);
        const int g = primitive_root(pr);
        if (ab.first && g && fft2r_smem(n, r1_, N, 4, sizeof(double2)) <= kFftSmemBudget) {
            kind_ = 3;
            ra_ = ab.first;
            rb_ = ab.second;
            std::vector<int> perm(2 * N);
            std::vector<long long> gp(N);   // g^s mod p
            long long v = 1;
            for (int t = 0; t < N; ++t) {
                gp[t] = v;
                v = v * g % pr;
            }
            for (int q = 0; q < N; ++q) perm[q] = int(gp[(N - q) % N]);   // a_q = x[g^-q]
            for (int m = 0; m < N; ++m) perm[N + m] = int(gp[m]);         // y[g^m]
            std::vector<double2> t64(3 * size_t(N));
            for (int t = 0; t < N; ++t) {
                const double a = -2.0 * kPi * double(t) / double(N);
                t64[t] = make_double2(std::cos(a), std::sin(a));
            }
            // Bh = DFT_N(b) / N, b_s = W_p^(g^s) (forward) or its conjugate (inverse)
            for (int k = 0; k < N; ++k) {
                double fr = 0, fi = 0, ir = 0, ii = 0;
                for (int t = 0; t < N; ++t) {
                    const double ab_ = -2.0 * kPi * double(gp[t]) / double(pr);
                    const double br = std::cos(ab_), bi = std::sin(ab_);
                    const double e = -2.0 * kPi * double((long long)t * k % N) / double(N);
                    const double er = std::cos(e), ei = std::sin(e);
                    fr += br * er - bi * ei;
                    fi += br * ei + bi * er;
                    ir += br * er + bi * ei;
                    ii += br * ei - bi * er;
                }
                t64[N + k] = make_double2(fr / N, fi / N);
                t64[2 * N + k] = make_double2(ir / N, ii / N);
            }
            upload_table(t64, rt64_, rt32_);
            rperm_.ensure(sizeof(int) * perm.size());
            MPM_CUDA(cudaMemcpy(rperm_.p, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice));
        }
    }
    // the streamed prime pass's table; lengths whose table and tile do not
    // fit in shared memory go to the general multi-pass kernel
    pp_total_ = pp_ld_ = 0;
    if (kind_ == 2) {
        std::vector<double2> q64;
        const int ld = append_prime_table(r2_, q64);
        if (fft2p_smem(n, 4, sizeof(double2), int(q64.size())) <= kFftSmemBudget) {
            pp_ld_ = ld;
            pp_total_ = int(q64.size());
            upload_table(q64, pp64_, pp32_);
        } else {
            kind_ = 0;
            r1_ = r2_ = 0;
        }
    }
}

void AxisFFT::upload_table(std::vector<double2> t64, DevBuf& d64, DevBuf& d32) {
    if (t64.empty()) t64.push_back(make_double2(0.0, 0.0));
    std::vector<float2> t32(t64.size());
    for (size_t k = 0; k < t64.size(); ++k) t32[k] = make_float2(float(t64[k].x), float(t64[k].y));
    d64.ensure(sizeof(double2) * t64.size());
    d32.ensure(sizeof(float2) * t32.size());
    MPM_CUDA(cudaMemcpy(d64.p, t64.data(), sizeof(double2) * t64.size(), cudaMemcpyHostToDevice));
    MPM_CUDA(cudaMemcpy(d32.p, t32.data(), sizeof(float2) * t32.size(), cudaMemcpyHostToDevice));
}

template <typename R>
void AxisFFT::launch_line(cplx<R>* data, size_t es, int ncols, size_t os, int nouter, int mode, const R* scale,
                          int sz, int sb, cudaStream_t s) const {
    if (f_.n <= 1 || nouter <= 0 || ncols <= 0) return;
    const int n = f_.n;
    LineScale<R> ks;
    ks.sc = scale;
    ks.nouter = nouter;
    ks.sz = sz;
    ks.sb = sb;
    const cplx<R>* tw = sizeof(R) == 4 ? reinterpret_cast<const cplx<R>*>(tw32_.p)
                                       : reinterpret_cast<const cplx<R>*>(tw64_.p);
    const int kind = path(ncols, mode);
    if (kind == 3) {
        // two-pass with a Rader prime pass
        const int N = r2_ - 1;
        const int L = 24;
        // wide butterfly classes hold more registers: smaller CTAs
        int cw = register_class(std::max(r1_, ra_)) > 8 ? 8 : 16;
        while (cw > 4 && (cw * L > (sizeof(R) == 8 ? 192 : kFft2MaxThreads) ||
                          fft2r_smem(n, r1_, N, cw, sizeof(cplx<R>)) > kFftSmemBudget))
            cw /= 2;
        const size_t shm = fft2r_smem(n, r1_, N, cw, sizeof(cplx<R>));
        if (shm > kFftSmemMax) throw std::runtime_error("FFT line does not fit in shared memory");
        const int ngroups = (ncols + cw - 1) / cw;
        const int nblocks = nouter * ngroups;
        const int cls = register_class(std::max(r1_, ra_));
        const cplx<R>* rt = sizeof(R) == 4 ? reinterpret_cast<const cplx<R>*>(rt32_.p)
                                           : reinterpret_cast<const cplx<R>*>(rt64_.p);
        const int* rp = rperm_.as<int>();
        auto go = [&](auto invc) {
            constexpr bool INV = decltype(invc)::value;
            if (cw == 16)
                launch2r_cw<R, INV, 16>(cls, nblocks, cw * L, shm, s, data, tw, rt, rp, r1_, r2_, ra_, rb_, es, ncols,
                                        os, ngroups);
            else if (cw == 8)
                launch2r_cw<R, INV, 8>(cls, nblocks, cw * L, shm, s, data, tw, rt, rp, r1_, r2_, ra_, rb_, es, ncols,
                                       os, ngroups);
            else
                launch2r_cw<R, INV, 4>(cls, nblocks, cw * L, shm, s, data, tw, rt, rp, r1_, r2_, ra_, rb_, es, ncols,
                                       os, ngroups);
        };
        if (mode == 1) go(std::true_type{});
        else go(std::false_type{});
        MPM_LAUNCH();
        return;
    }
    if (kind == 2) {
        // two-pass with a streamed prime pass
        const int half = (r2_ - 1) / 2;
        const int pc = fft2p_pc<R>();
        const int nitems = r1_ * ((half + pc - 1) / pc);
        const int L = std::min(sizeof(R) == 8 ? 24 : 32, std::max(16, nitems));
        int cw = 16;
        while (cw > 4 && (cw * L > kFft2MaxThreads ||
                          fft2p_smem(n, cw, sizeof(cplx<R>), pp_total_) > kFftSmemBudget))
            cw /= 2;
        const size_t shm = fft2p_smem(n, cw, sizeof(cplx<R>), pp_total_);
        const int ngroups = (ncols + cw - 1) / cw;
        const int nblocks = nouter * ngroups;
        const int cls = r1_ <= 8 ? 8 : 16;
        const cplx<R>* ptw = sizeof(R) == 4 ? reinterpret_cast<const cplx<R>*>(pp32_.p)
                                            : reinterpret_cast<const cplx<R>*>(pp64_.p);
        auto go = [&](auto invc) {
            constexpr bool INV = decltype(invc)::value;
            if (cw == 16)
                launch2p_cw<R, INV, 16>(cls, nblocks, cw * L, shm, s, data, tw, ptw, pp_total_, pp_ld_, r1_, r2_, es,
                                        ncols, os, ngroups);
            else if (cw == 8)
                launch2p_cw<R, INV, 8>(cls, nblocks, cw * L, shm, s, data, tw, ptw, pp_total_, pp_ld_, r1_, r2_, es,
                                       ncols, os, ngroups);
            else
                launch2p_cw<R, INV, 4>(cls, nblocks, cw * L, shm, s, data, tw, ptw, pp_total_, pp_ld_, r1_, r2_, es,
                                       ncols, os, ngroups);
        };
        if (mode == 1) go(std::true_type{});
        else go(std::false_type{});
        MPM_LAUNCH();
        return;
    }
    if (kind == 1) {
        // two-pass in-register transform
        // fp64 butterflies hold twice the registers: smaller CTAs keep two
        // of them resident per SM
        const int maxthr = sizeof(R) == 8 ? 192 : kFft2MaxThreads;
        int cw = 32;
        while (cw > 16 && (cw * r1_ > maxthr || fft2_smem(n, cw, sizeof(cplx<R>)) > kFftSmemBudget)) cw /= 2;
        if (cw * r1_ > kFft2MaxThreads) throw std::runtime_error("two-pass FFT: too many threads");
        const size_t shm = fft2_smem(n, cw, sizeof(cplx<R>));
        const int ngroups = (ncols + cw - 1) / cw;
        const int nblocks = nouter * ngroups;
        const int cls = register_class(r1_);
        auto go = [&](auto modec) {
            constexpr int MODE = decltype(modec)::value;
            if (cw == 32)
                launch2_cw<R, MODE, 32>(cls, nblocks, cw * r1_, shm, s, data, tw, r1_, r2_, es, ncols, os, ngroups, ks);
            else
                launch2_cw<R, MODE, 16>(cls, nblocks, cw * r1_, shm, s, data, tw, r1_, r2_, es, ncols, os, ngroups, ks);
        };
        if (mode == 2) go(std::integral_constant<int, 2>{});
        else if (mode == 1) go(std::integral_constant<int, 1>{});
        else go(std::integral_constant<int, 0>{});
        MPM_LAUNCH();
        return;
    }
    // the prime-pass tables go to shared memory when small (else the pass
    // indexes the line's own twiddles)
    FftFactors f = f_;
    int cw = pick_cw(n, sizeof(cplx<R>), ncols, 0);
    {
        // few lines in all (a batch of a few grid columns): fewer columns per
        // CTA, so that at least two CTAs per SM share the lines (a heuristic
        // on the first device's SM count)
        static const int sms = [] {
            int d = 0, v = 148;
            if (cudaGetDevice(&d) != cudaSuccess ||
                cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d) != cudaSuccess)
                v = 148;
            return v;
        }();
        while (cw > 4 && (long long)nouter * ((ncols + cw - 1) / cw) < 2LL * sms) cw /= 2;
    }
    // (only when that costs no columns per CTA)
    if (fft_smem(n, cw, sizeof(cplx<R>), f.pt_total) > kFftSmemBudget) f.pt_total = 0;
    const int pt_total = f.pt_total;
    const size_t shm = fft_smem(n, cw, sizeof(cplx<R>), pt_total);
    if (shm > kFftSmemMax) throw std::runtime_error("FFT line does not fit in shared memory");
    const int grd = nouter;
    int rsmall = 1;
    bool stream = false;
    for (int i = 0; i < f_.nf; ++i) {
        if (f_.r[i] > 16) stream = true;
        else rsmall = std::max(rsmall, f_.r[i]);
    }
    const int cls = rsmall <= 8 ? 8 : 16;
    const cplx<R>* ptw = sizeof(R) == 4 ? reinterpret_cast<const cplx<R>*>(pt32_.p)
                                        : reinterpret_cast<const cplx<R>*>(pt64_.p);
    if (mode == 2) launch<R, false, true>(cw, cls, stream, grd, shm, s, data, f, tw, es, ncols, os, ptw, ks);
    else if (mode == 1) launch<R, true, false>(cw, cls, stream, grd, shm, s, data, f, tw, es, ncols, os, ptw, ks);
    else launch<R, false, false>(cw, cls, stream, grd, shm, s, data, f, tw, es, ncols, os, ptw, ks);
    MPM_LAUNCH();
}

template <typename R>
void AxisFFT::run(cplx<R>* data, size_t es, int ncols, size_t os, int nouter, bool inverse, cudaStream_t s) const {
    launch_line<R>(data, es, ncols, os, nouter, inverse ? 1 : 0, nullptr, 1, 1, s);
}

template <typename R>
void AxisFFT::run_scaled(cplx<R>* data, size_t es, int ncols, size_t os, int nouter, const R* scale, int sz, int sb,
                         cudaStream_t s) const {
    if (!scale || sz <= 0 || sb <= 0) throw std::runtime_error("run_scaled: scale table and its strides required");
    launch_line<R>(data, es, ncols, os, nouter, 2, scale, sz, sb, s);
}

size_t slab_smem(int n, int Zs, int mc, size_t elem) { return (2 * size_t(n) * Zs * 3 * mc + n) * elem; }

bool AxisFFT::slab_ok(int Zs, bool fp64) const {
    if (kind_ != 1 || force_general_ || Zs < 1 || Zs > 16) return false;
    const int mc = fp64 ? slab_mc<double>(Zs == 1) : slab_mc<float>(Zs == 1);
    return slab_smem(f_.n, Zs, mc, fp64 ? sizeof(double2) : sizeof(float2)) <= kFftSmemBudget;
}

template <typename R>
void AxisFFT::run_slab(cplx<R>* data, int nx, int Zs, int M, const cplx<R>* taps, double kxu, double kyu,
                       cudaStream_t s) const {
    if (!slab_ok(Zs, sizeof(R) == 8)) throw std::runtime_error("run_slab: slab not supported by this axis");
    if (nx <= 0 || M <= 0) return;
    constexpr int MC1 = slab_mc<R>(true), MCS = slab_mc<R>(false);
    const int MC = Zs == 1 ? MC1 : MCS;
    const int n = f_.n;
    const size_t shm = slab_smem(n, Zs, MC, sizeof(cplx<R>));
    SlabArgs a;
    a.Nx = nx;
    a.Zs = Zs;
    a.M = M;
    a.nchunk = (M + MC - 1) / MC;
    a.kxu = kxu;
    a.kyu = kyu;
    const cplx<R>* tw = sizeof(R) == 4 ? reinterpret_cast<const cplx<R>*>(tw32_.p)
                                       : reinterpret_cast<const cplx<R>*>(tw64_.p);
    const int cls = register_class(r1_);
    auto go = [&](auto kern) {
        set_smem_limit(kern, shm);
        kern<<<nx * a.nchunk, kSlabThreads, shm, s>>>(data, tw, taps, r1_, r2_, a);
    };
    if (Zs == 1) {
        if (cls == 8) go(k_slab<R, MC1, 1, 8>);
        else if (cls == 12) go(k_slab<R, MC1, 1, 12>);
        else go(k_slab<R, MC1, 1, 16>);
    } else if (Zs <= 9) {
        if (cls == 8) go(k_slab<R, MCS, 9, 8>);
        else if (cls == 12) go(k_slab<R, MCS, 9, 12>);
        else go(k_slab<R, MCS, 9, 16>);
    } else {
        if (cls == 8) go(k_slab<R, MCS, 16, 8>);
        else if (cls == 12) go(k_slab<R, MCS, 16, 12>);
        else go(k_slab<R, MCS, 16, 16>);
    }
    MPM_LAUNCH();
}

template void AxisFFT::run_slab<float>(float2*, int, int, int, const float2*, double, double, cudaStream_t) const;
template void AxisFFT::run_slab<double>(double2*, int, int, int, const double2*, double, double, cudaStream_t) const;
template void AxisFFT::run<float>(float2*, size_t, int, size_t, int, bool, cudaStream_t) const;
template void AxisFFT::run<double>(double2*, size_t, int, size_t, int, bool, cudaStream_t) const;
template void AxisFFT::run_scaled<float>(float2*, size_t, int, size_t, int, const float*, int, int,
                                         cudaStream_t) const;
template void AxisFFT::run_scaled<double>(double2*, size_t, int, size_t, int, const double*, int, int,
                                          cudaStream_t) const;

}  // namespace mpm
