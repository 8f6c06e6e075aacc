// Polydisperse spectral-Ewald pieces shared by host and device code.
//
// Pair functions of two radii (a, b): the perpendicular and parallel
// real-space coefficients fd1, fd2 of the smoothed-sphere dipole field and
// the self value, restated from polydisperse_ewald_electric_field.cu:
// 1434-1627.  The reference writes eight exp/erfc terms per function; they
// pair up by two symmetries, which this file uses instead of the eight
// separate polynomials:
//   * the term of exp(-(r - s)^2 xi^2) is the term of exp(-(r + s)^2 xi^2)
//     at -r (s = a + b), the erfc((r - s) xi) term is minus the
//     erfc((r + s) xi) term at -r;
//   * the a - b terms are the a + b terms with a -> -a (a^3 -> -a^3 in the
//     prefactor included).
// One exception is kept: the reference's fd2 term of exp(-(r + a - b)^2 xi^2)
// has +4 (a - b)^2 (a^2 + 4ab + b^2) xi^4 in its r^1 coefficient where the
// symmetry gives -4; the difference is added explicitly (it vanishes for
// a == b).
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define MPM_HD __host__ __device__ __forceinline__
#else
#define MPM_HD inline
#endif

namespace mpm {
namespace poly {

constexpr double kPi_ = 3.14159265358979323846;
constexpr double kTableDr = 0.001;

// exp-weighted part of fd1 for radii (a, b) at signed distance r (a may be
// negative): the reference's first term, divided by its prefactor.
MPM_HD double e1(double r, double a, double b, double x) {
    const double x2 = x * x, x4 = x2 * x2, x5 = x4 * x;
    const double s = a + b;
    const double c3 = 4 * a * a * a - 3 * a * a * b - 3 * a * b * b + 4 * b * b * b;
    const double qm = a * a - 4 * a * b + b * b;
    const double r2 = r * r, r3 = r2 * r;
    const double poly = ((((4 * x4) * r - 4 * s * x4) * r + (16 * x2 + 8 * (-4 * a * a + a * b - 4 * b * b) * x4)) * r +
                         (-12 * s * x2 - 8 * c3 * x4)) * r2 +
                        r * (3 - 12 * (a * a - a * b + b * b) * x2 - 4 * s * s * qm * x4) + 3 * s + 4 * c3 * x2 +
                        4 * s * s * s * qm * x4;
    return poly / (1024.0 * kPi_ * std::sqrt(kPi_) * (a * a * a) * (b * b * b) * r3 * x5);
}

// erfc-weighted part of fd1 (the reference's fifth term).
MPM_HD double c1(double r, double a, double b, double x) {
    const double x2 = x * x, x4 = x2 * x2, x6 = x4 * x2;
    const double s = a + b, q2 = a * a + b * b, d2 = (a * a - b * b) * (a * a - b * b);
    const double qm = a * a - 4 * a * b + b * b;
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2;
    const double poly = -8 * r4 * r2 * x6 + 36 * r4 * x4 * (-1 + 2 * q2 * x2) + 128 * (a * a * a + b * b * b) * r3 * x6 +
                        r2 * (-18 * x2 + 72 * q2 * x4 + 72 * d2 * x6) + 3 - 18 * q2 * x2 - 36 * d2 * x4 -
                        8 * s * s * s * s * qm * x6;
    return poly / (2048.0 * kPi_ * (a * a * a) * (b * b * b) * r3 * x6);
}

// exp-weighted part of fd2.
MPM_HD double e2(double r, double a, double b, double x) {
    const double x2 = x * x, x4 = x2 * x2, x5 = x4 * x;
    const double s = a + b;
    const double c3 = 4 * a * a * a - 3 * a * a * b - 3 * a * b * b + 4 * b * b * b;
    const double c3b = a * a * a - 3 * a * a * b - 3 * a * b * b + b * b * b;
    const double qm = a * a - 4 * a * b + b * b;
    const double r2 = r * r, r3 = r2 * r;
    const double poly = ((((8 * x4) * r - 8 * s * x4) * r + (14 * x2 - 4 * (7 * a * a - 4 * a * b + 7 * b * b) * x4)) * r +
                         (-6 * s * x2 - 4 * c3b * x4)) * r2 +
                        r * (-3 + 12 * (a * a - a * b + b * b) * x2 + 4 * s * s * qm * x4) - 3 * s - 4 * c3 * x2 -
                        4 * s * s * s * qm * x4;
    return poly / (512.0 * kPi_ * std::sqrt(kPi_) * (a * a * a) * (b * b * b) * r3 * x5);
}

// erfc-weighted part of fd2.
MPM_HD double c2(double r, double a, double b, double x) {
    const double x2 = x * x, x4 = x2 * x2, x6 = x4 * x2;
    const double s = a + b, q2 = a * a + b * b, d2 = (a * a - b * b) * (a * a - b * b);
    const double qm = a * a - 4 * a * b + b * b;
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2;
    const double poly = -16 * r4 * r2 * x6 + 36 * r4 * x4 * (-1 + 2 * q2 * x2) + 64 * (a * a * a + b * b * b) * r3 * x6 -
                        3 + 18 * q2 * x2 + 36 * d2 * x4 + 8 * s * s * s * s * qm * x6;
    return poly / (1024.0 * kPi_ * (a * a * a) * (b * b * b) * r3 * x6);
}

// fd1(r), fd2(r) for radii a <= b (the table orientation) at r > 0.
MPM_HD void pair_functions(double r, double a, double b, double x, double& fd1, double& fd2) {
    const double x2 = x * x;
    double f1 = 0.0, f2 = 0.0;
    for (int sg = 0; sg < 2; ++sg) {
        const double aa = sg ? -a : a;
        const double s = aa + b;
        const double ep = std::exp(-(r + s) * (r + s) * x2), em = std::exp(-(r - s) * (r - s) * x2);
        const double cp = std::erfc((r + s) * x), cm = std::erfc((r - s) * x);
        f1 += e1(r, aa, b, x) * ep + e1(-r, aa, b, x) * em + c1(r, aa, b, x) * cp - c1(-r, aa, b, x) * cm;
        f2 += e2(r, aa, b, x) * ep + e2(-r, aa, b, x) * em + c2(r, aa, b, x) * cp - c2(-r, aa, b, x) * cm;
    }
    {   // the reference's fd2 r^1 coefficient of exp(-(r + a - b)^2 xi^2)
        const double t = a - b, x4 = x2 * x2, x5 = x4 * x;
        const double extra = 8 * t * t * (a * a + 4 * a * b + b * b) * x4 * r /
                             (512.0 * kPi_ * std::sqrt(kPi_) * (a * a * a) * (b * b * b) * r * r * r * x5);
        f2 += extra * std::exp(-(r + t) * (r + t) * x2);
    }
    // overlap / enclosure regularisation
    const double r3 = r * r * r, a3 = a * a * a, b3 = b * b * b;
    const double s = a + b, t = std::fabs(a - b);
    if (r < s && r >= t) {
        const double qm = a * a - 4 * a * b + b * b;
        f1 += (s - r) * (s - r) * (s - r) / (128.0 * kPi_ * a3 * b3 * r3) *
              (-r3 - 3 * s * r * r + 3 * qm * r + a3 - 3 * a * a * b - 3 * a * b * b + b3);
        f2 += -1.0 / (64.0 * kPi_ * a3 * b3 * r3) *
              (s * s * s * s * qm - 8 * (a3 + b3) * r3 + 9 * (a * a + b * b) * r3 * r - 2 * r3 * r3);
    } else if (r < b - a) {
        f1 += (r3 - b3) / (4.0 * kPi_ * b3 * r3);
        f2 += (r3 + 2 * b3) / (4.0 * kPi_ * b3 * r3);
    } else if (r < a - b) {
        f1 += (r3 - a3) / (4.0 * kPi_ * a3 * r3);
        f2 += (r3 + 2 * a3) / (4.0 * kPi_ * a3 * r3);
    }
    fd1 = f1;
    fd2 = f2;
}

// r = 0 entry of the (a, b) table: the self value.
MPM_HD double self_value(double a, double b, double x) {
    const double x2 = x * x, a3 = a * a * a, b3 = b * b * b;
    const double s = a + b, t = a - b;
    return 1.0 / (16.0 * kPi_ * std::sqrt(kPi_) * a3 * b3 * x2 * x) *
               ((1 - 2 * a * a * x2 + 2 * a * b * x2 - 2 * b * b * x2) * std::exp(-s * s * x2) +
                (-1 + 2 * a * a * x2 + 2 * a * b * x2 + 2 * b * b * x2) * std::exp(-t * t * x2)) +
           1.0 / (8.0 * kPi_ * a3 * b3) * ((a3 - b3) * std::erf(t * x) - (a3 + b3) * std::erf(s * x)) +
           (a3 < b3 ? a3 : b3) / (4.0 * kPi_ * a3 * b3);
}

// Table node k of the reference's r grid: 0, then 1 + (k-1) * 0.001.
MPM_HD double node(int k) { return k == 0 ? 0.0 : 1.0 + double(k - 1) * kTableDr; }

// Value the reference's linear table lookup returns at distance d
// (interpolate_table_gpu_polydisperse, :170-187) for a table of n nodes,
// evaluating only the nodes it reads.  Returns perp (fd1) and para (fd2).
MPM_HD void table_lookup(double d, double a, double b, double x, int n, double& perp, double& para) {
    double y0a, y0b, y1a, y1b;
    const double last = node(n - 1);
    if (d <= 0.0) {
        perp = para = self_value(a, b, x);
        return;
    }
    if (d >= last) {
        pair_functions(last, a, b, x, perp, para);
        return;
    }
    if (d < 1.0) {
        y0a = y0b = self_value(a, b, x);
        pair_functions(1.0, a, b, x, y1a, y1b);
        perp = y0a * (1.0 - d) + y1a * d;
        para = y0b * (1.0 - d) + y1b * d;
        return;
    }
    const int k = 1 + static_cast<int>((d - 1.0) / kTableDr);
    if (k >= n - 1) {
        pair_functions(last, a, b, x, perp, para);
        return;
    }
    const double r0 = node(k), r1 = node(k + 1);
    pair_functions(r0, a, b, x, y0a, y0b);
    pair_functions(r1, a, b, x, y1a, y1b);
    const double t = (d - r0) / (r1 - r0);
    perp = y0a * (1.0 - t) + y1a * t;
    para = y0b * (1.0 - t) + y1b * t;
}

}  // namespace poly
}  // namespace mpm
