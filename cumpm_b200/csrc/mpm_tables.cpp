// Closed-form real-space pair functions of the finite-size (unit sphere)
// spectral-Ewald split, tabulated for linear lookup.
//
// Every function has the shape
//   f(r) = sum_{s in {+2,-2,0}} [ A_s(r) exp(-(r+s)^2 xi^2) + B_s(r) erfc((r+s) xi) ]
//          + [r < 2] R(r)
// where the A/B polynomials and the overlap regularisation R follow the
// reference closed forms (monodisperse_ewald_electric_field.cu:132-459;
// self values :462-467).  The formulas are physics that must agree term by
// term for parity; the code layout here is this project's own.
#include "mpm_tables.h"

#include <cmath>

namespace mpm {

namespace {

constexpr double PI = 3.14159265358979323846;

struct Terms {
    double ep, em, e0, fp, fm, f0, reg;
};

inline double combine(double r, double xi, const Terms& t) {
    const double x2 = xi * xi;
    double v = t.ep * std::exp(-(r + 2.0) * (r + 2.0) * x2) + t.fp * std::erfc((r + 2.0) * xi) +
               t.em * std::exp(-(r - 2.0) * (r - 2.0) * x2) + t.fm * std::erfc((r - 2.0) * xi) +
               t.e0 * std::exp(-r * r * x2) + t.f0 * std::erfc(r * xi);
    if (r < 2.0) v += t.reg;
    return v;
}

struct Powers {
    double x, x2, x4, x5, x6, x7, x8, x9, x10;
    explicit Powers(double xi) {
        x = xi; x2 = xi * xi; x4 = x2 * x2; x5 = x4 * xi; x6 = x4 * x2; x7 = x6 * xi;
        x8 = x4 * x4; x9 = x8 * xi; x10 = x8 * x2;
    }
};

// dipole field, (I - rr) coefficient
Terms fd1_terms(double r, const Powers& p) {
    const double sp = std::pow(PI, 1.5);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3;
    const double x2 = p.x2, x4 = p.x4, x6 = p.x6;
    Terms t;
    const double ce = 1.0 / (1024.0 * sp * p.x5 * r3);
    t.ep = ce * (4 * x4 * r5 - 8 * x4 * r4 + 8 * x2 * (2 - 7 * x2) * r3 - 8 * x2 * (3 + 2 * x2) * r2 +
                 (3 - 12 * x2 + 32 * x4) * r + 2 * (3 + 4 * x2 - 32 * x4));
    t.em = ce * (4 * x4 * r5 + 8 * x4 * r4 + 8 * x2 * (2 - 7 * x2) * r3 + 8 * x2 * (3 + 2 * x2) * r2 +
                 (3 - 12 * x2 + 32 * x4) * r - 2 * (3 + 4 * x2 - 32 * x4));
    t.e0 = (-4 * x4 * r4 - 8 * x2 * (2 - 9 * x2) * r2 - 3 + 36 * x2) / (512.0 * sp * p.x5 * r2);
    const double cf = 1.0 / (2048.0 * PI * x6 * r3);
    t.fp = cf * (-8 * x6 * r6 - 36 * x4 * (1 - 4 * x2) * r4 + 256 * x6 * r3 - 18 * x2 * (1 - 8 * x2) * r2 + 3 -
                 36 * x2 + 256 * x6);
    t.fm = cf * (-8 * x6 * r6 - 36 * x4 * (1 - 4 * x2) * r4 - 256 * x6 * r3 - 18 * x2 * (1 - 8 * x2) * r2 + 3 -
                 36 * x2 + 256 * x6);
    t.f0 = (8 * x6 * r6 + 36 * x4 * (1 - 4 * x2) * r4 + 18 * x2 * (1 - 8 * x2) * r2 - 3 + 36 * x2) /
           (1024.0 * PI * x6 * r3);
    t.reg = -1.0 / (4 * PI * r3) + (1.0 - 9.0 * r / 16.0 + r3 / 32.0) / (4 * PI);
    return t;
}

// dipole field, rr coefficient
Terms fd2_terms(double r, const Powers& p) {
    const double sp = std::pow(PI, 1.5);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3;
    const double x2 = p.x2, x4 = p.x4, x6 = p.x6;
    Terms t;
    const double ce = 1.0 / (512.0 * sp * p.x5 * r3);
    t.ep = ce * (8 * x4 * r5 - 16 * x4 * r4 + 2 * x2 * (7 - 20 * x2) * r3 - 4 * x2 * (3 - 4 * x2) * r2 -
                 (3 - 12 * x2 + 32 * x4) * r - 2 * (3 + 4 * x2 - 32 * x4));
    t.em = ce * (8 * x4 * r5 + 16 * x4 * r4 + 2 * x2 * (7 - 20 * x2) * r3 + 4 * x2 * (3 - 4 * x2) * r2 -
                 (3 - 12 * x2 + 32 * x4) * r + 2 * (3 + 4 * x2 - 32 * x4));
    t.e0 = (-8 * x4 * r4 - 2 * x2 * (7 - 36 * x2) * r2 + 3 - 36 * x2) / (256.0 * sp * p.x5 * r2);
    const double cf = 1.0 / (1024.0 * PI * x6 * r3);
    t.fp = cf * (-16 * x6 * r6 - 36 * x4 * (1 - 4 * x2) * r4 + 128 * x6 * r3 - 3 + 36 * x2 - 256 * x6);
    t.fm = cf * (-16 * x6 * r6 - 36 * x4 * (1 - 4 * x2) * r4 - 128 * x6 * r3 - 3 + 36 * x2 - 256 * x6);
    t.f0 = (16 * x6 * r6 + 36 * x4 * (1 - 4 * x2) * r4 + 3 - 36 * x2) / (512.0 * PI * x6 * r3);
    t.reg = 1.0 / (2 * PI * r3) + (1.0 - 9.0 * r / 8.0 + r3 / 8.0) / (4 * PI);
    return t;
}

Terms fq1_terms(double r, const Powers& p) {
    const double sp = std::pow(PI, 1.5);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3, r7 = r6 * r, r8 = r4 * r4;
    const double x2 = p.x2, x4 = p.x4, x6 = p.x6, x8 = p.x8;
    Terms t;
    const double ce = 15.0 / (16384.0 * sp * p.x7 * r4);
    const double q = (3 - 8 * x2) * (3 - 8 * x2);
    t.ep = ce * (-24 * x6 * r7 - 4 * x4 * (9 - 8 * x2) * r5 + 8 * x4 * (3 - 8 * x2) * r4 + 48 * x6 * r6 +
                 2 * x2 * (21 - 80 * x2 + 64 * x4) * r3 - 4 * x2 * q * r2 -
                 (45 - 120 * x2 + 192 * x4 - 512 * x6) * r - 2 * (45 + 24 * x2 - 64 * x4 + 512 * x6));
    t.em = ce * (-24 * x6 * r7 - 4 * x4 * (9 - 8 * x2) * r5 - 8 * x4 * (3 - 8 * x2) * r4 - 48 * x6 * r6 +
                 2 * x2 * (21 - 80 * x2 + 64 * x4) * r3 + 4 * x2 * q * r2 -
                 (45 - 120 * x2 + 192 * x4 - 512 * x6) * r + 2 * (45 + 24 * x2 - 64 * x4 + 512 * x6));
    t.e0 = 15.0 / (8192.0 * sp * p.x7 * r3) *
           (24 * x6 * r6 + 4 * x4 * (9 - 32 * x2) * r4 - 2 * x2 * (21 - 128 * x2) * r2 + 45 - 480 * x2);
    const double base = 48 * x8 * r8 + 32 * x6 * (3 - 8 * x2) * r6 - 24 * x4 * (3 - 16 * x2) * r4 +
                        72 * x2 * (1 - 8 * x2) * r2;
    t.fp = 15.0 / (32768.0 * PI * x8 * r4) * (base - 45 + 480 * x2 + 4096 * x8);
    t.fm = t.fp;
    t.f0 = 15.0 / (16384.0 * PI * x8 * r4) * (-base + 45 - 480 * x2);
    t.reg = -15.0 / (4 * PI * r4) + 15.0 * r2 / (64 * PI) * (1.0 - 3.0 * r2 / 16.0);
    return t;
}

Terms fq2_terms(double r, const Powers& p) {
    const double sp = std::pow(PI, 1.5);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3, r7 = r6 * r, r8 = r4 * r4;
    const double x2 = p.x2, x4 = p.x4, x6 = p.x6, x8 = p.x8;
    Terms t;
    const double ce = 3.0 / (16384.0 * sp * p.x7 * r4);
    const double a = 45 - 120 * x2 + 192 * x4 - 512 * x6;
    const double b = 2 * (45 + 24 * x2 - 64 * x4 + 512 * x6);
    t.ep = ce * (-40 * x6 * r7 + 80 * x6 * r6 - 20 * x4 * (11 - 24 * x2) * r5 + 8 * x4 * (45 + 8 * x2) * r4 -
                 2 * x2 * (45 - 80 * x2 + 64 * x4) * r3 - 4 * x2 * (15 + 48 * x2 - 64 * x4) * r2 + a * r + b);
    t.em = ce * (-40 * x6 * r7 - 80 * x6 * r6 - 20 * x4 * (11 - 24 * x2) * r5 - 8 * x4 * (45 + 8 * x2) * r4 -
                 2 * x2 * (45 - 80 * x2 + 64 * x4) * r3 + 4 * x2 * (15 + 48 * x2 - 64 * x4) * r2 + a * r - b);
    t.e0 = 15.0 / (8192.0 * sp * p.x7 * r3) *
           (8 * x6 * r6 + 4 * x4 * (11 - 32 * x2) * r4 + 2 * x2 * (9 - 64 * x2) * r2 - 9 + 96 * x2);
    const double cf = 3.0 / (32768.0 * PI * x8 * r4);
    const double common = 80 * x8 * r8 + 160 * x6 * (3 - 8 * x2) * r6 + 120 * x4 * (3 - 16 * x2) * r4 -
                          120 * x2 * (1 - 8 * x2) * r2 + 45 - 480 * x2 - 4096 * x8;
    t.fp = cf * (common - 2048 * x8 * r5);
    t.fm = cf * (common + 2048 * x8 * r5);
    t.f0 = 15.0 / (16384.0 * PI * x8 * r4) *
           (-16 * x8 * r8 - 32 * x6 * (3 - 8 * x2) * r6 - 24 * x4 * (3 - 16 * x2) * r4 +
            24 * x2 * (1 - 8 * x2) * r2 - 9 + 96 * x2);
    t.reg = 3.0 / (4 * PI * r4) - 3.0 * r / (8 * PI) * (1.0 - 5.0 * r / 8.0 + 5.0 * r3 / 128.0);
    return t;
}

Terms fq3_terms(double r, const Powers& p) {
    const double sp = std::pow(PI, 1.5);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3;
    const double x2 = p.x2, x4 = p.x4, x6 = p.x6;
    Terms t;
    const double ce = 5.0 / (1024.0 * sp * p.x5 * r2);
    t.ep = ce * (4 * x4 * r5 - 8 * x4 * r4 + 16 * x2 * (1 - 2 * x2) * r3 - 24 * x2 * r2 + 3 * r + 6);
    t.em = ce * (4 * x4 * r5 + 8 * x4 * r4 + 16 * x2 * (1 - 2 * x2) * r3 + 24 * x2 * r2 + 3 * r - 6);
    t.e0 = 5.0 / (512.0 * sp * p.x5 * r) * (-4 * x4 * r4 - 16 * x2 * (1 - 3 * x2) * r2 - 3 + 24 * x2);
    const double cf = 5.0 / (2048.0 * PI * x6 * r2);
    const double common = -8 * x6 * r6 - 12 * x4 * (3 - 8 * x2) * r4 - 6 * x2 * (3 - 16 * x2) * r2 + 3 - 24 * x2;
    t.fp = cf * (common + 128 * x6 * r3);
    t.fm = cf * (common - 128 * x6 * r3);
    t.f0 = 5.0 / (1024.0 * PI * x6 * r2) *
           (8 * x6 * r6 + 12 * x4 * (3 - 8 * x2) * r4 + 6 * x2 * (3 - 16 * x2) * r2 - 3 + 24 * x2);
    t.reg = 5.0 * r / (8 * PI) * (1.0 - 3.0 * r / 4.0 + r3 / 16.0);
    return t;
}

Terms gq1_terms(double r, const Powers& p) {
    const double sp = std::pow(PI, 1.5);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3, r7 = r6 * r, r8 = r4 * r4;
    const double x2 = p.x2, x4 = p.x4, x6 = p.x6, x8 = p.x8;
    Terms t;
    const double ce = 75.0 / (16384.0 * sp * p.x7 * r3);
    t.ep = ce * (8 * x6 * r7 - 16 * x6 * r6 + (44 * x4 - 32 * x6) * r5 - (72 * x4 - 64 * x6) * r4 +
                 (18 * x2 + 32 * x4) * r3 + (12 * x2 - 64 * x4) * r2 - (9 + 24 * x2) * r - (18 - 48 * x2));
    t.em = ce * (8 * x6 * r7 + 16 * x6 * r6 + (44 * x4 - 32 * x6) * r5 + (72 * x4 - 64 * x6) * r4 +
                 (18 * x2 + 32 * x4) * r3 - (12 * x2 - 64 * x4) * r2 - (9 + 24 * x2) * r + (18 - 48 * x2));
    t.e0 = -75.0 / (8192.0 * sp * p.x7 * r2) *
           (8 * x6 * r6 + (44 * x4 - 64 * x6) * r4 + (18 * x2 - 64 * x4 + 128 * x6) * r2 - 9 + 48 * x2 - 192 * x4);
    const double poly = 16 * x8 * r8 + (96 * x6 - 128 * x8) * r6 + (72 * x4 - 192 * x6 + 256 * x8) * r4 -
                        (24 * x2 - 96 * x4 + 256 * x6) * r2 + 9 - 48 * x2 + 192 * x4;
    t.fp = -75.0 / (32768.0 * PI * x8 * r3) * poly;
    t.fm = t.fp;
    t.f0 = 75.0 / (16384.0 * PI * x8 * r3) * poly;
    t.reg = 75.0 * r * (4.0 - r2) * (4.0 - r2) / (1024 * PI);
    return t;
}

Terms gq2_terms(double r, const Powers& p) {
    const double sp = std::pow(PI, 1.5);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3, r7 = r6 * r, r8 = r4 * r4;
    const double r9 = r8 * r, r10 = r5 * r5;
    const double x2 = p.x2, x4 = p.x4, x6 = p.x6, x8 = p.x8, x10 = p.x10;
    Terms t;
    const double ce = 3.0 / (32768.0 * sp * p.x9 * r5);
    const double a6 = 1056 * x6 - 1216 * x8, a4 = 2160 * x4 - 4320 * x6 - 256 * x8;
    const double a2 = 360 * x2 - 1680 * x4 - 768 * x6 + 1024 * x8;
    const double a0 = 270 - 1080 * x2 - 192 * x4 + 512 * x6 - 4096 * x8;
    const double odd = -48 * x8 * r9 - (576 * x6 - 608 * x8) * r7 - (1536 * x4 - 2576 * x6 + 3968 * x8) * r5 -
                       (360 * x2 + 360 * x4 + 640 * x6 - 512 * x8) * r3 +
                       (135 + 180 * x2 + 480 * x4 - 768 * x6 + 2048 * x8) * r;
    const double even = 96 * x8 * r8 + a6 * r6 + a4 * r4 - a2 * r2 + a0;
    t.ep = ce * (odd + even);
    t.em = ce * (odd - even);
    t.e0 = 1.0 / (16384.0 * sp * p.x9 * r4) *
           (144 * x8 * r8 + (1728 * x6 - 2400 * x8) * r6 + (4608 * x4 - 13200 * x6 + 19200 * x8) * r4 +
            (1080 * x2 - 5400 * x4 + 19200 * x6) * r2 - 405 + 2700 * x2 - 14400 * x4);
    const double base = 288 * x10 * r10 + (3600 * x8 - 4800 * x10) * r8 +
                        (10800 * x6 - 28800 * x8 + 38400 * x10) * r6 + (5400 * x4 - 21600 * x6 + 57600 * x8) * r4 -
                        (1350 * x2 - 7200 * x4 + 28800 * x6) * r2 + 405 - 2700 * x2 + 14400 * x4;
    t.fp = (base + 49152 * x10 * r5 + 49152 * x10) / (65536.0 * PI * x10 * r5);
    t.fm = (base - 49152 * x10 * r5 + 49152 * x10) / (65536.0 * PI * x10 * r5);
    t.f0 = -base / (32768.0 * PI * x10 * r5);
    t.reg = -3.0 / (2 * PI) * (1.0 / r5 - 1.0 + 25.0 * r / 32.0 - 25.0 * r3 / 256.0 + 3.0 * r5 / 512.0);
    return t;
}

Terms gq3_terms(double r, const Powers& p) {
    const double sp = std::pow(PI, 1.5);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3, r7 = r6 * r, r8 = r4 * r4;
    const double r9 = r8 * r, r10 = r5 * r5;
    const double x2 = p.x2, x4 = p.x4, x6 = p.x6, x8 = p.x8, x10 = p.x10;
    Terms t;
    const double ce = -15.0 / (65536.0 * sp * p.x9 * r5);
    const double odd = 48 * x8 * r9 + (336 * x6 - 288 * x8) * r7 + (216 * x4 + 144 * x6 + 128 * x8) * r5 -
                       (180 * x2 - 120 * x4 + 640 * x6 - 512 * x8) * r3 +
                       (135 + 180 * x2 + 480 * x4 - 768 * x6 + 2048 * x8) * r;
    const double even = -96 * x8 * r8 - 576 * (x6 - x8) * r6 - (480 * x6 + 256 * x8) * r4 +
                        (720 * x4 + 768 * x6 - 1024 * x8) * r2 -
                        (-270 + 1080 * x2 + 192 * x4 - 512 * x6 + 4096 * x8);
    t.ep = ce * (odd + even);
    t.em = ce * (odd - even);
    t.e0 = 15.0 / (32768.0 * sp * p.x9 * r4) *
           (48 * x8 * r8 + (336 * x6 - 480 * x8) * r6 + (216 * x4 - 720 * x6 + 1280 * x8) * r4 -
            (180 * x2 - 840 * x4 + 2560 * x6) * r2 + 135 - 900 * x2 + 4800 * x4);
    const double base = -96 * x10 * r10 + (-720 * x8 + 960 * x10) * r8 -
                        (720 * x6 - 1920 * x8 + 2560 * x10) * r6 + (360 * x4 - 1440 * x6 + 3840 * x8) * r4 -
                        (270 * x2 - 1440 * x4 + 5760 * x6) * r2 + 135 - 900 * x2 + 4800 * x4;
    t.fp = -15.0 / (131072.0 * PI * x10 * r5) * (base + 16384 * x10);
    t.fm = t.fp;
    t.f0 = 15.0 / (65536.0 * PI * x10 * r5) * base;
    const double c4 = r2 - 4.0;
    t.reg = -15.0 * c4 * c4 * c4 * (3.0 * r4 + 6.0 * r2 + 8.0) / (2048 * PI * r5);
    return t;
}

Terms gq4_terms(double r, const Powers& p) {
    const double sp = std::pow(PI, 1.5);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3, r7 = r6 * r, r8 = r4 * r4;
    const double r9 = r8 * r, r10 = r5 * r5;
    const double x2 = p.x2, x4 = p.x4, x6 = p.x6, x8 = p.x8, x10 = p.x10;
    Terms t;
    const double ce = -15.0 / (65536.0 * sp * p.x9 * r5);
    const double odd = 144 * x8 * r9 + (288 * x6 + 96 * x8) * r7 - (432 * x4 - 912 * x6 + 896 * x8) * r5 +
                       (720 * x2 - 2280 * x4 + 4480 * x6 - 3584 * x8) * r3 -
                       (945 + 1260 * x2 + 3360 * x4 - 5376 * x6 + 14336 * x8) * r;
    const double even = -288 * x8 * r8 - (288 * x6 + 192 * x8) * r6 + (720 * x4 - 480 * x6 + 1792 * x8) * r4 -
                        (1080 * x2 + 2160 * x4 + 5376 * x6 - 7168 * x8) * r2 -
                        (1890 - 7560 * x2 - 1344 * x4 + 3584 * x6 - 28672 * x8);
    t.ep = ce * (odd + even);
    t.em = ce * (odd - even);
    t.e0 = 15.0 / (32768.0 * sp * p.x9 * r4) *
           (144 * x8 * r8 + (288 * x6 - 480 * x8) * r6 - (432 * x4 - 1200 * x6 + 1280 * x8) * r4 +
            (720 * x2 - 3000 * x4 + 6400 * x6) * r2 - 945 + 6300 * x2 - 33600 * x4);
    const double base = 288 * x10 * r10 + (720 * x8 - 960 * x10) * r8 -
                        (720 * x6 - 1920 * x8 + 2560 * x10) * r6 + (1080 * x4 - 4320 * x6 + 11520 * x8) * r4 -
                        (1350 * x2 - 7200 * x4 + 28800 * x6) * r2 + 945 - 6300 * x2 + 33600 * x4;
    t.fp = 15.0 / (131072.0 * PI * x10 * r5) * (base + 114688 * x10);
    t.fm = t.fp;
    t.f0 = -15.0 / (65536.0 * PI * x10 * r5) * base;
    t.reg = -15.0 * (3584.0 - 80.0 * r6 - 30.0 * r8 + 9.0 * r10) / (2048 * PI * r5);
    return t;
}

// polydisperse grad_quad_2 (polydisperse_ewald_electric_field.cu:1890-1924):
// the polydisperse field's own expression, lower in degree than gq2_terms
Terms gq2_poly_terms(double r, const Powers& p) {
    const double sp = std::pow(PI, 1.5);
    const double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r, r6 = r3 * r3, r7 = r6 * r, r8 = r4 * r4;
    const double x2 = p.x2, x4 = p.x4, x6 = p.x6, x8 = p.x8;
    Terms t;
    const double ce = -15.0 / (16384.0 * sp * p.x7 * r3);
    const double odd = 24 * x6 * r7 + (148 * x4 - 96 * x6) * r5 + (90 * x2 + 72 * x4 + 256 * x8) * r3 -
                       (45 + 120 * x2 - 192 * x4 + 512 * x6) * r;
    const double even = -48 * x6 * r6 - (264 * x4 - 192 * x6) * r4 + (60 * x2 - 144 * x4 + 512 * x8) * r2 -
                        2 * (45 + 24 * x2 - 64 * x4 + 512 * x6);
    t.ep = ce * (odd + even);
    t.em = ce * (odd - even);
    t.e0 = 75.0 / (8192.0 * sp * p.x7 * r2) *
           (8 * x6 * r6 + (44 * x4 - 64 * x6) * r4 + (18 * x2 - 48 * x4 + 128 * x6) * r2 - 9 + 40 * x2 - 192 * x4);
    const double base = 48 * x8 * r8 + (288 * x6 - 384 * x8) * r6 + (216 * x4 - 576 * x6 + 768 * x8) * r4 -
                        (72 * x2 - 288 * x4 + 768 * x6) * r2 + 45 - 240 * x2 + 960 * x4;
    const double cf = -15.0 / (32768.0 * PI * x8 * r3);
    t.fp = cf * (base - 4096 * x8 * r5 - 8192 * x8);
    t.fm = cf * (base + 4096 * x8 * r5 - 8192 * x8);
    t.f0 = 15.0 / (16384.0 * PI * x8 * r3) * base;
    t.reg = -45.0 * r / (32 * PI) * (1.0 - 5.0 * r2 / 12.0 + r4 / 16.0);
    return t;
}

// polydisperse grad_quad_3 (:1926-1967): gq3_terms with the r^5 and r^4
// terms of the exp(-(r+2)^2 xi^2) coefficient taken with the opposite sign
Terms gq3_poly_terms(double r, const Powers& p) {
    Terms t = gq3_terms(r, p);
    const double r2 = r * r, r4 = r2 * r2, r5 = r4 * r;
    const double ce = -15.0 / (65536.0 * std::pow(PI, 1.5) * p.x9 * r5);
    t.ep -= 2.0 * ce * ((216 * p.x4 + 144 * p.x6 + 128 * p.x8) * r5 - (480 * p.x6 + 256 * p.x8) * r4);
    return t;
}

// r = 0 entry of the gradient tables for the unit sphere
double gradient_self_value(double xi) {
    const double x2 = xi * xi, x4 = x2 * x2, x5 = x4 * xi;
    return 0.5 / PI *
           (3.0 * (3.0 - 10.0 * x2 + 20.0 * x4) / (8.0 * std::sqrt(PI) * x5) -
            3.0 * (3.0 + 2.0 * x2 + 4.0 * x4) * std::exp(-4.0 * x2) / (8.0 * std::sqrt(PI) * x5) +
            3.0 * std::erfc(2.0 * xi));
}

}  // namespace

MonoTables build_mono_tables(double xi) {
    MonoTables T;
    const Powers p(xi);
    T.r.resize(kTableSize);
    for (auto& v : T.f) v.resize(kTableSize);
    using Fn = Terms (*)(double, const Powers&);
    const Fn fns[T_COUNT] = {fd1_terms, fd2_terms, fq1_terms, fq2_terms, fq3_terms,
                             gq1_terms, gq2_terms, gq3_terms, gq4_terms};
    for (int k = 0; k < kTableSteps; ++k) {
        const double r = 1.0 + k * kTableDr;
        T.r[k + 1] = r;
        for (int f = 0; f < T_COUNT; ++f) T.f[f][k + 1] = combine(r, xi, fns[f](r, p));
    }
    const double x2 = p.x2;
    T.selfo = (-1.0 + 6.0 * x2 + (1.0 - 2.0 * x2) * std::exp(-4.0 * x2)) / (16.0 * std::pow(PI, 1.5) * x2 * xi) +
              std::erfc(2.0 * xi) / (4.0 * PI);
    T.self_grad = gradient_self_value(xi);
    T.r[0] = 0.0;
    T.f[T_FD1][0] = T.selfo;
    T.f[T_FD2][0] = T.selfo;
    T.f[T_FQ1][0] = T.f[T_FQ2][0] = T.f[T_FQ3][0] = 0.0;
    for (int f = T_GQ1; f <= T_GQ4; ++f) T.f[f][0] = T.self_grad;
    return T;
}

PolyQuadTables build_poly_quad_tables(double xi, int n_nodes) {
    if (n_nodes < 2) n_nodes = 2;
    PolyQuadTables T;
    const Powers p(xi);
    T.r.resize(n_nodes);
    for (auto& v : T.f) v.resize(n_nodes);
    using Fn = Terms (*)(double, const Powers&);
    const Fn fns[PQ_COUNT] = {fq1_terms, fq2_terms, fq3_terms, gq1_terms, gq2_poly_terms, gq3_poly_terms, gq4_terms};
    for (int k = 0; k + 1 < n_nodes; ++k) {
        const double r = 1.0 + k * kTableDr;
        T.r[k + 1] = r;
        for (int f = 0; f < PQ_COUNT; ++f) T.f[f][k + 1] = combine(r, xi, fns[f](r, p));
    }
    T.self_grad = gradient_self_value(xi);
    T.r[0] = 0.0;
    T.f[PQ_FQ1][0] = T.f[PQ_FQ2][0] = T.f[PQ_FQ3][0] = 0.0;
    for (int f = PQ_GQ1; f <= PQ_GQ4; ++f) T.f[f][0] = T.self_grad;
    return T;
}

double poly_quad_self_value(double a, double xi) {
    return gradient_self_value(xi * a) / (a * a * a * a * a);
}

double table_lookup(double r, const double* rt, const double* y, int n) {
    if (r <= 0.0) return y[0];
    if (r >= rt[n - 1]) return y[n - 1];
    if (r < 1.0) return y[0] * (1.0 - r) + y[1] * r;
    size_t idx = 1 + static_cast<size_t>((r - 1.0) / kTableDr);
    if (idx >= static_cast<size_t>(n - 1)) return y[n - 1];
    const double t = (r - rt[idx]) / (rt[idx + 1] - rt[idx]);
    return y[idx] * (1.0 - t) + y[idx + 1] * t;
}

}  // namespace mpm
