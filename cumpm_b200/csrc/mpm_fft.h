// Batched 1-D DFT along one axis of a grid whose batch index is innermost.
//
// The spectral-Ewald grids are stored [x][y][slot][b] with the right-hand
// sides innermost, so a transform along x or y sees, for every grid point,
// a contiguous row of independent columns.  Each CTA stages one line of a
// chunk of columns in shared memory and runs a mixed-radix Stockham
// autosort there (every radix pass computes each output as an r-term sum
// with table twiddles, so any prime factor works without Bluestein), then
// writes the line back in place.  Global loads and stores are row-coalesced.
// Unnormalised in both directions (the 1/V factor lives in the k-space
// scale, as in the reference's cuFFT use).
#pragma once

#include "mpm_common.cuh"

#include <vector>

namespace mpm {

constexpr int kFftMaxFactors = 16;

struct FftFactors {
    int n = 1;
    int nf = 0;
    int r[kFftMaxFactors] = {};
    // factors above 16 (streamed passes): offset and row length of their
    // W_r^(p q) table, rows q = 1..(r-1)/2, columns p = 1..(r-1)/2 (padded)
    int pt_off[kFftMaxFactors] = {};
    int pt_ld[kFftMaxFactors] = {};
    int pt_total = 0;     // entries of all tables together
};

class AxisFFT {
public:
    void init(int n);
    int n() const { return f_.n; }
    // transform `nouter` lines: line o, column c, element e lives at
    // data[o*os + e*es + c], c in [0, ncols)
    template <typename R>
    void run(cplx<R>* data, size_t es, int ncols, size_t os, int nouter, bool inverse, cudaStream_t s) const;
    // forward transform, multiplication of element e of line o, column c by
    // scale[(e * nouter + o) * sz + c / sb], inverse transform: the k-space
    // step of a convolution fused into one pass over the lines
    template <typename R>
    void run_scaled(cplx<R>* data, size_t es, int ncols, size_t os, int nouter, const R* scale, int sz, int sb,
                    cudaStream_t s) const;
    // whether one line of this length fits in shared memory
    static bool fits(int n, bool fp64);
    // the two-pass split n = r1 * r2: both in-register radices (r1 >= r2), or
    // r1 in-register and r2 a prime above 16 (streamed); (0, 0) if neither
    int split_r1() const { return r1_; }
    int split_r2() const { return r2_; }
    // run every length through the general multi-pass kernel (tests)
    void set_force_general(bool v) { force_general_ = v; }
    // kernel a transform of ncols columns takes: 0 general multi-pass,
    // 1 two-pass in registers, 2 two-pass with a streamed prime pass, 3
    // two-pass with a Rader prime pass (modes 0 forward, 1 inverse, 2
    // forward-scale-inverse; 2 has no prime variant)
    int path(int ncols, int mode) const {
        if (!r1_ || ncols < 16 || force_general_) return 0;
        if (kind_ >= 2 && mode == 2) return 0;
        return kind_;
    }
    // the Rader split p - 1 = A * B (0 when the prime pass is streamed)
    int rader_a() const { return ra_; }

    // The k-space step of the pruned (z-slab) monodisperse grid fused with
    // this axis's transforms, for the y axis: data is the grid
    // [x][y][slot][c][m] (Zs slots, 3 components, M right-hand sides), already
    // transformed along x.  For every (kx, chunk of right-hand sides) one CTA
    // loads its Ny x Zs x 3 x chunk values into shared memory, transforms
    // along y, applies the slab Green tensor of every (kx, ky) column as
    // three scalar Toeplitz kernels in z (taps [x][y][3][2 Zs - 1]:
    // t_n(d) = sum_kz kz^n S(k) / |k|^2 exp(2 pi i kz d / Nz), n = 0, 1, 2),
    //   a = kx E_x + ky E_y,  u = t0 * a + t1 * E_z,
    //   E_x <- kx u,  E_y <- ky u,  E_z <- t1 * a + t2 * E_z,
    // transforms back along y and stores: one HBM round trip for the y
    // transforms and the Green tensor.  kxu, kyu: the wavenumber of one
    // grid frequency along x and y (2 pi / L); nx: grid points along x.
    template <typename R>
    void run_slab(cplx<R>* data, int nx, int Zs, int M, const cplx<R>* taps, double kxu, double kyu,
                  cudaStream_t s) const;
    // whether run_slab handles this slab (two-pass in-register y transform,
    // Zs <= 16 slots, tile within the shared-memory budget)
    bool slab_ok(int Zs, bool fp64) const;

private:
    template <typename R>
    void launch_line(cplx<R>* data, size_t es, int ncols, size_t os, int nouter, int mode, const R* scale, int sz,
                     int sb, cudaStream_t s) const;
    static void upload_table(std::vector<double2> t64, DevBuf& d64, DevBuf& d32);
    FftFactors f_;
    int kind_ = 0, r1_ = 0, r2_ = 0;
    int ra_ = 0, rb_ = 0;   // Rader split of r2_ - 1
    DevBuf rt64_, rt32_;     // Rader tables: W_N^t, forward Bh, inverse Bh
    DevBuf rperm_;           // Rader index maps: g^-q, g^m
    bool force_general_ = false;
    DevBuf tw64_, tw32_;
    DevBuf pt64_, pt32_;   // prime-pass twiddle tables (see FftFactors)
    DevBuf pp64_, pp32_;   // the prime-streamed two-pass kernel's W_p^(p' q) table
    int pp_total_ = 0, pp_ld_ = 0;
};

}  // namespace mpm
