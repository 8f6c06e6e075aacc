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
    // the two-pass split n = r1 * r2 (r1 >= r2, in-register radices), or (0, 0)
    int split_r1() const { return r1_; }
    int split_r2() const { return r2_; }
    // run every length through the general multi-pass kernel (tests)
    void set_force_general(bool v) { force_general_ = v; }
    // whether a transform of ncols columns takes the two-pass kernel
    bool two_pass(int ncols) const { return r1_ && ncols >= 16 && !force_general_; }

private:
    template <typename R>
    void launch_line(cplx<R>* data, size_t es, int ncols, size_t os, int nouter, int mode, const R* scale, int sz,
                     int sb, cudaStream_t s) const;
    FftFactors f_;
    int r1_ = 0, r2_ = 0;
    bool force_general_ = false;
    DevBuf tw64_, tw32_;
    DevBuf pt64_, pt32_;   // prime-pass twiddle tables (see FftFactors)
};

}  // namespace mpm
