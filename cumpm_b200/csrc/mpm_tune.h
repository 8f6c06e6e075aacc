// Autotuner of the spectral-Ewald field: picks the splitting parameter xi,
// the grid, the Gaussian support and the spread tile for one particle
// configuration and one batch width by measurement on the device.
//
// The reference fixes all of them by rule from the user's xi and tolerance
// (grid N = ceil(1 + L kcut / pi), monodisperse_ewald_electric_field.cu:
// 546-616; polydisperse_ewald_electric_field.cu:2039-2112).  Any xi gives the
// same Ewald sum up to the truncation errors, so the tuner may move xi (the
// balance between the real-space pair sum and the reciprocal grid), round
// the grid up to sizes the line transforms handle fastest, trim the support
// and change the spread tile, and keeps a candidate only if its operator
// error, measured against a field of 1000x tighter tolerance on the same
// positions, stays within max(errortol, the rule's own error).
#pragma once

#include <vector>

#include "mpm_field.h"

namespace mpm {

struct FieldTuning {
    double xi = 0.0;
    int grid[3] = {0, 0, 0};   // 0: the rule
    int support = 0;           // 0: the rule
    int tile[2] = {0, 0};      // 0: 8 x 8
};

struct TuneReport {
    double apply_ms = 0, apply_ms_rule = 0;   // M-column apply: the pick, the rule
    double error = 0, error_rule = 0;         // relative operator error against the tight field
    double error_bound = 0;                   // acceptance bound
    int candidates = 0, accepted = 0;
};

// One stage-1 candidate: xi with its rule grid, support and cutoff.
struct XiCandidate {
    double xi;
    int grid[3];
    int support;
    double rc;
};

// smallest n' >= n whose prime factors are all 2, 3, 5 or 7
int tune_next_fast(int n);
// smallest n' >= n of the form 2^a 3^b
int tune_next_smooth23(int n);
// the xi candidates (base xi times fixed factors) for which the rules give a
// valid geometry: cutoff below half the box, stencil within the kernels'
// limit; host only
std::vector<XiCandidate> tune_xi_candidates(const FieldSpec& base);
// spread tiles (x, y) the kernels accept for a stencil half width `off`
std::vector<std::pair<int, int>> tune_tiles(int off);

// Measures candidates on the device (positions non-dimensional, host
// arrays) for a batch of M right-hand sides in the given arithmetic, and
// returns the fastest accepted one.  Direct fields have nothing to tune
// (the base is returned).
FieldTuning autotune(const FieldSpec& base, const double* x, const double* y, const double* z, int n, int M,
                     bool recip_fp32, bool real_fp32, cudaStream_t s, TuneReport* report);

// base with the tuning's overrides
FieldSpec apply_tuning(const FieldSpec& base, const FieldTuning& t);

}  // namespace mpm
