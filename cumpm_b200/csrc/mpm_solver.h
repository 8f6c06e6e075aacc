// Host driver of the self-consistent dipole/quadrupole solve.
//
// Mirrors the reference Dipole_Solver (dipole_solver.h, dipole_solver.cu):
// same constructor arguments, validation messages, non-dimensionalisation
// (length unit = smallest radius, permittivity unit = eps_m), initial-guess
// predictors, frequency loop and result storage/rescaling.  Differences:
// the K incident polarisations of a frequency (or, with batch_all, every
// frequency x polarisation pair) are solved as one batch on the device.
#pragma once

#include <complex>
#include <memory>
#include <string>
#include <vector>

#include "mpm_field.h"
#include "mpm_krylov.h"
#include "mpm_tune.h"

namespace mpm {

using cdouble = std::complex<double>;

enum Precision { PREC_AUTO = 0, PREC_MIXED = 1, PREC_DOUBLE = 2 };

struct DriverOptions {
    int restart = 50;
    int maxiter = 1000;
    bool batch_all = false;     // all frequencies x polarisations in one batch (mean-field guesses)
    bool refine = false;        // mixed precision + fp64 true-residual refinement
    double inner_tol = 1e-4;    // floor of one inner solve's reduction (see SolveOptions)
    bool real_fp32 = false;
};

class DipoleSolver {
public:
    DipoleSolver(std::vector<double> box, std::vector<std::vector<cdouble>> eps_p, std::vector<double> radius,
                 double eps_m, double xi, double tol, bool quiet, std::string guess_type, std::string solver_type,
                 std::string field_type, std::vector<std::vector<cdouble>> E0, bool solve_quadrupoles,
                 std::vector<int> quad_idxs, int precision);
    ~DipoleSolver();

    void compute(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z);

    // Field tuning (mpm_tune.h): a given one, or one measured on these
    // positions (physical units) for this solver's batch width and
    // arithmetic.  Either replaces the field; later frames use it.
    void set_tuning(const FieldTuning& t);
    FieldTuning autotune(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z,
                         TuneReport* report);
    bool tuned() const { return tuned_; }
    const FieldTuning& tuning() const { return tuning_; }

    std::vector<cdouble> get_eff_polarizability(bool physical) const;
    std::vector<cdouble> get_dipoles(bool physical) const;
    // the same values written straight into out (cap entries); returns the count
    size_t get_dipoles_into(bool physical, cdouble* out, size_t cap) const;
    std::vector<cdouble> get_quadrupoles(bool physical) const;

    size_t num_frames() const { return num_frames_; }
    size_t num_particles() const { return N_; }
    size_t num_quads() const { return Nq_; }
    size_t num_wavevectors() const { return eps_p_.size(); }
    size_t num_polarizations() const { return E0_.size(); }
    bool jacobi() const { return jacobi_; }
    void set_jacobi(bool on) { jacobi_ = on; }
    DriverOptions& options() { return opt_; }
    const SolveStats& last_stats() const { return last_stats_; }
    const std::vector<int>& all_iterations() const { return iters_; }
    Field* field() { return field_.get(); }

private:
    void set_dims(size_t n);
    void nondimensionalize();
    void setup(size_t n);               // first frame: dimensions, units, stream, batch solver
    FieldSpec field_spec() const;       // the field the reference's rules give
    std::vector<double> scaled(const std::vector<double>& v) const;
    std::vector<cdouble> mean_field_guess(size_t w) const;
    std::vector<cdouble> guess(const std::vector<cdouble>& fd, const std::vector<cdouble>& fq, size_t w) const;
    void solve_batch(const std::vector<size_t>& freqs, const std::vector<std::vector<cdouble>>& guesses,
                     std::vector<cdouble>& frame_cap, std::vector<cdouble>& frame_dip, std::vector<cdouble>& frame_quad);
    // batch_all with dipoles and uniform incident fields: the mean-field
    // guesses of frequencies 1..W-1 (and frequency 0's, from init) are built
    // on the device and the solution is written into the frame layout there
    bool device_batch_ok() const;
    void solve_all_device(const std::vector<cdouble>& init, std::vector<cdouble>& frame_cap,
                          std::vector<cdouble>& frame_dip);
    void print(const std::string& msg) const;

    std::vector<double> box_;
    std::vector<std::vector<cdouble>> eps_p_;
    std::vector<double> radius_;
    double eps_m_, xi_, tol_;
    bool quiet_;
    std::string guess_type_, solver_type_, field_type_;
    std::vector<std::vector<cdouble>> E0_;
    bool solve_quads_;
    std::vector<int> quad_idxs_;
    int precision_;
    bool jacobi_ = true;
    DriverOptions opt_;

    size_t N_ = 0, Nq_ = 0, num_frames_ = 0;
    double length_scale_ = 1.0, eps_scale_ = 1.0, vol_frac_ = 0.0;
    std::vector<cdouble> avg_dips_;
    // one vector per frame (appending a frame copies nothing already stored)
    std::vector<std::vector<cdouble>> dip_frames_, quad_frames_;
    std::vector<int> iters_;
    SolveStats last_stats_;

    FieldTuning tuning_;
    bool tuned_ = false;
    std::unique_ptr<Field> field_;
    std::unique_ptr<BatchSolver> solver_;
    cudaStream_t stream_ = nullptr;
    DevBuf dB_, dX_, dSC_;
    DevBuf dEps_, dRad_, dE0_, dInit_, dFrame_;   // device batch: eps (W x N), radii, E0 (K x 3), init, frame
    bool dev_eps_ = false;
    HostBuf hB_, hX_, hSC_;   // pinned staging of the batch's right-hand sides, guesses / solutions, self terms
    // frequencies whose right-hand sides and self terms dB_ / dSC_ hold (they
    // depend on nothing that changes between frames)
    std::vector<size_t> dev_freqs_;
    int indent_ = 0;
};

class NearField {
public:
    NearField(std::vector<double> box, std::vector<cdouble> E0, std::vector<double> radius, double xi, double errortol,
              std::string field_type);
    ~NearField();
    void set_dipoles(const std::vector<cdouble>& dip);
    void set_dipole_positions(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z);
    void set_field_points(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z);
    std::vector<double> calculate();

private:
    std::vector<double> box_;
    std::vector<cdouble> E0_;
    std::vector<double> radius_;
    double xi_, errortol_;
    std::string field_type_;
    size_t N_ = 0;
    std::vector<cdouble> dips_;
    std::vector<double> px_, py_, pz_, fx_, fy_, fz_;
    double length_scale_ = 1.0;
    FieldTuning tuning_;
    bool tuned_ = false;
    std::unique_ptr<Field> field_;
    cudaStream_t stream_ = nullptr;
    DevBuf dX_, dY_;
};

}  // namespace mpm
