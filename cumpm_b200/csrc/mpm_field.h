// Electric-field operator E = A(p) of the Mutual Polarization Method.
//
// One Field object replaces the reference's Electric_Field hierarchy
// (electric_field/electric_field.h:13-141) for the field kinds the solve
// uses:
//   * FIELD_MONO   periodic box, monodisperse spectral Ewald
//                  (monodisperse_ewald_electric_field.cu)
//   * FIELD_POLY   periodic box, polydisperse spectral Ewald, dipoles
//                  (polydisperse_ewald_electric_field.cu)
//   * FIELD_DIRECT open boundaries, all-pairs sum (direct_electric_field.cu)
// in either SOLVER_AX mode (the Krylov matvec: self terms, i != j) or
// INTERACTION_FIELD mode (field at arbitrary points, used by Near_Field).
//
// Unlike the reference, apply() takes M right-hand sides at once.  Moment
// and field vectors are device arrays in [row][M] layout (row = 3*i + c for
// dipoles, 3*N + 5*q + c for quadrupoles), complex128.
#pragma once

#include <cufft.h>
#include <memory>
#include <vector>

#include "mpm_common.cuh"
#include "mpm_fft.h"
#include "mpm_tables.h"

namespace mpm {

enum FieldKind { FIELD_DIRECT = 0, FIELD_MONO = 1, FIELD_POLY = 2 };

struct FieldSpec {
    int kind = FIELD_MONO;
    bool solver_ax = true;
    double box[3] = {0, 0, 0};
    double errortol = 1e-3;
    double xi = 0.5;
    std::vector<double> radius;       // per particle (direct, polydisperse) or empty
    bool quads = false;
    std::vector<int> quad_idxs;       // empty + quads => all particles
    // overrides of the spectral-Ewald rules (0: the rule), set by the
    // autotuner (mpm_tune.cu): grid points per axis, Gaussian support P,
    // spread tile in x and y (monodisperse)
    int grid[3] = {0, 0, 0};
    int support = 0;
    int tile[2] = {0, 0};
    // Bloch wavevector (x, y) of the periodic images (EELS zone sum):
    // k-space at k - b, a phase on every real-space pair; dipoles only
    double bloch[2] = {0.0, 0.0};
};

// Spectral-Ewald parameters (monodisperse_ewald_electric_field.cu:546-616).
struct EwaldGeom {
    double rc = 0, kcut = 0;
    int ng[3] = {0, 0, 0};
    double h[3] = {0, 0, 0};
    int P = 0;          // num_grid_gaussian (sets eta)
    int off = 0;        // stencil half width, stencil = 2*off+1 points
    double eta[3] = {0, 0, 0};
    double spread_const = 0;  // (2 xi^2/pi)^1.5 / sqrt(eta_x eta_y eta_z)
};

// grid / support: overrides of the rules (null / 0: the rule)
EwaldGeom make_ewald_geom(const double box[3], double errortol, double xi, const int* grid = nullptr,
                          int support = 0);

// Polydisperse parameters (polydisperse_ewald_electric_field.cu:2039-2112)
// and radius classes (:39-84).
struct PolyGeom {
    double rc = 0;
    int ng[3] = {0, 0, 0};
    double h[3] = {0, 0, 0};
    int P = 0;            // support points per dimension
    int off_min = 0;      // first offset, -floor((P-1)/2)
    double eta = 0;
    int table_n = 0;      // nodes of the reference's pair tables (r = 0, 1, 1.001, ...)
    std::vector<double> unique;  // sorted radius classes
    std::vector<int> cls;        // class of each particle
};

PolyGeom make_poly_geom(const double box[3], double errortol, double xi, const std::vector<double>& radii,
                        const int* grid = nullptr, int support = 0);

// Device-side description of the stored part of the grid.
struct GridView {
    int Nx, Ny, Nz;
    int Zs;        // stored z slots
    int z0;        // first stored plane (pruned layout)
    int pruned;    // 1: slots are the occupied planes z0..z0+Zs-1 (mod Nz)
    int off;       // stencil half width
    int S;         // stencil width
    // z extent of the stencils on the stored grid: S and off, or 1 and 0 for
    // a single layer (every particle the same z stencil, folded into the
    // k-space taps; the grid then holds one z slot)
    int Sz, offz;
    int layer;
};

struct PointSet {
    int n = 0;
    DevBuf xyz;     // double[3][n] SoA
    DevBuf base;    // int4[n] (wrapped gx, wrapped gy, z slot, wrapped gz)
    DevBuf w64;     // double[n][3][S]
    DevBuf w32;     // float[n][3][S]
    // spatial bins (spread sources only)
    DevBuf bin_key, bin_key_sorted, idx, idx_sorted, bin_start, bin_end, cub_tmp;
    int nb[3] = {1, 1, 1};
    int tile[3] = {8, 8, 8};
};

struct FieldStats {
    int pruned = 0;
    int z_slots = 0;
    long long num_pairs = 0;
    int grid[3] = {0, 0, 0};
    int stencil = 0;
    int slab_fused = 0;
    int single_layer = 0;
};

class Field {
public:
    explicit Field(const FieldSpec& spec);
    ~Field();
    Field(const Field&) = delete;
    Field& operator=(const Field&) = delete;

    // Host coordinate arrays (already non-dimensionalised).  In SOLVER_AX
    // mode the field points are the particles.
    void set_positions(const double* x, const double* y, const double* z, int n, cudaStream_t s);
    void set_field_points(const double* x, const double* y, const double* z, int n, cudaStream_t s);

    // Y = A X for M right-hand sides.  self_coef: device [N][M] complex (may
    // be null => zero), jacobi: apply diag(self_coef)^-1 to the result rows.
    // recip_fp32 / real_fp32 pick the arithmetic of the two halves.
    void apply(const double2* X, double2* Y, int M, const double2* self_coef, bool jacobi, bool recip_fp32,
               bool real_fp32, cudaStream_t s);

    // Same as apply(), but the reciprocal-space grid is the caller's scratch
    // (no allocation here); throws if it is smaller than grid_bytes(M).
    void apply_scratch(const double2* X, double2* Y, int M, const double2* self_coef, bool jacobi, bool recip_fp32,
                       bool real_fp32, void* scratch, size_t scratch_bytes, cudaStream_t s);
    size_t grid_bytes(int M, bool fp64) const;

    // Reciprocal-only / real-only parts (for split checks); same layout.
    void apply_part(const double2* X, double2* Y, int M, const double2* self_coef, bool recip_fp32,
                    bool real_fp32, int part, cudaStream_t s);

    // Gradients of the bilinear forms lam_m^T G p_m (G = this operator in
    // SOLVER_AX mode, without the caller's self coefficients), summed over
    // the M columns: gx[i][c] = sum_m d/dx_ic, ga[i] = sum_m d/da_i
    // (complex128, device).  Polydisperse and direct fields (mpm_adjoint.cu).
    void grad_bilinear(const double2* lam, const double2* p, int M, double2* gx, double2* ga, cudaStream_t s);

    // Bloch wavevector (non-dimensional): rebuilds the k-space tables and
    // pair phases at the next apply (Ewald fields, dipoles only)
    void set_bloch(double bx, double by);
    bool bloch_on() const { return spec_.bloch[0] != 0.0 || spec_.bloch[1] != 0.0; }

    int num_particles() const { return N_; }
    int num_targets() const { return spec_.solver_ax ? N_ : targets_.n; }
    int num_quads() const { return Nq_; }
    int rows_in() const { return 3 * N_ + 5 * Nq_; }
    int rows_out() const { return 3 * num_targets() + 5 * Nq_; }
    const FieldSpec& spec() const { return spec_; }
    const EwaldGeom& geom() const { return geom_; }
    FieldStats stats() const;
    const PolyGeom& poly_geom() const { return pgeom_; }
    double selfo() const { return tables_.selfo; }
    const int* quad_map_dev() const { return quad_map_.as<int>(); }
    const int* quad_idx_dev() const { return quad_idx_.as<int>(); }

private:
    void precalc(cudaStream_t s);
    void build_stencil(PointSet& ps, cudaStream_t s, bool bins);
    void build_pairs(cudaStream_t s);
    void choose_layout(cudaStream_t s);
    void build_column_kernel(cudaStream_t s);
    void build_slab_taps(cudaStream_t s);
    bool use_slab() const;   // pruned layout through AxisFFT::run_slab
    void build_scale(cudaStream_t s);
    void build_pair_phases(cudaStream_t s);
    void poly_build_scale();
    cufftHandle plan_for(int B, bool fp32);  // B columns per voxel
    // the real-space part already written into Y on another stream: the
    // contraction waits for `join`, adds, and scales by 1/s (jacobi_sc)
    struct RealOverlap {
        cudaEvent_t join;
        const double2* jacobi_sc;
    };
    template <typename R>
    void recip(const double2* X, double2* Y, int M, cudaStream_t s, const RealOverlap* ov = nullptr);
    template <typename R>
    void recip_on(const double2* X, double2* Y, int M, cplx<R>* grid, cudaStream_t s,
                  const RealOverlap* ov = nullptr);
    template <typename R> void transform(cplx<R>* grid, int B, bool inverse, cudaStream_t s);
    void build_spread_plan(cudaStream_t s);
    void real_part(const double2* X, double2* Y, int M, const double2* self_coef, bool jacobi, bool real_fp32,
                   bool add_recip, cudaStream_t s);
    void direct(const double2* X, double2* Y, int M, const double2* self_coef, bool jacobi, bool fp32,
                cudaStream_t s);
    // polydisperse pieces (mpm_poly.cu)
    void poly_init();
    void poly_precalc(cudaStream_t s);
    void poly_weights(PointSet& ps, const double* radius_dev, cudaStream_t s, bool bins);
    void poly_pair_coefs(cudaStream_t s);
    // Y == nullptr: stop after the inverse transform (grid = potential)
    template <typename R> void poly_recip_on(const double2* X, double2* Y, int M, cplx<R>* grid, cudaStream_t s);

    FieldSpec spec_;
    EwaldGeom geom_;
    MonoTables tables_;
    int N_ = 0, Nq_ = 0;
    PointSet sources_, targets_;
    GridView gv_{};
    bool precalc_dirty_ = true;
    std::vector<double> host_z_;    // source z coordinates (layout choice)

    DevBuf quad_idx_, quad_map_, radius_;
    // polydisperse quadrupoles: point weights of the sources, radius-1
    // quadrupole tables (r then 7 rows of table_n), per particle a^2 and
    // quadrupole self value
    DevBuf pqw64_, pqw32_, pqtab_, pqa2_, pqg2_;
    DevBuf tab_r_, tab_f_;          // double[kTableSize], double[T_COUNT][kTableSize]
    // CSR pairs by target
    DevBuf pair_off_, pair_cnt_, pair_src_, pair_T64_, pair_T32_, pair_Q_, cell_key_, cell_idx_, cell_key_s_,
        cell_idx_s_, cell_start_, cell_end_, cub_tmp_, pair_geo_, pair_ph64_, pair_ph32_;
    long long num_pairs_ = 0;
    // reciprocal space
    DevBuf grid_;                   // complex grid, sized for the largest use
    DevBuf scale64_, scale32_;      // full layout: per-voxel scale
    DevBuf colK64_, colK32_;        // pruned layout: per-column Toeplitz kernels (unfused path)
    DevBuf slabT64_, slabT32_;      // pruned layout: per-column scalar Toeplitz taps t0, t1, t2 (fused path)
    int slab_Z_ = -1;
    // single layer: the common z weights of every stencil (planes z0 ..
    // z0 + S - 1) and the (plane, offset) they were built for
    std::vector<double> layer_w_;
    long layer_key_g_ = -1;
    double layer_key_d_ = 0.0;
    bool layer_taps_ = false, layer_colK_ = false;   // layer taps / column kernel built for that key
    DevBuf layer_wd_;               // device copy of layer_w_ and its |DFT|^2 per kz
    // second stream for the real-space sum alongside the reciprocal chain
    cudaStream_t aux_ = nullptr;
    cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
    // per-frame spread plan (monodisperse): per tile candidates, 1-D weights,
    // column contributor lists; plan_cap_ = 0 when the plan is not in use
    DevBuf plan_nc_, plan_cid_, plan_w64_, plan_w32_, plan_lw64_, plan_lw32_, plan_lc_, plan_ln_, plan_cnt_;
    int plan_cap_ = 0;
    int colK_Z_ = -1;
    int scale_built_ = 0;
    struct PlanKey { int M; bool fp32; int pruned; int Zs; cufftHandle h; };  // M: columns per voxel
    std::vector<PlanKey> plans_;
    AxisFFT fftx_, ffty_, fftz_;    // in-house batched transforms (cuFFT only when a line is too long)
    bool own_fft_ = true;
    // polydisperse
    PolyGeom pgeom_;
    DevBuf pcls_, prad_, pself_, ptrad_;  // class per particle, class radii, self value per particle, target radii
    int pcand_cap_ = 0;                   // largest spread candidate count of a tile
    DevBuf ptoff_, ptlist_, ptmax_;       // per-tile spread candidate lists (CSR), their largest size
    DevBuf ptcnt_, ptclist_, ptruns_;     // per tile: candidates that cover it, their covered runs
    // adjoint: stacked [p | lam] columns, potential grid, per-pair table derivatives, self-value derivatives
    DevBuf adj_x_, adj_grid_, adj_part_, pair_dT_, pself_d_;
    long long pair_dT_for_ = -1;          // pair list the derivatives belong to
    int adj_frame_ = 0, pair_dT_frame_ = -1;
};

}  // namespace mpm
