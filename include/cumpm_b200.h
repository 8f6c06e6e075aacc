/*
 * cumpm_b200.h -- C ABI of the B200-native Mutual Polarization Method solve.
 *
 * Drop-in boundary for the reference cuMPM (TannerWilcoxson/cuMPM) hot path:
 * the self-consistent dipole/quadrupole solve behind cuMPM.dipole_solver and
 * cuMPM.Near_Field.  Every entry point returns an int status (MPM_OK on
 * success); mpm_last_error() gives the message of the last failure on the
 * calling thread.  Complex arrays are interleaved (re, im) doubles, i.e. the
 * memory layout of C99 double _Complex / std::complex<double> /
 * numpy.complex128.  No entry point terminates the process.
 *
 * Reference interfaces replaced (file:line in the reference project):
 *   mpm_solver_*  -> Dipole_Solver (src/cpp/dipole_solver.h:14-166,
 *                    bound in src/cpp/dipole_solver_bindings.cpp:80-178)
 *   mpm_near_*    -> Near_Field (src/cpp/near_field.h:12-58,
 *                    bound in src/cpp/near_field_bindings.cpp:8-25)
 *   mpm_field_*   -> Electric_Field / Monodisperse_Ewald_Electric_Field /
 *                    Direct_Electric_Field (src/cpp/electric_field/
 *                    electric_field.h:13-141, calculate() at
 *                    monodisperse_ewald_electric_field.cu:2485-2503 and
 *                    direct_electric_field.cu:555-559), here batched over M
 *                    right-hand sides on caller-owned device buffers
 *   mpm_batch_solve -> Numerical_Solver::solve (src/cpp/numerical_solver/
 *                    numerical_solver.h:34-40; GMRES gmres_solver.cu:56-208,
 *                    BiCGSTAB bicgstab_solver.cu:58-192), batched
 */
#ifndef CUMPM_B200_H
#define CUMPM_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MPM_API __attribute__((visibility("default")))
#else
#define MPM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define MPM_OK 0
#define MPM_ERR_INVALID 1   /* bad argument (maps to Python ValueError) */
#define MPM_ERR_RUNTIME 2   /* runtime/configuration error (RuntimeError) */
#define MPM_ERR_CUDA 3      /* CUDA / cuFFT failure */

/* precision (reference PrecisionMode, electric_field/direct_electric_field.h:10-16) */
#define MPM_PREC_AUTO 0     /* fp32 reciprocal space / fp32 direct sum */
#define MPM_PREC_MIXED 1
#define MPM_PREC_DOUBLE 2

/* field kinds and modes (reference FieldCalcMode, electric_field.h:8-11) */
#define MPM_FIELD_DIRECT 0
#define MPM_FIELD_MONO 1
#define MPM_FIELD_POLY 2    /* polydisperse Ewald, dipoles (radius per particle required) */
#define MPM_MODE_SOLVER_AX 0
#define MPM_MODE_INTERACTION 1

#define MPM_METHOD_GMRES 0
#define MPM_METHOD_BICGSTAB 1

typedef struct mpm_solver mpm_solver;
typedef struct mpm_near mpm_near;
typedef struct mpm_field mpm_field;

typedef struct mpm_solve_options {
    int method;        /* MPM_METHOD_* */
    int restart;       /* GMRES restart length (reference: 50) */
    int maxiter;       /* per right-hand side (reference: 1000) */
    double tol;        /* stop when |D^-1(b - A x)| < tol |b| (inner rule) */
    int jacobi;        /* diagonal (self-coefficient) preconditioning */
    int recip_fp32;    /* fp32 reciprocal space */
    int real_fp32;     /* fp32 real-space pair sum */
    int refine;        /* fp64 true-residual iterative refinement around fp32 solves */
    double inner_tol;  /* smallest relative reduction asked of one inner solve (0: 1e-4); a column's
                          inner solve also stops once its residual is below 0.5 tol |b| */
    int compact;       /* only still-iterating columns go through the operator (gathered batch) */
    int shifted;       /* refinement with GMRES: when the columns are one material's frequency sweep
                          (self coefficients one particle profile times a scalar, repeated right-hand
                          sides), solve the first correction on one Krylov space per distinct
                          right-hand side (shifted systems, from x = 0) */
} mpm_solve_options;

typedef struct mpm_solve_report {
    int matvecs;           /* batched operator applications */
    int refine_steps;
    int total_iterations;  /* sum over right-hand sides */
    int max_iterations;
    int num_converged;
    double max_rel_resid;  /* true fp64 |b-Ax|/|b| (refinement mode), else -1 */
    long long column_matvecs; /* right-hand-side columns that went through the operator */
    int reorth_steps;      /* GMRES steps that took a second projection pass */
    int shift_seeds;       /* seed columns of the shifted first correction (0: not used) */
    int fp64_matvecs;      /* fp64 true-residual matvecs of the refinement */
} mpm_solve_report;

typedef struct mpm_field_info {
    int kind, mode;
    int num_particles, num_targets, num_quads;
    int grid[3];
    int stencil;           /* Gaussian support per axis */
    int pruned;            /* 1: occupied-plane (slab) reciprocal transform */
    int z_slots;           /* stored z planes */
    long long num_pairs;   /* real-space (target, source) pairs */
    double rc, h[3], eta[3], selfo;
    int slab_fused;        /* 1: pruned layout whose y transforms and k-space step run as one fused pass */
    int single_layer;      /* 1: every particle has the same z stencil; the grid keeps one z slot */
} mpm_field_info;

MPM_API const char* mpm_last_error(void);
MPM_API const char* mpm_version(void);

/* ---- Dipole_Solver ------------------------------------------------------
 * eps: n_freq x eps_cols complex (eps_cols == 1 or number of particles).
 * radius: n_radius values (0 => 1.0 for every particle, 1 => shared).
 * E0: n_E0 vectors, vector k has E0_sizes[k] complex entries (3, 3N or
 *     3N+5Nq); n_E0 == 0 => three unit polarisations.
 * quad_idxs: n_quad_idxs particle indices (0 with solve_quads => all). */
MPM_API int mpm_solver_create(mpm_solver** out, const double box[3], const double* eps, int n_freq, int eps_cols,
                      const double* radius, int n_radius, double eps_m, double xi, double tol, int quiet,
                      const char* guess_type, const char* solver_type, const char* field_type, const double* E0,
                      const int* E0_sizes, int n_E0, int solve_quads, const int* quad_idxs, int n_quad_idxs,
                      int precision);
MPM_API void mpm_solver_destroy(mpm_solver* s);
/* one frame (reference Dipole_Solver::compute, dipole_solver.cu:495) */
MPM_API int mpm_solver_compute(mpm_solver* s, const double* x, const double* y, const double* z, int n);
/* dims: frames, wavevectors, particles, polarizations, quads */
MPM_API int mpm_solver_dims(const mpm_solver* s, int64_t dims[5]);
/* outputs sized frames*W*N*K*3, frames*W*Nq*K*5 and W*K*3 complex */
MPM_API int mpm_solver_get_dipoles(const mpm_solver* s, int physical, double* out, size_t n_complex);
MPM_API int mpm_solver_get_quadrupoles(const mpm_solver* s, int physical, double* out, size_t n_complex);
MPM_API int mpm_solver_get_eff_polarizability(const mpm_solver* s, int physical, double* out, size_t n_complex);
MPM_API int mpm_solver_set_jacobi(mpm_solver* s, int enable);
MPM_API int mpm_solver_get_jacobi(const mpm_solver* s, int* enable);
/* extras beyond the reference: restart, maxiter, all-frequency batching,
 * mixed-precision refinement */
MPM_API int mpm_solver_set_options(mpm_solver* s, int restart, int maxiter, int batch_all, int refine, double inner_tol,
                           int real_fp32);
/* iterations of every right-hand side solved so far, in solve order */
MPM_API int mpm_solver_iterations(const mpm_solver* s, int* out, size_t cap, size_t* n_out);

/* ---- Near_Field --------------------------------------------------------- */
MPM_API int mpm_near_create(mpm_near** out, const double box[3], const double E0[6], const double* radius, int n_radius,
                    double xi, double errortol, const char* field_type);
MPM_API void mpm_near_destroy(mpm_near* nf);
MPM_API int mpm_near_set_dipoles(mpm_near* nf, const double* dip, int n_complex);
MPM_API int mpm_near_set_dipole_positions(mpm_near* nf, const double* x, const double* y, const double* z, int n);
MPM_API int mpm_near_set_field_points(mpm_near* nf, const double* x, const double* y, const double* z, int n);
MPM_API int mpm_near_calculate(mpm_near* nf, double* intensity, int n);

/* ---- field operator on device buffers ----------------------------------
 * X, Y: device complex128 [rows][M], rows = 3*N (+ 5*Nq).  self_coef:
 * device complex128 [N][M] or NULL.  stream: cudaStream_t or NULL. */
MPM_API int mpm_field_create(mpm_field** out, int kind, int mode, const double box[3], double errortol, double xi,
                     const double* radius, int n_radius, int solve_quads, const int* quad_idxs, int n_quad_idxs);
MPM_API void mpm_field_destroy(mpm_field* f);
MPM_API int mpm_field_set_positions(mpm_field* f, const double* x, const double* y, const double* z, int n, void* stream);
MPM_API int mpm_field_set_field_points(mpm_field* f, const double* x, const double* y, const double* z, int n,
                               void* stream);
MPM_API int mpm_field_apply(mpm_field* f, const void* X, void* Y, int M, const void* self_coef, int jacobi, int recip_fp32,
                    int real_fp32, void* stream);
/* part 0: reciprocal space only; part 1: real space + self only */
MPM_API int mpm_field_apply_part(mpm_field* f, const void* X, void* Y, int M, const void* self_coef, int recip_fp32,
                         int real_fp32, int part, void* stream);
MPM_API int mpm_field_info_get(const mpm_field* f, mpm_field_info* info);
/* Bloch wavevector (kx, ky), non-dimensional, of the periodic images for
 * the EELS Brillouin-zone sum (the reference's Ewald base sets it,
 * ewald_electric_field_base.h:132-138): the k-space Green tensor at k - b
 * with the window deconvolution at k (monodisperse_ewald_electric_field.cu:
 * 1329-1331; the polydisperse scale likewise), and a phase
 * exp(-i (kx r_x + ky r_y)) on every real-space pair, r = source - target
 * (:1749-1756).  Ewald fields with dipoles only; (0, 0) restores the plain
 * operator.  Takes effect at the next apply. */
MPM_API int mpm_field_set_bloch(mpm_field* f, double kx, double ky);

/* Same result as mpm_field_apply, but this call allocates nothing.  No
 * counterpart in the reference.  For callers that cannot allocate device
 * memory while they solve (device memory handed to another allocator, or a
 * loop that must not enter the driver's allocator): the reciprocal-space
 * grid lives in a static 16 MiB device array of this library (held by every
 * GPU that loads it, until exit) instead of a cudaMalloc'd buffer.  The
 * field's per-frame data must already exist (mpm_field_set_positions is the
 * allocating set-up step).  The first call on a device looks up the array's
 * device address with that device current; make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race.
 * Returns MPM_ERR_INVALID if the grid for M right-hand sides exceeds
 * mpm_noalloc_scratch_bytes(). */
MPM_API int mpm_field_apply_noalloc(mpm_field* f, const void* X, void* Y, int M, const void* self_coef, int jacobi,
                                    int recip_fp32, int real_fp32, void* stream);
MPM_API size_t mpm_noalloc_scratch_bytes(void);

/* ---- field autotuner ---------------------------------------------------
 * No counterpart in the reference, which fixes these by rule from xi and the
 * tolerance (grid N = ceil(1 + L kcut / pi): monodisperse_ewald_electric_
 * field.cu:546-616, polydisperse_ewald_electric_field.cu:2039-2112; spread
 * tile 8 x 8).  A tuning overrides them; zeros keep the rule. */
typedef struct mpm_field_tuning {
    double xi;             /* Ewald splitting parameter (non-dimensional) */
    int grid[3];           /* grid points per axis, 0: the rule */
    int support;           /* Gaussian support P, 0: the rule */
    int tile[2];           /* spread tile in x and y (monodisperse), 0: 8 */
} mpm_field_tuning;

typedef struct mpm_tune_report {
    double apply_ms;       /* M-column apply of the pick (caller's arithmetic) */
    double apply_ms_rule;  /* the same for the rule configuration */
    double error;          /* relative operator error of the pick against a field of tolerance errortol/1000 */
    double error_rule;     /* the same for the rule configuration */
    double error_bound;    /* acceptance bound: max(errortol, error_rule) */
    int candidates, accepted;
} mpm_tune_report;

/* mpm_field_create with the tuning's xi and overrides */
MPM_API int mpm_field_create_tuned(mpm_field** out, int kind, int mode, const double box[3], double errortol,
                                   const mpm_field_tuning* tuning, const double* radius, int n_radius,
                                   int solve_quads, const int* quad_idxs, int n_quad_idxs);
/* Measures candidate (xi, grid, support, tile) settings of a SOLVER_AX
 * field on the device for the n positions (non-dimensional host arrays) and
 * a batch of M columns in the given arithmetic, and writes the fastest one
 * whose operator error stays within max(errortol, the rule's own error).  Direct fields: the rule (nothing to tune). */
MPM_API int mpm_field_autotune(int kind, const double box[3], double errortol, double xi, const double* radius,
                               int n_radius, int solve_quads, const int* quad_idxs, int n_quad_idxs, const double* x,
                               const double* y, const double* z, int n, int M, int recip_fp32, int real_fp32,
                               mpm_field_tuning* out, mpm_tune_report* report, void* stream);
/* Host only: the xi candidates of the tuner's first stage (xi times fixed
 * factors, those whose rule geometry is valid), with their rule grid,
 * support and cutoff; n_out = count (at most cap written). */
MPM_API int mpm_tune_xi_candidates(int kind, const double box[3], double errortol, double xi, const double* radius,
                                   int n_radius, double* xi_out, int* grid_out, int* support_out, double* rc_out,
                                   int cap, int* n_out);
/* Host only: smallest length >= n with prime factors in {2, 3, 5, 7}
 * (smooth23 = 0) or {2, 3} (smooth23 = 1). */
MPM_API int mpm_tune_next_size(int n, int smooth23);
/* Dipole solver: use this tuning for its field (before the first compute),
 * or tune it on the given positions (physical units, as compute takes them)
 * for the solver's batch width and arithmetic and keep the pick. */
MPM_API int mpm_solver_set_tuning(mpm_solver* s, const mpm_field_tuning* tuning);
MPM_API int mpm_solver_autotune(mpm_solver* s, const double* x, const double* y, const double* z, int n,
                                mpm_field_tuning* out, mpm_tune_report* report);

/* batched Krylov solve A X = B on device buffers (X holds the guess) */
MPM_API int mpm_batch_solve(mpm_field* f, const void* B, void* X, int M, const void* self_coef,
                    const mpm_solve_options* opt, mpm_solve_report* report, void* stream);

/* Gradient of the bilinear forms lam_m^T G p_m, summed over the M columns
 * (G = the field operator in SOLVER_AX mode without the caller's self
 * coefficients; polydisperse or direct field, dipoles): gx device
 * complex128 [N][3] = d/dx, ga device complex128 [N] = d/d(radius).  The
 * adjoint of a solve A p = b with A = G + diag(s) is complex-symmetric, so
 * with lam solving A lam = conj(c), dIm(c^H p)/dtheta = -Im(lam^T dA/dtheta p).
 * No counterpart in the reference (it has no gradients). */
MPM_API int mpm_field_grad(mpm_field* f, const void* lam, const void* p, int M, void* gx, void* ga, void* stream);

/* Batched 1-D DFT of the spectral-Ewald grids, the in-house replacement of
 * the reference's cuFFT plans (e.g. the cufftExecC2C / cufftExecZ2Z calls of
 * src/cpp/electric_field/polydisperse_ewald_electric_field.cu:2577-2627),
 * exposed for testing: line o, column c, element e at data[o*os + e*es + c] (complex64 or complex128, device memory), c < ncols.
 * mode 0 forward, 1 inverse (both unnormalised), 2 forward, multiplication of
 * element e of line o, column c by scale[(e*nouter + o)*sz + c/sb], inverse.
 * general != 0 forces the multi-pass kernel; split (optional, 2 ints)
 * receives the two-pass factorisation n = r1 * r2 that ran (r2 above 16 is
 * a prime handled by the streamed pass) or (0, 0) for the multi-pass kernel.  Synchronises
 * the stream before returning. */
MPM_API int mpm_line_fft(void* data, int fp64, int n, size_t es, int ncols, size_t os, int nouter, int mode,
                         const void* scale, int sz, int sb, int general, int* split, void* stream);

/* ---- measurement (no counterpart in the reference) -----------------------
 * Stage timers from CUDA events recorded on the launching stream, read
 * without adding synchronisation to the solve.  Stages: 0 spread, 1 forward
 * FFT, 2 k-space Green tensor, 3 inverse FFT, 4 contraction, 5 real space,
 * 6 direct sum, 7 Krylov vector work, 8 per-frame precalculation. */
MPM_API int mpm_profile_enable(int on);
MPM_API int mpm_profile_reset(void);
MPM_API int mpm_profile_read(double* ms, long long* count, int n);
/* kernel launches issued by this library since the last reset */
MPM_API long long mpm_kernel_launches(void);

/* ---- host-only helpers (no GPU needed) ---------------------------------- */
/* real-space tables: out has 10 x 9001 doubles (r, fd1, fd2, fq1, fq2, fq3,
 * gq1, gq2, gq3, gq4); selfo/self_grad may be NULL */
MPM_API int mpm_mono_tables(double xi, double* out, double* selfo, double* self_grad);
/* Ewald parameters for a box: grid[3], stencil, rc, h[3], eta[3] */
MPM_API int mpm_ewald_geometry(const double box[3], double errortol, double xi, int grid[3], int* stencil, double* rc,
                       double h[3], double eta[3]);
/* Polydisperse parameters (polydisperse_ewald_electric_field.cu:39-84,
 * 2039-2112): grid[3], support P, eta, rc, number of radius classes and the
 * class of each of the n radii (cls may be NULL). */
MPM_API int mpm_poly_geometry(const double box[3], double errortol, double xi, const double* radii, int n, int grid[3],
                              int* P, double* eta, double* rc, int* n_classes, int* cls);
/* Polydisperse real-space pair functions of radii a <= b at the n distances
 * r > 0 (helper_compute_pair_tables, polydisperse_ewald_electric_field.cu:
 * 1434-1627): fd1 (perpendicular), fd2 (parallel) and the r = 0 self value;
 * and, when lookup != 0, the reference's linear table lookup at r instead
 * (:170-187, table nodes 0, 1, 1.001, ... for cutoff rc). */
MPM_API int mpm_poly_pair_functions(double a, double b, double xi, double rc, int lookup, const double* r, int n,
                                    double* fd1, double* fd2, double* self_value);
/* Radius-1 quadrupole tables of the polydisperse field for cutoff rc
 * (computeRealSpaceTables, polydisperse_ewald_electric_field.cu:1690-2035):
 * n_nodes = ceil((max(rc, 1.001) - 1) / 0.001) + 1 nodes (0, 1, 1.001, ...);
 * out (cap doubles, at least 8 x n_nodes) gets r, fq1, fq2, fq3, gq1, gq2,
 * gq3, gq4, one row of n_nodes each.  out may be NULL to query n_nodes. */
MPM_API int mpm_poly_quad_tables(double xi, double rc, double* out, size_t cap, int* n_nodes);
/* Quadrupole self value of each of the n radii (:1690-1706). */
MPM_API int mpm_poly_quad_self(double xi, const double* radii, int n, double* out);

#ifdef __cplusplus
}
#endif

#endif /* CUMPM_B200_H */
