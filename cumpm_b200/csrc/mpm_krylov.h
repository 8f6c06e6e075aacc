// Batched device-resident Krylov solvers for A(omega) p = E0.
//
// Semantics per right-hand side follow the reference solvers:
//   GMRES    numerical_solver/gmres_solver.cu:56-208 (left Jacobi
//            preconditioning, restart 50, maxiter 1000, complex Givens,
//            stop when |D^-1 (b - A x)| < tol |b|)
//   BiCGSTAB numerical_solver/bicgstab_solver.cu:58-192 (unconjugated rho
//            dots, conjugated omega, same stop rule)
// but all M right-hand sides advance together: one batched matvec per step,
// all reductions on the device, the Hessenberg/Givens state per RHS on the
// device, and one small device->host flag read per step.  Arnoldi uses
// classical Gram-Schmidt with one re-orthogonalisation pass (CGS2), which
// spans the same Krylov space as the reference's modified Gram-Schmidt.
#pragma once

#include <vector>

#include "mpm_field.h"

namespace mpm {

enum SolverMethod { SOLVER_GMRES = 0, SOLVER_BICGSTAB = 1 };

struct SolveOptions {
    int method = SOLVER_GMRES;
    int restart = 50;
    int maxiter = 1000;
    double tol = 1e-3;
    bool jacobi = true;
    bool recip_fp32 = true;   // reference AUTO precision
    bool real_fp32 = false;
    // Mixed-precision refinement: inner solves with the fp32 operator, outer
    // true-residual check |b - A x| <= tol |b| with the fp64 operator.
    // The inner solve of column m stops once its residual is below half the
    // outer target, 0.5 tol |b_m|, or once it has reduced its own residual
    // by inner_tol, whichever comes first (inner_tol <= 0 means 1e-4): the
    // fp32 operator's rounding keeps one inner solve from reaching much
    // below that, and later rounds then stop as soon as the target is met.
    bool refine = false;
    double inner_tol = 1e-4;
    int max_refine = 20;
    // Only the columns still iterating go through the field operator
    // (gathered into a compact batch); converged columns cost nothing.
    bool compact = true;
    // Refinement with GMRES: when every column's self coefficients are one
    // particle profile times a scalar and right-hand sides repeat (a
    // frequency sweep of one material), solve the first correction of all
    // columns from x = 0 on one Krylov space per distinct right-hand side
    // (shifted systems).  The initial guess is then not used.
    bool shifted = true;
};

struct SolveStats {
    std::vector<int> iters;          // Krylov steps per RHS (all cycles)
    std::vector<int> converged;      // 1 if the stop rule was met
    std::vector<double> rel_resid;   // true |b - A x| / |b| (fp64 operator) when computed
    int matvecs = 0;                 // batched operator applications
    long long column_matvecs = 0;    // columns that went through the operator
    int refine_steps = 0;
    int reorth_steps = 0;            // GMRES steps that needed a second projection pass
    int shift_seeds = 0;             // seed columns of the shifted first correction (0: not used)
    int fp64_matvecs = 0;            // true-residual (fp64 operator) matvecs of the refinement
};

class BatchSolver {
public:
    BatchSolver();
    ~BatchSolver();
    BatchSolver(const BatchSolver&) = delete;
    BatchSolver& operator=(const BatchSolver&) = delete;
    // b, x: device [rows][M] (x holds the initial guess on entry).
    // sc: device [N][M] self coefficients.
    void solve(Field& F, const double2* b, double2* x, int M, const double2* sc, const SolveOptions& opt,
               SolveStats& st, cudaStream_t s);
    // true residual |b - A x| / |b| per RHS with the fp64 operator
    void true_residual(Field& F, const double2* b, const double2* x, int M, const double2* sc,
                       std::vector<double>& out, cudaStream_t s);

private:
    // x_zero: x is known to be zero on entry (skips the first matvec).
    // tolv: optional device per-column tolerance replacing opt.tol.
    // precond_rel: stop on |D^-1 r| < tol |D^-1 b| (a relative reduction of
    // the preconditioned residual, used by the inner solves of the
    // refinement) instead of the reference rule |D^-1 r| < tol |b|.
    void gmres(Field& F, const double2* b, double2* x, int M, const double2* sc, const SolveOptions& opt,
               SolveStats& st, bool recip32, bool real32, cudaStream_t s, bool x_zero = false,
               const double* tolv = nullptr, bool precond_rel = false);
    // Y = op(X) for the columns whose host flag is set (all when cols_ is
    // empty): gathers them into a compact batch when some are idle.
    // Returns the number of columns applied.
    int apply_cols(Field& F, const double2* X, double2* Y, int M, const double2* sc, bool jacobi, bool r32,
                   bool re32, const int* active, bool compact, cudaStream_t s);
    void bicgstab(Field& F, const double2* b, double2* x, int M, const double2* sc, const SolveOptions& opt,
                  SolveStats& st, bool recip32, bool real32, cudaStream_t s, bool x_zero = false,
                  const double* tolv = nullptr, bool precond_rel = false);
    // grp[m]: the seed (distinct right-hand side) of column m; f[m]: its
    // self-coefficient scale, sc[:, m] = f[m] sc[:, 0].  False when the
    // columns have no such structure or no repeated right-hand side.
    bool detect_shifts(const double2* b, const double2* sc, int rows, int N, int M, cudaStream_t s,
                       std::vector<int>& grp, std::vector<double2>& f);
    // x (the M columns but those with skip[m] set, device, may be null) from
    // x0 = 0 by GMRES on the seeds' Krylov spaces; stops each column at
    // |D^-1 r| < tolv[m] |D^-1 b|.  live (host, may be null) = !skip: seeds
    // with no live member are not iterated.
    void gmres_shifted(Field& F, const double2* b, double2* x, int M, const double2* sc, const SolveOptions& opt,
                       SolveStats& st, bool recip32, bool real32, cudaStream_t s, const double* tolv,
                       const std::vector<int>& grp, const std::vector<double2>& f, const int* skip,
                       const int* live);
    void dots(const double2* V, size_t vstride, int nvec, const double2* w, int rows, int M, int conj,
              double2* out, cudaStream_t s, int shift = -1);
    void norms(const double2* w, int rows, int M, double* out, cudaStream_t s);

    // reads the count and the nflags words that follow it into flag_
    int read_flags(const int* dflag, int nflags, cudaStream_t s);

    DevBuf V_, H_, g_, cs_, sn_, y_, h_, h2_, partial_, bnorm_, rnorm_, state_, w_, r_, bj_;
    DevBuf r0_, p_, v_, s_, t_, scal_, d_, rr_, xr_, flagdev_, tolv_;
    DevBuf cidx_, xc_, yc_, scc_;        // compact-batch gather buffers
    DevBuf bn2_, rn2_, convd_;           // refinement: |b|, true |r|, converged flags
    DevBuf sel_, rn64_;                  // refinement: columns re-checked in fp64, their |r|
    DevBuf dots_done_;                   // finished-CTA counters of the fused small dot kernel
    DevBuf shf_, shflag_, shmeta_, shsc_, shb_, shst_, hm_;   // shifted solve: detection, seeds, members
    int* flag_ = nullptr;                // pinned host words: count + per-column flags
    int flag_cap_ = 0;
    int* hidx_ = nullptr;                // pinned host column list for the gather
    int hidx_cap_ = 0;
    std::vector<int> cur_cols_;          // column list the device buffers hold
    const double2* cur_sc_ = nullptr;    // self coefficients gathered into scc_
};

}  // namespace mpm
