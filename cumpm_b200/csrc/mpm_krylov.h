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
    bool refine = false;
    double inner_tol = 1e-4;
    int max_refine = 20;
};

struct SolveStats {
    std::vector<int> iters;          // Krylov steps per RHS (all cycles)
    std::vector<int> converged;      // 1 if the stop rule was met
    std::vector<double> rel_resid;   // true |b - A x| / |b| (fp64 operator) when computed
    int matvecs = 0;                 // batched operator applications
    int refine_steps = 0;
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
    void gmres(Field& F, const double2* b, double2* x, int M, const double2* sc, const SolveOptions& opt,
               SolveStats& st, bool recip32, bool real32, cudaStream_t s);
    void bicgstab(Field& F, const double2* b, double2* x, int M, const double2* sc, const SolveOptions& opt,
                  SolveStats& st, bool recip32, bool real32, cudaStream_t s);
    void dots(const double2* V, size_t vstride, int nvec, const double2* w, int rows, int M, int conj,
              double2* out, cudaStream_t s);
    void norms(const double2* w, int rows, int M, double* out, cudaStream_t s);

    int read_flag(const int* dflag, cudaStream_t s);

    DevBuf V_, H_, g_, cs_, sn_, y_, h_, h2_, partial_, bnorm_, rnorm_, state_, w_, r_, bj_;
    DevBuf r0_, p_, v_, s_, t_, scal_, d_, rr_, xr_, flagdev_;
    int* flag_ = nullptr;  // pinned host word
};

}  // namespace mpm
