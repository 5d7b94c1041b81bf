// krylov.cuh -- device PCG and FGMRES(m) drivers.
#pragma once

#include "ladder.cuh"
#include "precond.cuh"

namespace hamlss {

// Solve status codes kept in device state (polled by the host).
enum : int { ST_RUN = 0, ST_CONV = 1, ST_MAXIT = 2, ST_RESTART = 3, ST_NONFINITE = 4,
             ST_ESCALATE = 5 };

struct SolveResult {
    int iterations = 0;
    int restarts = 0;
    int converged = 0;
    int status = HAMLSS_OK;
    double initial_residual = 0.0;
    double final_residual = 0.0;
    double device_time_s = 0.0;
    int escalate = 0;         // ESC_* when the device-side ladder test stopped the solve
    // set by solvers whose cost model is not the CG / FGMRES one (else left at -1)
    long long flops = -1, bytes = -1;
    int sstep_k = 0;          // s-step batch size (SStepCGSolver)
    long long comm_events = 0;
};

// CGSolver::solve (cg_solver.cpp:37-191) on device vectors.  T = double runs the FP64
// path; T = float is the FP32 inner solve of the mixed-precision scheme.  b, x have n
// entries of type T on the device.  `jac` (may be null) selects the fused Jacobi kernels.
template <typename T>
SolveResult cg_solve(Ctx& ctx, hamlss_mat* A, Prec* M, const T* b, T* x, double tol,
                     int max_iter, int check_every, Workspace& ws, const LadderCfg* lad = nullptr);

// FGMRESSolver::solve (fgmres_solver.cpp:165-241) with CGS2 Arnoldi; FP64.
// pipelined = true: PipelinedFGMRESSolver (pipelined_fgmres_solver.cpp:69-242), the same
// Arnoldi process with that solver's lucky-breakdown exit and cost model.
SolveResult fgmres_solve(Ctx& ctx, hamlss_mat* A, Prec* M, const double* b, double* x,
                         double tol, int max_iter, int restart, Workspace& ws,
                         const LadderCfg* lad = nullptr, bool pipelined = false);

// SStepCGSolver::solve (sstep_cg_solver.cpp:170-305): batches of k Newton-Chebyshev basis
// vectors, one Gram matrix per batch, a k x k Cholesky solve, x += B y, and the true
// residual.  k = params.sstep_k; the preconditioner is not applied (as in the reference).
SolveResult sstep_solve(Ctx& ctx, hamlss_mat* A, const double* b, double* x,
                        const hamlss_params& p, Workspace& ws);

// SparseMatrix::spectral_interval(steps) (sparse_matrix.cpp:451-479): Lanczos from the
// uniform vector, Gershgorin bounds of the tridiagonal.
void spectral_interval(Ctx& ctx, hamlss_mat* A, int steps, double* lo, double* hi);

// Mixed-precision PCG with reliable updates: FP32 iteration (values, vectors, M^-1),
// FP64 dot products and scalars, the residual replaced by the true FP64 one whenever the
// recursive one fell by `delta` since the last replacement and to confirm the stop test.
// x (FP64, device) is the initial guess and the result; *n_updates counts the updates.
SolveResult cg_reliable_solve(Ctx& ctx, hamlss_mat* A, Prec* M, const double* b, double* x, double tol,
                              int max_iter, int check_every, double delta, Workspace& ws,
                              const LadderCfg* lad, int* n_updates);

// Mixed precision: FP64 iterative refinement around an FP32 inner PCG / FGMRES.
SolveResult mixed_solve(Ctx& ctx, int solver, hamlss_mat* A, Prec* M, const double* b,
                        double* x, const hamlss_params& p, Workspace& ws, int* outer_iters,
                        const LadderCfg* lad = nullptr);

// ||b - A x|| / ||b|| in FP64 on the device (SolverBase::relative_residual,
// solver_base.cpp:9-17).
double true_relative_residual(Ctx& ctx, hamlss_mat* A, const double* b, const double* x,
                              Workspace& ws);

inline Workspace& workspace_of(hamlss_mat* A) { return A->ws; }

// AdaptiveSelector::extract_features + select_initial_state on the device.
int extract_features(Ctx& ctx, hamlss_mat* A, double feat[24], int* initial_state);

}  // namespace hamlss
