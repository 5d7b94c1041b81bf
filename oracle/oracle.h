/*
 * oracle.h -- CPU restatement of the HAMLSS solve path, used ONLY as a checker.
 *
 * Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load this code, and only to check or time against the device engine.  Nothing in
 * the engine (hybrid-sparse-pde-solver_b200/) links, calls or falls back to it.
 *
 * Every routine restates one function of the reference project (saumadeepsardar/
 * Hybrid-Sparse-PDE-Solver) and cites it as file:line.  Reductions run sequentially in
 * index order, which equals the reference's OpenMP reductions at OMP_NUM_THREADS=1.
 * The restatement is pinned against the reference itself (built from its sources by
 * oracle/Makefile into oracle/_ref/) by tests/test_oracle_pin.py, and against the
 * committed fixtures in tests/golden/.
 */
#ifndef HAMLSS_ORACLE_H
#define HAMLSS_ORACLE_H
#include <stdint.h>
#include "../include/hamlss.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- generators (sparse_matrix.cpp:288-350); arrays sized rows+1 / 5*rows ---- */
int64_t orc_poisson_2d(int32_t n, int32_t* rp, int32_t* ci, double* v);
int64_t orc_convdiff_2d(int32_t n, double eps, double bx, double by,
                        int32_t* rp, int32_t* ci, double* v);

/* ---- kernels ---- */
void   orc_spmv(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                const double* x, double* y);
double orc_dot(int32_t n, const double* a, const double* b);

/* ---- Jacobi (jacobi.cpp:13-51) ---- */
int  orc_jacobi_setup(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                      double omega, double* inv_diag);

/* ---- ILU(0) (ilu.cpp:41-89, :225-271) ---- */
int  orc_ilu0_factor(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                     double* lu);
int  orc_ilut_factor(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                     double drop_tol, int32_t fill_p, int32_t* out_rp, int32_t* out_ci,
                     double* out_lu, int64_t* nnz_out);
int  orc_ilu_apply(int32_t n, const int32_t* rp, const int32_t* ci, const double* lu,
                   const double* r, double* z);
/* level(i) = 1 + max level(j) over the strictly lower (which=0) or strictly upper
 * (which=1) columns j of row i; rows with none are level 0.  Returns the count. */
int32_t orc_levels(int32_t n, const int32_t* rp, const int32_t* ci, int which, int32_t* level);

/* ---- SA-AMG (amg.cpp) ---- */
int32_t orc_amg_aggregate(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                          double theta, int32_t* agg);
typedef struct orc_amg orc_amg;
orc_amg* orc_amg_setup(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                       const hamlss_params* p);
void     orc_amg_free(orc_amg* h);
int32_t  orc_amg_num_levels(const orc_amg* h);
/* which: 0 A, 1 P, 2 R.  Arrays may be NULL to query sizes. */
int      orc_amg_level(const orc_amg* h, int32_t level, int32_t which, int32_t* rows,
                       int32_t* cols, int32_t* nnz, int32_t* rp, int32_t* ci, double* v);
void     orc_amg_apply(const orc_amg* h, const double* r, double* z);

/* ---- generic preconditioner + solvers ---- */
typedef struct orc_prec orc_prec;
/* kind = HAMLSS_PREC_*; returns NULL for NONE and on error (*status set). */
orc_prec* orc_prec_setup(int kind, int32_t n, const int32_t* rp, const int32_t* ci,
                         const double* v, const hamlss_params* p, int* status);
void      orc_prec_free(orc_prec* M);
int       orc_prec_apply(const orc_prec* M, const double* r, double* z);

/* CGSolver::solve (cg_solver.cpp:37-191) and FGMRESSolver::solve (fgmres_solver.cpp:165-241).
 * Return value = converged (0/1), or a negative HAMLSS_ERR_* on failure. */
int orc_cg(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
           const orc_prec* M, const double* b, double* x, const hamlss_params* p,
           hamlss_stats* st);
int orc_fgmres(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
               const orc_prec* M, const double* b, double* x, const hamlss_params* p,
               hamlss_stats* st);
int  orc_pipelined_fgmres(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                          const orc_prec* M, const double* b, double* x,
                          const hamlss_params* p, hamlss_stats* st);
int  orc_sstep_cg(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                  const orc_prec* M, const double* b, double* x, const hamlss_params* p,
                  hamlss_stats* st);
void orc_spectral_interval(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                           int steps, double* lo, double* hi);

/* ---- adaptive selector (adaptive_selector.cpp:37-394) ---- */
int orc_extract_features(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                         double feat[24], int32_t* initial_state);
int orc_solve_adaptive(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                       const double* b, double* x, const hamlss_params* p, hamlss_stats* st,
                       hamlss_escalation* log, int32_t log_cap, int32_t* n_log,
                       int32_t* initial_state);

#ifdef __cplusplus
}
#endif
#endif
