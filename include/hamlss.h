/*
 * hamlss.h -- C ABI of the B200 sparse iterative solve engine.
 *
 * This is the drop-in boundary for the HAMLSS solve path (namespace `hsps` in the
 * reference C++17 code).  The reference has no FFI of its own: its path sits behind
 * plain C++ virtual classes.  Each entry point below replaces one of those calls and
 * cites it as `file:line` inside the reference project:
 *
 *   SparseMatrix / Vector        include/core/sparse_matrix.hpp:34-170, include/core/vector.hpp:16-69
 *   SolverBase::solve            include/solvers/solver_base.hpp:32-35
 *   PreconditionerBase           include/preconditioners/preconditioner_base.hpp:16-48
 *   SolverFactory                include/solvers/solver_factory.hpp:40-88
 *   AdaptiveSelector             include/adaptive/adaptive_selector.hpp:49-161
 *
 * Conventions
 *   - Every function returns an int status: HAMLSS_OK (0) or a negative error code.
 *     hamlss_last_error() returns a thread-local message for the last failure.
 *   - Non-convergence is NOT an error (as in the reference, where solve() returns
 *     false): the call returns HAMLSS_OK and stats->converged == 0.
 *   - Matrices are CSR with int32 row pointers / column indices and FP64 values,
 *     columns sorted inside each row (what SparseMatrix::from_coo produces).
 *   - Vector arguments are host pointers when `where == HAMLSS_HOST`, device
 *     pointers on the context's device when `where == HAMLSS_DEVICE`.
 *   - A context owns one CUDA stream.  Calls on one context are serialised by the
 *     caller; different contexts may be used from different threads.
 */
#ifndef HAMLSS_H
#define HAMLSS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
enum {
    HAMLSS_OK              = 0,
    HAMLSS_ERR_INVALID     = -1,  /* bad argument / unknown name (std::invalid_argument)        */
    HAMLSS_ERR_SIZE        = -2,  /* dimension mismatch (vector.cpp:42, sparse_matrix.cpp:69)    */
    HAMLSS_ERR_ZERO_DIAG   = -3,  /* Jacobi zero diagonal (jacobi.cpp:28-30)                     */
    HAMLSS_ERR_ZERO_PIVOT  = -4,  /* ILU near-zero pivot (ilu.cpp:65-67, ilu.cpp:257-259)        */
    HAMLSS_ERR_CUDA        = -5,  /* CUDA runtime failure                                         */
    HAMLSS_ERR_NOMEM       = -6,  /* device allocation failed                                     */
    HAMLSS_ERR_NOT_READY   = -7,  /* preconditioner used before setup                             */
    HAMLSS_ERR_TIMEOUT     = -8,  /* a bounded device-side wait ran out                           */
    HAMLSS_ERR_NONFINITE   = -9,  /* NaN / Inf in an input vector or matrix                       */
    HAMLSS_ERR_BUDGET      = -10, /* request does not fit the memory budget                       */
    HAMLSS_ERR_MALFORMED   = -11, /* CSR not well formed (row_ptr, bounds, unsorted columns)      */
    HAMLSS_ERR_CANCELLED   = -12  /* serving request cancelled before it ran                      */
};

enum { HAMLSS_HOST = 0, HAMLSS_DEVICE = 1 };

/* Same numeric values as hsps::SolverType / PrecondType / AdaptiveState
 * (include/core/types.hpp:30-54). */
enum { HAMLSS_SOLVER_CG = 0, HAMLSS_SOLVER_FGMRES = 1, HAMLSS_SOLVER_BICGSTAB = 2,
       HAMLSS_SOLVER_SSTEP_CG = 3, HAMLSS_SOLVER_ASYNC_FGMRES = 4,
       /* engine value: PipelinedFGMRESSolver (include/solvers/pipelined_fgmres_solver.hpp),
        * which has no SolverType of its own and reports FGMRES */
       HAMLSS_SOLVER_PIPELINED_FGMRES = 5 };
enum { HAMLSS_PREC_NONE = 0, HAMLSS_PREC_JACOBI = 1, HAMLSS_PREC_ILU = 2, HAMLSS_PREC_AMG = 3,
       HAMLSS_PREC_BLOCK_JACOBI = 4, HAMLSS_PREC_CHEBYSHEV = 5 };
enum { HAMLSS_STATE_EASY = 0, HAMLSS_STATE_MODERATE = 1, HAMLSS_STATE_HARD = 2 };

/* Arithmetic of the inner solve. */
enum { HAMLSS_FP64 = 0,        /* everything FP64, iteration-for-iteration like the reference      */
       HAMLSS_MIXED = 1 };     /* FP32 values/vectors inside an FP64 iterative-refinement loop      */

/* ------------------------------------------------------------------ parameters
 * Field-for-field mirror of hsps::SolverParams (include/core/types.hpp:119-143),
 * followed by engine fields that have no counterpart there.
 * hamlss_params_default() fills the reference defaults. */
typedef struct hamlss_params {
    double  tol;              /* 1e-8   relative residual tolerance              */
    int32_t max_iter;         /* 2000   Krylov iteration budget                  */
    int32_t restart_size;     /* 50     FGMRES restart length m                  */
    double  drop_tol;         /* 1e-4   ILU threshold; 0 selects ILU(0)          */
    int32_t amg_levels;       /* 10     maximum hierarchy depth                  */
    double  amg_strength;     /* 0.25                                            */
    double  amg_strong;       /* 0.25   strength threshold the factory forwards  */
    int32_t amg_smooth_pre;   /* 2                                               */
    int32_t amg_smooth_post;  /* 2                                               */
    int32_t stall_window;     /* 15                                              */
    double  stall_threshold;  /* 0.95                                            */
    int32_t verbose;          /* 0                                               */
    int32_t print_every;      /* 25                                              */
    int32_t sstep_k;          /* 1                                               */
    double  sstep_cond_tol;   /* 1e12                                            */
    int32_t async_enabled;    /* 0                                               */
    int32_t async_max_stale;  /* 3                                               */
    int32_t fill_per_row;     /* 0                                               */
    int32_t block_size;       /* 1                                               */
    int32_t record_hw_energy; /* 0  1: read the NVML energy counter around solves */
    /* ---- engine fields ---- */
    int32_t precision;        /* HAMLSS_FP64 (default) or HAMLSS_MIXED                       */
    double  ir_inner_tol;     /* relative reduction asked of each FP32 inner solve (1e-5)    */
    int32_t ir_max_outer;     /* cap on refinement steps (30)                                */
    double  amg_omega;        /* AMG Jacobi damping; reference value 0.67 (amg.hpp:101)      */
    int32_t amg_coarse_limit; /* direct solve at or below this many rows; reference 50       */
    double  jacobi_omega;     /* Jacobi preconditioner damping; reference 1.0 (jacobi.hpp:33) */
    int32_t ladder_mode;      /* 0: escalate when an attempt exhausts max_iter (reference)   */
                              /* 1: also escalate on the device-side stall / budget checks   */
                              /* 2: as 1, and end the top rung early on stall / divergence   */
                              /* 3: as 2, but the CG rung skips the windowed stall rule (its */
                              /*    residual is not monotone): divergence / budget only      */
    int32_t check_every;      /* iterations between device->host convergence polls (8)      */
    double  amg_stall_ratio;  /* 0: coarsen until amg_coarse_limit / amg_levels / no progress */
                              /* (reference); r in (0,1): also stop when n_c > r * n_f, the  */
                              /* coarsening having stalled, and solve that level densely     */
    double  ir_update;        /* mixed-precision PCG: FP32 iteration whose residual is        */
                              /* replaced by the true FP64 one when it fell by this factor   */
                              /* since the last replacement (reliable update), 1e-2; 0: FP64 */
                              /* refinement restarting an FP32 PCG (ir_inner_tol, _max_outer) */
} hamlss_params;

/* ----------------------------------------------------------------- statistics
 * Field-for-field mirror of hsps::SolverStats (include/core/types.hpp:91-114),
 * followed by engine fields. */
typedef struct hamlss_stats {
    int32_t iterations;
    double  initial_residual;
    double  final_residual;
    int32_t converged;
    double  solve_time_s;
    double  setup_time_s;
    double  energy_joules;    /* proxy model 2e-10 J/flop + 5e-9 J/byte (cg_solver.cpp:186-188) */
    int64_t flop_count;
    int64_t mem_bytes;
    int32_t solver_used;
    int32_t precond_used;
    int32_t state_used;
    int32_t restarts;
    double  energy_joules_hw; /* NVML total-energy delta around the solve (0 if unavailable) */
    double  rapl_start_j;
    double  rapl_end_j;
    int32_t sstep_k;
    int32_t async_mode;
    int64_t comm_bytes;
    double  comm_time_s;
    /* ---- engine fields ---- */
    double  true_residual;    /* ||b - A x|| / ||b|| in FP64 after the solve                 */
    int32_t outer_iterations; /* refinement steps (HAMLSS_MIXED), else 1                     */
    int32_t status;           /* 0 ok, else the HAMLSS_ERR_* that ended the solve            */
    double  device_time_s;    /* CUDA-event time of the solve on the context stream          */
} hamlss_stats;

/* Escalation log entry; mirrors hsps::EscalationRecord (adaptive_selector.hpp:38-44). */
typedef struct hamlss_escalation {
    int32_t at_iteration;
    int32_t from_state;
    int32_t to_state;
    double  residual_at_escalation;
    int32_t reason;           /* 0 attempt exhausted max_iter, 1 stall, 2 budget, 3 divergence */
} hamlss_escalation;

typedef struct hamlss_ctx  hamlss_ctx;
typedef struct hamlss_mat  hamlss_mat;
typedef struct hamlss_prec hamlss_prec;

/* ------------------------------------------------------------------- library */
const char* hamlss_version(void);
const char* hamlss_last_error(void);
void        hamlss_params_default(hamlss_params* p);

/* ------------------------------------------------------------------- context */
int hamlss_ctx_create(int device, hamlss_ctx** out);
int hamlss_ctx_destroy(hamlss_ctx* ctx);
int hamlss_ctx_synchronize(hamlss_ctx* ctx);
/* The context's cudaStream_t, as an opaque pointer, so callers can order their own work. */
int hamlss_ctx_stream(hamlss_ctx* ctx, void** stream);

/* Measurement support (no counterpart in the reference): when enabled, every engine
 * launch on this context is bracketed by a pair of CUDA events on the context stream and
 * tagged with its kernel family and the algorithmic bytes it must move.  Up to
 * max_launches launches are recorded; enabling again clears the record. */
int hamlss_profile_enable(hamlss_ctx* ctx, int enable, int32_t max_launches);
/* Totals per kernel family, at most `cap` families: names[i*32..] (NUL-terminated),
 * launches[i], total_ms[i] (sum of event-measured durations), total_bytes[i]
 * (algorithmic).  *count = number of families written.  Synchronises the stream. */
int hamlss_profile_read(hamlss_ctx* ctx, int32_t cap, char* names, int32_t* launches,
                        double* total_ms, double* total_bytes, int32_t* count);

/* Energy counter of CUDA device `device` (NVML's total energy since driver load, joules),
 * matched to the CUDA ordinal by PCI bus id.  Replaces NVMLMonitor::read_energy_j
 * (src/parallel/nvml_monitor.cpp:85-100).  Read only.  HAMLSS_ERR_NOT_READY when NVML or
 * the counter is not available for the device. */
int hamlss_energy_read(int device, double* joules);

/* -------------------------------------------------------------------- matrix
 * Replaces hsps::SparseMatrix(rows, cols, row_ptr, col_idx, values)
 * (sparse_matrix.cpp:22-27): a deep copy into device memory.  The engine keeps the
 * FP64 values and derives an FP32 copy on first use by a mixed-precision solve.
 * The CSR is validated on the device (row_ptr monotone, column bounds, sorted rows);
 * a malformed matrix returns HAMLSS_ERR_MALFORMED. */
int hamlss_mat_upload(hamlss_ctx* ctx, int32_t rows, int32_t cols, int32_t nnz,
                      const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                      int where, hamlss_mat** out);
int hamlss_mat_update_values(hamlss_mat* A, const double* values, int where);
int hamlss_mat_info(const hamlss_mat* A, int32_t* rows, int32_t* cols, int32_t* nnz);
int hamlss_mat_download(const hamlss_mat* A, int32_t* row_ptr, int32_t* col_idx, double* values);
int hamlss_mat_release(hamlss_mat* A);

/* y = A x.  Replaces SparseMatrix::spmv (sparse_matrix.cpp:68-87). */
int hamlss_spmv(hamlss_ctx* ctx, const hamlss_mat* A, const double* x, double* y, int where);

/* Vector BLAS-1 on device pointers.  Replace Vector::dot / norm2 / axpy / axpby / scale
 * (vector.cpp:39-89).  Results of reductions land in host memory. */
int hamlss_dot(hamlss_ctx* ctx, int32_t n, const double* x, const double* y, double* result);
int hamlss_norm2(hamlss_ctx* ctx, int32_t n, const double* x, double* result);
int hamlss_axpy(hamlss_ctx* ctx, int32_t n, double alpha, const double* x, double* y);
int hamlss_axpby(hamlss_ctx* ctx, int32_t n, double a, const double* x, double b, double* y);
int hamlss_scale(hamlss_ctx* ctx, int32_t n, double alpha, double* x);

/* x . y for callers that cannot let a library allocate device memory: an application that
 * reserves the GPU's memory for its own pool, or a latency-critical loop where cudaMalloc /
 * cudaFree would stall the whole device.  No counterpart in the reference (it has no
 * device memory); same kernel and same result as hamlss_dot, but no context and no
 * allocation of any kind.
 *   x, y    device pointers on the CURRENT device; result: host pointer (one double).
 *   stream  a cudaStream_t (NULL: the default stream); the call waits for it to finish.
 * The scratch (2048 partial sums, the result slot and a ticket: 16 KiB) is a fixed array
 * compiled into the library, which every GPU that loads the library holds until exit.
 * The first call on each device looks up that array's device address (make that first
 * call before any stream capture) and keeps it for the life of the process: after
 * cudaDeviceReset on a device the kept address is stale, so do not call this entry point
 * on a device that the process has reset.  All calls on a device share the array: calls whose
 * work may overlap on the GPU (other streams, other host threads) race; serialise them.
 * A launch that would need more than 2048 partial sums (a GPU with more than 256 SMs) is
 * refused with HAMLSS_ERR_SIZE. */
int hamlss_dot_noalloc(int32_t n, const double* x, const double* y, double* result, void* stream);

/* ------------------------------------------------------------ preconditioners
 * Replaces SolverFactory::make_precond (solver_factory.cpp:54-97) followed by
 * PreconditionerBase::setup.  kind = HAMLSS_PREC_*; HAMLSS_PREC_NONE yields *out == NULL
 * like the reference's nullptr.  HAMLSS_PREC_ILU with params->drop_tol > 0 or
 * fill_per_row > 0 is ILUT(drop_tol, fill_per_row) (ilu.cpp:31-36, 94-220), factored on
 * the device row by row in the reference's order; else ILU(0) (ilu.cpp:41-89).  An ILUT
 * work row that touches more than 512 columns is refused with HAMLSS_ERR_NOMEM.
 * fill_per_row is ILUPreconditioner::set_fill_per_row; SolverFactory::make_precond never
 * sets it (solver_factory.cpp:73-77), so callers that mirror the factory pass 0, and the
 * adaptive ladder (hamlss_solve_adaptive, the server) uses 0. */
int hamlss_precond_setup(hamlss_ctx* ctx, const hamlss_mat* A, int kind,
                         const hamlss_params* params, hamlss_prec** out, double* setup_time_s);
/* z = M^-1 r.  Replaces PreconditionerBase::apply (preconditioner_base.hpp:32). */
int hamlss_precond_apply(hamlss_ctx* ctx, const hamlss_prec* M, const double* r, double* z,
                         int where);
int hamlss_precond_type(const hamlss_prec* M, int32_t* kind);
int hamlss_precond_release(hamlss_prec* M);

/* --------------------------------------------------------------------- solve
 * Replaces SolverBase::solve (solver_base.hpp:32-35) for CGSolver (cg_solver.cpp:37-191),
 * FGMRESSolver (fgmres_solver.cpp:165-241), PipelinedFGMRESSolver
 * (pipelined_fgmres_solver.cpp:69-242; HAMLSS_SOLVER_PIPELINED_FGMRES) and SStepCGSolver
 * (sstep_cg_solver.cpp:170-305; HAMLSS_SOLVER_SSTEP_CG, batch size params->sstep_k in
 * [1, 32], FP64 whatever params->precision says, M recorded but not applied as in the
 * reference).  x holds the initial guess on entry and the solution on exit.  M may be
 * NULL (no preconditioner). */
int hamlss_solve(hamlss_ctx* ctx, int solver, const hamlss_mat* A, const hamlss_prec* M,
                 const double* b, double* x, int where, const hamlss_params* params,
                 hamlss_stats* stats);

/* Replaces AdaptiveSelector::solve (adaptive_selector.cpp:298-394): features, initial
 * state, then the CG+Jacobi -> FGMRES+ILU(0) -> FGMRES+AMG ladder with warm starts.
 * `log` receives up to `log_cap` escalation records; *n_log their count. */
int hamlss_solve_adaptive(hamlss_ctx* ctx, const hamlss_mat* A, const double* b, double* x,
                          int where, const hamlss_params* params, hamlss_stats* stats,
                          hamlss_escalation* log, int32_t log_cap, int32_t* n_log,
                          int32_t* initial_state);

/* AdaptiveSelector::extract_features + select_initial_state (adaptive_selector.cpp:37-233):
 * the 24-entry feature vector of MatrixFeatures::to_feature_vector (:418-446). */
int hamlss_extract_features(hamlss_ctx* ctx, const hamlss_mat* A, double features[24],
                            int32_t* initial_state);

/* ------------------------------------------------------------ batched solves
 * No counterpart in the reference, which solves one system per SolverBase::solve call
 * (include/solvers/solver_base.hpp:32-35); each system of a batch runs the reference's
 * algorithm for its method (CGSolver + JacobiPreconditioner, or FGMRESSolver +
 * ILUPreconditioner with drop_tol 0), all of them inside one persistent kernel.
 *
 * The `count` systems form ONE block-diagonal CSR: system k owns rows
 * [row_off[k], row_off[k+1]) and every entry of those rows has its column in the same
 * range (global row_ptr of row_off[count] + 1 entries, global column indices).  row_off is
 * host memory; row_ptr / col_idx / values follow `where`.  solver[k] is HAMLSS_SOLVER_CG
 * or HAMLSS_SOLVER_FGMRES, precond[k] HAMLSS_PREC_NONE, _JACOBI or (FGMRES only) _ILU.
 * Values are kept in FP64 and FP32: the systems are solved in FP32 inside an FP64
 * iterative-refinement loop to params->tol FP64 relative residual (params->max_iter inner
 * iterations, params->ir_max_outer refinement steps, params->restart_size <= 32).
 * A setup failure of one system (zero diagonal, zero pivot) is reported in its result and
 * does not stop the others. */
typedef struct hamlss_batch hamlss_batch;
typedef struct hamlss_batch_result {
    int32_t iterations;        /* inner Krylov iterations over all refinement steps */
    int32_t outer_iterations;  /* FP64 refinement steps                             */
    int32_t converged;
    int32_t status;            /* HAMLSS_OK or the HAMLSS_ERR_* of this system      */
    double  initial_residual;  /* ||b - A x0||                                      */
    double  final_residual;    /* FP64 ||b - A x|| / ||b||                          */
} hamlss_batch_result;

int hamlss_batch_create(hamlss_ctx* ctx, int32_t count, const int32_t* row_off,
                        const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                        const int32_t* solver, const int32_t* precond, int where,
                        const hamlss_params* params, hamlss_batch** out);
/* b, x: row_off[count] entries each (x = initial guess on entry).  results: `count`
 * entries (may be NULL); total (may be NULL): summed iterations, converged = all systems
 * converged, final_residual = the largest, device_time_s = the kernel's event time. */
int hamlss_batch_solve(hamlss_ctx* ctx, hamlss_batch* B, const double* b, double* x, int where,
                       hamlss_batch_result* results, hamlss_stats* total);
/* Team width (threads per system: 32, 64, 128, 256 or 512) of the four size classes
 * n <= 1024, <= 4096, <= 16384 and larger.  Results depend on the width only through the
 * order of the dot-product sums. */
int hamlss_batch_set_widths(hamlss_batch* B, const int32_t widths[4]);
int hamlss_batch_get_widths(const hamlss_batch* B, int32_t widths[4]);
/* Time every width for every size class present (solves of the batch itself, x0 = 0, on
 * internal buffers), keep the fastest, and record them in `cache_path` (may be NULL) keyed
 * by device, class, method mix and restart length; a cached key is reused without timing. */
int hamlss_batch_autotune(hamlss_ctx* ctx, hamlss_batch* B, const double* b, int where,
                          const char* cache_path, int32_t widths[4]);
int hamlss_batch_release(hamlss_batch* B);

/* ------------------------------------------------------------------ serving
 * No counterpart in the reference, which solves one system per synchronous
 * AdaptiveSelector::solve call (src/adaptive/adaptive_selector.cpp:298-394).  A server keeps
 * that per-request algorithm (the adaptive ladder; params->precision selects the FP64 or
 * the mixed-precision inner path) and runs many requests at once on one device:
 *   - admission: a request is admitted when its estimated device footprint fits
 *     hbm_budget_bytes beside those already admitted; one that could never fit is refused
 *     by submit with HAMLSS_ERR_BUDGET;
 *   - `slots` solve lanes (a worker thread and CUDA stream each) run admitted requests
 *     through the ladder concurrently, so their kernels overlap on the device;
 *   - requests with n <= batch_max_rows are coalesced: whenever the batch lane is free it
 *     solves every queued small request with the head's tolerance (up to batch_max_count)
 *     in one persistent launch -- CG + Jacobi for symmetric systems with a positive
 *     diagonal, FGMRES + ILU(0) for the rest, FP32 inside FP64 refinement.  A system that
 *     fails there continues on a solve lane through the full ladder.
 *   - when the ladder fails from the state the features chose, the rungs below it that it
 *     skipped are tried too (FGMRES + ILU(0); CG + Jacobi for symmetric systems with a
 *     positive diagonal), each from the request's initial guess.
 * Requests that arrive while others run are admitted as lanes and budget free up.  A
 * request's result does not depend on the other requests in flight.
 *
 * The caller's arrays (CSR, b, x) must stay valid and unmodified until the request is
 * finished; x holds the initial guess on submit and the solution once it is done.
 * Functions are thread-safe: any thread may submit, test, wait or cancel. */
typedef struct hamlss_server hamlss_server;
typedef struct hamlss_server_config {
    int32_t device;            /* CUDA device (0)                                           */
    int32_t slots;             /* concurrent solve lanes (4)                                */
    int64_t hbm_budget_bytes;  /* admission budget for request state (150e9)                */
    int32_t batch_max_rows;    /* coalesce requests with n <= this; 0 disables (16384)      */
    int32_t batch_max_count;   /* systems per coalesced launch (2048)                       */
    int32_t order;             /* solve-lane queue: 0 arrival order (a fitting request may  */
                               /* pass a head that does not fit, at most 8 times) (0); 1    */
                               /* fewest nonzeros first, a request passed 32 times leads    */
    int32_t large_rows;        /* requests with n >= large_rows are "large" (1048576)       */
    int32_t max_large;         /* large requests running at once; 0: no bound (1).  Others  */
                               /* pass a large head that waits for this bound, so one large */
                               /* solve at a time keeps its speed while small ones flow      */
} hamlss_server_config;

typedef struct hamlss_server_report {
    int64_t submitted, completed, failed, cancelled;
    int64_t coalesced;         /* completed in the batch lane                               */
    int64_t batches;           /* coalesced launches                                        */
    int64_t escalated;         /* moved from the batch lane to a solve lane                 */
    int64_t fallback;          /* solved by a rung below the ladder's failed start           */
    int64_t queued;            /* waiting now                                               */
    int32_t running, peak_running;
    int64_t admitted_bytes, peak_admitted_bytes;
    double  p50_latency_s, p99_latency_s, mean_latency_s, max_latency_s;  /* submit -> done */
    double  solves_per_s;      /* completed / (last completion - first submit)              */
} hamlss_server_report;

void hamlss_server_config_default(hamlss_server_config* config);
int hamlss_server_create(const hamlss_server_config* config, hamlss_server** out);
/* Queue one solve A x = b (host CSR, host b and x).  *request_id identifies it. */
int hamlss_server_submit(hamlss_server* server, int32_t n, int32_t nnz, const int32_t* row_ptr,
                         const int32_t* col_idx, const double* values, const double* b, double* x,
                         const hamlss_params* params, int64_t* request_id);
/* Wait for a request (timeout_s < 0: no limit).  Returns its status (HAMLSS_OK or the error
 * that ended it) and fills *stats; HAMLSS_ERR_TIMEOUT if it is still in flight.  A request
 * that has been waited for successfully or with an error is forgotten. */
int hamlss_server_wait(hamlss_server* server, int64_t request_id, double timeout_s,
                       hamlss_stats* stats);
/* *done = 1 once the request has finished (it can then be waited for without blocking). */
int hamlss_server_test(hamlss_server* server, int64_t request_id, int32_t* done);
/* Withdraw a request that has not started: its wait returns HAMLSS_ERR_CANCELLED. */
int hamlss_server_cancel(hamlss_server* server, int64_t request_id);
int hamlss_server_get_report(hamlss_server* server, hamlss_server_report* report);
/* Clear the counters and latency record (e.g. after a warm-up stream). */
int hamlss_server_reset_report(hamlss_server* server);
/* Finish the requests in flight, cancel the queued ones, release the lanes.  No other call
 * on this server may be in progress or follow. */
int hamlss_server_destroy(hamlss_server* server);

/* ------------------------------------------------------------- MatrixMarket
 * The .mtx files that feed the engine; same accepted formats and conversions as the
 * reference's MatrixMarketIO (include/utils/matrix_market_io.hpp:80-130,
 * src/utils/matrix_market_io.cpp): coordinate real / integer / pattern matrices,
 * symmetric and skew-symmetric storage expanded, entries sorted by (row, column) with
 * duplicates summed (SparseMatrix::from_coo, sparse_matrix.cpp:242-282); array or
 * coordinate vectors.  Host code; no device involved except in hamlss_mat_load_mtx. */
enum { HAMLSS_MTX_COORDINATE = 0, HAMLSS_MTX_ARRAY = 1 };
enum { HAMLSS_MTX_REAL = 0, HAMLSS_MTX_INTEGER = 1, HAMLSS_MTX_COMPLEX = 2, HAMLSS_MTX_PATTERN = 3 };
enum { HAMLSS_MTX_GENERAL = 0, HAMLSS_MTX_SYMMETRIC = 1, HAMLSS_MTX_SKEW = 2, HAMLSS_MTX_HERMITIAN = 3 };
/* MatrixMarketIO::read_header: banner and size line; entries = stored entries (array:
 * rows * cols).  Any output pointer may be NULL. */
int hamlss_mtx_read_header(const char* path, int32_t* format, int32_t* field, int32_t* symmetry,
                           int64_t* rows, int64_t* cols, int64_t* entries);
/* MatrixMarketIO::load_matrix into CSR.  Pass NULL arrays to learn rows / cols / nnz first
 * (the file is parsed again by the second call). */
int hamlss_mtx_read_matrix(const char* path, int32_t* rows, int32_t* cols, int32_t* nnz,
                           int32_t* row_ptr, int32_t* col_idx, double* values);
/* MatrixMarketIO::load_vector(path, expected_n): *n values (values may be NULL to query). */
int hamlss_mtx_read_vector(const char* path, int32_t expected_n, double* values, int32_t* n);
/* MatrixMarketIO::save_vector / save_matrix ("%.15e" values; comment may be NULL). */
int hamlss_mtx_write_vector(const char* path, int32_t n, const double* values, const char* comment);
int hamlss_mtx_write_matrix(const char* path, int32_t rows, int32_t cols, int32_t nnz,
                            const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                            const char* comment);
/* Parse a .mtx matrix and upload it to the context's device (hamlss_mat_upload). */
int hamlss_mat_load_mtx(hamlss_ctx* ctx, const char* path, hamlss_mat** out);

/* ------------------------------------------------------- inspection (parity)
 * Internals that the reference keeps private but that parity is checked on. */
/* Greedy aggregation of one matrix (amg.cpp:30-67): agg[rows]; returns the count. */
int hamlss_amg_aggregate(hamlss_ctx* ctx, const hamlss_mat* A, double theta,
                         int32_t* agg, int32_t* n_agg);
int hamlss_amg_num_levels(const hamlss_prec* M, int32_t* levels);
/* Level `l` of the hierarchy: which = 0 A, 1 P, 2 R.  Pass NULL arrays to query sizes. */
int hamlss_amg_level_matrix(const hamlss_prec* M, int32_t level, int32_t which,
                            int32_t* rows, int32_t* cols, int32_t* nnz,
                            int32_t* row_ptr, int32_t* col_idx, double* values);
/* ILU factor values in the factor's pattern (ilu.cpp's lu_val_): A's pattern for ILU(0). */
int hamlss_ilu_factors(const hamlss_prec* M, double* lu_values);
/* The L\U factor as CSR (ilu.cpp's lu_row_ptr_ / lu_col_ind_ / lu_val_; for ILUT each row
 * holds its kept L entries, then its U entries, both by ascending column).  *nnz receives
 * the entry count; row_ptr[rows + 1], col_idx[nnz], values[nnz] (host) are filled when
 * non-NULL. */
int hamlss_ilu_factor_csr(const hamlss_prec* M, int32_t* nnz, int32_t* row_ptr,
                          int32_t* col_idx, double* values);
/* Level sets of the lower (which = 0) or upper (which = 1) triangle of an ILU(0)
 * preconditioner: level[rows]; *n_levels their count. */
int hamlss_ilu_levels(const hamlss_prec* M, int32_t which, int32_t* level, int32_t* n_levels);

#ifdef __cplusplus
}
#endif
#endif /* HAMLSS_H */
