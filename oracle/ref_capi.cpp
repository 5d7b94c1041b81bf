// ref_capi.cpp -- C entry points over the REFERENCE implementation, for pinning only.
//
// Test infrastructure: compiled by oracle/Makefile together with the reference's own
// sources (read in place from the reference checkout, never copied) into
// oracle/_ref/libhsps_ref*.so.  tests/ use it to pin the oracle restatement and the
// device engine against the reference itself; bench.py's reference arm times it.
// The engine never links or calls it.
//
// The reference keeps the AMG hierarchy, the aggregation and the ILU factors private;
// this file opens them for inspection by compiling those headers with `private`
// mapped to `public`, which changes no layout or behaviour.

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <omp.h>

#include "core/sparse_matrix.hpp"
#include "core/vector.hpp"
#include "solvers/solver_factory.hpp"
#include "solvers/solver_base.hpp"
#include "solvers/cg_solver.hpp"
#include "solvers/fgmres_solver.hpp"
#include "solvers/pipelined_fgmres_solver.hpp"
#include "preconditioners/jacobi.hpp"
#define private public
#define protected public
#include "preconditioners/ilu.hpp"
#include "preconditioners/amg.hpp"
#include "adaptive/adaptive_selector.hpp"
#include "utils/matrix_market_io.hpp"
#undef private
#undef protected

#include "../include/hamlss.h"

using namespace hsps;

namespace {

SparseMatrix make_csr(int32_t n, const int32_t* rp, const int32_t* ci, const double* v) {
    int32_t nnz = rp[n];
    std::vector<Index> r(rp, rp + n + 1), c(ci, ci + nnz);
    std::vector<Real> vals(v, v + nnz);
    return SparseMatrix(n, n, r, c, vals);
}

SolverParams to_params(const hamlss_params* p) {
    SolverParams s;
    s.tol = p->tol;
    s.max_iter = p->max_iter;
    s.restart_size = p->restart_size;
    s.drop_tol = p->drop_tol;
    s.amg_levels = p->amg_levels;
    s.amg_strength = p->amg_strength;
    s.amg_strong = p->amg_strong;
    s.amg_smooth_pre = p->amg_smooth_pre;
    s.amg_smooth_post = p->amg_smooth_post;
    s.stall_window = p->stall_window;
    s.stall_threshold = p->stall_threshold;
    s.verbose = false;
    s.print_every = p->print_every;
    s.sstep_k = p->sstep_k;
    s.sstep_cond_tol = p->sstep_cond_tol;
    s.async_enabled = p->async_enabled != 0;
    s.async_max_stale = p->async_max_stale;
    s.fill_per_row = p->fill_per_row;
    s.block_size = p->block_size;
    return s;
}

void from_stats(const SolverStats& s, hamlss_stats* o) {
    std::memset(o, 0, sizeof(*o));
    o->iterations = s.iterations;
    o->initial_residual = s.initial_residual;
    o->final_residual = s.final_residual;
    o->converged = s.converged ? 1 : 0;
    o->solve_time_s = s.solve_time_s;
    o->setup_time_s = s.setup_time_s;
    o->energy_joules = s.energy_joules;
    o->flop_count = s.flop_count;
    o->mem_bytes = s.mem_bytes;
    o->solver_used = static_cast<int32_t>(s.solver_used);
    o->precond_used = static_cast<int32_t>(s.precond_used);
    o->state_used = static_cast<int32_t>(s.state_used);
    o->restarts = s.restarts;
    o->sstep_k = s.sstep_k;
    o->async_mode = s.async_mode ? 1 : 0;
    o->comm_bytes = s.comm_bytes;
    o->comm_time_s = s.comm_time_s;
}

int map_error(const std::exception& e) {
    std::string m = e.what();
    if (m.find("zero diagonal") != std::string::npos) return HAMLSS_ERR_ZERO_DIAG;
    if (m.find("pivot") != std::string::npos || m.find("U diagonal") != std::string::npos)
        return HAMLSS_ERR_ZERO_PIVOT;
    return HAMLSS_ERR_INVALID;
}

void copy_out(const SparseMatrix& A, int32_t* rows, int32_t* cols, int32_t* nnz,
              int32_t* rp, int32_t* ci, double* v) {
    if (rows) *rows = A.rows();
    if (cols) *cols = A.cols();
    if (nnz) *nnz = A.nnz();
    if (rp) std::memcpy(rp, A.row_ptr().data(), sizeof(int32_t) * (A.rows() + 1));
    if (ci && A.nnz()) std::memcpy(ci, A.col_idx().data(), sizeof(int32_t) * A.nnz());
    if (v && A.nnz()) std::memcpy(v, A.values().data(), sizeof(double) * A.nnz());
}

}  // namespace

extern "C" {

void ref_set_threads(int t) { omp_set_num_threads(t); }
int ref_max_threads(void) { return omp_get_max_threads(); }

int64_t ref_gen_poisson(int32_t n, int32_t* rp, int32_t* ci, double* v) {
    SparseMatrix A = SparseMatrix::poisson_2d(n);
    copy_out(A, nullptr, nullptr, nullptr, rp, ci, v);
    return A.nnz();
}

int64_t ref_gen_convdiff(int32_t n, double eps, double bx, double by,
                         int32_t* rp, int32_t* ci, double* v) {
    SparseMatrix A = SparseMatrix::convection_diffusion_2d(n, eps, bx, by);
    copy_out(A, nullptr, nullptr, nullptr, rp, ci, v);
    return A.nnz();
}

// SparseMatrix::from_coo: rows x cols, nz triples; output arrays sized rows+1 / nz.
int64_t ref_from_coo(int32_t rows, int32_t cols, int64_t nz, const int32_t* r,
                     const int32_t* c, const double* v, int32_t* rp, int32_t* ci, double* vo) {
    std::vector<Index> rv(r, r + nz), cv(c, c + nz);
    std::vector<Real> vv(v, v + nz);
    SparseMatrix A = SparseMatrix::from_coo(rows, cols, rv, cv, vv);
    copy_out(A, nullptr, nullptr, nullptr, rp, ci, vo);
    return A.nnz();
}

void ref_spmv(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
              const double* x, double* y) {
    SparseMatrix A = make_csr(n, rp, ci, v);
    Vector xv(std::vector<Real>(x, x + n)), yv(n);
    A.spmv(xv, yv);
    std::memcpy(y, yv.data(), sizeof(double) * n);
}

double ref_dot(int32_t n, const double* a, const double* b) {
    Vector av(std::vector<Real>(a, a + n)), bv(std::vector<Real>(b, b + n));
    return av.dot(bv);
}

// SolverFactory::make(solver, precond, A, params) then solver->solve(A, b, x, stats).
int ref_solve(int solver, int precond, int32_t n, const int32_t* rp, const int32_t* ci,
              const double* v, const double* b, double* x, const hamlss_params* p,
              hamlss_stats* st) {
    try {
        SparseMatrix A = make_csr(n, rp, ci, v);
        double setup = 0.0;
        auto pair = SolverFactory::make(static_cast<SolverType>(solver),
                                        static_cast<PrecondType>(precond), A, to_params(p), &setup);
        Vector bv(std::vector<Real>(b, b + n)), xv(std::vector<Real>(x, x + n));
        SolverStats s;
        s.setup_time_s = setup;
        bool ok = pair.first->solve(A, bv, xv, s);
        std::memcpy(x, xv.data(), sizeof(double) * n);
        from_stats(s, st);
        return ok ? 1 : 0;
    } catch (const std::exception& e) {
        return map_error(e);
    }
}

// PipelinedFGMRESSolver (no SolverType of its own): make_precond(precond), then solve.
int ref_pipelined_solve(int precond, int32_t n, const int32_t* rp, const int32_t* ci,
                        const double* v, const double* b, double* x, const hamlss_params* p,
                        hamlss_stats* st) {
    try {
        SparseMatrix A = make_csr(n, rp, ci, v);
        SolverParams sp = to_params(p);
        auto M = SolverFactory::make_precond(static_cast<PrecondType>(precond), A, sp);
        PipelinedFGMRESSolver s;
        s.set_params(sp);
        s.set_preconditioner(M);
        Vector bv(std::vector<Real>(b, b + n)), xv(std::vector<Real>(x, x + n));
        SolverStats out;
        bool ok = s.solve(A, bv, xv, out);
        std::memcpy(x, xv.data(), sizeof(double) * n);
        from_stats(out, st);
        return ok ? 1 : 0;
    } catch (const std::exception& e) {
        return map_error(e);
    }
}

// SparseMatrix::spectral_interval(steps).
void ref_spectral_interval(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                           int steps, double* lo, double* hi) {
    SparseMatrix A = make_csr(n, rp, ci, v);
    auto pr = A.spectral_interval(steps);
    *lo = pr.first;
    *hi = pr.second;
}

// make_precond(kind, A, params) then apply(r, z).
int ref_precond_apply(int kind, int32_t n, const int32_t* rp, const int32_t* ci,
                      const double* v, const hamlss_params* p, const double* r, double* z) {
    try {
        SparseMatrix A = make_csr(n, rp, ci, v);
        auto M = SolverFactory::make_precond(static_cast<PrecondType>(kind), A, to_params(p));
        Vector rv(std::vector<Real>(r, r + n)), zv(n);
        if (M) M->apply(rv, zv); else zv = rv;
        std::memcpy(z, zv.data(), sizeof(double) * n);
        return HAMLSS_OK;
    } catch (const std::exception& e) {
        return map_error(e);
    }
}

int32_t ref_amg_aggregate(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                          double theta, int32_t* agg) {
    SparseMatrix A = make_csr(n, rp, ci, v);
    AMGPreconditioner amg;
    amg.set_strength_thresh(theta);
    std::vector<Index> a = amg.aggregate(A);
    std::memcpy(agg, a.data(), sizeof(int32_t) * n);
    int32_t m = 0;
    for (Index x : a) m = x + 1 > m ? x + 1 : m;
    return m;
}

// Full AMG setup through the factory; returns an opaque handle.
void* ref_amg_setup(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                    const hamlss_params* p) {
    try {
        SparseMatrix A = make_csr(n, rp, ci, v);
        auto M = SolverFactory::make_precond(PrecondType::AMG, A, to_params(p));
        return new std::shared_ptr<PreconditionerBase>(M);
    } catch (...) {
        return nullptr;
    }
}

void ref_amg_free(void* h) { delete static_cast<std::shared_ptr<PreconditionerBase>*>(h); }

int32_t ref_amg_num_levels(void* h) {
    auto* amg = static_cast<AMGPreconditioner*>(static_cast<std::shared_ptr<PreconditionerBase>*>(h)->get());
    return amg->levels();
}

int ref_amg_level(void* h, int32_t level, int32_t which, int32_t* rows, int32_t* cols,
                  int32_t* nnz, int32_t* rp, int32_t* ci, double* v) {
    auto* amg = static_cast<AMGPreconditioner*>(static_cast<std::shared_ptr<PreconditionerBase>*>(h)->get());
    if (level < 0 || level >= amg->levels()) return HAMLSS_ERR_INVALID;
    const AMGLevel& L = amg->hierarchy_[level];
    const SparseMatrix& M = which == 0 ? L.A : which == 1 ? L.P : L.R;
    copy_out(M, rows, cols, nnz, rp, ci, v);
    return HAMLSS_OK;
}

void ref_amg_apply(void* h, int32_t n, const double* r, double* z) {
    auto* M = static_cast<std::shared_ptr<PreconditionerBase>*>(h)->get();
    Vector rv(std::vector<Real>(r, r + n)), zv(n);
    M->apply(rv, zv);
    std::memcpy(z, zv.data(), sizeof(double) * n);
}

int ref_ilu0_factor(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                    double* lu) {
    try {
        SparseMatrix A = make_csr(n, rp, ci, v);
        ILUPreconditioner ilu;
        ilu.set_drop_tol(0.0);
        ilu.setup(A);
        std::memcpy(lu, ilu.lu_val_.data(), sizeof(double) * rp[n]);
        return HAMLSS_OK;
    } catch (const std::exception& e) {
        return map_error(e);
    }
}

int ref_extract_features(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                         double* feat, int32_t* initial_state) {
    SparseMatrix A = make_csr(n, rp, ci, v);
    AdaptiveSelector sel;
    auto f = sel.extract_features(A);
    auto fv = f.to_feature_vector();
    std::memcpy(feat, fv.data(), sizeof(double) * fv.size());
    if (initial_state) *initial_state = static_cast<int32_t>(sel.select_initial_state(f));
    return HAMLSS_OK;
}

int ref_solve_adaptive(int32_t n, const int32_t* rp, const int32_t* ci, const double* v,
                       const double* b, double* x, const hamlss_params* p, hamlss_stats* st,
                       hamlss_escalation* log, int32_t log_cap, int32_t* n_log) {
    try {
        SparseMatrix A = make_csr(n, rp, ci, v);
        AdaptiveSelector sel(to_params(p));
        Vector bv(std::vector<Real>(b, b + n)), xv(std::vector<Real>(x, x + n));
        SolverStats s;
        bool ok = sel.solve(A, bv, xv, s);
        std::memcpy(x, xv.data(), sizeof(double) * n);
        from_stats(s, st);
        const auto& el = sel.escalation_log();
        *n_log = static_cast<int32_t>(el.size());
        for (int32_t i = 0; i < *n_log && i < log_cap; ++i) {
            log[i].at_iteration = el[i].at_iteration;
            log[i].from_state = static_cast<int32_t>(el[i].from_state);
            log[i].to_state = static_cast<int32_t>(el[i].to_state);
            log[i].residual_at_escalation = el[i].residual_at_escalation;
            log[i].reason = 0;
        }
        return ok ? 1 : 0;
    } catch (const std::exception& e) {
        return map_error(e);
    }
}

// ILUPreconditioner::setup with drop_tol > 0 or fill_per_row > 0 (setup_ilut): the L\U
// factor (row_ptr_, col_idx_, lu_val_).  *nnz first; the arrays when given.
int ref_ilut_factor(int32_t n, const int32_t* rp, const int32_t* ci, const double* v, double drop_tol,
                    int32_t fill_p, int32_t* frp, int32_t* fci, double* flu, int64_t* nnz) {
    try {
        SparseMatrix A = make_csr(n, rp, ci, v);
        ILUPreconditioner ilu;
        ilu.set_drop_tol(drop_tol);
        ilu.set_fill_per_row(fill_p);
        ilu.setup(A);
        *nnz = static_cast<int64_t>(ilu.col_idx_.size());
        if (frp) std::memcpy(frp, ilu.row_ptr_.data(), sizeof(int32_t) * (n + 1));
        if (fci && *nnz) std::memcpy(fci, ilu.col_idx_.data(), sizeof(int32_t) * (size_t)*nnz);
        if (flu && *nnz) std::memcpy(flu, ilu.lu_val_.data(), sizeof(double) * (size_t)*nnz);
        return 0;
    } catch (const std::exception& e) {
        return map_error(e);
    }
}

// MatrixMarketIO::load_matrix: rows / cols / nnz, then (when the arrays are given) the CSR.
int ref_mtx_load_matrix(const char* path, int32_t* rows, int32_t* cols, int32_t* nnz, int32_t* rp,
                        int32_t* ci, double* v) {
    try {
        SparseMatrix A = MatrixMarketIO::load_matrix(path);
        *rows = A.rows();
        *cols = A.cols();
        *nnz = A.nnz();
        if (rp) std::memcpy(rp, A.row_ptr().data(), sizeof(int32_t) * (A.rows() + 1));
        if (ci && A.nnz()) std::memcpy(ci, A.col_idx().data(), sizeof(int32_t) * A.nnz());
        if (v && A.nnz()) std::memcpy(v, A.values().data(), sizeof(double) * A.nnz());
        return 0;
    } catch (const std::exception& e) {
        return -1;
    }
}

// MatrixMarketIO::load_vector(path, expected_n): *n values (v may be null to query).
int ref_mtx_load_vector(const char* path, int32_t expected_n, double* v, int32_t* n) {
    try {
        Vector x = MatrixMarketIO::load_vector(path, expected_n);
        *n = static_cast<int32_t>(x.size());
        if (v && x.size()) std::memcpy(v, x.data(), sizeof(double) * x.size());
        return 0;
    } catch (const std::exception& e) {
        return -1;
    }
}

}  // extern "C"
