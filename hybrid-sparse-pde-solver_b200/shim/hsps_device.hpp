// hsps_device.hpp -- drop-in device solvers for the HAMLSS C++17 API (header only).
//
// Include this after the project's own headers (it is compiled against them, through
// the include path; nothing here redefines the hsps types) and link libhamlss_b200.so.
// Every class derives from the project's abstract interface, so existing call sites
// keep working:
//
//   hsps::SolverBase          -> hsps_b200::DeviceCGSolver, DeviceFGMRESSolver
//                                (include/solvers/solver_base.hpp:20-62)
//   hsps::PreconditionerBase  -> hsps_b200::DeviceJacobi, DeviceILU, DeviceAMG
//                                (include/preconditioners/preconditioner_base.hpp:16-48)
//   hsps::SolverFactory       -> hsps_b200::DeviceSolverFactory, same static signatures
//                                (include/solvers/solver_factory.hpp:40-88)
//   hsps::AdaptiveSelector    -> hsps_b200::DeviceAdaptiveSelector, same public surface
//                                (include/adaptive/adaptive_selector.hpp:49-161)
//
// Matrices are uploaded on first use and cached by identity: the SparseMatrix's address,
// dimensions, nnz and a 64-bit hash of its three arrays (so values edited in place are
// seen).  Errors come back as the exceptions the project throws: std::invalid_argument
// for unknown names / options, std::runtime_error for everything else; a solve that does
// not converge returns false, as before.
#pragma once

#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <ostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "adaptive/adaptive_selector.hpp"
#include "core/sparse_matrix.hpp"
#include "core/types.hpp"
#include "core/vector.hpp"
#include "preconditioners/preconditioner_base.hpp"
#include "solvers/solver_base.hpp"
#include "solvers/solver_factory.hpp"

#include "hamlss.h"

namespace hsps_b200 {

inline void check(int rc) {
    if (rc == HAMLSS_OK) return;
    std::string msg = hamlss_last_error();
    if (rc == HAMLSS_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

inline hamlss_params to_params(const hsps::SolverParams& s) {
    hamlss_params p;
    hamlss_params_default(&p);
    p.tol = s.tol;
    p.max_iter = s.max_iter;
    p.restart_size = s.restart_size;
    p.drop_tol = s.drop_tol;
    p.amg_levels = s.amg_levels;
    p.amg_strength = s.amg_strength;
    p.amg_strong = s.amg_strong;
    p.amg_smooth_pre = s.amg_smooth_pre;
    p.amg_smooth_post = s.amg_smooth_post;
    p.stall_window = s.stall_window;
    p.stall_threshold = s.stall_threshold;
    p.verbose = s.verbose ? 1 : 0;
    p.print_every = s.print_every;
    p.sstep_k = s.sstep_k;
    p.sstep_cond_tol = s.sstep_cond_tol;
    p.async_enabled = s.async_enabled ? 1 : 0;
    p.async_max_stale = s.async_max_stale;
    p.fill_per_row = s.fill_per_row;
    p.block_size = s.block_size;
    p.record_hw_energy = s.record_hw_energy ? 1 : 0;
    return p;
}

inline void to_stats(const hamlss_stats& h, hsps::SolverStats& s) {
    s.iterations = h.iterations;
    s.initial_residual = h.initial_residual;
    s.final_residual = h.final_residual;
    s.converged = h.converged != 0;
    s.solve_time_s = h.solve_time_s;
    s.setup_time_s += h.setup_time_s;
    s.energy_joules = h.energy_joules;
    s.flop_count = h.flop_count;
    s.mem_bytes = h.mem_bytes;
    s.solver_used = static_cast<hsps::SolverType>(h.solver_used);
    s.precond_used = static_cast<hsps::PrecondType>(h.precond_used);
    s.state_used = static_cast<hsps::AdaptiveState>(h.state_used);
    s.restarts = h.restarts;
    s.sstep_k = h.sstep_k;
    s.comm_bytes = h.comm_bytes;
    s.energy_joules_hw = h.energy_joules_hw;
    s.rapl_start_j = h.rapl_start_j;
    s.rapl_end_j = h.rapl_end_j;
}

// ------------------------------------------------------------------- device context
class Device {
public:
    static Device& get(int device = 0) {
        static std::mutex mu;
        static std::map<int, std::unique_ptr<Device>> all;
        std::lock_guard<std::mutex> g(mu);
        auto& d = all[device];
        if (!d) d.reset(new Device(device));
        return *d;
    }
    hamlss_ctx* ctx() const { return ctx_; }

    // Device copy of A (uploaded once per distinct content).
    hamlss_mat* matrix(const hsps::SparseMatrix& A) {
        std::lock_guard<std::mutex> g(mu_);
        Key k{&A, A.rows(), A.cols(), A.nnz(), content_hash(A)};
        auto it = cache_.find(k);
        if (it != cache_.end()) return it->second.get();
        // drop stale entries of the same object
        for (auto e = cache_.begin(); e != cache_.end();)
            e = (e->first.addr == &A) ? cache_.erase(e) : std::next(e);
        hamlss_mat* m = nullptr;
        check(hamlss_mat_upload(ctx_, A.rows(), A.cols(), A.nnz(), A.row_ptr().data(),
                                A.col_idx().data(), A.values().data(), HAMLSS_HOST, &m));
        cache_.emplace(k, MatPtr(m, &hamlss_mat_release));
        return m;
    }

    static uint64_t content_hash(const hsps::SparseMatrix& A) {
        uint64_t h = 1469598103934665603ULL;
        auto mix = [&h](const void* p, size_t bytes) {
            const unsigned char* c = static_cast<const unsigned char*>(p);
            size_t i = 0;
            for (; i + 8 <= bytes; i += 8) {
                uint64_t w;
                std::memcpy(&w, c + i, 8);
                h = (h ^ w) * 1099511628211ULL;
                h ^= h >> 29;
            }
            for (; i < bytes; ++i) h = (h ^ c[i]) * 1099511628211ULL;
        };
        mix(A.row_ptr().data(), A.row_ptr().size() * sizeof(int));
        mix(A.col_idx().data(), A.col_idx().size() * sizeof(int));
        mix(A.values().data(), A.values().size() * sizeof(double));
        return h;
    }

private:
    explicit Device(int device) { check(hamlss_ctx_create(device, &ctx_)); }
    struct Key {
        const void* addr;
        int rows, cols, nnz;
        uint64_t hash;
        bool operator<(const Key& o) const {
            if (addr != o.addr) return addr < o.addr;
            if (hash != o.hash) return hash < o.hash;
            if (rows != o.rows) return rows < o.rows;
            if (cols != o.cols) return cols < o.cols;
            return nnz < o.nnz;
        }
    };
    using MatPtr = std::unique_ptr<hamlss_mat, int (*)(hamlss_mat*)>;
    hamlss_ctx* ctx_ = nullptr;
    std::mutex mu_;
    std::map<Key, MatPtr> cache_;
};

// --------------------------------------------------------------- preconditioners
class DevicePreconditioner : public hsps::PreconditionerBase {
public:
    explicit DevicePreconditioner(hsps::PrecondType t) : hsps::PreconditionerBase(t) {}
    ~DevicePreconditioner() override { if (h_) hamlss_precond_release(h_); }

    double setup(const hsps::SparseMatrix& A) override {
        Device& d = Device::get();
        if (h_) { hamlss_precond_release(h_); h_ = nullptr; }
        hamlss_params p = params();
        double t = 0.0;
        check(hamlss_precond_setup(d.ctx(), d.matrix(A), static_cast<int>(type_), &p, &h_, &t));
        n_ = A.rows();
        ready_ = true;
        return t;
    }

    void apply(const hsps::Vector& r, hsps::Vector& z) const override {
        if (!ready_) throw std::runtime_error("preconditioner used before setup");
        if (z.size() != r.size()) z.resize(r.size());
        check(hamlss_precond_apply(Device::get().ctx(), h_, r.data(), z.data(), HAMLSS_HOST));
    }

    hamlss_prec* handle() const { return h_; }

protected:
    virtual hamlss_params params() const {
        hamlss_params p;
        hamlss_params_default(&p);
        return p;
    }
    hamlss_prec* h_ = nullptr;
    int n_ = 0;
};

class DeviceJacobi : public DevicePreconditioner {
public:
    DeviceJacobi() : DevicePreconditioner(hsps::PrecondType::JACOBI) {}
    const char* energy_tier() const override { return "CHEAP"; }
    void set_omega(hsps::Real w) { omega_ = w; }

protected:
    hamlss_params params() const override {
        hamlss_params p = DevicePreconditioner::params();
        p.jacobi_omega = omega_;
        return p;
    }
    hsps::Real omega_ = 1.0;
};

// ILU(0), or ILUT(drop_tol, fill_per_row) when either is > 0 (ilu.cpp:31-36), factored on
// the device in the project's order (bit-identical factors).
class DeviceILU : public DevicePreconditioner {
public:
    DeviceILU() : DevicePreconditioner(hsps::PrecondType::ILU) {}
    const char* energy_tier() const override { return "MODERATE"; }
    void set_drop_tol(hsps::Real t) { drop_ = t; }
    void set_fill_per_row(int p) { fill_ = p; }

protected:
    hamlss_params params() const override {
        hamlss_params p = DevicePreconditioner::params();
        p.drop_tol = drop_;
        p.fill_per_row = fill_;
        return p;
    }
    hsps::Real drop_ = 0.0;
    int fill_ = 0;
};

class DeviceAMG : public DevicePreconditioner {
public:
    DeviceAMG() : DevicePreconditioner(hsps::PrecondType::AMG) {}
    const char* energy_tier() const override { return "EXPENSIVE"; }
    void set_max_levels(int n) { p_.amg_levels = n; }
    void set_strength_thresh(hsps::Real t) { p_.amg_strong = t; }
    void set_smooth_pre(int n) { p_.amg_smooth_pre = n; }
    void set_smooth_post(int n) { p_.amg_smooth_post = n; }
    void set_coarse_limit(int n) { p_.amg_coarse_limit = n; }
    void set_omega(hsps::Real w) { p_.amg_omega = w; }
    int levels() const {
        int32_t l = 0;
        if (h_) check(hamlss_amg_num_levels(h_, &l));
        return l;
    }

protected:
    hamlss_params params() const override { return p_; }
    hamlss_params p_ = [] { hamlss_params p; hamlss_params_default(&p); return p; }();
};

// ------------------------------------------------------------------------ solvers
class DeviceSolver : public hsps::SolverBase {
public:
    explicit DeviceSolver(hsps::SolverType t, int engine_id = -1)
        : hsps::SolverBase(t), engine_id_(engine_id < 0 ? static_cast<int>(t) : engine_id) {}

    bool solve(const hsps::SparseMatrix& A, const hsps::Vector& b, hsps::Vector& x,
               hsps::SolverStats& stats) override {
        const int n = A.rows();
        if (b.size() != n) throw std::runtime_error("solve: b size != rows");
        if (x.size() != n) x.resize(n, hsps::REAL_ZERO);     // cg_solver.cpp:49
        hamlss_prec* M = nullptr;
        if (precond_) {
            auto* dp = dynamic_cast<DevicePreconditioner*>(precond_.get());
            if (!dp)
                throw std::invalid_argument("device solvers need a device preconditioner "
                                            "(DeviceJacobi / DeviceILU / DeviceAMG)");
            M = dp->handle();
        }
        Device& d = Device::get();
        hamlss_params p = to_params(params_);
        p.precision = precision_;
        adjust(p);
        hamlss_stats st;
        check(hamlss_solve(d.ctx(), engine_id_, d.matrix(A), M, b.data(), x.data(), HAMLSS_HOST, &p,
                           &st));
        to_stats(st, stats);
        true_residual_ = st.true_residual;
        return stats.converged;
    }

    // Engine option: HAMLSS_MIXED runs FP32 inner solves inside FP64 refinement.
    void set_precision(int prec) { precision_ = prec; }
    double last_true_residual() const { return true_residual_; }

protected:
    virtual void adjust(hamlss_params&) const {}
    int engine_id_;
    int precision_ = HAMLSS_FP64;
    double true_residual_ = 0.0;
};

class DeviceCGSolver : public DeviceSolver {
public:
    DeviceCGSolver() : DeviceSolver(hsps::SolverType::CG) {}
};

class DeviceFGMRESSolver : public DeviceSolver {
public:
    DeviceFGMRESSolver() : DeviceSolver(hsps::SolverType::FGMRES) {}
};

// PipelinedFGMRESSolver (include/solvers/pipelined_fgmres_solver.hpp:44-74): a SolverBase of
// type FGMRES, like the project's class.
class DevicePipelinedFGMRESSolver : public DeviceSolver {
public:
    DevicePipelinedFGMRESSolver()
        : DeviceSolver(hsps::SolverType::FGMRES, HAMLSS_SOLVER_PIPELINED_FGMRES) {}
};

// SStepCGSolver(k) (include/solvers/sstep_cg_solver.hpp:57-60); the preconditioner is
// recorded, not applied, as in the project.
class DeviceSStepCGSolver : public DeviceSolver {
public:
    explicit DeviceSStepCGSolver(int k = 4) : DeviceSolver(hsps::SolverType::SSTEP_CG), k_(k) {}

protected:
    void adjust(hamlss_params& p) const override { p.sstep_k = k_; }
    int k_;
};

// ------------------------------------------------------------------------ factory
struct DeviceSolverFactory {
    static std::unique_ptr<hsps::SolverBase> make_solver(hsps::SolverType t, const hsps::SolverParams& p) {
        std::unique_ptr<hsps::SolverBase> s;
        switch (t) {
            case hsps::SolverType::CG: s = std::make_unique<DeviceCGSolver>(); break;
            case hsps::SolverType::FGMRES:
            case hsps::SolverType::BICGSTAB: s = std::make_unique<DeviceFGMRESSolver>(); break;
            case hsps::SolverType::SSTEP_CG:                     // solver_factory.cpp:38-40
                s = std::make_unique<DeviceSStepCGSolver>(p.sstep_k);
                break;
            default: throw std::invalid_argument("SolverFactory: solver type not provided on the device");
        }
        s->set_params(p);
        return s;
    }

    static std::shared_ptr<hsps::PreconditionerBase> make_precond(hsps::PrecondType t,
                                                                  const hsps::SparseMatrix& A,
                                                                  const hsps::SolverParams& p,
                                                                  double* setup_time_s = nullptr) {
        std::shared_ptr<DevicePreconditioner> M;
        switch (t) {
            case hsps::PrecondType::NONE:
                if (setup_time_s) *setup_time_s = 0.0;
                return nullptr;
            case hsps::PrecondType::JACOBI: M = std::make_shared<DeviceJacobi>(); break;
            case hsps::PrecondType::ILU: {
                auto ilu = std::make_shared<DeviceILU>();
                ilu->set_drop_tol(p.drop_tol);                 // solver_factory.cpp:75
                M = ilu;
                break;
            }
            case hsps::PrecondType::AMG: {
                auto amg = std::make_shared<DeviceAMG>();
                amg->set_max_levels(p.amg_levels);              // solver_factory.cpp:83-86
                amg->set_strength_thresh(p.amg_strong);
                amg->set_smooth_pre(p.amg_smooth_pre);
                amg->set_smooth_post(p.amg_smooth_post);
                M = amg;
                break;
            }
            default: throw std::invalid_argument("SolverFactory: unknown PrecondType");
        }
        double t0 = M->setup(A);
        if (setup_time_s) *setup_time_s = t0;
        return M;
    }

    static hsps::SolverPrecondPair make(hsps::SolverType st, hsps::PrecondType pt,
                                        const hsps::SparseMatrix& A, const hsps::SolverParams& p,
                                        double* setup_time_s = nullptr) {
        double t = 0.0;
        auto M = make_precond(pt, A, p, &t);
        if (setup_time_s) *setup_time_s = t;
        auto s = make_solver(st, p);
        if (M) s->set_preconditioner(M);
        return {std::move(s), M};
    }

    static hsps::SolverPrecondPair make(const std::string& sname, const std::string& pname,
                                        const hsps::SparseMatrix& A, const hsps::SolverParams& p,
                                        double* setup_time_s = nullptr) {
        return make(hsps::SolverFactory::parse_solver(sname), hsps::SolverFactory::parse_precond(pname),
                    A, p, setup_time_s);
    }

    static hsps::SolverPrecondPair make_for_state(hsps::AdaptiveState s, const hsps::SparseMatrix& A,
                                                  const hsps::SolverParams& p,
                                                  double* setup_time_s = nullptr) {
        switch (s) {
            case hsps::AdaptiveState::EASY:
                return make(hsps::SolverType::CG, hsps::PrecondType::JACOBI, A, p, setup_time_s);
            case hsps::AdaptiveState::MODERATE:
                return make(hsps::SolverType::FGMRES, hsps::PrecondType::ILU, A, p, setup_time_s);
            case hsps::AdaptiveState::HARD:
                return make(hsps::SolverType::FGMRES, hsps::PrecondType::AMG, A, p, setup_time_s);
        }
        throw std::invalid_argument("SolverFactory: unknown AdaptiveState");
    }
};

// --------------------------------------------------------------- adaptive selector
class DeviceAdaptiveSelector {
public:
    explicit DeviceAdaptiveSelector(const hsps::SolverParams& p = {}) : params_(p) {}

    bool solve(const hsps::SparseMatrix& A, const hsps::Vector& b, hsps::Vector& x,
               hsps::SolverStats& stats) {
        const int n = A.rows();
        if (x.size() != n) x.resize(n, hsps::REAL_ZERO);
        Device& d = Device::get();
        hamlss_params p = to_params(params_);
        p.ladder_mode = ladder_mode_;
        p.precision = precision_;
        hamlss_stats st;
        hamlss_escalation log[16];
        int32_t nlog = 0, init = 0;
        check(hamlss_solve_adaptive(d.ctx(), d.matrix(A), b.data(), x.data(), HAMLSS_HOST, &p, &st, log,
                                    16, &nlog, &init));
        stats = hsps::SolverStats{};
        to_stats(st, stats);
        esc_log_.clear();
        for (int i = 0; i < nlog && i < 16; ++i) {
            hsps::EscalationRecord e;
            e.at_iteration = log[i].at_iteration;
            e.from_state = static_cast<hsps::AdaptiveState>(log[i].from_state);
            e.to_state = static_cast<hsps::AdaptiveState>(log[i].to_state);
            e.residual_at_escalation = log[i].residual_at_escalation;
            e.reason = log[i].reason == 0 ? "convergence stall / budget exhausted"
                     : log[i].reason == 1 ? "stall (device check)"
                     : log[i].reason == 2 ? "budget (device check)" : "divergence (device check)";
            esc_log_.push_back(e);
        }
        current_state_ = static_cast<hsps::AdaptiveState>(st.state_used);
        return stats.converged;
    }

    // The 24 features of MatrixFeatures::to_feature_vector and the initial state.
    std::vector<double> feature_vector(const hsps::SparseMatrix& A, hsps::AdaptiveState* init = nullptr) {
        Device& d = Device::get();
        std::vector<double> f(24);
        int32_t s = 0;
        check(hamlss_extract_features(d.ctx(), d.matrix(A), f.data(), &s));
        if (init) *init = static_cast<hsps::AdaptiveState>(s);
        return f;
    }

    hsps::AdaptiveState select_initial_state(const hsps::SparseMatrix& A) {
        hsps::AdaptiveState s;
        feature_vector(A, &s);
        return s;
    }

    // Same rule as the project's should_escalate (adaptive_selector.cpp:238-267).
    bool should_escalate(hsps::AdaptiveState st, int iteration, hsps::Real now,
                         const std::vector<hsps::Real>& hist) const {
        const int w = params_.stall_window;
        if (hist.size() >= 2 && now > 10.0 * hist[0]) return true;
        if ((int)hist.size() >= w) {
            hsps::Real prev = hist[hist.size() - w];
            if (prev > hsps::REAL_EPS && now / prev > params_.stall_threshold) return true;
        }
        if (st == hsps::AdaptiveState::EASY && iteration > params_.max_iter * 4 / 10) return true;
        if (st == hsps::AdaptiveState::MODERATE && iteration > params_.max_iter * 7 / 10) return true;
        return false;
    }

    const std::vector<hsps::EscalationRecord>& escalation_log() const { return esc_log_; }
    hsps::AdaptiveState current_state() const { return current_state_; }
    void print_summary(std::ostream& os) const {
        os << "\n=== Adaptive Selector Summary (device) ===\n"
           << "  Final state     : " << hsps::to_string(current_state_) << "\n"
           << "  Escalations     : " << esc_log_.size() << "\n";
        for (size_t i = 0; i < esc_log_.size(); ++i)
            os << "  [" << i << "] iter " << esc_log_[i].at_iteration << "  "
               << hsps::to_string(esc_log_[i].from_state) << " -> "
               << hsps::to_string(esc_log_[i].to_state) << "  rel_res="
               << esc_log_[i].residual_at_escalation << "\n";
    }

    // Engine options: 1 = escalate on the device-side stall / budget / divergence test.
    void set_ladder_mode(int m) { ladder_mode_ = m; }
    void set_precision(int prec) { precision_ = prec; }

private:
    hsps::SolverParams params_;
    hsps::AdaptiveState current_state_ = hsps::AdaptiveState::EASY;
    std::vector<hsps::EscalationRecord> esc_log_;
    int ladder_mode_ = 0;
    int precision_ = HAMLSS_FP64;
};

}  // namespace hsps_b200
