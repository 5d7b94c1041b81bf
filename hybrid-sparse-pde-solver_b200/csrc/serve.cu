// serve.cu -- the continuous-batching request loop behind hamlss_server_* (hamlss.h).
//
// The reference has no serving layer: every solve is one synchronous SolverBase::solve or
// AdaptiveSelector::solve call (include/solvers/solver_base.hpp:32-35,
// src/adaptive/adaptive_selector.cpp:298-394).  The server keeps the same per-request
// algorithm (the adaptive CG+Jacobi -> FGMRES+ILU(0) -> FGMRES+AMG ladder) and adds:
//
//   admission   a request is admitted once its estimated device footprint fits the HBM
//               budget next to the requests already admitted; one that can never fit is
//               refused at submit time (HAMLSS_ERR_BUDGET).  Queue order (config.order):
//               0 (default) arrival order, where a request that fits may pass a head that
//               does not, at most kMaxBypass times; 1 fewest nonzeros first -- the least
//               work first, which keeps the median latency down under steady load but
//               leaves the largest requests to the end of a burst -- where a request passed
//               kMaxAgeBypass times leads and is passed by nobody.  In both orders at most
//               max_large requests of large_rows rows or more run at once (default 1):
//               under processor sharing a large solve next to three others runs several
//               times slower and sets the tail latency, while the requests that pass the
//               waiting large one are short.
//   solve lanes `slots` worker threads, each with its own engine context (its own CUDA
//               stream), take admitted requests and run the adaptive ladder on them; their
//               kernels overlap on the device.
//   coalescing  small requests (n <= batch_max_rows) go to the batch lane instead: each time
//               the lane is free it takes every queued small request that shares the head's
//               tolerance (up to batch_max_count) and solves them in ONE persistent launch
//               (hamlss_batch_*), FP32 inner iterations inside FP64 refinement to the request's
//               tolerance.  Symmetric systems with a positive diagonal run CG + Jacobi, the
//               rest FGMRES + ILU(0): the ladder's first two rungs.  A system that fails there
//               escalates to a solve lane and runs the full ladder.
//
// Requests that arrive while others are on the device are queued and admitted as lanes
// and budget free up.  A request's result does not depend on what else is in flight: the
// batch kernel's arithmetic depends only on the system and its size class, and the solve
// lanes run the same deterministic code as a lone hamlss_solve_adaptive call.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"

namespace {

constexpr int kMaxBypass = 8;           // how often queued requests may pass the head
constexpr int kMaxAgeBypass = 32;       // fewest-nonzeros order: passes before a request leads
constexpr int kBatchMaxRestart = 32;    // the batch kernel's FGMRES restart limit

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int fail(int code, const std::string& m) { return hamlss::set_last_error(code, m); }

enum class St { Queued, Running, Done };

struct Request {
    int64_t id = 0;
    int32_t n = 0, nnz = 0;
    const int32_t* rp = nullptr;
    const int32_t* ci = nullptr;
    const double* v = nullptr;
    const double* b = nullptr;
    double* x = nullptr;
    hamlss_params p{};
    int64_t footprint = 0;
    bool small = false;         // goes to the batch lane first
    bool spd_like = false;      // symmetric with a positive diagonal
    bool escalated = false;     // failed in the batch lane, re-queued for a solve lane
    bool coalesced = false;     // finished in the batch lane
    int bypassed = 0;
    St state = St::Queued;
    int status = HAMLSS_OK;
    std::string err;
    hamlss_stats stats{};
    double t_submit = 0.0, t_done = 0.0;
};

// Device footprint of one request while it is admitted (bytes, an upper estimate):
// CSR (int32 row_ptr + int32 col_idx + FP64 values), its FP32 copy and the diagonal;
// Krylov workspace (eight FP64 and eight FP32 vectors, the FGMRES basis V and Z of
// 2m+1 vectors); ILU(0) factors plus level-ordered L and U copies; an AMG hierarchy
// (operators of the coarse levels, P and R) bounded by twice the fine operator.
int64_t footprint_of(int64_t n, int64_t nnz, int m) {
    const int64_t csr = 4 * (n + 1) + 12 * nnz;
    const int64_t f32 = 4 * nnz + 8 * n;
    const int64_t ws = 8 * 8 * n + 8 * 4 * n + (int64_t)(2 * m + 1) * 8 * n + 64 * 1024;
    const int64_t ilu = 8 * nnz + 2 * (12 * nnz + 4 * n) + 16 * n;
    const int64_t amg = 2 * (csr + f32) + 4 * 8 * n;
    return csr + f32 + 8 * n + ws + std::max(ilu, amg) + (1 << 20);
}

// Footprint of a request solved in the batch lane: the block's share of the batch's
// CSR (FP64 + FP32), factors, level sets and per-system vectors.
int64_t footprint_small(int64_t n, int64_t nnz, int m) {
    return 4 * (n + 1) + 12 * nnz + 4 * nnz + 8 * nnz + 16 * n + 8 * n * (2 * m + 12) + 4096;
}

// Symmetric values and a positive diagonal (columns sorted within each row).
bool spd_like(int n, const int32_t* rp, const int32_t* ci, const double* v) {
    for (int i = 0; i < n; ++i) {
        bool diag = false;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            if (j == i) {
                if (!(v[k] > 0.0)) return false;
                diag = true;
                continue;
            }
            const int32_t* lo = ci + rp[j];
            const int32_t* hi = ci + rp[j + 1];
            const int32_t* it = std::lower_bound(lo, hi, i);
            if (it == hi || *it != i || v[it - ci] != v[k]) return false;
        }
        if (!diag) return false;
    }
    return true;
}

bool same_batch_key(const hamlss_params& a, const hamlss_params& b) {
    return a.tol == b.tol && a.max_iter == b.max_iter && a.ir_max_outer == b.ir_max_outer &&
           a.ir_inner_tol == b.ir_inner_tol && a.ir_update == b.ir_update &&
           std::min(a.restart_size, kBatchMaxRestart) == std::min(b.restart_size, kBatchMaxRestart);
}

}  // namespace

struct hamlss_server {
    hamlss_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work;   // lanes wait for work or budget
    std::condition_variable cv_done;   // callers wait for results
    std::deque<Request*> big_q, small_q;
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    int64_t next_id = 1;
    int64_t admitted = 0, peak_admitted = 0;
    int running = 0, peak_running = 0;
    int running_large = 0;              // admitted requests with n >= cfg.large_rows
    bool stop = false;
    std::vector<hamlss_ctx*> ctxs;
    std::vector<std::thread> threads;
    // report counters
    int64_t n_submitted = 0, n_completed = 0, n_failed = 0, n_cancelled = 0;
    int64_t n_coalesced = 0, n_batches = 0, n_escalated = 0, n_fallback = 0;
    std::vector<double> latencies;
    double t_first = -1.0, t_last = 0.0;

    bool is_large(const Request* r) const { return r->n >= cfg.large_rows; }
    // a large request waits while max_large of them run (others may pass it meanwhile)
    bool large_blocked(const Request* r) const {
        return cfg.max_large > 0 && is_large(r) && running_large >= cfg.max_large;
    }

    // ---- queue selection (mu held)
    Request* pick(std::deque<Request*>& q) {
        if (cfg.order == 1 && !q.empty()) {
            // fewest nonzeros first (the least work first keeps the median latency low when
            // the lanes are busy); a request passed kMaxAgeBypass times goes first, and while
            // it does not fit nobody passes it
            Request* h = q.front();
            if (h->bypassed >= kMaxAgeBypass && !large_blocked(h)) {
                if (admitted + h->footprint > cfg.hbm_budget_bytes) return nullptr;
                q.pop_front();
                admit(h);
                return h;
            }
            long best = -1;
            for (size_t i = 0; i < q.size(); ++i)
                if (admitted + q[i]->footprint <= cfg.hbm_budget_bytes && !large_blocked(q[i]) &&
                    (best < 0 || q[i]->nnz < q[(size_t)best]->nnz))
                    best = (long)i;
            if (best < 0) return nullptr;
            for (long j = 0; j < best; ++j) ++q[(size_t)j]->bypassed;
            Request* r = q[(size_t)best];
            q.erase(q.begin() + best);
            admit(r);
            return r;
        }
        Request* head = nullptr;          // the first request not held by max_large
        for (size_t i = 0; i < q.size(); ++i) {
            Request* r = q[i];
            if (large_blocked(r)) continue;
            if (admitted + r->footprint <= cfg.hbm_budget_bytes) {
                if (head) ++head->bypassed;
                q.erase(q.begin() + (long)i);
                admit(r);
                return r;
            }
            if (!head && r->bypassed >= kMaxBypass) return nullptr;  // head waits, nobody passes
            if (!head) head = r;
        }
        return nullptr;
    }
    void admit(Request* r) {
        if (is_large(r)) ++running_large;
        admitted += r->footprint;
        peak_admitted = std::max(peak_admitted, admitted);
        r->state = St::Running;
        ++running;
        peak_running = std::max(peak_running, running);
    }
    void retire(Request* r, bool requeue) {
        if (is_large(r)) --running_large;
        admitted -= r->footprint;
        --running;
        if (requeue) {
            r->state = St::Queued;
            r->footprint = footprint_of(r->n, r->nnz, r->p.restart_size);
            big_q.push_front(r);     // escalations go first: they have waited already
        } else {
            r->state = St::Done;
            r->t_done = now_s();
            t_last = std::max(t_last, r->t_done);
            if (r->status == HAMLSS_OK) {
                ++n_completed;
                latencies.push_back(r->t_done - r->t_submit);
            } else {
                ++n_failed;
            }
            if (r->coalesced) ++n_coalesced;
            cv_done.notify_all();
        }
        cv_work.notify_all();
    }

    void solve_lane(hamlss_ctx* ctx);
    void batch_lane(hamlss_ctx* ctx);
};

// A solve lane: one engine context, one request at a time through the adaptive ladder.
void hamlss_server::solve_lane(hamlss_ctx* ctx) {
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] { return stop || (r = pick(big_q)) != nullptr; });
            if (!r) return;
        }
        hamlss_mat* A = nullptr;
        hamlss_stats st;
        std::memset(&st, 0, sizeof(st));
        std::vector<double> x0(r->x, r->x + r->n);
        int rc = hamlss_mat_upload(ctx, r->n, r->n, r->nnz, r->rp, r->ci, r->v, HAMLSS_HOST, &A);
        int init = 0;
        bool fell_back = false;
        if (rc == HAMLSS_OK) {
            int nlog = 0;
            rc = hamlss_solve_adaptive(ctx, A, r->b, r->x, HAMLSS_HOST, &r->p, &st, nullptr, 0,
                                       &nlog, &init);
        }
        // The ladder climbs from the state the features pick; when it fails at the top (no
        // convergence, or a preconditioner that could not be set up), try the rungs below
        // that it skipped (FGMRES + ILU(0), then CG + Jacobi for symmetric systems with a
        // positive diagonal), each from the original x0.
        const bool setup_failed = A && (rc == HAMLSS_ERR_NOMEM || rc == HAMLSS_ERR_ZERO_PIVOT ||
                                        rc == HAMLSS_ERR_TIMEOUT || rc == HAMLSS_ERR_ZERO_DIAG);
        if (setup_failed) {
            rc = HAMLSS_OK;
            st.converged = 0;
            std::memcpy(r->x, x0.data(), sizeof(double) * r->n);
        }
        for (int state = init - 1; rc == HAMLSS_OK && !st.converged && state >= 0; --state) {
            if (state == HAMLSS_STATE_EASY && !spd_like(r->n, r->rp, r->ci, r->v)) continue;
            const int kind = state == HAMLSS_STATE_EASY ? HAMLSS_PREC_JACOBI : HAMLSS_PREC_ILU;
            const int solver = state == HAMLSS_STATE_EASY ? HAMLSS_SOLVER_CG : HAMLSS_SOLVER_FGMRES;
            hamlss_prec* M = nullptr;
            double setup = 0.0;
            hamlss_params q = r->p;
            q.fill_per_row = 0;              // the ladder's factory-made ILU (drop_tol only)
            if (hamlss_precond_setup(ctx, A, kind, &q, &M, &setup) != HAMLSS_OK) continue;
            std::vector<double> x(x0);
            hamlss_stats s2;
            std::memset(&s2, 0, sizeof(s2));
            const int rc2 = hamlss_solve(ctx, solver, A, M, r->b, x.data(), HAMLSS_HOST, &r->p, &s2);
            hamlss_precond_release(M);
            if (rc2 == HAMLSS_OK && s2.converged) {
                std::memcpy(r->x, x.data(), sizeof(double) * r->n);
                s2.setup_time_s = setup;
                s2.state_used = state;
                s2.iterations += st.iterations;       // work spent on the failed ladder too
                st = s2;
                fell_back = true;
            }
        }
        std::string msg = rc == HAMLSS_OK ? std::string() : std::string(hamlss_last_error());
        if (A) hamlss_mat_release(A);
        std::lock_guard<std::mutex> g(mu);
        if (fell_back) ++n_fallback;
        r->status = rc;
        r->err = msg;
        r->stats = st;
        r->stats.status = rc;
        retire(r, false);
    }
}

// The batch lane: every free moment, coalesce the queued small requests into one launch.
void hamlss_server::batch_lane(hamlss_ctx* ctx) {
    std::vector<int32_t> row_off, rp, ci, solver, precond;
    std::vector<double> v, bb, xb;
    for (;;) {
        std::vector<Request*> take;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_work.wait(lk, [&] {
                if (stop) return true;
                if (small_q.empty()) return false;
                const hamlss_params key = small_q.front()->p;
                for (size_t i = 0; i < small_q.size() && (int)take.size() < cfg.batch_max_count;) {
                    Request* r = small_q[i];
                    if (!same_batch_key(r->p, key) ||
                        admitted + r->footprint > cfg.hbm_budget_bytes) {
                        ++i;
                        continue;
                    }
                    small_q.erase(small_q.begin() + (long)i);
                    admit(r);
                    take.push_back(r);
                }
                return !take.empty();
            });
            if (take.empty()) return;
            ++n_batches;
        }
        // block-diagonal CSR of the taken systems (global rows and columns)
        const int cnt = (int)take.size();
        row_off.assign(cnt + 1, 0);
        int64_t N = 0, NZ = 0;
        for (int k = 0; k < cnt; ++k) {
            N += take[k]->n;
            NZ += take[k]->nnz;
            row_off[k + 1] = (int32_t)N;
        }
        rp.resize(N + 1);
        ci.resize(NZ);
        v.resize(NZ);
        bb.resize(N);
        xb.resize(N);
        solver.resize(cnt);
        precond.resize(cnt);
        int64_t nz0 = 0;
        for (int k = 0; k < cnt; ++k) {
            const Request* r = take[k];
            const int32_t r0 = row_off[k];
            for (int i = 0; i < r->n; ++i) rp[r0 + i] = (int32_t)(r->rp[i] + nz0);
            for (int e = 0; e < r->nnz; ++e) ci[nz0 + e] = r->ci[e] + r0;
            std::memcpy(v.data() + nz0, r->v, sizeof(double) * r->nnz);
            std::memcpy(bb.data() + r0, r->b, sizeof(double) * r->n);
            std::memcpy(xb.data() + r0, r->x, sizeof(double) * r->n);
            solver[k] = r->spd_like ? HAMLSS_SOLVER_CG : HAMLSS_SOLVER_FGMRES;
            precond[k] = r->spd_like ? HAMLSS_PREC_JACOBI : HAMLSS_PREC_ILU;
            nz0 += r->nnz;
        }
        rp[N] = (int32_t)NZ;
        hamlss_params p = take[0]->p;
        p.restart_size = std::min(p.restart_size, kBatchMaxRestart);
        hamlss_batch* B = nullptr;
        std::vector<hamlss_batch_result> res(cnt);
        hamlss_stats tot;
        std::memset(&tot, 0, sizeof(tot));
        const double t0 = now_s();
        int rc = hamlss_batch_create(ctx, cnt, row_off.data(), rp.data(), ci.data(), v.data(),
                                     solver.data(), precond.data(), HAMLSS_HOST, &p, &B);
        if (rc == HAMLSS_OK)
            rc = hamlss_batch_solve(ctx, B, bb.data(), xb.data(), HAMLSS_HOST, res.data(), &tot);
        const double wall = now_s() - t0;
        if (B) hamlss_batch_release(B);
        std::lock_guard<std::mutex> g(mu);
        for (int k = 0; k < cnt; ++k) {
            Request* r = take[k];
            const hamlss_batch_result& o = res[k];
            if (rc != HAMLSS_OK || o.status != HAMLSS_OK || !o.converged) {
                r->escalated = true;
                ++n_escalated;
                retire(r, true);
                continue;
            }
            std::memcpy(r->x, xb.data() + row_off[k], sizeof(double) * r->n);
            hamlss_stats& s = r->stats;
            std::memset(&s, 0, sizeof(s));
            s.iterations = o.iterations;
            s.outer_iterations = o.outer_iterations;
            s.initial_residual = o.initial_residual;
            s.final_residual = o.final_residual;
            s.true_residual = o.final_residual;
            s.converged = 1;
            s.solve_time_s = wall;
            s.device_time_s = tot.device_time_s;
            s.solver_used = solver[k];
            s.precond_used = precond[k];
            s.state_used = r->spd_like ? HAMLSS_STATE_EASY : HAMLSS_STATE_MODERATE;
            r->coalesced = true;
            r->status = HAMLSS_OK;
            retire(r, false);
        }
    }
}

extern "C" {

void hamlss_server_config_default(hamlss_server_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->device = 0;
    c->slots = 4;
    c->hbm_budget_bytes = 150LL * 1000 * 1000 * 1000;
    c->batch_max_rows = 16384;
    c->batch_max_count = 2048;
    c->order = 0;
    c->large_rows = 1 << 20;
    c->max_large = 1;
}

int hamlss_server_create(const hamlss_server_config* config, hamlss_server** out) {
    if (!out) return fail(HAMLSS_ERR_INVALID, "null argument");
    *out = nullptr;
    hamlss_server_config c;
    if (config) c = *config;
    else hamlss_server_config_default(&c);
    if (c.slots < 1 || c.slots > 64) return fail(HAMLSS_ERR_INVALID, "slots must be in [1, 64]");
    if (c.order != 0 && c.order != 1) return fail(HAMLSS_ERR_INVALID, "order must be 0 or 1");
    if (c.large_rows < 1 || c.max_large < 0)
        return fail(HAMLSS_ERR_INVALID, "large_rows >= 1 and max_large >= 0");
    if (c.hbm_budget_bytes <= 0) return fail(HAMLSS_ERR_INVALID, "hbm_budget_bytes must be > 0");
    if (c.batch_max_rows < 0 || (c.batch_max_rows > 0 && c.batch_max_count < 1))
        return fail(HAMLSS_ERR_INVALID, "batch_max_rows >= 0 and batch_max_count >= 1");
    auto* s = new hamlss_server();
    s->cfg = c;
    const int nctx = c.slots + (c.batch_max_rows > 0 ? 1 : 0);
    for (int i = 0; i < nctx; ++i) {
        hamlss_ctx* h = nullptr;
        int rc = hamlss_ctx_create(c.device, &h);
        if (rc != HAMLSS_OK) {
            std::string m = hamlss_last_error();
            for (auto* x : s->ctxs) hamlss_ctx_destroy(x);
            delete s;
            return fail(rc, m);
        }
        s->ctxs.push_back(h);
    }
    for (int i = 0; i < c.slots; ++i)
        s->threads.emplace_back([s, i] { s->solve_lane(s->ctxs[i]); });
    if (c.batch_max_rows > 0)
        s->threads.emplace_back([s, nctx] { s->batch_lane(s->ctxs[nctx - 1]); });
    *out = s;
    return HAMLSS_OK;
}

int hamlss_server_submit(hamlss_server* s, int32_t n, int32_t nnz, const int32_t* row_ptr,
                         const int32_t* col_idx, const double* values, const double* b, double* x,
                         const hamlss_params* params, int64_t* request_id) {
    if (!s || !row_ptr || !col_idx || !values || !b || !x || !request_id)
        return fail(HAMLSS_ERR_INVALID, "null argument");
    if (n <= 0 || nnz < 0 || row_ptr[0] != 0 || row_ptr[n] != nnz)
        return fail(HAMLSS_ERR_MALFORMED, "row_ptr must run from 0 to nnz over n rows");
    auto r = std::make_unique<Request>();
    r->n = n;
    r->nnz = nnz;
    r->rp = row_ptr;
    r->ci = col_idx;
    r->v = values;
    r->b = b;
    r->x = x;
    if (params) r->p = *params;
    else hamlss_params_default(&r->p);
    r->small = s->cfg.batch_max_rows > 0 && n <= s->cfg.batch_max_rows;
    if (r->small) {
        for (int i = 0; i < n; ++i)
            if (row_ptr[i + 1] < row_ptr[i])
                return fail(HAMLSS_ERR_MALFORMED, "row_ptr is not monotone");
        for (int32_t e = 0; e < nnz; ++e)
            if (col_idx[e] < 0 || col_idx[e] >= n)
                return fail(HAMLSS_ERR_MALFORMED, "column index out of range");
        r->spd_like = spd_like(n, row_ptr, col_idx, values);
        r->footprint = footprint_small(n, nnz, std::min(r->p.restart_size, kBatchMaxRestart));
    } else {
        r->footprint = footprint_of(n, nnz, r->p.restart_size);
    }
    const int64_t big = footprint_of(n, nnz, r->p.restart_size);
    if (big > s->cfg.hbm_budget_bytes)
        return fail(HAMLSS_ERR_BUDGET, "request needs an estimated " + std::to_string(big) +
                                           " bytes, more than the server's HBM budget");
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) return fail(HAMLSS_ERR_CANCELLED, "server is shutting down");
    r->id = s->next_id++;
    r->t_submit = now_s();
    if (s->t_first < 0) s->t_first = r->t_submit;
    ++s->n_submitted;
    *request_id = r->id;
    Request* raw = r.get();
    s->reqs[r->id] = std::move(r);
    (raw->small ? s->small_q : s->big_q).push_back(raw);
    s->cv_work.notify_all();
    return HAMLSS_OK;
}

int hamlss_server_wait(hamlss_server* s, int64_t id, double timeout_s, hamlss_stats* stats) {
    if (!s) return fail(HAMLSS_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(HAMLSS_ERR_INVALID, "unknown request id");
    Request* r = it->second.get();
    auto done = [&] { return r->state == St::Done; };
    if (timeout_s < 0) s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done))
        return fail(HAMLSS_ERR_TIMEOUT, "request still in flight");
    if (stats) *stats = r->stats;
    const int rc = r->status;
    std::string msg = r->err;
    s->reqs.erase(it);
    if (rc != HAMLSS_OK) return fail(rc, msg.empty() ? "request failed" : msg);
    return HAMLSS_OK;
}

int hamlss_server_test(hamlss_server* s, int64_t id, int32_t* done) {
    if (!s || !done) return fail(HAMLSS_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(HAMLSS_ERR_INVALID, "unknown request id");
    *done = it->second->state == St::Done ? 1 : 0;
    return HAMLSS_OK;
}

int hamlss_server_cancel(hamlss_server* s, int64_t id) {
    if (!s) return fail(HAMLSS_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(HAMLSS_ERR_INVALID, "unknown request id");
    Request* r = it->second.get();
    if (r->state != St::Queued) return fail(HAMLSS_ERR_INVALID, "request already running or done");
    for (auto* q : {&s->big_q, &s->small_q}) {
        auto pos = std::find(q->begin(), q->end(), r);
        if (pos != q->end()) q->erase(pos);
    }
    r->state = St::Done;
    r->status = HAMLSS_ERR_CANCELLED;
    r->err = "cancelled before it ran";
    r->stats.status = HAMLSS_ERR_CANCELLED;
    ++s->n_cancelled;
    s->cv_done.notify_all();
    s->cv_work.notify_all();
    return HAMLSS_OK;
}

int hamlss_server_get_report(hamlss_server* s, hamlss_server_report* rep) {
    if (!s || !rep) return fail(HAMLSS_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    std::memset(rep, 0, sizeof(*rep));
    rep->submitted = s->n_submitted;
    rep->completed = s->n_completed;
    rep->failed = s->n_failed;
    rep->cancelled = s->n_cancelled;
    rep->coalesced = s->n_coalesced;
    rep->batches = s->n_batches;
    rep->escalated = s->n_escalated;
    rep->fallback = s->n_fallback;
    rep->queued = (int64_t)(s->big_q.size() + s->small_q.size());
    rep->running = s->running;
    rep->peak_running = s->peak_running;
    rep->admitted_bytes = s->admitted;
    rep->peak_admitted_bytes = s->peak_admitted;
    if (!s->latencies.empty()) {
        std::vector<double> l = s->latencies;
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) {
            // nearest-rank percentile
            size_t k = (size_t)std::ceil(q * (double)l.size());
            return l[std::min(l.size() - 1, k ? k - 1 : 0)];
        };
        double sum = 0.0;
        for (double t : l) sum += t;
        rep->p50_latency_s = pct(0.50);
        rep->p99_latency_s = pct(0.99);
        rep->mean_latency_s = sum / (double)l.size();
        rep->max_latency_s = l.back();
        const double span = s->t_last - s->t_first;
        rep->solves_per_s = span > 0 ? (double)s->n_completed / span : 0.0;
    }
    return HAMLSS_OK;
}

int hamlss_server_reset_report(hamlss_server* s) {
    if (!s) return fail(HAMLSS_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    s->n_submitted = s->n_completed = s->n_failed = s->n_cancelled = 0;
    s->n_coalesced = s->n_batches = s->n_escalated = s->n_fallback = 0;
    s->latencies.clear();
    s->t_first = -1.0;
    s->t_last = 0.0;
    s->peak_admitted = s->admitted;
    s->peak_running = s->running;
    return HAMLSS_OK;
}

int hamlss_server_destroy(hamlss_server* s) {
    if (!s) return HAMLSS_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        for (auto* q : {&s->big_q, &s->small_q}) {
            for (Request* r : *q) {
                r->state = St::Done;
                r->status = HAMLSS_ERR_CANCELLED;
                r->err = "server destroyed before the request ran";
            }
            q->clear();
        }
        s->cv_work.notify_all();
        s->cv_done.notify_all();
    }
    for (auto& t : s->threads) t.join();
    for (auto* c : s->ctxs) hamlss_ctx_destroy(c);
    delete s;
    return HAMLSS_OK;
}

}  // extern "C"
