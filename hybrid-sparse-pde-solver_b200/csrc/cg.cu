// cg.cu -- preconditioned CG on the device (CGSolver::solve, cg_solver.cpp:37-191).
//
// One CG trip of the reference = 1 SpMV, 3 dots, 3 axpy, M^-1.  Here it is two fused
// launches with Jacobi, three plus M^-1 otherwise:
//   K1  q = A p with p = z + beta p_old formed on the fly (p written for own rows), p.q
//   K2  x += alpha p, r -= alpha q, ||r||^2 (and for Jacobi z = D^-1 r, r.z)
//   [M^-1 r -> z ; K3 r.z]                      (non-Jacobi preconditioners)
// All scalars (rho, alpha, beta, rel) live in device memory; the last block of each
// reduction computes them, including the reference's convergence test on the recursive
// residual (:133, :143) and both breakdown restarts (:109-120, :157-167).  The host only
// polls the state once per chunk of trips.  Element updates use separate multiply and
// add in FP64, in the reference's operand order, so only the dot summation order differs.
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "krylov.cuh"

namespace hamlss {

namespace {

constexpr double kEps = 2.220446049250313e-16;

struct CgState {
    double bnorm, r0, rel, tol, rho, rho_old, alpha, beta, pq;
    int iter, max_iter, halt, status, restart_kind, early;
    int halt_stage;     // launch of the trip that set halt: 1 = K1, 2 = K2, 3 = K3
                        // (reliable-update PCG: 3 = the update, 4 = K3)
    // reliable-update PCG (mixed precision) only
    double scale;       // 1 / ||b||: the FP32 vectors hold r / ||b|| and the FP32 iterate
    double rmax;        // largest recursive relative residual since the last update
    double delta;       // update when the residual fell below delta * rmax
    int skip_ru;        // gate of the update launches: 0 only in a trip that updates
    int ru_final;       // the pending update confirms the stop test
    unsigned long long ru_mask;   // bit (iter % 64) of each trip whose update ran
    LadderDev lad;
};

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }

// ---------------------------------------------------------------- init: r = b - A x
template <typename T>
struct EpiInitRes {
    const T* b;
    T* r;
    HAMLSS_NO_LOAD
    __device__ __forceinline__ void prefetch(int r0, int r1) const { l2_prefetch_rows(b, r0, r1); }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        double bi = (double)b[i];
        T ri = (T)__dsub_rn(bi, ax);
        r[i] = ri;
        acc[0] += bi * bi;
        acc[1] += (double)ri * (double)ri;
    }
};

struct FinInit {
    CgState* s;
    bool first;   // false for a breakdown restart: keep bnorm and the initial residual
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        if (!first) return;
        double bn = sqrt(t[0]), r0 = sqrt(t[1]);
        s->bnorm = bn;
        s->r0 = r0;
        if (!isfinite(bn) || !isfinite(r0)) { s->status = ST_NONFINITE; s->halt = 1; return; }
        if (bn < kEps) { s->status = ST_CONV; s->early = 1; s->rel = r0; s->halt = 1; return; }
        double rel = r0 / bn;
        s->rel = rel;
        if (rel < s->tol) { s->status = ST_CONV; s->early = 2; s->halt = 1; }
    }
};

// ------------------------------------------------------- rho = r.z after (re)start
template <typename T, bool JAC>
struct BodyRho {
    const T* r;
    const T* z;      // unused for JAC
    const T* dinv;   // JAC only
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&acc)[NV]) const {
        double ri = (double)r[i];
        double zi = JAC ? (double)(T)dmul((double)dinv[i], ri) : (double)z[i];
        acc[0] += ri * zi;
    }
};

struct FinRho {
    CgState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        s->rho = t[0];
        s->rho_old = t[0];
        s->beta = 0.0;
    }
};

// ------------------------------------------------------------- K1: q = A p, p.q
template <typename T, bool JAC>
struct XP {
    const T* z;       // or r when JAC
    const T* dinv;
    const T* pold;
    const CgState* s;
    double beta;
    __device__ __forceinline__ void load() { beta = s->beta; }
    __device__ __forceinline__ T p(int j) const {
        double zj = JAC ? (double)(T)dmul((double)__ldg(&dinv[j]), (double)__ldg(&z[j]))
                        : (double)__ldg(&z[j]);
        return (T)dadd(zj, dmul(beta, (double)__ldg(&pold[j])));
    }
    __device__ __forceinline__ double operator()(int j) const { return (double)p(j); }
};

template <typename T, bool JAC>
struct EpiQ {
    XP<T, JAC> xp;
    T* pnew;
    T* q;
    __device__ __forceinline__ void load() { xp.load(); }
    // the rows' own z (or r), D^-1 and p_old: read by the gathers of the tile and by p_i
    __device__ __forceinline__ void prefetch(int r0, int r1) const {
        l2_prefetch_rows(xp.z, r0, r1);
        if (JAC) l2_prefetch_rows(xp.dinv, r0, r1);
        l2_prefetch_rows(xp.pold, r0, r1);
    }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        T pi = xp.p(i);
        T qi = (T)ax;
        pnew[i] = pi;
        q[i] = qi;
        acc[0] += (double)pi * (double)qi;
    }
};

struct FinPQ {
    CgState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        double pq = t[0];
        s->pq = pq;
        if (fabs(pq) < kEps * 1e6 * fabs(s->rho)) {
            s->iter += 1;
            if (s->iter >= s->max_iter) s->status = ST_MAXIT;
            else { s->status = ST_RESTART; s->restart_kind = 1; }
            s->halt = 1;
            s->halt_stage = 1;
            return;
        }
        s->alpha = s->rho / pq;
    }
};

// --------------------------------------- K2: x += a p, r -= a q, |r|^2 (+ Jacobi r.z)
template <typename T, bool JAC>
struct BodyUpd {
    T* x;
    T* r;
    const T* p;
    const T* q;
    const T* dinv;
    const CgState* s;
    double alpha;
    __device__ __forceinline__ void load() { alpha = s->alpha; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&acc)[NV]) const {
        x[i] = (T)dadd((double)x[i], dmul(alpha, (double)p[i]));
        T ri = (T)dadd((double)r[i], dmul(-alpha, (double)q[i]));
        r[i] = ri;
        double rd = (double)ri;
        acc[0] += rd * rd;
        if constexpr (JAC) {
            double zi = (double)(T)dmul((double)dinv[i], rd);
            acc[1] += rd * zi;
        }
    }
};

// rho update + second breakdown check + trip accounting (shared by K2/JAC and K3)
__device__ __forceinline__ void rho_step(CgState* s, double rz, int stage) {
    double rho_old = s->rho;
    s->rho_old = rho_old;
    s->rho = rz;
    if (fabs(rho_old) < kEps * 1e8 * fabs(rz)) {
        s->iter += 1;
        if (s->iter >= s->max_iter) s->status = ST_MAXIT;
        else { s->status = ST_RESTART; s->restart_kind = 2; }
        s->halt = 1;
        s->halt_stage = stage;
        return;
    }
    s->beta = rz / rho_old;
    s->iter += 1;
    if (s->iter >= s->max_iter) { s->status = ST_MAXIT; s->halt = 1; s->halt_stage = stage; }
}

template <bool JAC>
struct FinUpd {
    CgState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        double rel = sqrt(t[0]) / s->bnorm;
        s->rel = rel;
        int st = ST_RUN;
        if (rel < s->tol) st = ST_CONV;
        else if (!isfinite(rel)) st = ST_NONFINITE;
        else if (ladder_check(&s->lad, s->iter, rel)) st = ST_ESCALATE;
        if (st != ST_RUN) { s->iter += 1; s->status = st; s->halt = 1; s->halt_stage = 2; return; }
        if constexpr (JAC) rho_step(s, t[1], 2);
    }
};

template <typename T>
struct BodyRz {
    const T* r;
    const T* z;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&acc)[NV]) const {
        acc[0] += (double)r[i] * (double)z[i];
    }
};

struct FinRz {
    CgState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const { rho_step(s, t[0], 3); }
};

template <typename T>
struct BodyFill {
    T* a;
    T val;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const { a[i] = val; }
};

template <typename T>
Csr<T> csr_of(Ctx& ctx, hamlss_mat* A);
template <>
Csr<double> csr_of<double>(Ctx&, hamlss_mat* A) { return A->A.f64(); }
template <>
Csr<float> csr_of<float>(Ctx& ctx, hamlss_mat* A) { return A->A.f32(ctx.lane.stream); }

template <typename T>
T* wvec(Workspace& ws, int k, size_t n);
template <>
double* wvec<double>(Workspace& ws, int k, size_t n) { ws.d[k].ensure(n); return ws.d[k].p; }
template <>
float* wvec<float>(Workspace& ws, int k, size_t n) { ws.f[k].ensure(n); return ws.f[k].p; }

template <typename T>
const T* jacobi_diag(Ctx& ctx, Prec* M);
template <>
const double* jacobi_diag<double>(Ctx&, Prec* M) { return static_cast<JacobiPrec*>(M)->inv.p; }
template <>
const float* jacobi_diag<float>(Ctx& ctx, Prec* M) {
    auto* J = static_cast<JacobiPrec*>(M);
    J->prepare32(ctx);
    return J->inv32.p;
}

template <typename T>
void precond_apply(Ctx& ctx, Prec* M, const T* r, T* z, const int* gate);
template <>
void precond_apply<double>(Ctx& ctx, Prec* M, const double* r, double* z, const int* gate) {
    M->apply(ctx, ctx.lane, r, z, gate);
}
template <>
void precond_apply<float>(Ctx& ctx, Prec* M, const float* r, float* z, const int* gate) {
    M->apply32(ctx, ctx.lane, r, z, gate);
}

template <typename T, bool JAC>
SolveResult cg_impl(Ctx& ctx, hamlss_mat* A, Prec* M, const T* b, T* x, double tol,
                    int max_iter, int check_every, Workspace& ws, const LadderCfg* lad) {
    const int n = A->A.n;
    const Lane& L = ctx.lane;
    const int sm = ctx.sm_count;
    cudaStream_t st = L.stream;
    Csr<T> Ad = csr_of<T>(ctx, A);
    T* r = wvec<T>(ws, 0, n);
    T* z = M && !JAC ? wvec<T>(ws, 1, n) : r;     // no preconditioner: z aliases r
    T* p[2] = {wvec<T>(ws, 2, n), wvec<T>(ws, 3, n)};
    T* q = wvec<T>(ws, 4, n);
    const T* dinv = JAC ? jacobi_diag<T>(ctx, M) : nullptr;
    const double wb = (double)sizeof(T) * n;     // bytes of one vector
    ws.state.ensure(sizeof(CgState));
    CgState* s = reinterpret_cast<CgState*>(ws.state.p);
    int* halt = &s->halt;

    CgState h0{};
    h0.tol = tol;
    h0.max_iter = max_iter;
    h0.lad = ladder_init(lad);
    HAMLSS_CUDA(cudaMemcpyAsync(s, &h0, sizeof(CgState), cudaMemcpyHostToDevice, st));
    launch_vec<0>(sm, L, n, BodyFill<T>{p[0], T(0)});
    launch_vec<0>(sm, L, n, BodyFill<T>{p[1], T(0)});
    HAMLSS_CUDA(cudaEventRecord(ctx.ev0, st));

    auto restart_seq = [&](bool first) {
        launch_spmv<T, 2>(sm, L, Ad, XVec<T>{x}, EpiInitRes<T>{b, r}, FinInit{s, first},
                          first ? nullptr : halt, "cg_residual", 3.0 * wb);
        if (!JAC && M) precond_apply<T>(ctx, M, r, z, halt);
        launch_vec<1>(sm, L, n, BodyRho<T, JAC>{r, z, dinv}, FinRho{s}, halt, "cg_dot", 2.0 * wb);
    };
    auto poll = [&](CgState& h) {
        HAMLSS_CUDA(cudaMemcpyAsync(ctx.host_poll.p, s, sizeof(CgState), cudaMemcpyDeviceToHost, st));
        HAMLSS_CUDA(cudaStreamSynchronize(st));
        std::memcpy(&h, ctx.host_poll.p, sizeof(CgState));
    };

    SolveResult res;
    CgState h{};
    restart_seq(true);
    poll(h);
    const bool run = !h.halt && max_iter > 0;
    int parity = 0;
    int chunk = std::max(1, check_every);
    // Launch positions of each trip in the engine profiler: its K1, K2, the rest, its end.
    struct TripMarks { size_t k1, k2, rest, end; };
    std::vector<TripMarks> trips;
    int poll_iter = h.iter;
    double poll_rel = h.rel;
    while (run) {
        const int iter0 = h.iter;
        trips.clear();
        for (int t = 0; t < chunk; ++t) {
            TripMarks tm;
            tm.k1 = prof_pos(L.prof);
            T* pold = p[parity];
            T* pnew = p[parity ^ 1];
            XP<T, JAC> xp{JAC ? r : z, dinv, pold, s, 0.0};
            launch_spmv<T, 1>(sm, L, Ad, xp, EpiQ<T, JAC>{xp, pnew, q}, FinPQ{s}, halt,
                              "cg_spmv", (JAC ? 5.0 : 4.0) * wb);
            tm.k2 = prof_pos(L.prof);
            launch_vec<JAC ? 2 : 1>(sm, L, n, BodyUpd<T, JAC>{x, r, pnew, q, dinv, s, 0.0},
                                    FinUpd<JAC>{s}, halt, "cg_update", (JAC ? 7.0 : 6.0) * wb);
            tm.rest = prof_pos(L.prof);
            if (!JAC) {
                if (M) precond_apply<T>(ctx, M, r, z, halt);
                launch_vec<1>(sm, L, n, BodyRz<T>{r, z}, FinRz{s}, halt, "cg_dot", 2.0 * wb);
            }
            tm.end = prof_pos(L.prof);
            trips.push_back(tm);
            parity ^= 1;
        }
        poll(h);
        if (h.halt) {
            // every trip increments iter once, the halting one included; the launches the
            // gate skipped are booked as "gated", with no bytes
            const int ran = std::max(1, std::min((int)trips.size(), h.iter - iter0));
            const TripMarks& last = trips[ran - 1];
            const size_t from = h.halt_stage == 1 ? last.k2 : h.halt_stage == 2 ? last.rest : last.end;
            prof_gated(L.prof, from, trips.back().end);
        }
        if (h.status == ST_RESTART) {
            res.restarts++;
            CgState hh = h;
            hh.status = ST_RUN;
            hh.halt = 0;
            hh.halt_stage = 0;
            HAMLSS_CUDA(cudaMemcpyAsync(s, &hh, sizeof(CgState), cudaMemcpyHostToDevice, st));
            restart_seq(false);
            poll_iter = h.iter;
            poll_rel = h.rel;
            continue;
        }
        if (h.halt) break;
        // Trips until the next poll: as many as the residual's decay since the previous
        // poll (or since the start) predicts are left before the stop test passes, at most
        // twice the last chunk and 64 -- so that few trips are issued past convergence.
        int grow = std::min(chunk * 2, 64);
        double rate = 0.0;
        if (h.iter > poll_iter && h.rel > 0.0 && poll_rel > h.rel)
            rate = std::log(h.rel / poll_rel) / (h.iter - poll_iter);
        else if (h.iter > 0 && h.rel > 0.0 && h.r0 > 0.0 && h.bnorm > 0.0 && h.r0 / h.bnorm > h.rel)
            rate = std::log(h.rel / (h.r0 / h.bnorm)) / h.iter;
        if (rate < 0.0 && h.rel > tol) {
            // with a preconditioner a trip is costly next to a poll: aim a little short and
            // let the next poll take the last trips (fewer trips issued past the stop)
            const double need = std::ceil(std::log(tol / h.rel) / rate * (JAC ? 1.0 : 0.75));
            if (need < grow) grow = std::max(1, (int)need);
        }
        chunk = std::max(1, std::min(grow, max_iter - h.iter));
        poll_iter = h.iter;
        poll_rel = h.rel;
    }
    HAMLSS_CUDA(cudaEventRecord(ctx.ev1, st));
    HAMLSS_CUDA(cudaEventSynchronize(ctx.ev1));
    float ms = 0.f;
    HAMLSS_CUDA(cudaEventElapsedTime(&ms, ctx.ev0, ctx.ev1));
    res.device_time_s = ms * 1e-3;
    res.iterations = h.iter;
    res.initial_residual = h.r0;
    res.final_residual = h.rel;
    res.converged = h.status == ST_CONV;
    if (h.status == ST_NONFINITE) res.status = HAMLSS_ERR_NONFINITE;
    if (h.status == ST_ESCALATE) res.escalate = h.lad.reason;
    return res;
}

// ------------------------------------------------ reliable-update mixed-precision PCG
//
// PCG whose iteration runs in FP32 -- SpMV on FP32 values, FP32 vectors, the FP32
// V-cycle or Jacobi -- with the dot products and alpha, beta in FP64, and whose
// residual is replaced by the true FP64 residual b - A x ("reliable update") whenever the
// recursive one has fallen by a factor delta since the last replacement, and once more to
// confirm the stop test.  The FP32 iterate y accumulates the corrections since the last
// update; an update folds it into the FP64 x (x += ||b|| y, y = 0) and recomputes
// r = (b - A x) / ||b|| with FP64 values.  Unlike restarted refinement the search
// direction p is kept across updates, so the iteration count stays that of FP64 PCG, and
// the result is certified by an FP64 residual like every mixed-precision solve.
// Per trip: K1 and K2 as in cg_impl (FP32); [fold, FP64 residual] when due (gated by
// skip_ru); [M^-1 r, K3] (non-Jacobi).

struct BodyBnorm {
    const double* b;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&acc)[NV]) const { acc[0] += b[i] * b[i]; }
};

struct FinScale {
    CgState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        const double bn = sqrt(t[0]);
        s->bnorm = bn;
        s->scale = (bn >= kEps && isfinite(bn)) ? 1.0 / bn : 1.0;
    }
};

// x += ||b|| y ; y = 0
struct BodyFold {
    double* x;
    float* y;
    const CgState* s;
    double bn;
    __device__ __forceinline__ void load() { bn = s->bnorm; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const {
        x[i] = dadd(x[i], dmul(bn, (double)y[i]));
        y[i] = 0.0f;
    }
};

// r = (b - A x) / ||b|| in FP64, stored in FP32; ||r||^2 (and r.D^-1 r for Jacobi, as
// K2 forms it)
template <bool JAC>
struct EpiRelRes {
    const double* b;
    float* r;
    const float* dinv;
    const CgState* s;
    double scale;
    __device__ __forceinline__ void load() { scale = s->scale; }
    __device__ __forceinline__ void prefetch(int r0, int r1) const { l2_prefetch_rows(b, r0, r1); }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        const float ri = (float)(__dsub_rn(b[i], ax) * scale);
        r[i] = ri;
        const double rd = (double)ri;
        acc[0] += rd * rd;
        if constexpr (JAC) acc[1] += rd * (double)(float)dmul((double)dinv[i], rd);
    }
};

// start / breakdown restart: the relative residual of x, stop tests as FinInit
struct FinStartRU {
    CgState* s;
    bool first;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        const double rel = sqrt(t[0]);
        s->rel = rel;
        s->rmax = rel;
        if (!first) return;
        const double bn = s->bnorm;
        s->r0 = rel * bn;
        if (!isfinite(bn) || !isfinite(rel)) { s->status = ST_NONFINITE; s->halt = 1; return; }
        if (bn < kEps) { s->status = ST_CONV; s->early = 1; s->rel = 0.0; s->halt = 1; return; }
        if (rel < s->tol) { s->status = ST_CONV; s->early = 2; s->halt = 1; }
    }
};

// K2's finaliser: stop tests on the recursive residual decide whether this trip updates
template <bool JAC>
struct FinUpdRU {
    CgState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        const double rel = sqrt(t[0]);
        s->rel = rel;
        int st = ST_RUN;
        if (!isfinite(rel)) st = ST_NONFINITE;
        else if (ladder_check(&s->lad, s->iter, rel)) st = ST_ESCALATE;
        if (st != ST_RUN) { s->iter += 1; s->status = st; s->halt = 1; s->halt_stage = 2; return; }
        if (rel > s->rmax) s->rmax = rel;
        const bool fin = rel < s->tol;
        if (fin || rel < s->delta * s->rmax) {
            s->skip_ru = 0;
            s->ru_final = fin ? 1 : 0;
            return;                              // the update finishes the trip
        }
        if constexpr (JAC) rho_step(s, t[1], 2);
    }
};

// the update's finaliser: the true residual decides convergence; otherwise the trip goes
// on with the replaced residual
template <bool JAC>
struct FinRU {
    CgState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        const double rel = sqrt(t[0]);
        s->skip_ru = 1;
        s->ru_mask |= 1ull << (s->iter & 63);
        s->rel = rel;
        s->rmax = rel;
        if (!isfinite(rel)) { s->iter += 1; s->status = ST_NONFINITE; s->halt = 1; s->halt_stage = 3; return; }
        if (rel < s->tol) { s->iter += 1; s->status = ST_CONV; s->halt = 1; s->halt_stage = 3; return; }
        if constexpr (JAC) rho_step(s, t[1], 3);
    }
};

template <bool JAC>
struct FinRzRU {
    CgState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const { rho_step(s, t[0], 4); }
};

template <bool JAC>
SolveResult cg_reliable_impl(Ctx& ctx, hamlss_mat* A, Prec* M, const double* b, double* x, double tol,
                             int max_iter, int check_every, double delta, Workspace& ws,
                             const LadderCfg* lad, int* n_updates) {
    const int n = A->A.n;
    const Lane& L = ctx.lane;
    const int sm = ctx.sm_count;
    cudaStream_t st = L.stream;
    Csr<float> A32 = A->A.f32(st);
    Csr<double> A64 = A->A.f64();
    float* r = wvec<float>(ws, 0, n);
    float* z = M && !JAC ? wvec<float>(ws, 1, n) : r;
    float* p[2] = {wvec<float>(ws, 2, n), wvec<float>(ws, 3, n)};
    float* q = wvec<float>(ws, 4, n);
    float* y = wvec<float>(ws, 5, n);
    const float* dinv = JAC ? jacobi_diag<float>(ctx, M) : nullptr;
    const double w4 = 4.0 * n, w8 = 8.0 * n;
    ws.state.ensure(sizeof(CgState));
    CgState* s = reinterpret_cast<CgState*>(ws.state.p);
    int* halt = &s->halt;
    int* skip_ru = &s->skip_ru;

    CgState h0{};
    h0.tol = tol;
    h0.max_iter = max_iter;
    h0.delta = delta;
    h0.skip_ru = 1;
    h0.lad = ladder_init(lad);
    HAMLSS_CUDA(cudaMemcpyAsync(s, &h0, sizeof(CgState), cudaMemcpyHostToDevice, st));
    HAMLSS_CUDA(cudaMemsetAsync(p[0], 0, sizeof(float) * n, st));
    HAMLSS_CUDA(cudaMemsetAsync(p[1], 0, sizeof(float) * n, st));
    HAMLSS_CUDA(cudaMemsetAsync(y, 0, sizeof(float) * n, st));
    HAMLSS_CUDA(cudaEventRecord(ctx.ev0, st));
    launch_vec<1>(sm, L, n, BodyBnorm{b}, FinScale{s}, nullptr, "vec", w8);

    // (re)start: fold y into x, r = (b - A x) / ||b|| in FP64, z = M^-1 r, rho = r.z, beta = 0
    auto restart_seq = [&](bool first) {
        const int* g = first ? nullptr : halt;
        if (!first) launch_vec<0>(sm, L, n, BodyFold{x, y, s, 0.0}, NoFin{}, g, "mixed_fold", 2.0 * w8 + 2.0 * w4);
        launch_spmv<double, 1>(sm, L, A64, XVec<double>{x}, EpiRelRes<false>{b, r, nullptr, s, 0.0},
                               FinStartRU{s, first}, g, "mixed_residual", 2.0 * w8 + w4);
        if (!JAC && M) precond_apply<float>(ctx, M, r, z, halt);
        launch_vec<1>(sm, L, n, BodyRho<float, JAC>{r, z, dinv}, FinRho{s}, halt, "cg_dot", 2.0 * w4);
    };
    auto poll = [&](CgState& h) {
        HAMLSS_CUDA(cudaMemcpyAsync(ctx.host_poll.p, s, sizeof(CgState), cudaMemcpyDeviceToHost, st));
        HAMLSS_CUDA(cudaStreamSynchronize(st));
        std::memcpy(&h, ctx.host_poll.p, sizeof(CgState));
    };

    SolveResult res;
    CgState h{};
    restart_seq(true);
    poll(h);
    const bool run = !h.halt && max_iter > 0;
    int parity = 0;
    int chunk = std::max(1, check_every);
    struct TripMarks { size_t k1, k2, ru, rest, end; int iter; };
    std::vector<TripMarks> trips;
    int poll_iter = h.iter;
    double poll_rel = h.rel;
    int updates = 0;
    while (run) {
        const int iter0 = h.iter;
        trips.clear();
        for (int t = 0; t < chunk; ++t) {
            TripMarks tm;
            tm.iter = iter0 + t;
            tm.k1 = prof_pos(L.prof);
            float* pold = p[parity];
            float* pnew = p[parity ^ 1];
            XP<float, JAC> xp{JAC ? r : z, dinv, pold, s, 0.0};
            launch_spmv<float, 1>(sm, L, A32, xp, EpiQ<float, JAC>{xp, pnew, q}, FinPQ{s}, halt,
                                  "cg_spmv", (JAC ? 5.0 : 4.0) * w4);
            tm.k2 = prof_pos(L.prof);
            launch_vec<JAC ? 2 : 1>(sm, L, n, BodyUpd<float, JAC>{y, r, pnew, q, dinv, s, 0.0},
                                    FinUpdRU<JAC>{s}, halt, "cg_update", (JAC ? 7.0 : 6.0) * w4);
            tm.ru = prof_pos(L.prof);
            launch_vec<0>(sm, L, n, BodyFold{x, y, s, 0.0}, NoFin{}, skip_ru, "mixed_fold", 2.0 * w8 + 2.0 * w4);
            launch_spmv<double, JAC ? 2 : 1>(sm, L, A64, XVec<double>{x}, EpiRelRes<JAC>{b, r, dinv, s, 0.0},
                                             FinRU<JAC>{s}, skip_ru, "mixed_residual",
                                             2.0 * w8 + (JAC ? 2.0 : 1.0) * w4);
            tm.rest = prof_pos(L.prof);
            if (!JAC) {
                if (M) precond_apply<float>(ctx, M, r, z, halt);
                launch_vec<1>(sm, L, n, BodyRz<float>{r, z}, FinRzRU<JAC>{s}, halt, "cg_dot", 2.0 * w4);
            }
            tm.end = prof_pos(L.prof);
            trips.push_back(tm);
            parity ^= 1;
        }
        poll(h);
        HAMLSS_CUDA(cudaMemsetAsync(&s->ru_mask, 0, sizeof(unsigned long long), st));
        const int ran = h.halt ? std::max(1, std::min((int)trips.size(), h.iter - iter0)) : (int)trips.size();
        if (L.prof) {
            // updates that did not run, and everything the halt gate skipped
            for (int k = 0; k < ran; ++k)
                if (!((h.ru_mask >> (trips[k].iter & 63)) & 1ull)) prof_gated(L.prof, trips[k].ru, trips[k].rest);
            if (h.halt) {
                const TripMarks& last = trips[ran - 1];
                const size_t from = h.halt_stage == 1 ? last.k2 : h.halt_stage == 2 ? last.ru
                                  : h.halt_stage == 3 ? last.rest : last.end;
                prof_gated(L.prof, from, last.end);
                prof_gated(L.prof, last.end, trips.back().end);
            }
        }
        for (int k = 0; k < ran; ++k) updates += (int)((h.ru_mask >> (trips[k].iter & 63)) & 1ull);
        if (h.status == ST_RESTART) {
            res.restarts++;
            CgState hh = h;
            hh.status = ST_RUN;
            hh.halt = 0;
            hh.halt_stage = 0;
            hh.skip_ru = 1;
            hh.ru_mask = 0;
            HAMLSS_CUDA(cudaMemcpyAsync(s, &hh, sizeof(CgState), cudaMemcpyHostToDevice, st));
            restart_seq(false);
            poll_iter = h.iter;
            poll_rel = h.rel;
            continue;
        }
        if (h.halt) break;
        int grow = std::min(chunk * 2, 64);
        double rate = 0.0;
        if (h.iter > poll_iter && h.rel > 0.0 && poll_rel > h.rel)
            rate = std::log(h.rel / poll_rel) / (h.iter - poll_iter);
        else if (h.iter > 0 && h.rel > 0.0 && h.r0 > 0.0 && h.bnorm > 0.0 && h.r0 / h.bnorm > h.rel)
            rate = std::log(h.rel / (h.r0 / h.bnorm)) / h.iter;
        if (rate < 0.0 && h.rel > tol) {
            // with a preconditioner a trip is costly next to a poll: aim a little short and
            // let the next poll take the last trips (fewer trips issued past the stop)
            const double need = std::ceil(std::log(tol / h.rel) / rate * (JAC ? 1.0 : 0.75));
            if (need < grow) grow = std::max(1, (int)need);
        }
        chunk = std::max(1, std::min(grow, max_iter - h.iter));
        poll_iter = h.iter;
        poll_rel = h.rel;
    }
    // the FP32 iterate's corrections since the last update join x (zeros after a
    // converged update)
    launch_vec<0>(sm, L, n, BodyFold{x, y, s, 0.0}, NoFin{}, nullptr, "mixed_fold", 2.0 * w8 + 2.0 * w4);
    HAMLSS_CUDA(cudaEventRecord(ctx.ev1, st));
    HAMLSS_CUDA(cudaEventSynchronize(ctx.ev1));
    float ms = 0.f;
    HAMLSS_CUDA(cudaEventElapsedTime(&ms, ctx.ev0, ctx.ev1));
    res.device_time_s = ms * 1e-3;
    res.iterations = h.iter;
    res.initial_residual = h.r0;
    res.final_residual = h.rel;
    res.converged = h.status == ST_CONV;
    *n_updates = updates;
    if (h.status == ST_NONFINITE) res.status = HAMLSS_ERR_NONFINITE;
    if (h.status == ST_ESCALATE) res.escalate = h.lad.reason;
    return res;
}

}  // namespace

template <typename T>
SolveResult cg_solve(Ctx& ctx, hamlss_mat* A, Prec* M, const T* b, T* x, double tol,
                     int max_iter, int check_every, Workspace& ws, const LadderCfg* lad) {
    if (M && M->kind == HAMLSS_PREC_JACOBI)
        return cg_impl<T, true>(ctx, A, M, b, x, tol, max_iter, check_every, ws, lad);
    return cg_impl<T, false>(ctx, A, M, b, x, tol, max_iter, check_every, ws, lad);
}

SolveResult cg_reliable_solve(Ctx& ctx, hamlss_mat* A, Prec* M, const double* b, double* x, double tol,
                              int max_iter, int check_every, double delta, Workspace& ws,
                              const LadderCfg* lad, int* n_updates) {
    if (M) M->prepare32(ctx);
    if (M && M->kind == HAMLSS_PREC_JACOBI)
        return cg_reliable_impl<true>(ctx, A, M, b, x, tol, max_iter, check_every, delta, ws, lad, n_updates);
    return cg_reliable_impl<false>(ctx, A, M, b, x, tol, max_iter, check_every, delta, ws, lad, n_updates);
}

template SolveResult cg_solve<double>(Ctx&, hamlss_mat*, Prec*, const double*, double*, double,
                                      int, int, Workspace&, const LadderCfg*);
template SolveResult cg_solve<float>(Ctx&, hamlss_mat*, Prec*, const float*, float*, double, int,
                                     int, Workspace&, const LadderCfg*);

}  // namespace hamlss
