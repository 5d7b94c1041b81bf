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

#include "krylov.cuh"

namespace hamlss {

namespace {

constexpr double kEps = 2.220446049250313e-16;

struct CgState {
    double bnorm, r0, rel, tol, rho, rho_old, alpha, beta, pq;
    int iter, max_iter, halt, status, restart_kind, early;
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
__device__ __forceinline__ void rho_step(CgState* s, double rz) {
    double rho_old = s->rho;
    s->rho_old = rho_old;
    s->rho = rz;
    if (fabs(rho_old) < kEps * 1e8 * fabs(rz)) {
        s->iter += 1;
        if (s->iter >= s->max_iter) s->status = ST_MAXIT;
        else { s->status = ST_RESTART; s->restart_kind = 2; }
        s->halt = 1;
        return;
    }
    s->beta = rz / rho_old;
    s->iter += 1;
    if (s->iter >= s->max_iter) { s->status = ST_MAXIT; s->halt = 1; }
}

template <bool JAC>
struct FinUpd {
    CgState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        double rel = sqrt(t[0]) / s->bnorm;
        s->rel = rel;
        if (rel < s->tol) { s->iter += 1; s->status = ST_CONV; s->halt = 1; return; }
        if (!isfinite(rel)) { s->iter += 1; s->status = ST_NONFINITE; s->halt = 1; return; }
        if (ladder_check(&s->lad, s->iter, rel)) { s->iter += 1; s->status = ST_ESCALATE; s->halt = 1; return; }
        if constexpr (JAC) rho_step(s, t[1]);
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
    __device__ void operator()(const double (&t)[NV]) const { rho_step(s, t[0]); }
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
    while (run) {
        for (int t = 0; t < chunk; ++t) {
            T* pold = p[parity];
            T* pnew = p[parity ^ 1];
            XP<T, JAC> xp{JAC ? r : z, dinv, pold, s, 0.0};
            launch_spmv<T, 1>(sm, L, Ad, xp, EpiQ<T, JAC>{xp, pnew, q}, FinPQ{s}, halt,
                              "cg_spmv", (JAC ? 5.0 : 4.0) * wb);
            launch_vec<JAC ? 2 : 1>(sm, L, n, BodyUpd<T, JAC>{x, r, pnew, q, dinv, s, 0.0},
                                    FinUpd<JAC>{s}, halt, "cg_update", (JAC ? 7.0 : 6.0) * wb);
            if (!JAC) {
                if (M) precond_apply<T>(ctx, M, r, z, halt);
                launch_vec<1>(sm, L, n, BodyRz<T>{r, z}, FinRz{s}, halt, "cg_dot", 2.0 * wb);
            }
            parity ^= 1;
        }
        poll(h);
        if (h.status == ST_RESTART) {
            res.restarts++;
            CgState hh = h;
            hh.status = ST_RUN;
            hh.halt = 0;
            HAMLSS_CUDA(cudaMemcpyAsync(s, &hh, sizeof(CgState), cudaMemcpyHostToDevice, st));
            restart_seq(false);
            continue;
        }
        if (h.halt) break;
        chunk = std::min(chunk * 2, 64);
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

}  // namespace

template <typename T>
SolveResult cg_solve(Ctx& ctx, hamlss_mat* A, Prec* M, const T* b, T* x, double tol,
                     int max_iter, int check_every, Workspace& ws, const LadderCfg* lad) {
    if (M && M->kind == HAMLSS_PREC_JACOBI)
        return cg_impl<T, true>(ctx, A, M, b, x, tol, max_iter, check_every, ws, lad);
    return cg_impl<T, false>(ctx, A, M, b, x, tol, max_iter, check_every, ws, lad);
}

template SolveResult cg_solve<double>(Ctx&, hamlss_mat*, Prec*, const double*, double*, double,
                                      int, int, Workspace&, const LadderCfg*);
template SolveResult cg_solve<float>(Ctx&, hamlss_mat*, Prec*, const float*, float*, double, int,
                                     int, Workspace&, const LadderCfg*);

}  // namespace hamlss
