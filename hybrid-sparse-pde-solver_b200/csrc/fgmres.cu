// fgmres.cu -- restarted flexible GMRES on the device (FGMRESSolver, fgmres_solver.cpp).
//
// Per inner step j (all launches gated by the cycle's halt flag, no host round trip):
//   z_j = M^-1 v_j                        preconditioner
//   w   = A z_j                           SpMV
//   h   = V_j^T w                         multi-dot, one pass over v_0..v_j and w
//   w  -= V_j h ; h' = V_j^T w            fused update + second multi-dot (CGS2)
//   w  -= V_j h' ; ||w||^2                fused update + norm; the last block then forms
//                                         column j of H, applies the stored Givens
//                                         rotations, makes the new one, updates g and
//                                         tests |g_{j+1}| < tol ||b|| (fgmres_solver.cpp:126-148)
//   v_{j+1} = w / ||w||
// The cycle ends with the triangular solve for y (:57-66) and x += Z y, both on the
// device; the host polls between groups of inner steps (sized by the decay of the
// residual estimate) and at the end of each cycle.  Classical Gram-Schmidt applied twice
// replaces the reference's modified Gram-Schmidt (:122-125): same subspace, three passes
// over V instead of 2(j+1) dependent dot/axpy pairs.
#include <cmath>
#include <cstring>
#include <vector>

#include "krylov.cuh"

namespace hamlss {

namespace {

constexpr double kEps = 2.220446049250313e-16;

struct GmState {
    double bnorm, tol_abs, beta, res, inv_beta, hn_inv, hn;
    int jcount, halt, status, m, iter_base, pipelined;
    LadderDev lad;
};

// Device-side small arrays, laid out in ws.small: H (m+1) x m row-major, cs, sn, g, y,
// h1, h2.
struct GmArrays {
    double* H;
    double* cs;
    double* sn;
    double* g;
    double* y;
    double* h1;
    double* h2;
    int m;
};

struct BodyBB {
    const double* b;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&acc)[NV]) const { acc[0] += b[i] * b[i]; }
};

struct FinBnorm {
    GmState* s;
    double tol;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        double bn = sqrt(t[0]);
        s->bnorm = bn;
        s->tol_abs = tol * bn;
        if (!isfinite(bn)) s->status = ST_NONFINITE;
    }
};

// r = b - A x and ||r||^2
struct EpiRes {
    const double* b;
    double* r;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        double ri = __dsub_rn(b[i], ax);
        r[i] = ri;
        acc[0] += ri * ri;
    }
};

struct FinCycleStart {
    GmState* s;
    GmArrays a;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        double beta = sqrt(t[0]);
        s->beta = beta;
        s->res = beta;
        s->jcount = 0;
        if (!isfinite(beta)) { s->status = ST_NONFINITE; s->halt = 1; return; }
        if (beta < s->tol_abs) { s->halt = 1; return; }
        s->inv_beta = 1.0 / beta;
        for (int k = 0; k <= a.m; ++k) a.g[k] = 0.0;
        a.g[0] = beta;
    }
};

struct BodyScaleV0 {
    const double* r;
    double* v0;
    const GmState* s;
    double inv;
    __device__ __forceinline__ void load() { inv = s->inv_beta; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const { v0[i] = __dmul_rn(r[i], inv); }
};

// Multi-dot family over the basis V (nv vectors of length n, leading dimension ld).
// MODE 0: acc_k = v_k . w
// MODE 1: w -= sum_k hp_k v_k (stored), then acc_k = v_k . w
// MODE 2: w -= sum_k hp_k v_k (stored), then acc_0 = w . w
template <int NV, int MODE, typename Fin>
__global__ void __launch_bounds__(256)
k_mdot(int n, int nv, const double* __restrict__ V, long long ld, double* w,
       const double* __restrict__ hprev, Reducer red, Fin fin, const int* gate) {
    constexpr int NR = (MODE == 2) ? 1 : NV;
    __shared__ double hp[NV];
    __shared__ double rsh[8 * NR];
    if (gate && *(volatile const int*)gate) return;
    if (MODE >= 1) {
        for (int k = threadIdx.x; k < NV; k += blockDim.x) hp[k] = (k < nv) ? hprev[k] : 0.0;
        __syncthreads();
    }
    double acc[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) acc[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double wi = w[i];
        if (MODE >= 1) {
#pragma unroll
            for (int k = 0; k < NV; ++k)
                if (k < nv) wi -= hp[k] * __ldg(&V[k * ld + i]);
            w[i] = wi;
        }
        if (MODE <= 1) {
#pragma unroll
            for (int k = 0; k < NV; ++k)
                if (k < nv) acc[k] += __ldg(&V[k * ld + i]) * wi;
        } else {
            acc[0] += wi * wi;
        }
    }
    double tot[NR];
    if (grid_reduce<NR>(red, acc, rsh, tot)) fin(tot);
}

template <int NV>
struct FinH1 {
    GmArrays a;
    int j;
    __device__ void operator()(const double (&t)[NV]) const {
        for (int k = 0; k <= j && k < NV; ++k) { a.h1[k] = t[k]; a.H[k * a.m + j] = t[k]; }
    }
};

template <int NV>
struct FinH2 {
    GmArrays a;
    int j;
    __device__ void operator()(const double (&t)[NV]) const {
        for (int k = 0; k <= j && k < NV; ++k) { a.h2[k] = t[k]; a.H[k * a.m + j] += t[k]; }
    }
};

// compute_givens / apply_givens (fgmres_solver.cpp:36-51)
__device__ void givens(double f, double g, double& cs, double& sn, double& r) {
    if (fabs(g) < kEps) { cs = 1.0; sn = 0.0; r = f; }
    else if (fabs(f) < kEps) { cs = 0.0; sn = 1.0; r = g; }
    else { double t = sqrt(f * f + g * g); cs = f / t; sn = g / t; r = t; }
}
__device__ void rot(double& dx, double& dy, double cs, double sn) {
    double t = cs * dx + sn * dy;
    dy = -sn * dx + cs * dy;
    dx = t;
}

struct FinNorm {
    GmState* s;
    GmArrays a;
    int j;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        const int m = a.m;
        double hn = sqrt(t[0]);
        s->hn = hn;
        a.H[(j + 1) * m + j] = hn;
        s->hn_inv = (hn > kEps) ? 1.0 / hn : 0.0;
        // PipelinedFGMRESSolver leaves the cycle on a lucky breakdown before rotating
        // column j (pipelined_fgmres_solver.cpp:117-123)
        if (s->pipelined && !(hn > kEps)) { s->jcount = j + 1; s->halt = 1; return; }
        for (int i = 0; i < j; ++i) rot(a.H[i * m + j], a.H[(i + 1) * m + j], a.cs[i], a.sn[i]);
        double r;
        givens(a.H[j * m + j], a.H[(j + 1) * m + j], a.cs[j], a.sn[j], r);
        a.H[j * m + j] = r;
        a.H[(j + 1) * m + j] = 0.0;
        rot(a.g[j], a.g[j + 1], a.cs[j], a.sn[j]);
        double res = fabs(a.g[j + 1]);
        s->res = res;
        s->jcount = j + 1;
        if (!isfinite(res)) { s->status = ST_NONFINITE; s->halt = 1; return; }
        if (res < s->tol_abs) { s->halt = 1; return; }
        if (ladder_check(&s->lad, s->iter_base + j, res / s->bnorm)) { s->status = ST_ESCALATE; s->halt = 1; }
    }
};

struct BodyNextV {
    const double* w;
    double* v;
    const GmState* s;
    double inv;
    __device__ __forceinline__ void load() { inv = s->hn_inv; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const {
        v[i] = (inv != 0.0) ? __dmul_rn(w[i], inv) : 0.0;
    }
};

// solve_hessenberg (fgmres_solver.cpp:57-66) for the steps actually taken
__global__ void k_backsolve(GmState* s, GmArrays a) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int k = s->jcount, m = a.m;
    for (int i = k - 1; i >= 0; --i) {
        double t = a.g[i];
        for (int c = i + 1; c < k; ++c) t -= a.H[i * m + c] * a.y[c];
        a.y[i] = (fabs(a.H[i * m + i]) > kEps) ? (t / a.H[i * m + i]) : 0.0;
    }
}

// x += sum_i y_i z_i in the reference's order (x.axpy(y[i], Z[i]) for i = 0..k-1)
__global__ void __launch_bounds__(256)
k_update_x(int n, double* x, const double* __restrict__ Z, long long ld, const GmState* s,
           const double* __restrict__ y) {
    const int k = s->jcount;
    if (k == 0) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double xi = x[i];
        for (int c = 0; c < k; ++c) xi = __dadd_rn(xi, __dmul_rn(y[c], Z[c * ld + i]));
        x[i] = xi;
    }
}

template <int NV>
void launch_mdot_t(Ctx& ctx, int mode, int n, int nv, const double* V, long long ld, double* w,
                   const double* hprev, GmState* s, const GmArrays& a, int j, const int* gate) {
    const Lane& L = ctx.lane;
    int blocks = std::max(1, std::min(ceil_div(n, 256), ctx.sm_count * 4));
    L.red_check(blocks, mode == 2 ? 1 : NV);
    ProfScope ps(L, "gmres_mdot", 8.0 * n * (nv + (mode == 0 ? 1 : 2)));
    if (mode == 0)
        k_mdot<NV, 0, FinH1<NV>><<<blocks, 256, 0, L.stream>>>(n, nv, V, ld, w, hprev, L.red(),
                                                                FinH1<NV>{a, j}, gate);
    else if (mode == 1)
        k_mdot<NV, 1, FinH2<NV>><<<blocks, 256, 0, L.stream>>>(n, nv, V, ld, w, hprev, L.red(),
                                                                FinH2<NV>{a, j}, gate);
    else
        k_mdot<NV, 2, FinNorm><<<blocks, 256, 0, L.stream>>>(n, nv, V, ld, w, hprev, L.red(),
                                                              FinNorm{s, a, j}, gate);
    HAMLSS_LAUNCH_CHECK();
}

void launch_mdot(Ctx& ctx, int mode, int n, int nv, const double* V, long long ld, double* w,
                 const double* hprev, GmState* s, const GmArrays& a, int j, const int* gate) {
    if (nv <= 4) launch_mdot_t<4>(ctx, mode, n, nv, V, ld, w, hprev, s, a, j, gate);
    else if (nv <= 8) launch_mdot_t<8>(ctx, mode, n, nv, V, ld, w, hprev, s, a, j, gate);
    else if (nv <= 16) launch_mdot_t<16>(ctx, mode, n, nv, V, ld, w, hprev, s, a, j, gate);
    else if (nv <= 32) launch_mdot_t<32>(ctx, mode, n, nv, V, ld, w, hprev, s, a, j, gate);
    else if (nv <= 64) launch_mdot_t<64>(ctx, mode, n, nv, V, ld, w, hprev, s, a, j, gate);
    else fail(HAMLSS_ERR_INVALID, "FGMRES restart length above 63 is not supported");
}

}  // namespace

SolveResult fgmres_solve(Ctx& ctx, hamlss_mat* A, Prec* M, const double* b, double* x,
                         double tol, int max_iter, int restart, Workspace& ws,
                         const LadderCfg* lad, bool pipelined) {
    const int n = A->A.n;
    const int m = std::max(1, std::min(restart, n));
    if (m > 63) fail(HAMLSS_ERR_INVALID, "FGMRES restart length above 63 is not supported");
    const Lane& L = ctx.lane;
    const int sm = ctx.sm_count;
    cudaStream_t st = L.stream;
    const long long ld = ((long long)n + 31) / 32 * 32;      // keep every basis vector 256-B aligned
    const bool flex = M != nullptr;
    ws.basis.ensure((size_t)ld * (size_t)(m + 1 + (flex ? m : 0)));
    double* V = ws.basis.p;
    double* Z = flex ? V + ld * (m + 1) : V;
    double* w = (ws.d[0].ensure(n), ws.d[0].p);
    double* r = (ws.d[1].ensure(n), ws.d[1].p);
    ws.small.ensure((size_t)(m + 1) * m + 6 * (m + 1) + 64);
    GmArrays a;
    a.m = m;
    a.H = ws.small.p;
    a.cs = a.H + (size_t)(m + 1) * m;
    a.sn = a.cs + (m + 1);
    a.g = a.sn + (m + 1);
    a.y = a.g + (m + 1);
    a.h1 = a.y + (m + 1);
    a.h2 = a.h1 + (m + 1);
    HAMLSS_CUDA(cudaMemsetAsync(ws.small.p, 0, sizeof(double) * ((size_t)(m + 1) * m + 6 * (m + 1)), st));
    ws.state.ensure(sizeof(GmState));
    GmState* s = reinterpret_cast<GmState*>(ws.state.p);
    GmState h0{};
    h0.m = m;
    h0.pipelined = pipelined ? 1 : 0;
    h0.lad = ladder_init(lad);
    HAMLSS_CUDA(cudaMemcpyAsync(s, &h0, sizeof(h0), cudaMemcpyHostToDevice, st));
    HAMLSS_CUDA(cudaEventRecord(ctx.ev0, st));

    auto poll = [&](GmState& h) {
        HAMLSS_CUDA(cudaMemcpyAsync(ctx.host_poll.p, s, sizeof(GmState), cudaMemcpyDeviceToHost, st));
        HAMLSS_CUDA(cudaStreamSynchronize(st));
        std::memcpy(&h, ctx.host_poll.p, sizeof(GmState));
    };

    SolveResult res;
    GmState h{};
    launch_vec<1>(sm, L, n, BodyBB{b}, FinBnorm{s, tol}, nullptr, "vec", 8.0 * n);
    poll(h);
    if (h.status == ST_NONFINITE) { res.status = HAMLSS_ERR_NONFINITE; return res; }
    if (h.bnorm < kEps) {           // fgmres_solver.cpp:179-183
        res.converged = 1;
        res.final_residual = 0.0;
        if (pipelined) res.flops = res.bytes = 0;
        return res;
    }
    int total = 0, cycles = 0;
    int sub = std::max(1, std::min(m, 8));       // inner steps issued before the first poll
    // Launch positions of each inner step in the engine profiler: its start, its last
    // launch (v_{j+1} = w / ||w||) and its end.
    struct StepMarks { size_t start, next_v, end; };
    std::vector<StepMarks> steps;
    while (total < max_iter) {
        const int cm = std::min(m, max_iter - total);
        HAMLSS_CUDA(cudaMemsetAsync(&s->halt, 0, sizeof(int), st));
        HAMLSS_CUDA(cudaMemcpyAsync(&s->iter_base, &total, sizeof(int), cudaMemcpyHostToDevice, st));
        launch_spmv<double, 1>(sm, L, A->A.f64(), XVec<double>{x}, EpiRes{b, r}, FinCycleStart{s, a},
                               nullptr, "gmres_residual", 24.0 * n);
        const size_t v0_mark = prof_pos(L.prof);
        launch_vec<0>(sm, L, n, BodyScaleV0{r, V, s, 0.0}, NoFin{}, &s->halt, "vec", 16.0 * n);
        steps.clear();
        // Inner steps go out in groups; the host polls between groups and stops issuing
        // once the device's test has ended the cycle.  The group size follows the decay of
        // |g_{j+1}| (monotone in GMRES) since the previous poll.
        int j = 0, poll_j = 0;
        double poll_res = -1.0;
        bool halted = false;
        while (j < cm && !halted) {
            const int jend = std::min(cm, j + sub);
            for (; j < jend; ++j) {
                StepMarks sm_;
                sm_.start = prof_pos(L.prof);
                double* vj = V + ld * j;
                double* zj = Z + ld * j;
                if (flex) M->apply(ctx, L, vj, zj, &s->halt);
                launch_spmv<double, 0>(sm, L, A->A.f64(), XVec<double>{zj}, EpiStore<double>{w}, NoFin{},
                                       &s->halt, "spmv");
                launch_mdot(ctx, 0, n, j + 1, V, ld, w, nullptr, s, a, j, &s->halt);
                launch_mdot(ctx, 1, n, j + 1, V, ld, w, a.h1, s, a, j, &s->halt);
                launch_mdot(ctx, 2, n, j + 1, V, ld, w, a.h2, s, a, j, &s->halt);
                sm_.next_v = prof_pos(L.prof);
                launch_vec<0>(sm, L, n, BodyNextV{w, V + ld * (j + 1), s, 0.0}, NoFin{}, &s->halt, "vec",
                              16.0 * n);
                sm_.end = prof_pos(L.prof);
                steps.push_back(sm_);
            }
            if (j >= cm) break;                    // the cycle's own poll follows
            poll(h);
            halted = h.halt != 0;
            if (!halted && h.bnorm > 0.0) {
                const double res = h.res;
                int grow = std::min(2 * sub, m);
                if (poll_res > res && res > 0.0 && h.jcount > poll_j) {
                    const double rate = std::log(res / poll_res) / (h.jcount - poll_j);
                    const double need = std::ceil(std::log(h.tol_abs / res) / rate);
                    if (need >= 0.0 && need < grow) grow = std::max(1, (int)need);
                }
                sub = grow;
                poll_j = h.jcount;
                poll_res = res;
            }
        }
        {
            ProfScope ps(L, "gmres_small", 0.0);
            k_backsolve<<<1, 32, 0, st>>>(s, a);
            HAMLSS_LAUNCH_CHECK();
        }
        const size_t upd_mark = prof_pos(L.prof);
        {
            ProfScope ps(L, "gmres_update", 8.0 * n * (2 + cm));
            k_update_x<<<std::max(1, std::min(ceil_div(n, 256), sm * 8)), 256, 0, st>>>(n, x, Z, ld, s, a.y);
            HAMLSS_LAUNCH_CHECK();
        }
        poll(h);
        if (L.prof && h.halt) {
            // launches the gate skipped: after a stop at cycle start, every inner step;
            // after a stop in step jcount - 1, that step's v_{j+1} and the later steps
            const size_t end = steps.empty() ? v0_mark + 1 : steps.back().end;
            const size_t from = h.jcount == 0 ? v0_mark
                              : (size_t)h.jcount <= steps.size() ? steps[h.jcount - 1].next_v : end;
            prof_gated(L.prof, from, end);
        }
        if (L.prof && upd_mark < L.prof->pos())       // x += Z y over the steps taken
            L.prof->marks[upd_mark].bytes = h.jcount ? 8.0 * n * (2 + h.jcount) : 0.0;
        if (h.status == ST_NONFINITE) { res.status = HAMLSS_ERR_NONFINITE; break; }
        total += h.jcount;
        ++cycles;
        if (h.status == ST_ESCALATE) {       // device ladder test fired inside the cycle
            res.escalate = h.lad.reason;
            res.final_residual = h.res / h.bnorm;
            break;
        }
        double rel = h.res / h.bnorm;
        if (rel < tol || h.jcount == 0) {          // fgmres_solver.cpp:221-225
            res.converged = rel < tol;
            res.final_residual = rel;
            break;
        }
    }
    // max_iter exhausted: final_residual stays 0 as in the reference (:197-226)
    HAMLSS_CUDA(cudaEventRecord(ctx.ev1, st));
    HAMLSS_CUDA(cudaEventSynchronize(ctx.ev1));
    float ms = 0.f;
    HAMLSS_CUDA(cudaEventElapsedTime(&ms, ctx.ev0, ctx.ev1));
    res.device_time_s = ms * 1e-3;
    res.iterations = total;
    res.restarts = cycles - 1;                     // fgmres_solver.cpp:231
    res.initial_residual = 0.0;
    if (pipelined) {
        // (inner steps + 1 primer) SpMVs per cycle plus 4n per step
        // (pipelined_fgmres_solver.cpp:207-212)
        const long long nn = n, nz = A->A.nnz;
        const long long spmv = (long long)total + cycles;
        res.flops = spmv * 2 * nz + (long long)total * 4 * nn;
        res.bytes = spmv * ((nn + 1 + nz) * 4 + nz * 8 + nn * 16) + (long long)total * 4 * nn * 8;
    }
    return res;
}

}  // namespace hamlss
