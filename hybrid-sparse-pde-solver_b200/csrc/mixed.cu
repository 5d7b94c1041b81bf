// mixed.cu -- mixed-precision solves.
//
// PCG: by default the reliable-update PCG of cg.cu (FP32 iteration, residual refreshed in
// FP64; ir_update > 0).  With ir_update = 0, and for FGMRES, FP32 inner solves inside an
// FP64 iterative-refinement loop:
//
//   repeat:  r = b - A x            FP64 values, FP64 vectors (true residual)
//            stop when ||r|| / ||b|| < tol
//            s = ||r||, solve A d = r / s in FP32 (values, vectors, V-cycle) to a relative
//            reduction max(ir_inner_tol, 0.5 tol / rel); the CG scalars alpha, beta and
//            all dot products stay FP64
//            x += s d                FP64
// Every result is therefore certified by an FP64 residual; iterations reported are the
// inner iterations summed over refinement steps.  For FGMRES the Krylov vectors,
// Hessenberg and Givens data stay FP64 and the preconditioner runs in FP32 (flexible
// GMRES accepts the inexact inner solve).
#include <chrono>
#include <cmath>
#include <cstring>

#include "krylov.cuh"

namespace hamlss {

namespace {

struct EpiRes64 {
    const double* b;
    double* r;
    HAMLSS_NO_LOAD
    __device__ __forceinline__ void prefetch(int r0, int r1) const { l2_prefetch_rows(b, r0, r1); }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        double bi = b[i];
        double ri = __dsub_rn(bi, ax);
        r[i] = ri;
        acc[0] += bi * bi;
        acc[1] += ri * ri;
    }
};

struct FinStore2 {
    double* out;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const { out[0] = t[0]; out[1] = t[1]; }
};

struct BodyToF32 {
    const double* r;
    float* r32;
    const double* scale;   // device scalar: 1/||r||
    double inv;
    __device__ __forceinline__ void load() { inv = *scale; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const {
        r32[i] = (float)(r[i] * inv);
    }
};

struct BodyCorrect {
    double* x;
    const float* d;
    double s;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const { x[i] += s * (double)d[i]; }
};

template <typename A, typename B>
struct BodyConv {
    const A* a;
    B* b;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const { b[i] = (B)a[i]; }
};

// Runs an FP32 preconditioner on FP64 vectors (for FP64 FGMRES with an FP32 M^-1).
struct Prec32Adapter : Prec {
    Prec* inner;
    DBuf<float> r32, z32;
    void apply(Ctx& ctx, const Lane& L, const double* r, double* z, const int* gate) override {
        r32.ensure(n);
        z32.ensure(n);
        launch_vec<0>(ctx.sm_count, L, n, BodyConv<double, float>{r, r32.p}, NoFin{}, gate, "vec", 12.0 * n);
        inner->apply32(ctx, L, r32.p, z32.p, gate);
        launch_vec<0>(ctx.sm_count, L, n, BodyConv<float, double>{z32.p, z}, NoFin{}, gate, "vec", 12.0 * n);
    }
};

}  // namespace

SolveResult mixed_solve(Ctx& ctx, int solver, hamlss_mat* A, Prec* M, const double* b, double* x,
                        const hamlss_params& p, Workspace& ws, int* outer_iters,
                        const LadderCfg* lad) {
    const int n = A->A.n;
    const Lane& L = ctx.lane;
    cudaStream_t st = L.stream;
    if (M && !M->has32()) fail(HAMLSS_ERR_INVALID, "preconditioner has no FP32 path");
    if (M) M->prepare32(ctx);
    if (solver == HAMLSS_SOLVER_FGMRES) {
        Prec32Adapter ad;
        ad.inner = M;
        ad.n = n;
        ad.kind = M ? M->kind : HAMLSS_PREC_NONE;
        *outer_iters = 1;
        return fgmres_solve(ctx, A, M ? &ad : nullptr, b, x, p.tol, p.max_iter, p.restart_size, ws, lad);
    }
    if (p.ir_update > 0.0) {
        // reliable updates: one FP32 PCG whose residual is refreshed in FP64 (cg.cu)
        int updates = 0;
        SolveResult r = cg_reliable_solve(ctx, A, M, b, x, p.tol, p.max_iter, p.check_every,
                                          std::min(p.ir_update, 0.5), ws, lad, &updates);
        *outer_iters = updates;
        return r;
    }
    // buffers: FP64 residual in d[5]; FP32 rhs / correction in f[5], f[6]; scalars in small
    ws.d[5].ensure(n);
    ws.f[5].ensure(n);
    ws.f[6].ensure(n);
    ws.small.ensure(4096);
    double* r = ws.d[5].p;
    float* r32 = ws.f[5].p;
    float* d32 = ws.f[6].p;
    double* sc = ws.small.p + 4000;      // [0] b.b, [1] r.r, [2] 1/||r||
    // the inner CG uses ws.f[0..4] and ws.state, disjoint from the buffers above
    SolveResult res;
    const auto t0 = std::chrono::steady_clock::now();
    int total = 0, outer = 0;
    double rel = 0.0, bn = 0.0;
    for (;;) {
        launch_spmv<double, 2>(ctx.sm_count, L, A->A.f64(), XVec<double>{x}, EpiRes64{b, r},
                               FinStore2{sc}, nullptr, "ir_residual", 24.0 * n);
        double h[2];
        HAMLSS_CUDA(cudaMemcpyAsync(h, sc, sizeof(h), cudaMemcpyDeviceToHost, st));
        HAMLSS_CUDA(cudaStreamSynchronize(st));
        bn = std::sqrt(h[0]);
        double rn = std::sqrt(h[1]);
        if (!std::isfinite(bn) || !std::isfinite(rn)) { res.status = HAMLSS_ERR_NONFINITE; break; }
        if (outer == 0) res.initial_residual = rn;
        if (bn < 2.220446049250313e-16) { res.converged = 1; rel = rn; break; }
        rel = rn / bn;
        if (rel < p.tol) { res.converged = 1; break; }
        if (outer >= p.ir_max_outer || total >= p.max_iter) break;
        double inv = 1.0 / rn;
        HAMLSS_CUDA(cudaMemcpyAsync(sc + 2, &inv, sizeof(double), cudaMemcpyHostToDevice, st));
        launch_vec<0>(ctx.sm_count, L, n, BodyToF32{r, r32, sc + 2, 0.0}, NoFin{}, nullptr, "vec", 12.0 * n);
        HAMLSS_CUDA(cudaMemsetAsync(d32, 0, sizeof(float) * n, st));
        double inner_tol = std::max(p.ir_inner_tol, 0.5 * p.tol / rel);
        SolveResult ir = cg_solve<float>(ctx, A, M, r32, d32, inner_tol, p.max_iter - total,
                                         p.check_every, ws, lad);
        if (ir.status != HAMLSS_OK) { res.status = ir.status; break; }
        total += ir.iterations;
        if (ir.escalate) { res.escalate = ir.escalate; }
        launch_vec<0>(ctx.sm_count, L, n, BodyCorrect{x, d32, rn}, NoFin{}, nullptr, "vec", 20.0 * n);
        ++outer;
        if (ir.iterations == 0 || res.escalate) break;    // no progress possible / escalate
    }
    HAMLSS_CUDA(cudaStreamSynchronize(st));
    res.iterations = total;
    res.final_residual = rel;
    // the loop synchronises on every refinement step, so wall time is the device time
    res.device_time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *outer_iters = outer;
    return res;
}

}  // namespace hamlss
