// sstep.cu -- SStepCGSolver (sstep_cg_solver.cpp:170-305) on the device.
//
// One batch of k steps:
//   B_0 = r / ||r||; B_j = (A - theta_{j-1}) B_{j-1}, normalised     k-1 fused SpMV + norm
//                                                                     launches, k-1 scales
//   [r, B_0 .. B_{k-1}]^T [r, B_0 .. B_{k-1}]                         one DGEMM: the Gram
//                                                                     matrix and r . B_i
//   G y = (r . B_i) by Cholesky (k x k, on the host)                  one device->host copy
//   x += sum_i y_i B_i ; r = b - A x ; ||r||                          two launches, one poll
// The shifts theta_j are the Chebyshev nodes of the Lanczos interval of A (20 steps,
// sparse_matrix.cpp:451-479); an ill-conditioned Gram matrix (diagonal ratio above
// sstep_cond_tol) halves k for the batch; a failed Cholesky takes one steepest-descent
// step instead.  The preconditioner is not applied, as in the reference.
//
// The update minimises ||r - B y|| over the basis and adds B y to x: a projected
// Richardson step.  It converges only when the spectrum of A lies inside (0, 2) roughly
// (e.g. a unit-diagonal scaling of an M-matrix); elsewhere the residual grows every batch
// until it overflows, and the loop ends on the non-finite residual exactly as the
// reference's `while (... && rel_res > tol)` does.  Reproduced, not repaired.
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dense_lu.cuh"
#include "krylov.cuh"

namespace hamlss {

namespace {

constexpr double kEps = 2.220446049250313e-16;
constexpr int kMaxS = 32;            // largest batch size accepted

struct SsState {
    double nrm2;                     // ||B_j||^2 of the last basis vector
    double inv;                      // 1 / ||B_j|| (1 when ||B_j|| <= eps)
    double rr;                       // ||r||^2
    double rap;                      // r . Ap (steepest-descent fallback)
    double bb;                       // ||b||^2
};

// Every reduction below either accumulates into the launch's grid reduction or, when
// `terms` is set (systems of at most kSeqRows rows), stores its per-row terms
// (terms[i], terms[n + i]) for k_seq_sum to add in row order -- the reference's
// single-thread summation, bit for bit: the s-step update amplifies last-bit differences.
struct BodyBB {
    const double* b;
    double* terms;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&acc)[NV]) const {
        const double t = __dmul_rn(b[i], b[i]);
        if (terms) terms[i] = t;
        else acc[0] += t;
    }
};

struct FinBB {
    SsState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const { s->bb = t[0]; }
};

// B_j = A B_{j-1} - theta B_{j-1} (tmp = A B_{j-1}; B_j = tmp; B_j.axpy(-theta, B_{j-1}))
// and ||B_j||^2
struct EpiNewton {
    const double* prev;
    double* out;
    double mtheta;
    double* terms;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        const double v = __dadd_rn(ax, __dmul_rn(mtheta, prev[i]));
        out[i] = v;
        const double t = __dmul_rn(v, v);
        if (terms) terms[i] = t;
        else acc[0] += t;
    }
};

struct FinNorm2 {
    SsState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        s->nrm2 = t[0];
        const double nj = sqrt(t[0]);
        s->inv = (nj > kEps) ? 1.0 / nj : 1.0;
    }
};

// B_j *= 1 / ||B_j|| when ||B_j|| > eps (Vector::scale)
struct BodyScaleDev {
    double* v;
    const SsState* s;
    double inv;
    __device__ __forceinline__ void load() { inv = s->inv; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const { v[i] = __dmul_rn(v[i], inv); }
};

struct BodyScale {
    const double* src;
    double* dst;
    double a;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const { dst[i] = __dmul_rn(src[i], a); }
};

struct BodyCopy {
    const double* src;
    double* dst;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const { dst[i] = src[i]; }
};

// r = b - A x, ||r||^2
struct EpiResid {
    const double* b;
    double* r;
    double* terms;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        const double ri = __dsub_rn(b[i], ax);
        r[i] = ri;
        const double t = __dmul_rn(ri, ri);
        if (terms) terms[i] = t;
        else acc[0] += t;
    }
};

struct FinRR {
    SsState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const { s->rr = t[0]; }
};

// Ap = A r; r . r and r . Ap
struct EpiAp {
    const double* r;
    double* ap;
    double* terms;
    int n;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        ap[i] = ax;
        const double ri = r[i];
        const double t0 = __dmul_rn(ri, ri), t1 = __dmul_rn(ri, ax);
        if (terms) {
            terms[i] = t0;
            terms[n + i] = t1;
        } else {
            acc[0] += t0;
            acc[1] += t1;
        }
    }
};

struct FinRrRap {
    SsState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        s->rr = t[0];
        s->rap = t[1];
    }
};

// x += alpha r ; r -= alpha Ap ; ||r||^2
struct BodySteep {
    double* x;
    double* r;
    const double* ap;
    double alpha;
    double* terms;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&acc)[NV]) const {
        const double ri = r[i];
        x[i] = __dadd_rn(x[i], __dmul_rn(alpha, ri));
        const double rn = __dadd_rn(ri, __dmul_rn(-alpha, ap[i]));
        r[i] = rn;
        const double t = __dmul_rn(rn, rn);
        if (terms) terms[i] = t;
        else acc[0] += t;
    }
};

// The stored terms of NV reductions added in row order by one thread each (separate
// adds from 0.0), then handed to the reduction's finaliser.
constexpr int kSeqRows = 1 << 15;

template <int NV, typename Fin>
__global__ void k_seq_sum(int n, const double* __restrict__ terms, Fin fin) {
    __shared__ double tot[NV];
    if (threadIdx.x < NV) {
        double acc = 0.0;
        for (int i = 0; i < n; ++i) acc = __dadd_rn(acc, terms[(size_t)threadIdx.x * n + i]);
        tot[threadIdx.x] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[NV];
        for (int k = 0; k < NV; ++k) t[k] = tot[k];
        fin(t);
    }
}

struct Coeffs {
    double y[kMaxS];
};

// x += y_i B_i for i = 0..k-1 in that order (x.axpy(y[i], B[i]))
__global__ void __launch_bounds__(256)
k_sstep_update(int n, int k, double* x, const double* __restrict__ B, long long ld, Coeffs c) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double xi = x[i];
        for (int q = 0; q < k; ++q) xi = __dadd_rn(xi, __dmul_rn(c.y[q], B[q * ld + i]));
        x[i] = xi;
    }
}

// chebyshev_shifts (sstep_cg_solver.cpp:26-37)
std::vector<double> chebyshev_shifts(double lo, double hi, int k) {
    std::vector<double> t(k);
    const double c = 0.5 * (lo + hi), h = 0.5 * (hi - lo);
    for (int j = 0; j < k; ++j) t[j] = c + h * std::cos(M_PI * (2.0 * j + 1.0) / (2.0 * k));
    return t;
}

// gram_condition_estimate (sstep_cg_solver.cpp:108-119)
double gram_cond(const std::vector<double>& G, int k, int ldg) {
    double mx = 0.0, mn = INFINITY;
    for (int i = 0; i < k; ++i) {
        const double d = std::fabs(G[(size_t)i * ldg + i]);
        mx = std::max(mx, d);
        if (d > kEps) mn = std::min(mn, d);
    }
    if (mn >= mx) return 1.0;
    return mx / mn;
}

// local_lstsq (sstep_cg_solver.cpp:125-164): Cholesky of G, two triangular solves
bool cholesky_solve(const std::vector<double>& G, int ldg, const std::vector<double>& rhs, int k,
                    std::vector<double>& y) {
    std::vector<double> L((size_t)k * k, 0.0);
    for (int i = 0; i < k; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = G[(size_t)i * ldg + j];
            for (int l = 0; l < j; ++l) s -= L[(size_t)i * k + l] * L[(size_t)j * k + l];
            if (i == j) {
                if (s <= 0.0) return false;
                L[(size_t)i * k + j] = std::sqrt(s);
            } else {
                L[(size_t)i * k + j] = s / L[(size_t)j * k + j];
            }
        }
    std::vector<double> z(k, 0.0);
    for (int i = 0; i < k; ++i) {
        double s = rhs[i];
        for (int j = 0; j < i; ++j) s -= L[(size_t)i * k + j] * z[j];
        z[i] = s / L[(size_t)i * k + i];
    }
    y.assign(k, 0.0);
    for (int i = k - 1; i >= 0; --i) {
        double s = z[i];
        for (int j = i + 1; j < k; ++j) s -= L[(size_t)j * k + i] * y[j];
        y[i] = s / L[(size_t)i * k + i];
    }
    return true;
}

}  // namespace


SolveResult sstep_solve(Ctx& ctx, hamlss_mat* A, const double* b, double* x, const hamlss_params& p,
                        Workspace& ws) {
    const int n = A->A.n;
    const long long nz = A->A.nnz;
    if (p.sstep_k < 1 || p.sstep_k > kMaxS)
        fail(HAMLSS_ERR_INVALID, "sstep_k must be in [1, 32]");
    const int k = std::min(p.sstep_k, std::max(1, n / 10));     // sstep_cg_solver.cpp:179
    const Lane& L = ctx.lane;
    const int sm = ctx.sm_count;
    cudaStream_t st = L.stream;
    SolveResult res;
    HAMLSS_CUDA(cudaEventRecord(ctx.ev0, st));
    // spectral interval for the shifts (sstep_cg_solver.cpp:182-184)
    double lo = 0.0, hi = 0.0;
    {
        ProfScope ps(L, "sstep_setup", 0.0);
        spectral_interval(ctx, A, 20, &lo, &hi);
    }
    const double lam_min = std::max(lo, kEps);
    const double lam_max = std::max(hi, lam_min * 2.0);
    // Y = [r, B_0 .. B_{k-1}] as columns of ld entries; Ap for the fallback step
    const long long ld = ((long long)n + 31) / 32 * 32;
    if (ld > INT_MAX) fail(HAMLSS_ERR_SIZE, "s-step basis larger than 2^31 rows");
    ws.basis.ensure((size_t)ld * (size_t)(k + 1));
    double* Y = ws.basis.p;
    double* r = Y;
    auto Bcol = [&](int i) { return Y + ld * (i + 1); };
    double* ap = (ws.d[3].ensure(n), ws.d[3].p);
    ws.state.ensure(sizeof(SsState));
    SsState* s = reinterpret_cast<SsState*>(ws.state.p);
    ws.small.ensure((size_t)(kMaxS + 1) * (kMaxS + 1));
    double* Gd = ws.small.p;
    HAMLSS_CUDA(cudaMemsetAsync(s, 0, sizeof(SsState), st));
    auto poll = [&](SsState& h) {
        HAMLSS_CUDA(cudaMemcpyAsync(ctx.host_poll.p, s, sizeof(SsState), cudaMemcpyDeviceToHost, st));
        HAMLSS_CUDA(cudaStreamSynchronize(st));
        std::memcpy(&h, ctx.host_poll.p, sizeof(SsState));
    };
    const long long spmv_f = 2 * nz;
    const long long spmv_b = ((long long)n + 1 + nz) * 4 + nz * 8 + (long long)n * 16;
    // r = b - A x, ||b|| (sstep_cg_solver.cpp:186-195)
    SsState h{};
    // small systems: every reduction in row order (k_seq_sum), as the reference sums
    DBuf<double> term_buf;
    double* terms = nullptr;
    if (n <= kSeqRows) {
        term_buf.ensure(2 * (size_t)std::max(n, 1));
        terms = term_buf.p;
    }
    auto seq1 = [&](auto fin) {
        if (!terms) return;
        k_seq_sum<1><<<1, 32, 0, st>>>(n, terms, fin);
        HAMLSS_LAUNCH_CHECK();
    };
    launch_spmv<double, 1>(sm, L, A->A.f64(), XVec<double>{x}, EpiResid{b, r, terms}, FinRR{s}, nullptr,
                           "sstep_residual", 24.0 * n);
    seq1(FinRR{s});
    launch_vec<1>(sm, L, n, BodyBB{b, terms}, FinBB{s}, nullptr, "vec", 8.0 * n);
    seq1(FinBB{s});
    poll(h);
    const double r0 = std::sqrt(h.rr);
    const double bnorm = std::sqrt(h.bb);
    res.initial_residual = r0;
    res.flops = 0;
    res.bytes = 0;
    if (bnorm < kEps) {
        res.converged = 1;
        res.final_residual = 0.0;
        return res;
    }
    double rel = r0 / bnorm;
    double rnorm = r0;
    if (rel < p.tol) {
        res.converged = 1;
        res.final_residual = rel;
        return res;
    }
    res.sstep_k = k;
    long long flops = 0, bytes = 0;
    int total = 0;
    std::vector<double> G;
    DBuf<double> gram_part;
    auto build = [&](int kb) {
        // build_basis (sstep_cg_solver.cpp:44-66)
        const std::vector<double> th = chebyshev_shifts(lam_min, lam_max, kb);
        if (rnorm > kEps) launch_vec<0>(sm, L, n, BodyScale{r, Bcol(0), 1.0 / rnorm}, NoFin{}, nullptr, "vec", 16.0 * n);
        else launch_vec<0>(sm, L, n, BodyCopy{r, Bcol(0)}, NoFin{}, nullptr, "vec", 16.0 * n);
        for (int j = 1; j < kb; ++j) {
            launch_spmv<double, 1>(sm, L, A->A.f64(), XVec<double>{Bcol(j - 1)},
                                   EpiNewton{Bcol(j - 1), Bcol(j), -th[j - 1], terms}, FinNorm2{s}, nullptr,
                                   "sstep_basis", 24.0 * n);
            seq1(FinNorm2{s});
            launch_vec<0>(sm, L, n, BodyScaleDev{Bcol(j), s, 0.0}, NoFin{}, nullptr, "vec", 16.0 * n);
        }
        // gram_matrix (:71-80) and rhs_ls[i] = r . B[i] (:228-230): one (kb+1)^2 Gram matrix
        {
            ProfScope ps(L, "sstep_gram", 8.0 * (double)n * (kb + 1));
            gram_part.ensure((size_t)gram_partials(ctx, kb + 1));
            gram_matrix(ctx, n, kb + 1, Y, (long long)ld, Gd, gram_part.p);
        }
        G.assign((size_t)(kb + 1) * (kb + 1), 0.0);
        HAMLSS_CUDA(cudaMemcpyAsync(G.data(), Gd, sizeof(double) * G.size(), cudaMemcpyDeviceToHost, st));
        HAMLSS_CUDA(cudaStreamSynchronize(st));
    };
    while (total < p.max_iter && rel > p.tol) {
        int kb = k;
        build(kb);
        flops += (long long)kb * spmv_f;
        bytes += (long long)kb * spmv_b;
        // G[i][j] = B_i . B_j sits at (i + 1, j + 1) of the (kb+1)^2 product
        auto gram = [&](int kk) {
            std::vector<double> g((size_t)kk * kk);
            for (int i = 0; i < kk; ++i)
                for (int j = 0; j < kk; ++j) g[(size_t)i * kk + j] = G[(size_t)(i + 1) * (kk + 1) + (j + 1)];
            return g;
        };
        std::vector<double> Gk = gram(kb);
        const double cond = gram_cond(Gk, kb, kb);
        if (cond > p.sstep_cond_tol && kb > 1) {
            kb = std::max(1, kb / 2);
            build(kb);
            Gk = gram(kb);
        }
        ++res.comm_events;
        std::vector<double> rhs(kb);
        for (int i = 0; i < kb; ++i) rhs[i] = G[(size_t)0 * (kb + 1) + (i + 1)];
        flops += (long long)kb * 2 * n;
        std::vector<double> y;
        if (!cholesky_solve(Gk, kb, rhs, kb, y)) {
            // one steepest-descent step (sstep_cg_solver.cpp:236-250)
            launch_spmv<double, 2>(sm, L, A->A.f64(), XVec<double>{r}, EpiAp{r, ap, terms, n}, FinRrRap{s},
                                   nullptr, "sstep_fallback", 32.0 * n);
            if (terms) {
                k_seq_sum<2><<<1, 32, 0, st>>>(n, terms, FinRrRap{s});
                HAMLSS_LAUNCH_CHECK();
            }
            poll(h);
            double rn2 = h.rr;
            if (std::fabs(h.rap) > kEps) {
                const double alpha = h.rr / h.rap;
                launch_vec<1>(sm, L, n, BodySteep{x, r, ap, alpha, terms}, FinRR{s}, nullptr, "vec", 40.0 * n);
                seq1(FinRR{s});
                poll(h);
                rn2 = h.rr;
            }
            ++total;
            rnorm = std::sqrt(rn2);
            rel = rnorm / bnorm;
            if (p.verbose)
                std::fprintf(stderr, "  s-step CG: Cholesky failed, steepest step (r.Ap = %.3e)  iters=%d  rel_res=%.4e\n",
                             h.rap, total, rel);
            continue;
        }
        Coeffs c{};
        for (int i = 0; i < kb; ++i) c.y[i] = y[i];
        {
            ProfScope ps(L, "sstep_update", 8.0 * (double)n * (kb + 2));
            k_sstep_update<<<std::max(1, std::min(ceil_div(n, 256), sm * 8)), 256, 0, st>>>(
                n, kb, x, Bcol(0), ld, c);
            HAMLSS_LAUNCH_CHECK();
        }
        // exact residual every batch (:255-264)
        launch_spmv<double, 1>(sm, L, A->A.f64(), XVec<double>{x}, EpiResid{b, r, terms}, FinRR{s}, nullptr,
                               "sstep_residual", 24.0 * n);
        seq1(FinRR{s});
        flops += spmv_f;
        bytes += spmv_b;
        poll(h);
        rnorm = std::sqrt(h.rr);
        rel = rnorm / bnorm;
        total += kb;
        if (p.verbose)                                   // sstep_cg_solver.cpp:268-272
            std::fprintf(stderr, "  s-step CG: iters=%d  k=%d  kappa(G)=%.4e  rel_res=%.4e\n", total, kb,
                         cond, rel);
    }
    HAMLSS_CUDA(cudaEventRecord(ctx.ev1, st));
    HAMLSS_CUDA(cudaEventSynchronize(ctx.ev1));
    float ms = 0.f;
    HAMLSS_CUDA(cudaEventElapsedTime(&ms, ctx.ev0, ctx.ev1));
    res.device_time_s = ms * 1e-3;
    res.iterations = total;
    res.final_residual = rel;
    res.converged = rel < p.tol;
    res.flops = flops;
    res.bytes = bytes;
    return res;
}

}  // namespace hamlss
