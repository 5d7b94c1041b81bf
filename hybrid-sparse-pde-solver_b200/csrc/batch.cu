// batch.cu -- see batch.cuh.  Setup kernels, the persistent team solver, the autotuner.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

#include "batch.cuh"
#include "ilu_row.cuh"
#include "scan.cuh"

namespace hamlss {

namespace {

constexpr double kEps = 2.220446049250313e-16;
constexpr int kGroup = 8;               // accumulators per multi-dot group
constexpr int kMaxPhases = kBatchClasses;

struct Phase {
    int begin, end, width;              // systems order[begin, end), team width
};

struct BArgs {
    int nphase;
    Phase ph[kMaxPhases];
    const int* order;
    int* tickets;
    const BProb* prob;
    const int* rp;
    const int* ci;
    const double* v64;
    const float* v32;
    const float* dinv;
    const float* lu;
    const int* dpos;
    const int* lptrL;
    const int* lordL;
    const int* lptrU;
    const int* lordU;
    const int* pstatus;
    const double* b;
    double* x;
    double* r64;
    float* work;
    hamlss_batch_result* out;
    double tol, inner_tol;
    int max_iter, max_outer, m;
};

// ------------------------------------------------------------------ shared layout
// Per team (doubles): red[nw * R] | res[R] | H[(m+1) m] | cs[m] | sn[m] | g[m+1] | y[m] | slot
__host__ __device__ inline int team_stride(int W, int m) {
    const int R = m + 2;
    return (W / 32) * R + R + (m + 1) * m + 4 * m + 1 + 2;
}
inline size_t batch_smem(int W, int m) {
    return sizeof(double) * (size_t)(kBatchThreads / W) * team_stride(W, m);
}

struct Team {
    int W, lt, id, wit, R, m;
    double* red;
    double* res;
    double* H;
    double* cs;
    double* sn;
    double* g;
    double* y;
    int* slot;

    __device__ void init(int width, int mm, double* smem) {
        W = width;
        m = mm;
        R = m + 2;
        id = threadIdx.x / W;
        lt = threadIdx.x - id * W;
        wit = lt >> 5;
        double* base = smem + (size_t)id * team_stride(W, m);
        red = base;
        res = red + (W / 32) * R;
        H = res + R;
        cs = H + (m + 1) * m;
        sn = cs + m;
        g = sn + m;
        y = g + m + 1;
        slot = reinterpret_cast<int*>(y + m);
    }
    // team barrier: a warp syncs itself; wider teams use named barrier id + 1 (0 is the
    // CTA barrier), at most kBatchThreads / 64 = 8 of them
    __device__ __forceinline__ void sync() const {
        if (W == 32) __syncwarp();
        else asm volatile("bar.sync %0, %1;" ::"r"(id + 1), "r"(W) : "memory");
    }
    // stage one value for slot k of a team-wide sum (every lane of every warp calls it)
    __device__ __forceinline__ void put(double v, int k) const {
        v = warp_sum(v);
        if ((threadIdx.x & 31) == 0) red[wit * R + k] = v;
    }
    // finish nv staged sums; every thread may then read res[0, nv)
    __device__ __forceinline__ void finish(int nv) const {
        sync();
        if (lt < nv) {
            double s = 0.0;
            for (int w = 0; w < W / 32; ++w) s += red[w * R + lt];
            res[lt] = s;
        }
        sync();
    }
};

// FP64 row product in the reference's operation order (sparse_matrix.cpp:80-86)
__device__ __forceinline__ double row_ax64(int g, const BArgs& a, const double* x) {
    double s = 0.0;
    for (int k = __ldg(&a.rp[g]); k < __ldg(&a.rp[g + 1]); ++k)
        s = __dadd_rn(s, __dmul_rn(__ldg(&a.v64[k]), x[__ldg(&a.ci[k])]));
    return s;
}

// FP32 row product over a local vector (column c lives at v[c - row0])
__device__ __forceinline__ float row_ax32(int g, int row0, const BArgs& a, const float* v) {
    float s = 0.f;
    for (int k = __ldg(&a.rp[g]); k < __ldg(&a.rp[g + 1]); ++k)
        s = __fmaf_rn(__ldg(&a.v32[k]), v[__ldg(&a.ci[k]) - row0], s);
    return s;
}

// ---------------------------------------------------------------- inner PCG (FP32)
struct CgZ {
    const float* R;
    const float* dinv;     // null: no preconditioner
    __device__ __forceinline__ float operator()(int i) const {
        return dinv ? __fmul_rn(__ldg(&dinv[i]), R[i]) : R[i];
    }
};

__device__ int inner_cg(const Team& T, const BArgs& a, const BProb& P, float* w, double itol,
                        int maxit) {
    const int n = P.n, r0 = P.row0;
    float* R = w;
    float* Pa = w + n;
    float* Pb = w + 2 * (size_t)n;
    float* Q = w + 3 * (size_t)n;
    float* D = w + 4 * (size_t)n;
    const CgZ z{R, P.method == BM_CG_JAC ? a.dinv + r0 : nullptr};
    double rz = 0.0, rr = 0.0;
    for (int i = T.lt; i < n; i += T.W) {
        const float r = R[i];
        rz += (double)r * (double)z(i);
        rr += (double)r * (double)r;
        Pa[i] = 0.f;
    }
    T.put(rz, 0);
    T.put(rr, 1);
    T.finish(2);
    double rho = T.res[0];
    const double rn0 = sqrt(T.res[1]);
    if (!(rn0 > 0.0)) return 0;
    float beta = 0.f;
    const float* pold = Pa;
    float* pnew = Pb;
    int it = 0;
    while (it < maxit) {
        // q = A p with p = z + beta p_old formed on the fly; p.q
        double pq = 0.0;
        for (int i = T.lt; i < n; i += T.W) {
            const int g = r0 + i;
            float s = 0.f;
            for (int k = __ldg(&a.rp[g]); k < __ldg(&a.rp[g + 1]); ++k) {
                const int j = __ldg(&a.ci[k]) - r0;
                s = __fmaf_rn(__ldg(&a.v32[k]), __fmaf_rn(beta, pold[j], z(j)), s);
            }
            const float pi = __fmaf_rn(beta, pold[i], z(i));
            pnew[i] = pi;
            Q[i] = s;
            pq += (double)pi * (double)s;
        }
        T.put(pq, 0);
        T.finish(1);
        pq = T.res[0];
        if (!(fabs(pq) > kEps * 1e6 * fabs(rho))) break;        // breakdown or NaN
        const float af = (float)(rho / pq);
        rr = 0.0;
        rz = 0.0;
        for (int i = T.lt; i < n; i += T.W) {
            D[i] = __fmaf_rn(af, pnew[i], D[i]);
            const float r = __fmaf_rn(-af, Q[i], R[i]);
            R[i] = r;
            rr += (double)r * (double)r;
            rz += (double)r * (double)z(i);
        }
        T.put(rr, 0);
        T.put(rz, 1);
        T.finish(2);
        ++it;
        const double rel = sqrt(T.res[0]) / rn0;
        if (!(rel >= itol)) break;                               // converged or NaN
        if (!(fabs(rho) > 0.0)) break;
        beta = (float)(T.res[1] / rho);
        rho = T.res[1];
        const float* t = pold;
        pold = pnew;
        pnew = const_cast<float*>(t);
    }
    return it;
}

// ------------------------------------------------------------- preconditioner (FP32)
// z = M^-1 v for the FGMRES systems; ends with a team barrier.
__device__ void bprec(const Team& T, const BArgs& a, const BProb& P, const float* v, float* z,
                      float* Y) {
    const int n = P.n, r0 = P.row0;
    if (P.method == BM_GM_ILU) {
        // L y = v (unit lower, ilu.cpp:225-239), level by level
        for (int l = 0; l < P.nlevL; ++l) {
            const int b = __ldg(&a.lptrL[P.levL + l]), e = __ldg(&a.lptrL[P.levL + l + 1]);
            for (int t = b + T.lt; t < e; t += T.W) {
                const int g = __ldg(&a.lordL[t]);
                float s = v[g - r0];
                // columns are sorted, so the entries left of the diagonal are exactly c < g
                const int d = __ldg(&a.dpos[g]);
                for (int p = __ldg(&a.rp[g]); p < d; ++p)
                    s = __fmaf_rn(-__ldg(&a.lu[p]), Y[__ldg(&a.ci[p]) - r0], s);
                Y[g - r0] = s;
            }
            T.sync();
        }
        // U z = y (ilu.cpp:244-262), level by level
        for (int l = 0; l < P.nlevU; ++l) {
            const int b = __ldg(&a.lptrU[P.levU + l]), e = __ldg(&a.lptrU[P.levU + l + 1]);
            for (int t = b + T.lt; t < e; t += T.W) {
                const int g = __ldg(&a.lordU[t]);
                const int d = __ldg(&a.dpos[g]);
                float s = Y[g - r0];
                for (int p = d + 1; p < __ldg(&a.rp[g + 1]); ++p)
                    s = __fmaf_rn(-__ldg(&a.lu[p]), z[__ldg(&a.ci[p]) - r0], s);
                z[g - r0] = __fdiv_rn(s, __ldg(&a.lu[d]));
            }
            T.sync();
        }
        return;
    }
    const float* dv = P.method == BM_GM_JAC ? a.dinv + r0 : nullptr;
    for (int i = T.lt; i < n; i += T.W) z[i] = dv ? __fmul_rn(__ldg(&dv[i]), v[i]) : v[i];
    T.sync();
}

// Team sums of V_k . w for k < nv (w read from W), staged in groups of kGroup.
__device__ void multi_dot(const Team& T, const float* V, size_t n, int nv, const float* W) {
    for (int g0 = 0; g0 < nv; g0 += kGroup) {
        double acc[kGroup];
#pragma unroll
        for (int q = 0; q < kGroup; ++q) acc[q] = 0.0;
        for (int i = T.lt; i < (int)n; i += T.W) {
            const double wi = W[i];
#pragma unroll
            for (int q = 0; q < kGroup; ++q)
                if (g0 + q < nv) acc[q] += (double)V[(size_t)(g0 + q) * n + i] * wi;
        }
#pragma unroll
        for (int q = 0; q < kGroup; ++q)
            if (g0 + q < nv) T.put(acc[q], g0 + q);
    }
    T.finish(nv);
}

// ------------------------------------------------------------- inner FGMRES (FP32)
__device__ int inner_gmres(const Team& T, const BArgs& a, const BProb& P, float* w, double itol,
                           int maxit) {
    const int n = P.n, r0 = P.row0, m = a.m;
    const size_t nn = (size_t)n;
    float* R = w;
    float* D = w + nn;
    float* Wv = w + 2 * nn;
    float* Y = w + 3 * nn;
    float* V = w + 4 * nn;
    float* Z = w + (4 + (size_t)m + 1) * nn;
    int it = 0;
    double beta0 = -1.0;
    while (it < maxit) {
        // v0 = R - A D
        double bb = 0.0;
        for (int i = T.lt; i < n; i += T.W) {
            float s = R[i];
            if (beta0 >= 0.0) s -= row_ax32(r0 + i, r0, a, D);
            V[i] = s;
            bb += (double)s * (double)s;
        }
        T.put(bb, 0);
        T.finish(1);
        const double beta = sqrt(T.res[0]);
        if (beta0 < 0.0) beta0 = beta;
        if (!(beta > itol * beta0)) break;                      // converged, zero rhs or NaN
        const float inv = (float)(1.0 / beta);
        for (int i = T.lt; i < n; i += T.W) V[i] = __fmul_rn(V[i], inv);
        if (T.lt == 0) {
            T.g[0] = beta;
            for (int k = 1; k <= m; ++k) T.g[k] = 0.0;
        }
        T.sync();
        int jend = 0;
        bool done = false;
        for (int j = 0; j < m && it < maxit; ++j) {
            const float* Vj = V + (size_t)j * nn;
            float* Zj = Z + (size_t)j * nn;
            bprec(T, a, P, Vj, Zj, Y);
            // w = A z_j ; h = V^T w
            for (int i = T.lt; i < n; i += T.W) Wv[i] = row_ax32(r0 + i, r0, a, Zj);
            multi_dot(T, V, nn, j + 1, Wv);
            if (T.lt <= j) T.H[T.lt * m + j] = T.res[T.lt];
            T.sync();
            // w -= V h ; h2 = V^T w   (classical Gram-Schmidt, second pass)
            for (int i = T.lt; i < n; i += T.W) {
                float wi = Wv[i];
                for (int k = 0; k <= j; ++k) wi = __fmaf_rn(-(float)T.H[k * m + j], V[(size_t)k * nn + i], wi);
                Wv[i] = wi;
            }
            multi_dot(T, V, nn, j + 1, Wv);
            // w -= V h2 ; ||w||^2
            double ww = 0.0;
            for (int i = T.lt; i < n; i += T.W) {
                float wi = Wv[i];
                for (int k = 0; k <= j; ++k) wi = __fmaf_rn(-(float)T.res[k], V[(size_t)k * nn + i], wi);
                Wv[i] = wi;
                ww += (double)wi * (double)wi;
            }
            // H[k][j] += h2[k]: res still holds h2 until the next finish
            T.sync();
            if (T.lt <= j) T.H[T.lt * m + j] += T.res[T.lt];
            T.put(ww, m + 1);
            T.sync();
            if (T.lt == 0) {
                double s = 0.0;
                for (int q = 0; q < T.W / 32; ++q) s += T.red[q * T.R + m + 1];
                T.res[m + 1] = s;
            }
            T.sync();
            const double hn = sqrt(T.res[m + 1]);
            float* Vn = V + (size_t)(j + 1) * nn;
            const float sc = hn > kEps ? (float)(1.0 / hn) : 0.f;     // fgmres_solver.cpp:129-131
            for (int i = T.lt; i < n; i += T.W) Vn[i] = __fmul_rn(Wv[i], sc);
            if (T.lt == 0) {
                double* H = T.H;
                H[(j + 1) * m + j] = hn;
                for (int k = 0; k < j; ++k) {          // previous rotations (fgmres_solver.cpp:134-138)
                    const double t = T.cs[k] * H[k * m + j] + T.sn[k] * H[(k + 1) * m + j];
                    H[(k + 1) * m + j] = -T.sn[k] * H[k * m + j] + T.cs[k] * H[(k + 1) * m + j];
                    H[k * m + j] = t;
                }
                const double x1 = H[j * m + j], x2 = H[(j + 1) * m + j];
                double c, s;
                if (x2 == 0.0) { c = 1.0; s = 0.0; }
                else if (fabs(x2) > fabs(x1)) { const double t = x1 / x2; s = 1.0 / sqrt(1.0 + t * t); c = s * t; }
                else { const double t = x2 / x1; c = 1.0 / sqrt(1.0 + t * t); s = c * t; }
                T.cs[j] = c;
                T.sn[j] = s;
                H[j * m + j] = c * x1 + s * x2;
                H[(j + 1) * m + j] = 0.0;
                T.g[j + 1] = -s * T.g[j];
                T.g[j] = c * T.g[j];
            }
            T.sync();
            ++it;
            jend = j + 1;
            if (!(fabs(T.g[j + 1]) >= itol * beta0)) { done = true; break; }
        }
        // y = H^-1 g (fgmres_solver.cpp:57-66), D += Z y
        if (T.lt == 0) {
            for (int k = jend - 1; k >= 0; --k) {
                double s = T.g[k];
                for (int l = k + 1; l < jend; ++l) s -= T.H[k * m + l] * T.y[l];
                const double d = T.H[k * m + k];
                T.y[k] = fabs(d) > 0.0 ? s / d : 0.0;
            }
        }
        T.sync();
        for (int i = T.lt; i < n; i += T.W) {
            float d = D[i];
            for (int k = 0; k < jend; ++k) d = __fmaf_rn((float)T.y[k], Z[(size_t)k * nn + i], d);
            D[i] = d;
        }
        T.sync();
        if (done || jend == 0) break;
    }
    return it;
}

// ------------------------------------------------------ one system: FP64 refinement
__device__ void solve_one(const Team& T, const BArgs& a, int k) {
    const BProb P = a.prob[k];
    const int n = P.n, r0 = P.row0;
    float* w = a.work + P.w0;
    const bool cg = P.method == BM_CG_JAC || P.method == BM_CG_NONE;
    float* R = w;
    float* D = cg ? w + 4 * (size_t)n : w + (size_t)n;
    int status = a.pstatus[k];
    int total = 0, outer = 0, conv = 0;
    double rel = 0.0, rinit = 0.0;
    while (status == HAMLSS_OK) {
        double bb = 0.0, rr = 0.0;
        for (int i = T.lt; i < n; i += T.W) {
            const int g = r0 + i;
            const double bi = a.b[g];
            const double ri = __dsub_rn(bi, row_ax64(g, a, a.x));
            a.r64[g] = ri;
            bb += bi * bi;
            rr += ri * ri;
        }
        T.put(bb, 0);
        T.put(rr, 1);
        T.finish(2);
        const double bn = sqrt(T.res[0]), rn = sqrt(T.res[1]);
        if (outer == 0) rinit = rn;
        if (!isfinite(bn) || !isfinite(rn)) { status = HAMLSS_ERR_NONFINITE; break; }
        if (bn < kEps) { conv = 1; rel = rn; break; }       // cg_solver.cpp:60-64
        rel = rn / bn;
        if (rel < a.tol) { conv = 1; break; }
        if (outer >= a.max_outer || total >= a.max_iter) break;
        const double inv = 1.0 / rn;
        for (int i = T.lt; i < n; i += T.W) {
            R[i] = (float)(a.r64[r0 + i] * inv);
            D[i] = 0.f;
        }
        T.sync();
        const double itol = fmax(a.inner_tol, 0.5 * a.tol / rel);
        const int its = cg ? inner_cg(T, a, P, w, itol, a.max_iter - total)
                           : inner_gmres(T, a, P, w, itol, a.max_iter - total);
        total += its;
        for (int i = T.lt; i < n; i += T.W) a.x[r0 + i] += rn * (double)D[i];
        T.sync();
        ++outer;
        if (its == 0) break;
    }
    if (T.lt == 0) {
        hamlss_batch_result o;
        o.iterations = total;
        o.outer_iterations = outer;
        o.converged = conv;
        o.status = status;
        o.initial_residual = rinit;
        o.final_residual = rel;
        a.out[k] = o;
    }
    T.sync();
}

__global__ void __launch_bounds__(kBatchThreads) k_batch_solve(BArgs a) {
    extern __shared__ double smem[];
    for (int p = 0; p < a.nphase; ++p) {
        Team T;
        T.init(a.ph[p].width, a.m, smem);
        const int cnt = a.ph[p].end - a.ph[p].begin;
        for (;;) {
            if (T.lt == 0) *T.slot = atomicAdd(&a.tickets[p], 1);
            T.sync();
            const int q = *T.slot;
            T.sync();
            if (q >= cnt) break;
            solve_one(T, a, a.order[a.ph[p].begin + q]);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ setup kernels
__global__ void k_prob_rows(int count, const BProb* __restrict__ prob, int* prow) {
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        const BProb P = prob[k];
        for (int i = threadIdx.x; i < P.n; i += blockDim.x) prow[P.row0 + i] = k;
    }
}

// columns inside the own block; diagonal; Jacobi inverse; FP32 values
__global__ void k_batch_rows(int N, const int* __restrict__ prow, const BProb* __restrict__ prob,
                             const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ v, double omega, float* v32, int* dpos,
                             float* dinv, int* pstatus, int* bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int k = prow[i];
        const BProb P = prob[k];
        int d = -1;
        for (int q = rp[i]; q < rp[i + 1]; ++q) {
            const int c = ci[q];
            if (c < P.row0 || c >= P.row0 + P.n) atomicMin(bad, i);
            if (c == i) d = q;
            v32[q] = (float)v[q];
        }
        dpos[i] = d;
        const double a = d >= 0 ? v[d] : 0.0;
        const bool jac = P.method == BM_CG_JAC || P.method == BM_GM_JAC;
        if (jac && fabs(a) < kEps) pstatus[k] = HAMLSS_ERR_ZERO_DIAG;     // jacobi.cpp:28-30
        dinv[i] = fabs(a) < kEps ? 0.f : (float)(omega / a);
    }
}

__global__ void k_level_max(int N, const int* __restrict__ prow, const BProb* __restrict__ prob,
                            const int* __restrict__ lvL, const int* __restrict__ lvU, int* nL, int* nU) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int k = prow[i];
        if (prob[k].method != BM_GM_ILU) continue;
        atomicMax(&nL[k], lvL[i] + 1);
        atomicMax(&nU[k], lvU[i] + 1);
    }
}

template <bool FILL>
__global__ void k_level_bucket(int N, const int* __restrict__ prow, const BProb* __restrict__ prob,
                               const int* __restrict__ lvL, const int* __restrict__ lvU, int* cL, int* cU,
                               int* ordL, int* ordU) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int k = prow[i];
        const BProb P = prob[k];
        if (P.method != BM_GM_ILU) continue;
        const int sl = P.levL + lvL[i], su = P.levU + lvU[i];
        if (FILL) {
            ordL[atomicAdd(&cL[sl], 1)] = i;
            ordU[atomicAdd(&cU[su], 1)] = i;
        } else {
            atomicAdd(&cL[sl], 1);
            atomicAdd(&cU[su], 1);
        }
    }
}

// ILU(0) of the ILU systems, one block per system, level by level (ilu.cpp:41-89);
// then the backward-sweep diagonal check (ilu.cpp:257-259).
__global__ void k_batch_ilu(int nsys, const int* __restrict__ sys, const BProb* __restrict__ prob,
                            const int* __restrict__ lptrL, const int* __restrict__ lordL,
                            const int* __restrict__ rp, const int* __restrict__ ci,
                            const int* __restrict__ dpos, double* lu, int* zp, int* pstatus) {
    for (int s = blockIdx.x; s < nsys; s += gridDim.x) {
        const int k = sys[s];
        const BProb P = prob[k];
        for (int l = 0; l < P.nlevL; ++l) {
            for (int t = lptrL[P.levL + l] + threadIdx.x; t < lptrL[P.levL + l + 1]; t += blockDim.x)
                ilu_row(lordL[t], rp, ci, dpos, lu, &zp[k]);
            __syncthreads();
        }
        for (int i = threadIdx.x; i < P.n; i += blockDim.x) {
            const int d = dpos[P.row0 + i];
            if (d < 0 || fabs(lu[d]) < kEps) atomicMin(&zp[k], P.row0 + i);
        }
        __syncthreads();
        if (threadIdx.x == 0 && zp[k] != INT_MAX && pstatus[k] == HAMLSS_OK) pstatus[k] = HAMLSS_ERR_ZERO_PIVOT;
        __syncthreads();
    }
}

__global__ void k_d2f_batch(const double* __restrict__ a, float* b, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

int klass_of(int n) {
    if (n <= 1024) return 0;
    if (n <= 4096) return 1;
    if (n <= 16384) return 2;
    return 3;
}

bool valid_width(int w) {
    for (int c : kBatchWidths)
        if (c == w) return true;
    return false;
}

}  // namespace

Batch::~Batch() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
}

std::unique_ptr<Batch> batch_create(Ctx& ctx, hamlss_ctx* h, int count, const int* row_off,
                                    const int* rp, const int* ci, const double* v,
                                    const int* solver, const int* precond, int where,
                                    const hamlss_params& p) {
    if (count <= 0 || !row_off || !rp || !ci || !v || !solver || !precond)
        fail(HAMLSS_ERR_INVALID, "batch: null argument or empty batch");
    if (p.restart_size < 1 || p.restart_size > kBatchMaxM)
        fail(HAMLSS_ERR_INVALID, "batch: restart_size must be in [1, 32]");
    if (row_off[0] != 0) fail(HAMLSS_ERR_MALFORMED, "batch: row_off[0] must be 0");
    for (int k = 0; k < count; ++k)
        if (row_off[k + 1] <= row_off[k]) fail(HAMLSS_ERR_MALFORMED, "batch: empty or decreasing system");
    auto B = std::make_unique<Batch>();
    B->ctx = h;
    B->count = count;
    B->N = row_off[count];
    B->m = p.restart_size;
    B->params = p;
    B->row_off.assign(row_off, row_off + count + 1);
    cudaStream_t s = ctx.lane.stream;
    const int N = B->N;
    // structure
    B->rp.ensure(N + 1);
    if (where == HAMLSS_HOST) B->rp.upload(rp, N + 1, s);
    else HAMLSS_CUDA(cudaMemcpyAsync(B->rp.p, rp, sizeof(int) * (N + 1), cudaMemcpyDeviceToDevice, s));
    int ends[2];
    HAMLSS_CUDA(cudaMemcpyAsync(&ends[0], B->rp.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    HAMLSS_CUDA(cudaMemcpyAsync(&ends[1], B->rp.p + N, sizeof(int), cudaMemcpyDeviceToHost, s));
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    if (ends[0] != 0 || ends[1] < 0) fail(HAMLSS_ERR_MALFORMED, "batch: row_ptr must start at 0");
    const int nnz = ends[1];
    B->nnz = nnz;
    B->ci.ensure(std::max(nnz, 1));
    B->v64.ensure(std::max(nnz, 1));
    if (where == HAMLSS_HOST) {
        B->ci.upload(ci, nnz, s);
        B->v64.upload(v, nnz, s);
    } else if (nnz) {
        HAMLSS_CUDA(cudaMemcpyAsync(B->ci.p, ci, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s));
        HAMLSS_CUDA(cudaMemcpyAsync(B->v64.p, v, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, s));
    }
    if (validate_csr(ctx, Csr<double>{N, N, nnz, B->rp.p, B->ci.p, B->v64.p}) != HAMLSS_OK)
        fail(HAMLSS_ERR_MALFORMED, "batch: CSR not well formed (row_ptr, column bounds or unsorted rows)");
    // systems
    B->hprob.resize(count);
    bool any_ilu = false;
    for (int k = 0; k < count; ++k) {
        BProb& P = B->hprob[k];
        P.row0 = row_off[k];
        P.n = row_off[k + 1] - row_off[k];
        P.klass = klass_of(P.n);
        if (solver[k] == HAMLSS_SOLVER_CG) {
            if (precond[k] == HAMLSS_PREC_JACOBI) P.method = BM_CG_JAC;
            else if (precond[k] == HAMLSS_PREC_NONE) P.method = BM_CG_NONE;
            else fail(HAMLSS_ERR_INVALID, "batch: CG systems take NONE or JACOBI");
        } else if (solver[k] == HAMLSS_SOLVER_FGMRES) {
            if (precond[k] == HAMLSS_PREC_ILU) P.method = BM_GM_ILU;
            else if (precond[k] == HAMLSS_PREC_JACOBI) P.method = BM_GM_JAC;
            else if (precond[k] == HAMLSS_PREC_NONE) P.method = BM_GM_NONE;
            else fail(HAMLSS_ERR_INVALID, "batch: FGMRES systems take NONE, JACOBI or ILU");
        } else {
            fail(HAMLSS_ERR_INVALID, "batch: solver must be CG or FGMRES");
        }
        any_ilu |= P.method == BM_GM_ILU;
        P.levL = P.levU = P.nlevL = P.nlevU = 0;
    }
    // work vectors
    long long off = 0;
    for (auto& P : B->hprob) {
        P.w0 = off;
        const bool cg = P.method == BM_CG_JAC || P.method == BM_CG_NONE;
        long long len = (cg ? 5LL : 2LL * B->m + 5) * P.n;
        off += (len + 63) / 64 * 64;
    }
    B->work.ensure(std::max<long long>(off, 1));
    B->prob.ensure(count);
    B->prob.upload(B->hprob.data(), count, s);
    const int g = std::max(1, std::min(ceil_div(N, 256), ctx.sm_count * 8));
    DBuf<int> prow(N), bad(1);
    k_prob_rows<<<std::min(count, ctx.sm_count * 8), 256, 0, s>>>(count, B->prob.p, prow.p);
    int init = INT_MAX;
    bad.upload(&init, 1, s);
    B->pstatus.ensure(count);
    B->pstatus.zero(s);
    B->v32.ensure(std::max(nnz, 1));
    B->dpos.ensure(N);
    B->dinv.ensure(N);
    k_batch_rows<<<g, 256, 0, s>>>(N, prow.p, B->prob.p, B->rp.p, B->ci.p, B->v64.p, p.jacobi_omega,
                                   B->v32.p, B->dpos.p, B->dinv.p, B->pstatus.p, bad.p);
    HAMLSS_LAUNCH_CHECK();
    int hbad = 0;
    bad.download(&hbad, 1, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    if (hbad != INT_MAX)
        fail(HAMLSS_ERR_MALFORMED, "batch: row " + std::to_string(hbad) + " reaches outside its system");
    // ILU(0) of the ILU systems
    B->lu.ensure(std::max(nnz, 1));
    if (any_ilu) {
        DBuf<int> dpos2, lvL, lvU;
        int nlL = 0, nlU = 0;
        pattern_levels(ctx, N, nnz, B->rp.p, B->ci.p, dpos2, lvL, lvU, &nlL, &nlU);
        DBuf<int> nL(count), nU(count);
        nL.zero(s);
        nU.zero(s);
        k_level_max<<<g, 256, 0, s>>>(N, prow.p, B->prob.p, lvL.p, lvU.p, nL.p, nU.p);
        HAMLSS_LAUNCH_CHECK();
        std::vector<int> hL(count), hU(count);
        nL.download(hL.data(), count, s);
        nU.download(hU.data(), count, s);
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        long long tl = 0, tu = 0;
        std::vector<int> sys;
        for (int k = 0; k < count; ++k) {
            BProb& P = B->hprob[k];
            if (P.method != BM_GM_ILU) continue;
            sys.push_back(k);
            P.levL = (int)tl;
            P.nlevL = hL[k];
            P.levU = (int)tu;
            P.nlevU = hU[k];
            tl += hL[k];
            tu += hU[k];
        }
        if (tl >= INT_MAX || tu >= INT_MAX) fail(HAMLSS_ERR_NOMEM, "batch: too many levels");
        B->prob.upload(B->hprob.data(), count, s);
        B->lptrL.ensure(tl + 1);
        B->lptrU.ensure(tu + 1);
        B->lptrL.zero(s);
        B->lptrU.zero(s);
        k_level_bucket<false><<<g, 256, 0, s>>>(N, prow.p, B->prob.p, lvL.p, lvU.p, B->lptrL.p, B->lptrU.p,
                                                nullptr, nullptr);
        HAMLSS_LAUNCH_CHECK();
        long long rowsL = exclusive_scan(ctx, B->lptrL.p, (int)tl + 1);
        exclusive_scan(ctx, B->lptrU.p, (int)tu + 1);
        B->lordL.ensure(std::max<long long>(rowsL, 1));
        B->lordU.ensure(std::max<long long>(rowsL, 1));
        DBuf<int> fL(tl + 1), fU(tu + 1);
        HAMLSS_CUDA(cudaMemcpyAsync(fL.p, B->lptrL.p, sizeof(int) * (tl + 1), cudaMemcpyDeviceToDevice, s));
        HAMLSS_CUDA(cudaMemcpyAsync(fU.p, B->lptrU.p, sizeof(int) * (tu + 1), cudaMemcpyDeviceToDevice, s));
        k_level_bucket<true><<<g, 256, 0, s>>>(N, prow.p, B->prob.p, lvL.p, lvU.p, fL.p, fU.p, B->lordL.p,
                                               B->lordU.p);
        HAMLSS_LAUNCH_CHECK();
        DBuf<double> lu64(std::max(nnz, 1));
        if (nnz)
            HAMLSS_CUDA(cudaMemcpyAsync(lu64.p, B->v64.p, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, s));
        DBuf<int> dsys(sys.size()), zp(count);
        dsys.upload(sys.data(), sys.size(), s);
        std::vector<int> zinit(count, INT_MAX);
        zp.upload(zinit.data(), count, s);
        k_batch_ilu<<<std::min<int>((int)sys.size(), ctx.sm_count * 16), 256, 0, s>>>(
            (int)sys.size(), dsys.p, B->prob.p, B->lptrL.p, B->lordL.p, B->rp.p, B->ci.p, B->dpos.p, lu64.p,
            zp.p, B->pstatus.p);
        HAMLSS_LAUNCH_CHECK();
        if (nnz) k_d2f_batch<<<g, 256, 0, s>>>(lu64.p, B->lu.p, nnz);
        HAMLSS_LAUNCH_CHECK();
        HAMLSS_CUDA(cudaStreamSynchronize(s));
    } else {
        B->lptrL.ensure(1);
        B->lptrU.ensure(1);
        B->lordL.ensure(1);
        B->lordU.ensure(1);
    }
    // schedule: classes largest first, longest system first inside a class
    std::vector<int> ord(count);
    for (int k = 0; k < count; ++k) ord[k] = k;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
        const BProb& a = B->hprob[x];
        const BProb& b = B->hprob[y];
        if (a.klass != b.klass) return a.klass > b.klass;
        return a.n > b.n;
    });
    B->order.ensure(count);
    B->order.upload(ord.data(), count, s);
    B->tickets.ensure(kMaxPhases);
    B->r64.ensure(N);
    B->xb.ensure(N);
    B->bb.ensure(N);
    B->out.ensure(count);
    HAMLSS_CUDA(cudaEventCreate(&B->e0));
    HAMLSS_CUDA(cudaEventCreate(&B->e1));
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    return B;
}

double batch_run(Ctx& ctx, Batch& B, const double* b, double* x, unsigned class_mask) {
    cudaStream_t s = ctx.lane.stream;
    BArgs a{};
    // phases in schedule order (classes descending), each a contiguous run of `order`
    int pos = 0;
    a.nphase = 0;
    std::vector<int> per(kBatchClasses, 0);
    for (const auto& P : B.hprob) per[P.klass]++;
    int wmin = kBatchThreads;
    for (int c = kBatchClasses - 1; c >= 0; --c) {
        if (!per[c]) continue;
        if (class_mask & (1u << c)) {
            a.ph[a.nphase++] = Phase{pos, pos + per[c], B.width[c]};
            wmin = std::min(wmin, B.width[c]);
        }
        pos += per[c];
    }
    if (a.nphase == 0) return 0.0;
    a.order = B.order.p;
    a.tickets = B.tickets.p;
    a.prob = B.prob.p;
    a.rp = B.rp.p;
    a.ci = B.ci.p;
    a.v64 = B.v64.p;
    a.v32 = B.v32.p;
    a.dinv = B.dinv.p;
    a.lu = B.lu.p;
    a.dpos = B.dpos.p;
    a.lptrL = B.lptrL.p;
    a.lordL = B.lordL.p;
    a.lptrU = B.lptrU.p;
    a.lordU = B.lordU.p;
    a.pstatus = B.pstatus.p;
    a.b = b;
    a.x = x;
    a.r64 = B.r64.p;
    a.work = B.work.p;
    a.out = B.out.p;
    a.tol = B.params.tol;
    a.inner_tol = B.params.ir_inner_tol;
    a.max_iter = B.params.max_iter;
    a.max_outer = B.params.ir_max_outer;
    a.m = B.m;
    const size_t smem = batch_smem(wmin, B.m);
    static DeviceOnce raised;            // the device's opt-in maximum, so no call lowers it
    raised(ctx.device, [&] {
        int optin = 0;
        HAMLSS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx.device));
        HAMLSS_CUDA(cudaFuncSetAttribute(k_batch_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    });
    int per_sm = occupancy_blocks(k_batch_solve, kBatchThreads, smem);
    const int blocks = std::max(1, per_sm * ctx.sm_count);
    HAMLSS_CUDA(cudaMemsetAsync(B.tickets.p, 0, sizeof(int) * kMaxPhases, s));
    // algorithmic bytes of one launch are not a fixed figure (iteration counts differ per
    // system); the profiler records the launch with 0 bytes
    ProfScope ps(ctx.lane, "batch_solve", 0.0);
    HAMLSS_CUDA(cudaEventRecord(B.e0, s));
    k_batch_solve<<<blocks, kBatchThreads, smem, s>>>(a);
    HAMLSS_LAUNCH_CHECK();
    HAMLSS_CUDA(cudaEventRecord(B.e1, s));
    HAMLSS_CUDA(cudaEventSynchronize(B.e1));
    float ms = 0.f;
    HAMLSS_CUDA(cudaEventElapsedTime(&ms, B.e0, B.e1));
    B.last_ms = ms;
    return ms;
}

void batch_autotune(Ctx& ctx, Batch& B, const double* b_dev, const char* cache_path, int* widths_out) {
    cudaStream_t s = ctx.lane.stream;
    cudaDeviceProp prop;
    HAMLSS_CUDA(cudaGetDeviceProperties(&prop, ctx.device));
    std::string dev(prop.name);
    for (auto& c : dev)
        if (c == ' ') c = '_';
    // method mix per class: bit 0 CG systems present, bit 1 FGMRES systems present
    int mix[kBatchClasses] = {0, 0, 0, 0}, per[kBatchClasses] = {0, 0, 0, 0};
    for (const auto& P : B.hprob) {
        mix[P.klass] |= (P.method == BM_CG_JAC || P.method == BM_CG_NONE) ? 1 : 2;
        per[P.klass]++;
    }
    auto key = [&](int c) {
        std::ostringstream o;
        o << dev << " class" << c << " mix" << mix[c] << " m" << B.m;
        return o.str();
    };
    std::map<std::string, int> cache;
    if (cache_path) {
        std::ifstream f(cache_path);
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream is(line);
            std::string d, c, mx, mm;
            int w = 0;
            if (is >> d >> c >> mx >> mm >> w && valid_width(w)) cache[d + " " + c + " " + mx + " " + mm] = w;
        }
    }
    B.xt.ensure(B.N);
    bool changed = false;
    for (int c = 0; c < kBatchClasses; ++c) {
        if (!per[c]) continue;
        auto it = cache.find(key(c));
        if (it != cache.end()) { B.width[c] = it->second; continue; }
        double best = 1e300;
        int bw = B.width[c];
        for (int w : kBatchWidths) {
            B.width[c] = w;
            HAMLSS_CUDA(cudaMemsetAsync(B.xt.p, 0, sizeof(double) * B.N, s));
            batch_run(ctx, B, b_dev, B.xt.p, 1u << c);      // warm
            HAMLSS_CUDA(cudaMemsetAsync(B.xt.p, 0, sizeof(double) * B.N, s));
            double ms = batch_run(ctx, B, b_dev, B.xt.p, 1u << c);
            if (ms < best) { best = ms; bw = w; }
        }
        B.width[c] = bw;
        cache[key(c)] = bw;
        changed = true;
    }
    if (cache_path && changed) {
        std::ofstream f(cache_path, std::ios::trunc);
        for (auto& kv : cache) f << kv.first << " " << kv.second << "\n";
    }
    for (int c = 0; c < kBatchClasses; ++c) widths_out[c] = B.width[c];
}

}  // namespace hamlss
