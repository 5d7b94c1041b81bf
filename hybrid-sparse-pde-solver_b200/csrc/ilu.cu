// ilu.cu -- ILU(0) on the device (ILUPreconditioner, ilu.cpp:41-89 and :225-271).
//
// Setup, all on the device:
//   1. level sets of the lower and upper triangles: level(i) = 1 + max level(j) over the
//      strictly lower (upper) columns j of row i.  Computed by a frontier sweep (Kahn's
//      order) inside ONE cooperative kernel, one grid barrier per level; the frontiers,
//      laid end to end, are the rows grouped by level.
//   2. the factorisation, level by level of the lower sets: each row runs the reference's
//      IKJ elimination (same pivots, same update order, separate multiply and subtract),
//      so the factor values equal the reference's lu_val_ bit for bit.
//   3. level-ordered copies of L (strictly lower part) and U (diagonal + upper part), so
//      the rows of one level are contiguous in memory.
// Apply: forward then backward sweep, one level per barrier.  With at most a few
// thousand rows per level (the natural-order 5-point grids here have <= n_side rows per
// level) one thread block per sweep is fastest: a block barrier costs far less than a
// grid barrier, and rows of the next level are prefetched while the current one waits.
// The arithmetic per row is the reference's (ilu.cpp:230-237, :249-260), so z is
// bit-identical to ILUPreconditioner::apply.
#include <cooperative_groups.h>

#include <cmath>
#include <cstring>

#include "ilu_row.cuh"
#include "krylov.cuh"
#include "scan.cuh"

namespace cg = cooperative_groups;

namespace hamlss {

namespace {

constexpr double kEps = 2.220446049250313e-16;

// ---------------------------------------------------------------- pattern helpers
// dpos[i] = position of a_ii in row i (-1 if absent); lcnt[i] = # columns < i;
// ucnt[i] = # columns > i.
__global__ void k_row_info(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           int* dpos, int* lcnt, int* ucnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int s = rp[i], e = rp[i + 1], d = -1, lo = 0, hi = 0;
        for (int k = s; k < e; ++k) {
            int c = ci[k];
            if (c < i) ++lo;
            else if (c == i) d = k;
            else ++hi;
        }
        dpos[i] = d;
        lcnt[i] = lo;
        ucnt[i] = hi;
    }
}

// column counts of the pattern (for the transpose)
__global__ void k_col_count(int n, const int* __restrict__ rp, const int* __restrict__ ci, int* cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; ++k) atomicAdd(&cnt[ci[k]], 1);
}

__global__ void k_col_fill(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           int* fillpos, int* trow) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; ++k) trow[atomicAdd(&fillpos[ci[k]], 1)] = i;
}

// single-block exclusive scan of n+1 ints in place (setup only)
__global__ void k_scan_inplace(int* a, int count) {
    __shared__ int carry;
    __shared__ int buf[1024];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < count; base += 1024) {
        int i = base + threadIdx.x;
        int v = i < count ? a[i] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            int t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
            __syncthreads();
            buf[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < count) a[i] = buf[threadIdx.x] - v + carry;   // exclusive
        __syncthreads();
        if (threadIdx.x == 1023) carry += buf[1023];
        __syncthreads();
    }
}

// Kahn frontier sweep over the dependency DAG of one triangle.
//   LOWER: row i depends on columns j < i of row i; dependents of j are the rows i > j
//          holding column j (transpose entries below the diagonal).
//   UPPER: mirror image.
// indeg must hold the dependency counts; on exit order[] lists the rows level by level,
// lptr[l] is where level l starts, level[i] is the level of row i, *nlev the count.
template <bool LOWER>
__global__ void k_levels(int n, const int* __restrict__ trp, const int* __restrict__ trow,
                         int* indeg, int* order, int* lptr, int* cnt, int* level, int* nlev) {
    cg::grid_group grid = cg::this_grid();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    for (int i = tid; i < n; i += nth)
        if (indeg[i] == 0) order[atomicAdd(&cnt[0], 1)] = i;
    grid.sync();
    int start = 0;
    for (int l = 0;; ++l) {
        const int c = *(volatile int*)&cnt[l];
        if (c == 0) {
            if (tid == 0) { *nlev = l; lptr[l] = start; }
            break;
        }
        if (tid == 0) lptr[l] = start;
        const int next = start + c;
        for (int t = tid; t < c; t += nth) {
            const int i = order[start + t];
            level[i] = l;
            for (int k = trp[i]; k < trp[i + 1]; ++k) {
                const int d = trow[k];
                if (LOWER ? (d > i) : (d < i)) {
                    if (atomicSub(&indeg[d], 1) == 1) order[next + atomicAdd(&cnt[l + 1], 1)] = d;
                }
            }
        }
        start = next;
        grid.sync();
    }
}

__global__ void k_ilu_factor_block(int nlev, const int* __restrict__ order, const int* __restrict__ lptr,
                                   const int* __restrict__ rp, const int* __restrict__ ci,
                                   const int* __restrict__ dpos, double* lu, int* status) {
    for (int l = 0; l < nlev; ++l) {
        const int b = lptr[l], e = lptr[l + 1];
        for (int t = b + threadIdx.x; t < e; t += blockDim.x) ilu_row(order[t], rp, ci, dpos, lu, status);
        __syncthreads();
    }
}

__global__ void k_ilu_factor_grid(int nlev, const int* __restrict__ order, const int* __restrict__ lptr,
                                  const int* __restrict__ rp, const int* __restrict__ ci,
                                  const int* __restrict__ dpos, double* lu, int* status) {
    cg::grid_group grid = cg::this_grid();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    for (int l = 0; l < nlev; ++l) {
        const int b = lptr[l], e = lptr[l + 1];
        for (int t = b + tid; t < e; t += nth) ilu_row(order[t], rp, ci, dpos, lu, status);
        grid.sync();
    }
}

// Level-ordered L / U copies.  Lrp/Urp are prefix sums of per-slot counts in order.
__global__ void k_perm_counts(int n, const int* __restrict__ order, const int* __restrict__ cnt,
                              int* out) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        out[t] = cnt[order[t]];
}

template <typename T>
__global__ void k_fill_L(int n, const int* __restrict__ order, const int* __restrict__ rp,
                         const int* __restrict__ ci, const double* __restrict__ lu,
                         const int* __restrict__ Lrp, int* Lci, T* Lv) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = order[t];
        int o = Lrp[t];
        for (int p = rp[i]; p < rp[i + 1]; ++p) {
            const int j = ci[p];
            if (j >= i) break;
            Lci[o] = j;
            Lv[o] = (T)lu[p];
            ++o;
        }
    }
}

// U copy: the diagonal (1.0 if absent, as backward_sub assumes, ilu.cpp:251) then the
// upper entries.  bad[0] receives the smallest row with |u_ii| < eps (ilu.cpp:257-259).
template <typename T>
__global__ void k_fill_U(int n, const int* __restrict__ order, const int* __restrict__ rp,
                         const int* __restrict__ ci, const double* __restrict__ lu,
                         const int* __restrict__ Urp, int* Uci, T* Uv, T* Ud, int* bad) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = order[t];
        int o = Urp[t];
        double d = 1.0;
        for (int p = rp[i]; p < rp[i + 1]; ++p) {
            const int j = ci[p];
            if (j == i) { d = lu[p]; continue; }
            if (j > i) { Uci[o] = j; Uv[o] = (T)lu[p]; ++o; }
        }
        Ud[t] = (T)d;
        if (bad && fabs(d) < kEps) atomicMin(bad, i);
    }
}

// ------------------------------------------------------------------------ sweeps
template <typename T>
struct IluLevels {
    int n, nlevL, nlevU;
    const int* ordL;
    const int* lptrL;
    const int* Lrp;
    const int* Lci;
    const T* Lv;
    const int* ordU;
    const int* lptrU;
    const int* Urp;
    const int* Uci;
    const T* Uv;
    const T* Ud;
};

template <typename T>
__device__ __forceinline__ T sub_mul(T s, T a, T b);
template <>
__device__ __forceinline__ double sub_mul<double>(double s, double a, double b) {
    return __dsub_rn(s, __dmul_rn(a, b));
}
template <>
__device__ __forceinline__ float sub_mul<float>(float s, float a, float b) {
    return __fsub_rn(s, __fmul_rn(a, b));
}

// L y = r (unit lower, forward_sub) then U z = y (backward_sub); one block.
template <typename T, int NT>
__global__ void __launch_bounds__(NT)
k_ilu_apply_block(IluLevels<T> F, const T* __restrict__ r, T* y, T* z, const int* gate) {
    if (gate && *(volatile const int*)gate) return;
    for (int l = 0; l < F.nlevL; ++l) {
        const int b = F.lptrL[l], e = F.lptrL[l + 1];
        for (int t = b + threadIdx.x; t < e; t += NT) {
            const int i = F.ordL[t];
            T s = r[i];
            for (int o = F.Lrp[t]; o < F.Lrp[t + 1]; ++o) s = sub_mul<T>(s, F.Lv[o], __ldcg(&y[F.Lci[o]]));
            y[i] = s;
        }
        __syncthreads();
    }
    for (int l = 0; l < F.nlevU; ++l) {
        const int b = F.lptrU[l], e = F.lptrU[l + 1];
        for (int t = b + threadIdx.x; t < e; t += NT) {
            const int i = F.ordU[t];
            T s = __ldcg(&y[i]);
            for (int o = F.Urp[t]; o < F.Urp[t + 1]; ++o) s = sub_mul<T>(s, F.Uv[o], __ldcg(&z[F.Uci[o]]));
            z[i] = s / F.Ud[t];
        }
        __syncthreads();
    }
}

// Same sweeps with the whole grid (cooperative launch) for matrices with wide levels.
template <typename T>
__global__ void k_ilu_apply_grid(IluLevels<T> F, const T* __restrict__ r, T* y, T* z, const int* gate) {
    if (gate && *(volatile const int*)gate) return;
    cg::grid_group grid = cg::this_grid();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    for (int l = 0; l < F.nlevL; ++l) {
        const int b = F.lptrL[l], e = F.lptrL[l + 1];
        for (int t = b + tid; t < e; t += nth) {
            const int i = F.ordL[t];
            T s = r[i];
            for (int o = F.Lrp[t]; o < F.Lrp[t + 1]; ++o) s = sub_mul<T>(s, F.Lv[o], __ldcg(&y[F.Lci[o]]));
            y[i] = s;
        }
        grid.sync();
    }
    for (int l = 0; l < F.nlevU; ++l) {
        const int b = F.lptrU[l], e = F.lptrU[l + 1];
        for (int t = b + tid; t < e; t += nth) {
            const int i = F.ordU[t];
            T s = __ldcg(&y[i]);
            for (int o = F.Urp[t]; o < F.Urp[t + 1]; ++o) s = sub_mul<T>(s, F.Uv[o], __ldcg(&z[F.Uci[o]]));
            z[i] = s / F.Ud[t];
        }
        grid.sync();
    }
}

template <typename K>
int coop_blocks(Ctx& ctx, K kernel, int threads) {
    int per = occupancy_blocks(kernel, threads);
    return std::max(1, std::min(per, 4) * ctx.sm_count);
}

template <typename K, typename... Args>
void coop_launch(Ctx& ctx, K kernel, int blocks, int threads, Args... args) {
    void* ptrs[] = {(void*)&args...};
    HAMLSS_CUDA(cudaLaunchCooperativeKernel((const void*)kernel, dim3(blocks), dim3(threads), ptrs, 0,
                                            ctx.lane.stream));
}

}  // namespace

// ---------------------------------------------------------------------- the object
struct IluPrec : Prec {
    hamlss_mat* A = nullptr;
    DBuf<int> dpos, lcnt, ucnt, trp, trow, indeg, cnt, levelL, levelU, nlev;
    DBuf<int> ordL, lptrL, ordU, lptrU, Lrp, Lci, Urp, Uci;
    DBuf<double> lu, Lv, Uv, Ud;
    DBuf<float> Lv32, Uv32, Ud32;
    DBuf<double> y;
    DBuf<float> y32;
    int nlevL = 0, nlevU = 0, nnzL = 0, nnzU = 0;
    int bad_diag_row = -1;       // backward_sub would throw on this row
    bool f32_ready = false;
    bool wide = false;

    IluLevels<double> view64() const {
        return IluLevels<double>{n, nlevL, nlevU, ordL.p, lptrL.p, Lrp.p, Lci.p, Lv.p,
                                 ordU.p, lptrU.p, Urp.p, Uci.p, Uv.p, Ud.p};
    }
    IluLevels<float> view32() const {
        return IluLevels<float>{n, nlevL, nlevU, ordL.p, lptrL.p, Lrp.p, Lci.p, Lv32.p,
                                ordU.p, lptrU.p, Urp.p, Uci.p, Uv32.p, Ud32.p};
    }

    void check_apply() const {
        if (bad_diag_row >= 0)
            fail(HAMLSS_ERR_ZERO_PIVOT,
                 "ILU backward sub: near-zero U diagonal at row " + std::to_string(bad_diag_row));
    }

    template <typename T>
    void run(Ctx& ctx, const Lane& L, const IluLevels<T>& F, const T* r, T* yb, T* z, const int* gate) {
        check_apply();
        if (!n) return;
        ProfScope ps(L, "ilu_sweep", (double)sizeof(T) * (nnzL + nnzU + 4.0 * n) + 4.0 * (nnzL + nnzU + 4.0 * n));
        if (!wide) {
            k_ilu_apply_block<T, 1024><<<1, 1024, 0, L.stream>>>(F, r, yb, z, gate);
            HAMLSS_LAUNCH_CHECK();
        } else {
            static const int blocks = coop_blocks(ctx, k_ilu_apply_grid<T>, 256);
            void* args[] = {(void*)&F, (void*)&r, (void*)&yb, (void*)&z, (void*)&gate};
            HAMLSS_CUDA(cudaLaunchCooperativeKernel((const void*)k_ilu_apply_grid<T>, dim3(blocks),
                                                    dim3(256), args, 0, L.stream));
        }
    }

    void apply(Ctx& ctx, const Lane& L, const double* r, double* z, const int* gate) override {
        run<double>(ctx, L, view64(), r, y.p, z, gate);
    }
    void prepare32(Ctx& ctx) override {
        if (f32_ready) return;
        cudaStream_t s = ctx.lane.stream;
        Lv32.ensure(nnzL); Uv32.ensure(nnzU); Ud32.ensure(n); y32.ensure(n);
        int g = std::max(1, std::min(ceil_div(n, 256), ctx.sm_count * 8));
        if (n) {
            k_fill_L<float><<<g, 256, 0, s>>>(n, ordL.p, A->A.rp.p, A->A.ci.p, lu.p, Lrp.p, Lci.p, Lv32.p);
            k_fill_U<float><<<g, 256, 0, s>>>(n, ordU.p, A->A.rp.p, A->A.ci.p, lu.p, Urp.p, Uci.p, Uv32.p,
                                              Ud32.p, nullptr);
            HAMLSS_LAUNCH_CHECK();
        }
        f32_ready = true;
    }
    void apply32(Ctx& ctx, const Lane& L, const float* r, float* z, const int* gate) override {
        prepare32(ctx);
        run<float>(ctx, L, view32(), r, y32.p, z, gate);
    }
    bool has32() const override { return true; }
};

std::unique_ptr<Prec> make_ilu0(Ctx& ctx, hamlss_mat* A) {
    auto P = std::make_unique<IluPrec>();
    P->kind = HAMLSS_PREC_ILU;
    P->A = A;
    const int n = A->A.n;
    const int nnz = A->A.nnz;
    P->n = n;
    if (A->A.n != A->A.m) fail(HAMLSS_ERR_SIZE, "ILU needs a square matrix");
    cudaStream_t s = ctx.lane.stream;
    AllocScope scope(s);                 // setup buffers from the stream-ordered pool
    const int g = std::max(1, std::min(ceil_div(n, 256), ctx.sm_count * 8));
    const int* rp = A->A.rp.p;
    const int* ci = A->A.ci.p;
    P->lu.ensure(nnz);
    P->y.ensure(n);
    if (nnz) HAMLSS_CUDA(cudaMemcpyAsync(P->lu.p, A->A.v.p, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, s));
    if (n == 0) return P;
    P->dpos.ensure(n); P->lcnt.ensure(n); P->ucnt.ensure(n);
    k_row_info<<<g, 256, 0, s>>>(n, rp, ci, P->dpos.p, P->lcnt.p, P->ucnt.p);
    HAMLSS_LAUNCH_CHECK();
    // transpose of the pattern: counts per column, exclusive scan over n+1 slots
    P->trp.ensure(n + 1); P->trow.ensure(nnz);
    HAMLSS_CUDA(cudaMemsetAsync(P->trp.p, 0, sizeof(int) * (n + 1), s));
    k_col_count<<<g, 256, 0, s>>>(n, rp, ci, P->trp.p);
    k_scan_inplace<<<1, 1024, 0, s>>>(P->trp.p, n + 1);
    HAMLSS_LAUNCH_CHECK();
    {
        DBuf<int> fill(n);
        HAMLSS_CUDA(cudaMemcpyAsync(fill.p, P->trp.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
        k_col_fill<<<g, 256, 0, s>>>(n, rp, ci, fill.p, P->trow.p);
        HAMLSS_LAUNCH_CHECK();
        HAMLSS_CUDA(cudaStreamSynchronize(s));
    }
    // level sets
    P->indeg.ensure(n); P->cnt.ensure(n + 2); P->nlev.ensure(2);
    P->ordL.ensure(n); P->lptrL.ensure(n + 1); P->levelL.ensure(n);
    P->ordU.ensure(n); P->lptrU.ensure(n + 1); P->levelU.ensure(n);
    {
        int lb = coop_blocks(ctx, k_levels<true>, 256);
        HAMLSS_CUDA(cudaMemcpyAsync(P->indeg.p, P->lcnt.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
        HAMLSS_CUDA(cudaMemsetAsync(P->cnt.p, 0, sizeof(int) * (n + 2), s));
        coop_launch(ctx, k_levels<true>, lb, 256, n, (const int*)P->trp.p, (const int*)P->trow.p,
                    P->indeg.p, P->ordL.p, P->lptrL.p, P->cnt.p, P->levelL.p, P->nlev.p);
        HAMLSS_CUDA(cudaMemcpyAsync(P->indeg.p, P->ucnt.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
        HAMLSS_CUDA(cudaMemsetAsync(P->cnt.p, 0, sizeof(int) * (n + 2), s));
        coop_launch(ctx, k_levels<false>, lb, 256, n, (const int*)P->trp.p, (const int*)P->trow.p,
                    P->indeg.p, P->ordU.p, P->lptrU.p, P->cnt.p, P->levelU.p, P->nlev.p + 1);
        int hl[2];
        HAMLSS_CUDA(cudaMemcpyAsync(hl, P->nlev.p, sizeof(hl), cudaMemcpyDeviceToHost, s));
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        P->nlevL = hl[0];
        P->nlevU = hl[1];
    }
    P->wide = (double)n / std::max(1, std::min(P->nlevL, P->nlevU)) > 4096.0;
    // factorisation
    {
        DBuf<int> status(1);
        int init = 0x7fffffff;
        status.upload(&init, 1, s);
        if (!P->wide) {
            k_ilu_factor_block<<<1, 1024, 0, s>>>(P->nlevL, P->ordL.p, P->lptrL.p, rp, ci, P->dpos.p,
                                                 P->lu.p, status.p);
            HAMLSS_LAUNCH_CHECK();
        } else {
            int fb = coop_blocks(ctx, k_ilu_factor_grid, 256);
            coop_launch(ctx, k_ilu_factor_grid, fb, 256, P->nlevL, (const int*)P->ordL.p,
                        (const int*)P->lptrL.p, rp, ci, (const int*)P->dpos.p, P->lu.p, status.p);
        }
        int h = 0;
        status.download(&h, 1, s);
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        if (h != 0x7fffffff)
            fail(HAMLSS_ERR_ZERO_PIVOT, "ILU(0): near-zero pivot at row " + std::to_string(h));
    }
    // level-ordered factor copies
    {
        P->Lrp.ensure(n + 1); P->Urp.ensure(n + 1);
        HAMLSS_CUDA(cudaMemsetAsync(P->Lrp.p, 0, sizeof(int) * (n + 1), s));
        HAMLSS_CUDA(cudaMemsetAsync(P->Urp.p, 0, sizeof(int) * (n + 1), s));
        k_perm_counts<<<g, 256, 0, s>>>(n, P->ordL.p, P->lcnt.p, P->Lrp.p);
        k_perm_counts<<<g, 256, 0, s>>>(n, P->ordU.p, P->ucnt.p, P->Urp.p);
        k_scan_inplace<<<1, 1024, 0, s>>>(P->Lrp.p, n + 1);
        k_scan_inplace<<<1, 1024, 0, s>>>(P->Urp.p, n + 1);
        HAMLSS_LAUNCH_CHECK();
        int h[2];
        HAMLSS_CUDA(cudaMemcpyAsync(&h[0], P->Lrp.p + n, sizeof(int), cudaMemcpyDeviceToHost, s));
        HAMLSS_CUDA(cudaMemcpyAsync(&h[1], P->Urp.p + n, sizeof(int), cudaMemcpyDeviceToHost, s));
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        P->nnzL = h[0];
        P->nnzU = h[1];
        P->Lci.ensure(P->nnzL); P->Lv.ensure(P->nnzL);
        P->Uci.ensure(P->nnzU); P->Uv.ensure(P->nnzU); P->Ud.ensure(n);
        DBuf<int> bad(1);
        int init = 0x7fffffff;
        bad.upload(&init, 1, s);
        k_fill_L<double><<<g, 256, 0, s>>>(n, P->ordL.p, rp, ci, P->lu.p, P->Lrp.p, P->Lci.p, P->Lv.p);
        k_fill_U<double><<<g, 256, 0, s>>>(n, P->ordU.p, rp, ci, P->lu.p, P->Urp.p, P->Uci.p, P->Uv.p,
                                           P->Ud.p, bad.p);
        HAMLSS_LAUNCH_CHECK();
        int hb = 0;
        bad.download(&hb, 1, s);
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        P->bad_diag_row = hb != 0x7fffffff ? hb : -1;
    }
    P->trow.release();
    P->indeg.release();
    return P;
}

// Level sets of the strictly lower and strictly upper dependency DAGs of a square CSR
// pattern (the definitions make_ilu0 uses), without factorising.  The batched solver
// calls this on its block-diagonal matrix: blocks never depend on one another, so every
// row's level is its level inside its own system.
void pattern_levels(Ctx& ctx, int n, int nnz, const int* rp, const int* ci, DBuf<int>& dpos,
                    DBuf<int>& levelL, DBuf<int>& levelU, int* nlevL, int* nlevU) {
    cudaStream_t s = ctx.lane.stream;
    dpos.ensure(std::max(n, 1));
    levelL.ensure(std::max(n, 1));
    levelU.ensure(std::max(n, 1));
    *nlevL = *nlevU = 0;
    if (n == 0) return;
    const int g = std::max(1, std::min(ceil_div(n, 256), ctx.sm_count * 8));
    DBuf<int> lcnt(n), ucnt(n), trp(n + 1), trow(std::max(nnz, 1)), fill(n), indeg(n), cnt(n + 2),
        order(n), lptr(n + 1), nl(2);
    k_row_info<<<g, 256, 0, s>>>(n, rp, ci, dpos.p, lcnt.p, ucnt.p);
    HAMLSS_CUDA(cudaMemsetAsync(trp.p, 0, sizeof(int) * (n + 1), s));
    k_col_count<<<g, 256, 0, s>>>(n, rp, ci, trp.p);
    HAMLSS_LAUNCH_CHECK();
    exclusive_scan(ctx, trp.p, n + 1);
    HAMLSS_CUDA(cudaMemcpyAsync(fill.p, trp.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    k_col_fill<<<g, 256, 0, s>>>(n, rp, ci, fill.p, trow.p);
    HAMLSS_LAUNCH_CHECK();
    const int lb = coop_blocks(ctx, k_levels<true>, 256);
    HAMLSS_CUDA(cudaMemcpyAsync(indeg.p, lcnt.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    HAMLSS_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (n + 2), s));
    coop_launch(ctx, k_levels<true>, lb, 256, n, (const int*)trp.p, (const int*)trow.p, indeg.p,
                order.p, lptr.p, cnt.p, levelL.p, nl.p);
    HAMLSS_CUDA(cudaMemcpyAsync(indeg.p, ucnt.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    HAMLSS_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (n + 2), s));
    coop_launch(ctx, k_levels<false>, lb, 256, n, (const int*)trp.p, (const int*)trow.p, indeg.p,
                order.p, lptr.p, cnt.p, levelU.p, nl.p + 1);
    int h[2];
    HAMLSS_CUDA(cudaMemcpyAsync(h, nl.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    *nlevL = h[0];
    *nlevU = h[1];
}

// Inspection entry points (hamlss.h).
int ilu_copy_factors(const Prec* M, double* out, cudaStream_t s) {
    auto* P = dynamic_cast<const IluPrec*>(M);
    if (!P) return HAMLSS_ERR_INVALID;
    if (P->A->A.nnz) P->lu.download(out, P->A->A.nnz, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    return HAMLSS_OK;
}

int ilu_copy_levels(const Prec* M, int which, int* level, int* nlev, cudaStream_t s) {
    auto* P = dynamic_cast<const IluPrec*>(M);
    if (!P) return HAMLSS_ERR_INVALID;
    if (P->n) (which == 0 ? P->levelL : P->levelU).download(level, P->n, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    *nlev = which == 0 ? P->nlevL : P->nlevU;
    return HAMLSS_OK;
}

}  // namespace hamlss
