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

#include <climits>
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
//
// One level's critical path is a barrier plus the loads of the vector being solved for; the
// rest of a row's inputs (its index, right-hand side, columns, values, diagonal) do not
// depend on the sweep, so they are fetched ahead in a three-stage pipeline: stage 1 (row
// index, row bounds) two levels ahead, stage 2 (rhs, up to kIluPre columns and values, the
// diagonal) one level ahead, while the current level computes.  The level pointers sit in
// shared memory.  A thread pipelines its first row of each level; rows beyond the block
// width and rows longer than kIluPre take the plain path.  The block's own stores are read
// back with ordinary loads after the barrier (block scope), and every row sums in its
// stored (ascending column) order, so results are bit-identical to the plain loop.
constexpr int kIluPre = 4;
constexpr int kIluLptrSmem = 4096;

template <typename T>
struct IluStage2 {
    int t, i, o0, cnt;
    T rv, d;
    int c[kIluPre];
    T v[kIluPre];
};

template <typename T, bool DIV, int NT>
__device__ __forceinline__ void ilu_sweep_block(int nlev, const int* __restrict__ lptr_g, const int* s_lptr,
                                                const int* __restrict__ ord, const int* __restrict__ rp,
                                                const int* __restrict__ ci, const T* __restrict__ v,
                                                const T* __restrict__ dg, const T* rhs, T* out) {
    auto lptr = [&](int l) { return l < kIluLptrSmem ? s_lptr[l] : __ldg(&lptr_g[l]); };
    const int tid = threadIdx.x;
    // stage 1 of a level: (t, i, o0, cnt) of this thread's first row, t = -1 if none
    auto stage1 = [&](int l, int& t, int& i, int& o0, int& cnt) {
        t = -1;
        if (l < nlev) {
            const int b = lptr(l), e = lptr(l + 1);
            if (b + tid < e) {
                t = b + tid;
                i = ord[t];
                o0 = rp[t];
                cnt = rp[t + 1] - o0;
            }
        }
    };
    auto stage2 = [&](IluStage2<T>& q, int t, int i, int o0, int cnt) {
        q.t = t;
        if (t < 0) return;
        q.i = i;
        q.o0 = o0;
        q.cnt = cnt;
        q.rv = rhs[i];
        if (DIV) q.d = dg[t];
#pragma unroll
        for (int k = 0; k < kIluPre; ++k)
            if (k < cnt) {
                q.c[k] = ci[o0 + k];
                q.v[k] = v[o0 + k];
            }
    };
    int t1, i1, o1, c1;                  // stage 1 of level l + 1
    IluStage2<T> cur;
    {
        int t0, i0, o0, c0;
        stage1(0, t0, i0, o0, c0);
        stage2(cur, t0, i0, o0, c0);
        stage1(1, t1, i1, o1, c1);
    }
    for (int l = 0; l < nlev; ++l) {
        IluStage2<T> nxt;
        stage2(nxt, t1, i1, o1, c1);     // level l + 1, in flight while level l computes
        int t2, i2, o2, c2;
        stage1(l + 2, t2, i2, o2, c2);   // level l + 2
        if (cur.t >= 0) {
            T s = cur.rv;
            if (cur.cnt <= kIluPre) {
#pragma unroll
                for (int k = 0; k < kIluPre; ++k)
                    if (k < cur.cnt) s = sub_mul<T>(s, cur.v[k], out[cur.c[k]]);
            } else {
                for (int o = cur.o0; o < cur.o0 + cur.cnt; ++o) s = sub_mul<T>(s, v[o], out[ci[o]]);
            }
            out[cur.i] = DIV ? s / cur.d : s;
            // rows of this level beyond the block width
            const int e = lptr(l + 1);
            for (int t = cur.t + NT; t < e; t += NT) {
                const int i = ord[t];
                T s2 = rhs[i];
                for (int o = rp[t]; o < rp[t + 1]; ++o) s2 = sub_mul<T>(s2, v[o], out[ci[o]]);
                out[i] = DIV ? s2 / dg[t] : s2;
            }
        }
        __syncthreads();
        cur = nxt;
        t1 = t2; i1 = i2; o1 = o2; c1 = c2;
    }
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT)
k_ilu_apply_block(IluLevels<T> F, const T* __restrict__ r, T* y, T* z, const int* gate) {
    __shared__ int s_lptr[kIluLptrSmem];
    if (gate && *(volatile const int*)gate) return;
    for (int l = threadIdx.x; l <= F.nlevL && l < kIluLptrSmem; l += NT) s_lptr[l] = F.lptrL[l];
    __syncthreads();
    ilu_sweep_block<T, false, NT>(F.nlevL, F.lptrL, s_lptr, F.ordL, F.Lrp, F.Lci, F.Lv, nullptr, r, y);
    for (int l = threadIdx.x; l <= F.nlevU && l < kIluLptrSmem; l += NT) s_lptr[l] = F.lptrU[l];
    __syncthreads();
    ilu_sweep_block<T, true, NT>(F.nlevU, F.lptrU, s_lptr, F.ordU, F.Urp, F.Uci, F.Uv, F.Ud, y, z);
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

// ------------------------------------------------------------------------- ILUT
// ILUT(tau, p) (ilu.cpp:94-220) on the device.  The reference eliminates row by row with
// a dense work row; row i needs the finished U rows of the pivots k < i it eliminates.
// Here one warp takes one row at a time, rows claimed in increasing order (atomic ticket,
// cooperative launch: every claimed row belongs to a running warp, so a row only waits on
// rows that can finish); the work row's touched columns live in the warp's shared memory
// (column, value, active flag) and the pending pivots in a min-heap, so the columns are
// visited in the reference's ascending order and every value gets the reference's
// operations (separate multiply and subtract, the same division, the same drops).  The
// keep-largest selection is the reference's heap select (make_heap / pop_heap over the
// row in column order).  Each finished row is published (entries, counts, then a done
// flag after a fence, then a count of finished rows); a wait on a done flag gives up when
// no row at all has finished for about a second (the kernel records *err, every warp
// stops, and the host fails with HAMLSS_ERR_TIMEOUT).
constexpr int kIlutWarps = 4;
constexpr int kIlutCap = 512;            // touched columns a work row may hold
// per warp: columns, values, flags, pending heap, and a row buffer of kIlutCap + 1 entries
constexpr size_t kIlutWarpBytes = (size_t)kIlutCap * (4 + 8 + 1 + 4) + 16 * ((size_t)kIlutCap + 1);
constexpr long long kIlutWaitCycles = 2000000000LL;

struct IlutArgs {
    int n, fill_p;
    double drop_tol;
    const int* rp;
    const int* ci;
    const double* v;
    const int* off;                      // capacity offsets: row i's L at off[i], U at off[i] + max(keep, 1)
    int* ecol;
    double* eval;
    int* lcnt;
    int* ucnt;
    int* done;
    int* ticket;
    int* err;                            // 1 bounded wait ran out, 2 work row overflow
    int* finished;                       // rows published so far
};

struct IlutEntry {
    int col;
    double val;
};

__device__ __forceinline__ bool ilut_first(const IlutEntry& a, const IlutEntry& b) {
    return fabs(a.val) > fabs(b.val);
}

__device__ void ilut_adjust(IlutEntry* h, int hole, int len, IlutEntry value) {
    const int top = hole;
    int child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (ilut_first(h[child], h[child - 1])) --child;
        h[hole] = h[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        h[hole] = h[child - 1];
        hole = child - 1;
    }
    int parent = (hole - 1) / 2;
    while (hole > top && ilut_first(h[parent], value)) {
        h[hole] = h[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    h[hole] = value;
}

// keep_largest (ilu.cpp:186-197) on a row in column order: heap select, then column order.
__device__ void ilut_keep(IlutEntry* row, int* len, int keep) {
    if (keep <= 0 || *len <= keep) return;
    for (int parent = (keep - 2) / 2; keep >= 2; --parent) {
        ilut_adjust(row, parent, keep, row[parent]);
        if (parent == 0) break;
    }
    for (int t = keep; t < *len; ++t)
        if (ilut_first(row[t], row[0])) {
            IlutEntry v = row[t];
            row[t] = row[0];
            ilut_adjust(row, 0, keep, v);
        }
    *len = keep;
    for (int a = 1; a < keep; ++a) {                 // insertion sort by column
        IlutEntry x = row[a];
        int b = a - 1;
        while (b >= 0 && row[b].col > x.col) { row[b + 1] = row[b]; --b; }
        row[b + 1] = x;
    }
}

__device__ __forceinline__ void heap_push(int* h, int& nh, int x) {
    int c = nh++;
    h[c] = x;
    while (c > 0 && h[(c - 1) / 2] > h[c]) {
        const int t = h[c];
        h[c] = h[(c - 1) / 2];
        h[(c - 1) / 2] = t;
        c = (c - 1) / 2;
    }
}

__device__ __forceinline__ int heap_pop(int* h, int& nh) {
    const int top = h[0];
    h[0] = h[--nh];
    for (int c = 0;;) {
        const int l = 2 * c + 1, r = l + 1;
        int m = c;
        if (l < nh && h[l] < h[m]) m = l;
        if (r < nh && h[r] < h[m]) m = r;
        if (m == c) break;
        const int t = h[c];
        h[c] = h[m];
        h[m] = t;
        c = m;
    }
    return top;
}

// The work-row slots that are active, at least tau in magnitude and below (lower) or above
// column i, gathered by the warp into dst[0..count) and sorted by column (warp bitonic sort;
// columns are distinct).  dst must hold the next power of two >= count entries.
__device__ int ilut_gather_sorted(const int* scol, const double* sval, const unsigned char* sact, int nt,
                                  int i, double tau, bool lower, IlutEntry* dst, int lane) {
    int cnt = 0;
    for (int b0 = 0; b0 < nt; b0 += 32) {
        const int t = b0 + lane;
        bool take = false;
        int c = 0;
        double v = 0.0;
        if (t < nt) {
            c = scol[t];
            v = sval[t];
            take = sact[t] && fabs(v) >= tau && (lower ? c < i : c > i);
        }
        const unsigned m = __ballot_sync(0xffffffffu, take);
        if (take) {
            const int q = cnt + __popc(m & ((1u << lane) - 1u));
            dst[q].col = c;
            dst[q].val = v;
        }
        cnt += __popc(m);
    }
    int N = 1;
    while (N < cnt) N <<= 1;
    for (int t = cnt + lane; t < N; t += 32) {
        dst[t].col = INT_MAX;
        dst[t].val = 0.0;
    }
    __syncwarp();
    for (int kk = 2; kk <= N; kk <<= 1)
        for (int jj = kk >> 1; jj > 0; jj >>= 1) {
            for (int t = lane; t < N; t += 32) {
                const int p = t ^ jj;
                if (p > t) {
                    const IlutEntry x = dst[t], y = dst[p];
                    if ((x.col > y.col) == ((t & kk) == 0)) {
                        dst[t] = y;
                        dst[p] = x;
                    }
                }
            }
            __syncwarp();
        }
    return cnt;
}

__global__ void __launch_bounds__(32 * kIlutWarps) k_ilut_rows(IlutArgs a) {
    extern __shared__ unsigned char ilut_smem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned char* base = ilut_smem + (size_t)wid * kIlutWarpBytes;
    int* scol = reinterpret_cast<int*>(base);
    double* sval = reinterpret_cast<double*>(base + 4 * kIlutCap);
    unsigned char* sact = base + 12 * kIlutCap;
    int* heap = reinterpret_cast<int*>(base + 13 * kIlutCap);
    IlutEntry* row = reinterpret_cast<IlutEntry*>(base + 17 * kIlutCap);
    for (;;) {
        int i = 0;
        if (lane == 0) i = *(volatile int*)a.err ? a.n : atomicAdd(a.ticket, 1);
        i = __shfl_sync(0xffffffffu, i, 0);
        if (i >= a.n) break;
        const int rs = a.rp[i], re = a.rp[i + 1], orig = re - rs;
        const int keep = orig + a.fill_p;
        const int half = keep > 1 ? keep : 1;        // capacity of each half of the row
        int nt = min(orig, kIlutCap);
        bool overflow = orig > kIlutCap;
        for (int t = lane; t < nt; t += 32) {
            scol[t] = a.ci[rs + t];
            sval[t] = a.v[rs + t];
            sact[t] = 1;
        }
        __syncwarp();
        double tau = 0.0;
        int nh = 0;
        if (lane == 0) {
            double norm = 0.0;
            for (int t = 0; t < nt; ++t) norm = __dadd_rn(norm, __dmul_rn(sval[t], sval[t]));
            tau = a.drop_tol * sqrt(norm);
            for (int t = 0; t < nt; ++t)
                if (scol[t] < i) heap_push(heap, nh, scol[t]);
        }
        tau = __shfl_sync(0xffffffffu, tau, 0);
        nh = __shfl_sync(0xffffffffu, nh, 0);
        while (nh > 0) {
            int k = 0;
            if (lane == 0) k = heap_pop(heap, nh);
            k = __shfl_sync(0xffffffffu, k, 0);
            nh = __shfl_sync(0xffffffffu, nh, 0);
            // slot of column k
            int sk = -1;
            for (int b0 = 0; b0 < nt && sk < 0; b0 += 32) {
                const int t = b0 + lane;
                const unsigned m = __ballot_sync(0xffffffffu, t < nt && scol[t] == k);
                if (m) sk = b0 + __ffs(m) - 1;
            }
            if (sk < 0 || !sact[sk]) continue;
            const double wk = sval[sk];
            if (fabs(wk) < tau) {
                __syncwarp();
                if (lane == 0) { sval[sk] = 0.0; sact[sk] = 0; }
                __syncwarp();
                continue;
            }
            // row k must be finished
            if (lane == 0) {
                const volatile int* d = a.done + k;
                if (*d == 0) {
                    int seen = *(volatile int*)a.finished;
                    long long t0 = clock64();
                    while (*d == 0) {
                        if (*(volatile int*)a.err) break;
                        const int now = *(volatile int*)a.finished;
                        if (now != seen) {
                            seen = now;
                            t0 = clock64();
                        } else if (clock64() - t0 > kIlutWaitCycles) {
                            atomicExch(a.err, 1);
                            break;
                        }
                        __nanosleep(64);
                    }
                }
                __threadfence();
            }
            __syncwarp();
            const int kk = __ldcg(&a.rp[k + 1]) - __ldcg(&a.rp[k]) + a.fill_p;
            const int us = __ldcg(&a.off[k]) + (kk > 1 ? kk : 1);
            const int ul = __ldcg(&a.ucnt[k]);
            const double ukk = (ul > 0 && __ldcg(&a.ecol[us]) == k) ? __ldcg(&a.eval[us]) : 0.0;
            if (fabs(ukk) < 2.220446049250313e-16) {
                __syncwarp();
                if (lane == 0) sact[sk] = 0;
                __syncwarp();
                continue;
            }
            const double lik = wk / ukk;
            __syncwarp();
            if (lane == 0) sval[sk] = lik;
            __syncwarp();
            for (int q0 = 0; q0 < ul; q0 += 32) {
                const int q = q0 + lane;
                int j = -1;
                double prod = 0.0;
                if (q < ul) {
                    j = __ldcg(&a.ecol[us + q]);
                    if (j <= k) j = -1;
                    else prod = __dmul_rn(lik, __ldcg(&a.eval[us + q]));
                }
                int slot = -1;
                if (j >= 0)
                    for (int t = 0; t < nt; ++t)
                        if (scol[t] == j) { slot = t; break; }
                const unsigned need = __ballot_sync(0xffffffffu, j >= 0 && slot < 0);
                if (j >= 0 && slot < 0) {
                    slot = nt + __popc(need & ((1u << lane) - 1u));
                    if (slot < kIlutCap) {
                        scol[slot] = j;
                        sval[slot] = 0.0;
                        sact[slot] = 0;
                    }
                }
                nt += __popc(need);
                if (nt > kIlutCap) { overflow = true; nt = kIlutCap; }
                bool push = false;
                if (j >= 0 && slot < kIlutCap) {
                    if (!sact[slot] && fabs(prod) >= tau) {
                        sact[slot] = 1;
                        push = j < i;
                    }
                    sval[slot] = __dsub_rn(sval[slot], prod);
                }
                __syncwarp();
                unsigned pm = __ballot_sync(0xffffffffu, push);
                while (pm) {
                    const int l = __ffs(pm) - 1;
                    const int jj = __shfl_sync(0xffffffffu, j, l);
                    if (lane == 0) heap_push(heap, nh, jj);
                    pm &= pm - 1;
                }
                nh = __shfl_sync(0xffffffffu, nh, 0);
                __syncwarp();
            }
        }
        // collect L and U (the warp gathers and sorts by column; lane 0 applies the fill
        // limit, a sequential heap select) and publish the row
        int nl = ilut_gather_sorted(scol, sval, sact, nt, i, tau, true, row, lane);
        if (lane == 0) ilut_keep(row, &nl, keep);
        nl = __shfl_sync(0xffffffffu, nl, 0);
        __syncwarp();
        const int o = a.off[i];
        for (int t = lane; t < nl; t += 32) {
            a.ecol[o + t] = row[t].col;
            a.eval[o + t] = row[t].val;
        }
        __syncwarp();                                  // row[] is reused for U
        double diag = 0.0;
        for (int b0 = 0; b0 < nt; b0 += 32) {
            const int t = b0 + lane;
            const unsigned m = __ballot_sync(0xffffffffu, t < nt && scol[t] == i);
            if (m) {
                diag = __shfl_sync(0xffffffffu, t < nt ? sval[t] : 0.0, __ffs(m) - 1);
                break;
            }
        }
        if (fabs(diag) < 2.220446049250313e-16) diag = (diag >= 0 ? 1.0 : -1.0) * 2.220446049250313e-16 * 1e6;
        int nu = 1 + ilut_gather_sorted(scol, sval, sact, nt, i, tau, false, row + 1, lane);
        if (lane == 0) {
            row[0].col = i;
            row[0].val = diag;
            ilut_keep(row, &nu, keep);
        }
        nu = __shfl_sync(0xffffffffu, nu, 0);
        __syncwarp();
        for (int t = lane; t < nu; t += 32) {
            a.ecol[o + half + t] = row[t].col;
            a.eval[o + half + t] = row[t].val;
        }
        if (lane == 0) {
            a.lcnt[i] = nl;
            a.ucnt[i] = nu;
            if (overflow) atomicExch(a.err, 2);
        }
        __threadfence();                               // every lane's entries, then the flag
        __syncwarp();
        if (lane == 0) {
            *(volatile int*)(a.done + i) = 1;
            atomicAdd(a.finished, 1);
        }
        __syncwarp();
    }
}

// Capacity per row (2 * (row length + fill_p)): L in the first half, U in the second.
__global__ void k_ilut_caps(int n, const int* __restrict__ rp, int fill_p, int* cap) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int keep = rp[i + 1] - rp[i] + fill_p;
        cap[i] = 2 * (keep > 1 ? keep : 1);
    }
}

__global__ void k_ilut_counts(int n, const int* __restrict__ lcnt, const int* __restrict__ ucnt, int* cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        cnt[i] = lcnt[i] + ucnt[i];
}

// Compact the capacity layout into the L\U CSR (row: L entries, then U entries).
__global__ void k_ilut_compact(int n, const int* __restrict__ rp, int fill_p, const int* __restrict__ off,
                               const int* __restrict__ lcnt, const int* __restrict__ ucnt,
                               const int* __restrict__ ecol, const double* __restrict__ eval,
                               const int* __restrict__ frp, int* fci, double* flu) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int keep = rp[i + 1] - rp[i] + fill_p;
        const int half = keep > 1 ? keep : 1;
        int o = frp[i];
        for (int t = 0; t < lcnt[i]; ++t, ++o) { fci[o] = ecol[off[i] + t]; flu[o] = eval[off[i] + t]; }
        for (int t = 0; t < ucnt[i]; ++t, ++o) { fci[o] = ecol[off[i] + half + t]; flu[o] = eval[off[i] + half + t]; }
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
    // pattern of the factor: A's for ILU(0); the factor's own (frp, fci) for ILUT
    const int* prp = nullptr;
    const int* pci = nullptr;
    int pnnz = 0;
    DBuf<int> frp, fci;
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
            k_fill_L<float><<<g, 256, 0, s>>>(n, ordL.p, prp, pci, lu.p, Lrp.p, Lci.p, Lv32.p);
            k_fill_U<float><<<g, 256, 0, s>>>(n, ordU.p, prp, pci, lu.p, Urp.p, Uci.p, Uv32.p,
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

namespace {
void finish_ilu(Ctx& ctx, IluPrec* P, bool factorise);
}  // namespace

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
    P->prp = A->A.rp.p;
    P->pci = A->A.ci.p;
    P->pnnz = nnz;
    P->lu.ensure(nnz);
    if (nnz) HAMLSS_CUDA(cudaMemcpyAsync(P->lu.p, A->A.v.p, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, s));
    finish_ilu(ctx, P.get(), true);
    return P;
}

std::unique_ptr<Prec> make_ilut(Ctx& ctx, hamlss_mat* A, double drop_tol, int fill_p) {
    auto P = std::make_unique<IluPrec>();
    P->kind = HAMLSS_PREC_ILU;
    P->A = A;
    const int n = A->A.n;
    P->n = n;
    if (A->A.n != A->A.m) fail(HAMLSS_ERR_SIZE, "ILU needs a square matrix");
    if (fill_p < 0) fail(HAMLSS_ERR_INVALID, "ILUT: fill_per_row must be >= 0");
    cudaStream_t s = ctx.lane.stream;
    AllocScope scope(s);
    const int g = std::max(1, std::min(ceil_div(n, 256), ctx.sm_count * 8));
    // capacity layout: row i owns 2 * max(row length + fill_p, 1) slots
    DBuf<int> off(n + 1), lcnt(std::max(n, 1)), ucnt(std::max(n, 1)), done(std::max(n, 1)), flags(3);
    HAMLSS_CUDA(cudaMemsetAsync(off.p + n, 0, sizeof(int), s));
    if (n) k_ilut_caps<<<g, 256, 0, s>>>(n, A->A.rp.p, fill_p, off.p);
    HAMLSS_LAUNCH_CHECK();
    const long long total = exclusive_scan(ctx, off.p, n + 1);
    if (total > INT_MAX) fail(HAMLSS_ERR_NOMEM, "ILUT: factor capacity exceeds 2^31 entries");
    DBuf<int> ecol(std::max<long long>(total, 1));
    DBuf<double> eval(std::max<long long>(total, 1));
    lcnt.zero(s);
    ucnt.zero(s);
    done.zero(s);
    flags.zero(s);
    if (n) {
        static DeviceOnce raised;
        raised(ctx.device, [] {
            HAMLSS_CUDA(cudaFuncSetAttribute(k_ilut_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)(kIlutWarpBytes * kIlutWarps)));
        });
        const size_t smem = kIlutWarpBytes * kIlutWarps;
        int per = 0;
        HAMLSS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_ilut_rows, 32 * kIlutWarps, smem));
        const int blocks = std::max(1, std::min(std::max(per, 1) * ctx.sm_count, ceil_div(n, kIlutWarps)));
        IlutArgs a;
        a.n = n;
        a.fill_p = fill_p;
        a.drop_tol = drop_tol;
        a.rp = A->A.rp.p;
        a.ci = A->A.ci.p;
        a.v = A->A.v.p;
        a.off = off.p;
        a.ecol = ecol.p;
        a.eval = eval.p;
        a.lcnt = lcnt.p;
        a.ucnt = ucnt.p;
        a.done = done.p;
        a.ticket = flags.p;
        a.err = flags.p + 1;
        a.finished = flags.p + 2;
        void* args[] = {&a};
        HAMLSS_CUDA(cudaLaunchCooperativeKernel((const void*)k_ilut_rows, dim3(blocks), dim3(32 * kIlutWarps),
                                                args, smem, s));
        int h[2] = {0, 0};
        flags.download(h, 2, s);
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        if (h[1] == 1) fail(HAMLSS_ERR_TIMEOUT, "ILUT: a bounded wait for an earlier row ran out");
        if (h[1] == 2) fail(HAMLSS_ERR_NOMEM, "ILUT: a work row touched more than 512 columns");
    }
    // compact into the L\U CSR
    P->frp.ensure(n + 1);
    HAMLSS_CUDA(cudaMemsetAsync(P->frp.p + n, 0, sizeof(int), s));
    if (n) k_ilut_counts<<<g, 256, 0, s>>>(n, lcnt.p, ucnt.p, P->frp.p);
    HAMLSS_LAUNCH_CHECK();
    const long long fnnz = exclusive_scan(ctx, P->frp.p, n + 1);
    P->fci.ensure(std::max<long long>(fnnz, 1));
    P->lu.ensure(std::max<long long>(fnnz, 1));
    if (n)
        k_ilut_compact<<<g, 256, 0, s>>>(n, A->A.rp.p, fill_p, off.p, lcnt.p, ucnt.p, ecol.p, eval.p,
                                          P->frp.p, P->fci.p, P->lu.p);
    HAMLSS_LAUNCH_CHECK();
    P->prp = P->frp.p;
    P->pci = P->fci.p;
    P->pnnz = (int)fnnz;
    finish_ilu(ctx, P.get(), false);
    return P;
}

std::unique_ptr<Prec> make_ilu(Ctx& ctx, hamlss_mat* A, const hamlss_params& p) {
    if (p.drop_tol > 0.0 || p.fill_per_row > 0) return make_ilut(ctx, A, p.drop_tol, p.fill_per_row);
    return make_ilu0(ctx, A);
}

namespace {
// Pattern information, level sets, (for ILU(0)) the factorisation, and the level-ordered
// L / U copies of an ILU preconditioner whose pattern (prp, pci, pnnz) and values (lu)
// are set.
void finish_ilu(Ctx& ctx, IluPrec* P, bool factorise) {
    const int n = P->n;
    const int nnz = P->pnnz;
    cudaStream_t s = ctx.lane.stream;
    const int g = std::max(1, std::min(ceil_div(n, 256), ctx.sm_count * 8));
    const int* rp = P->prp;
    const int* ci = P->pci;
    P->y.ensure(n);
    if (n == 0) return;
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
    // factorisation (ILU(0); ILUT arrives factored)
    if (factorise) {
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
}
}  // namespace

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
    if (P->pnnz) P->lu.download(out, P->pnnz, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    return HAMLSS_OK;
}

int ilu_factor_csr(const Prec* M, int* nnz, int* rp, int* ci, double* v, cudaStream_t s) {
    auto* P = dynamic_cast<const IluPrec*>(M);
    if (!P) return HAMLSS_ERR_INVALID;
    *nnz = P->pnnz;
    if (rp) HAMLSS_CUDA(cudaMemcpyAsync(rp, P->prp, sizeof(int) * (P->n + 1), cudaMemcpyDeviceToHost, s));
    if (ci && P->pnnz) HAMLSS_CUDA(cudaMemcpyAsync(ci, P->pci, sizeof(int) * P->pnnz, cudaMemcpyDeviceToHost, s));
    if (v && P->pnnz) P->lu.download(v, P->pnnz, s);
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
