// spmv.cuh -- the CSR SpMV kernel template every solver kernel is built from.
//
// Layout: CSR, int32 row_ptr / col_idx, values in T (double or float), columns sorted per
// row.  Scheduling: one warp owns a tile of 32 consecutive rows and lane l sums row
// tile+l in column order, reading it straight from global memory four entries at a time
// (consecutive rows are contiguous, so a warp's loads cover whole cache lines that L1
// keeps for the next entries; measured 1.5x faster than staging the tile through shared
// memory on the 5-point operator).  A persistent grid walks the tiles.  For FP32 operands
// with longer rows, groups of lanes share a row instead (gsz below).
//
// Fusion: the kernel is parameterised by
//   XOp  x(j)            -> value of the multiplied vector at column j (may be computed on
//                           the fly, e.g. p_j = z_j + beta * p_old_j)
//   Epi  epi(i, ax, acc) -> consumes (A x)_i for own row i; may write vectors and add into
//                           the NRED per-thread accumulators
//   Fin  fin(tot)        -> runs once, in the last block, on the grid-wide sums of acc
// so SpMV + following dot / residual / update / smoother step cost one pass over A.
// Row sums follow the reference's order (sparse_matrix.cpp:80-86); for double they use
// separate multiply and add, so A x is bit-identical to the reference's spmv.
#pragma once

#include "common.cuh"

namespace hamlss {

constexpr int kSpmvThreads = 256;             // 8 warps per block
constexpr int kSpmvWarps = kSpmvThreads / 32;

template <typename T>
__device__ __forceinline__ double mul_add(double acc, T a, double x) {
    return acc + (double)a * x;
}
template <>
__device__ __forceinline__ double mul_add<double>(double acc, double a, double x) {
    return __dadd_rn(acc, __dmul_rn(a, x));
}

// Sum of row `row` of A against x(), by one lane: the row's loads are issued four at a
// time, then summed in column order -- the reference's order (sparse_matrix.cpp:80-86).
template <typename T, typename XOp>
__device__ __forceinline__ double lane_row_sum(int row, const int* __restrict__ rp,
                                               const int* __restrict__ ci, const T* __restrict__ v,
                                               const XOp& x) {
    const int rs = __ldg(&rp[row]), re = __ldg(&rp[row + 1]);
    double sum = 0.0;
    int k = rs;
    for (; k + 4 <= re; k += 4) {
        const T a0 = __ldg(&v[k]), a1 = __ldg(&v[k + 1]), a2 = __ldg(&v[k + 2]), a3 = __ldg(&v[k + 3]);
        const int c0 = __ldg(&ci[k]), c1 = __ldg(&ci[k + 1]), c2 = __ldg(&ci[k + 2]), c3 = __ldg(&ci[k + 3]);
        const double x0 = x(c0), x1 = x(c1), x2 = x(c2), x3 = x(c3);
        sum = mul_add<T>(sum, a0, x0);
        sum = mul_add<T>(sum, a1, x1);
        sum = mul_add<T>(sum, a2, x2);
        sum = mul_add<T>(sum, a3, x3);
    }
    for (; k < re; ++k) sum = mul_add<T>(sum, __ldg(&v[k]), x(__ldg(&ci[k])));
    return sum;
}

// L2 prefetch of [p, p + bytes) by one thread (cp.async.bulk.prefetch.L2), trimmed to
// the whole 16-byte granules inside the range so it never touches memory outside it.
// Functors of the bulk-copy SpMV (spmv_stream.cuh) call it from prefetch(r0, r1) for the
// vector slices a row tile will read.
__device__ __forceinline__ void l2_prefetch(const void* p, size_t bytes) {
    uintptr_t a = reinterpret_cast<uintptr_t>(p);
    uintptr_t lo = (a + 15) & ~(uintptr_t)15, hi = (a + bytes) & ~(uintptr_t)15;
    while (hi > lo) {
        const uintptr_t chunk = (hi - lo) > (1u << 20) ? (1u << 20) : (hi - lo);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((unsigned)chunk) : "memory");
        lo += chunk;
    }
}
template <typename T>
__device__ __forceinline__ void l2_prefetch_rows(const T* v, int r0, int r1) {
    if (v && r1 > r0) l2_prefetch(v + r0, (size_t)(r1 - r0) * sizeof(T));
}

struct NoFin {
    template <int NV>
    __device__ void operator()(const double (&)[NV]) const {}
};

// gate: when non-null and *gate != 0 the whole launch is a no-op (the solve it belongs
// to has stopped; the flag is only written by earlier kernels on the same stream).
// gsz > 1 (FP32 operands only, see spmv_group_size): groups of gsz lanes share a row,
// stride over its nonzeros and add their partial sums with shuffles -- coalesced loads for
// rows of 8 and more nonzeros, at the price of the reference's summation order.
template <typename T, int NRED, typename XOp, typename Epi, typename Fin>
__global__ void __launch_bounds__(kSpmvThreads)
k_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ v,
       XOp xop, Epi epi, Reducer red, Fin fin, const int* gate, int gsz, int skip_len) {
    __shared__ double rsh[kSpmvWarps * (NRED > 0 ? NRED : 1)];
    if (gate && *(volatile const int*)gate) return;
    XOp xop_l = xop;
    Epi epi_l = epi;
    xop_l.load();
    epi_l.load();
    const int wid = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int ntiles = (n + 31) >> 5;
    double acc[NRED > 0 ? NRED : 1];
#pragma unroll
    for (int k = 0; k < (NRED > 0 ? NRED : 1); ++k) acc[k] = 0.0;
    if (gsz > 1) {
        const int per_warp = 32 / gsz, sub = lane / gsz, gl = lane - sub * gsz;
        const int stride = gridDim.x * kSpmvWarps * per_warp;
        for (int base = (blockIdx.x * kSpmvWarps + wid) * per_warp; base < n; base += stride) {
            int row = base + sub;
            // rows longer than skip_len are left to k_spmv_rows_seq
            if (row < n && __ldg(&rp[row + 1]) - __ldg(&rp[row]) > skip_len) row = n;
            double sum = 0.0;
            if (row < n) {
                const int rs = __ldg(&rp[row]), re = __ldg(&rp[row + 1]);
                for (int k = rs + gl; k < re; k += gsz) sum = mul_add<T>(sum, __ldg(&v[k]), xop_l(__ldg(&ci[k])));
            }
            for (int o = gsz >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (row < n && gl == 0) epi_l(row, sum, acc);
        }
    } else {
        for (int t = blockIdx.x * kSpmvWarps + wid; t < ntiles; t += gridDim.x * kSpmvWarps) {
            const int row = (t << 5) + lane;
            if (row < n && __ldg(&rp[row + 1]) - __ldg(&rp[row]) <= skip_len)
                epi_l(row, lane_row_sum<T>(row, rp, ci, v, xop_l), acc);
        }
    }
    if constexpr (NRED > 0) {
        double tot[NRED];
        if (grid_reduce<NRED>(red, acc, rsh, tot)) fin(tot);
    }
}

// FP32 operators with long rows (the dense-ish coarse AMG levels, hundreds of entries a
// row): G lanes per row (G = 32: a warp), each lane keeping four entries' loads in flight
// (entries k, k + G, k + 2G, k + 3G) into four partial sums, combined by shuffles.  No
// bit-exactness requirement applies to FP32 operands, so the order is free.
template <typename T, int NRED, typename XOp, typename Epi, typename Fin, int G>
__global__ void __launch_bounds__(256)
k_spmv_long(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ v,
            XOp xop, Epi epi, Reducer red, Fin fin, const int* gate) {
    __shared__ double rsh[8 * (NRED > 0 ? NRED : 1)];
    if (gate && *(volatile const int*)gate) return;
    XOp xop_l = xop;
    Epi epi_l = epi;
    xop_l.load();
    epi_l.load();
    const int lane = threadIdx.x & 31, sub = lane / G, gl = lane - sub * G;
    constexpr int kRows = 32 / G;                  // rows per warp
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    double acc[NRED > 0 ? NRED : 1];
#pragma unroll
    for (int k = 0; k < (NRED > 0 ? NRED : 1); ++k) acc[k] = 0.0;
    for (int base = gw * kRows; base < n; base += nw * kRows) {
        const int row = base + sub;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (row < n) {
            const int rs = __ldg(&rp[row]), re = __ldg(&rp[row + 1]);
            int k = rs + gl;
            for (; k + 3 * G < re; k += 4 * G) {
                const T a0 = __ldg(&v[k]), a1 = __ldg(&v[k + G]), a2 = __ldg(&v[k + 2 * G]),
                        a3 = __ldg(&v[k + 3 * G]);
                const int c0 = __ldg(&ci[k]), c1 = __ldg(&ci[k + G]), c2 = __ldg(&ci[k + 2 * G]),
                          c3 = __ldg(&ci[k + 3 * G]);
                s0 += (double)a0 * xop_l(c0);
                s1 += (double)a1 * xop_l(c1);
                s2 += (double)a2 * xop_l(c2);
                s3 += (double)a3 * xop_l(c3);
            }
            for (; k < re; k += G) s0 += (double)__ldg(&v[k]) * xop_l(__ldg(&ci[k]));
        }
        double sum = (s0 + s1) + (s2 + s3);
#pragma unroll
        for (int o = G >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (row < n && gl == 0) epi_l(row, sum, acc);
    }
    if constexpr (NRED > 0) {
        double tot[NRED];
        if (grid_reduce<NRED>(red, acc, rsh, tot)) fin(tot);
    }
}

// Rows far longer than the matrix's average (a skewed row-length profile), one warp per
// listed row: the lanes load 32 entries at a time (the next 32 already in flight while the
// current ones are added) and form the products a_ij * x_j, and lane 0 adds them to the
// row's sum in column order with separate multiply and add -- the reference's order
// (sparse_matrix.cpp:80-86), so FP64 results are bit-identical to one lane per row, while
// a row of many thousand entries no longer holds one lane of a tile for all of them.
constexpr int kSeqRowWarps = 8;

template <typename T, typename XOp, typename Epi>
__global__ void __launch_bounds__(32 * kSeqRowWarps)
k_spmv_rows_seq(const int* __restrict__ rows, int nrows, const int* __restrict__ rp,
                const int* __restrict__ ci, const T* __restrict__ v, XOp xop, Epi epi) {
    __shared__ double prod[kSeqRowWarps][32];
    XOp xop_l = xop;
    Epi epi_l = epi;
    xop_l.load();
    epi_l.load();
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* pw = prod[wid];
    for (int r = blockIdx.x * kSeqRowWarps + wid; r < nrows; r += gridDim.x * kSeqRowWarps) {
        const int row = rows[r];
        const int rs = __ldg(&rp[row]), re = __ldg(&rp[row + 1]);
        double sum = 0.0;
        T a = T(0);
        double x = 0.0;
        if (rs + lane < re) {
            a = __ldg(&v[rs + lane]);
            x = xop_l(__ldg(&ci[rs + lane]));
        }
        for (int kb = rs; kb < re; kb += 32) {
            const double p = __dmul_rn((double)a, x);
            const int kn = kb + 32 + lane;                // the next 32, in flight meanwhile
            a = T(0);
            x = 0.0;
            if (kn < re) {
                a = __ldg(&v[kn]);
                x = xop_l(__ldg(&ci[kn]));
            }
            pw[lane] = p;
            __syncwarp();
            if (lane == 0) {
                const int cnt = min(32, re - kb);
                for (int j = 0; j < cnt; ++j) sum = __dadd_rn(sum, pw[j]);
            }
            __syncwarp();
        }
        double none[1];
        if (lane == 0) epi_l(row, sum, none);
    }
}

// Elementwise kernel with the same reduction / finalize machinery (no matrix).
template <int NRED, typename Body, typename Fin>
__global__ void __launch_bounds__(256)
k_vec(int n, Body body, Reducer red, Fin fin, const int* gate) {
    __shared__ double rsh[8 * (NRED > 0 ? NRED : 1)];
    if (gate && *(volatile const int*)gate) return;
    Body b = body;
    b.load();
    double acc[NRED > 0 ? NRED : 1];
#pragma unroll
    for (int k = 0; k < (NRED > 0 ? NRED : 1); ++k) acc[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        b(i, acc);
    if constexpr (NRED > 0) {
        double tot[NRED];
        if (grid_reduce<NRED>(red, acc, rsh, tot)) fin(tot);
    }
}

// ------------------------------------------------------------------ common operators
// Operators may read device scalars once per launch in load() (called at kernel entry,
// after the gate check).
#define HAMLSS_NO_LOAD \
    __device__ __forceinline__ void load() {}

template <typename T>
struct XVec {
    const T* x;
    HAMLSS_NO_LOAD
    __device__ __forceinline__ double operator()(int j) const { return (double)__ldg(&x[j]); }
};

template <typename T>
struct EpiStore {
    T* y;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&)[NV]) const { y[i] = (T)ax; }
};

}  // namespace hamlss
