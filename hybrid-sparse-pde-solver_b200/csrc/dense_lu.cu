// dense_lu.cu -- blocked LU with partial pivoting and the explicit inverse, for the
// coarsest AMG level when it is too large for the one-block elimination in amg.cu.
//
// The reference solves its coarsest level by dense Gaussian elimination with partial
// pivoting (amg.cpp:260-291).  Coarse operators of the smoothed-aggregation hierarchy
// become dense, and when the hierarchy is cut where coarsening stalls the coarsest level
// can hold thousands of rows.  Blocked for the GPU (row-major n x n, nb = 64), first
// without interchanges -- diagonal block factored in shared memory, the inverses of its
// two triangles formed by the same kernel (64 x 64 each), L21 = A21 U11^-1 and
// U12 = L11^-1 A12 as DGEMMs, A22 by DGEMM, no grid-wide synchronisation -- and, if a pivot falls below
// 1e-10 of the largest entry, again with partial pivoting as the reference does:
//   panel     columns [k0, k0+nb): one cooperative kernel over all SMs, one column at a
//             time -- pivot search (largest |a_ij|, first index on ties, like the
//             reference), row swap inside the panel, multipliers l = a_ij * (1/a_jj),
//             rank-1 update of the panel's remaining columns; two grid barriers a column
//   swaps     the panel's row interchanges applied to every other column
//   U12       L11^-1 A12, one thread per column (unit lower triangular solve)
//   trailing  A22 -= L21 U12, a DGEMM on the FP64 tensor cores (k_dgemm below)
// The inverse solves A X = I: X = P I, then L Y = X and U X = Y, blocked the same way
// (each 64-row block multiplied by its diagonal block's inverse, DGEMM update of the
// rest): every step is a GEMM, where column-per-thread triangular solves were a long
// dependent chain per launch.
#include <vector>
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "dense_lu.cuh"

namespace cg = cooperative_groups;

namespace hamlss {

namespace {

constexpr int kNb = 64;
constexpr int kPanelThreads = 256;

__device__ __forceinline__ bool better(double v, int i, double bv, int bi) {
    return v > bv || (v == bv && i < bi);
}

// Panel factorisation, cooperative.  Rows [k0, n) go to warps round-robin; lane c holds
// panel columns c and c + 32 of its row.  cand_v / cand_i: one slot per block.
__global__ void __launch_bounds__(kPanelThreads)
k_lu_panel(int n, int k0, int kb, double* M, int* piv, double* cand_v, int* cand_i, int* singular) {
    cg::grid_group grid = cg::this_grid();
    __shared__ double prow[kNb], jrow[kNb];
    __shared__ double wv[kPanelThreads / 32];
    __shared__ int wi[kPanelThreads / 32];
    __shared__ int s_p;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nwb = blockDim.x >> 5;
    const int gw = blockIdx.x * nwb + wib, W = gridDim.x * nwb;
    // candidate for column k0 (before any update of this panel)
    auto block_candidate = [&](double v, int idx) {
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, v, o);
            const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
            if (better(ov, oi, v, idx)) { v = ov; idx = oi; }
        }
        if (lane == 0) { wv[wib] = v; wi[wib] = idx; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double bv = -1.0;
            int bi = INT_MAX;
            for (int w = 0; w < nwb; ++w)
                if (better(wv[w], wi[w], bv, bi)) { bv = wv[w]; bi = wi[w]; }
            cand_v[blockIdx.x] = bv;
            cand_i[blockIdx.x] = bi;
        }
        __syncthreads();
    };
    {
        double v = -1.0;
        int idx = INT_MAX;
        for (int i = k0 + gw; i < n; i += W)
            if (lane == 0) {
                const double a = fabs(M[(size_t)i * n + k0]);
                if (better(a, i, v, idx)) { v = a; idx = i; }
            }
        block_candidate(v, idx);
    }
    grid.sync();
    for (int jj = 0; jj < kb; ++jj) {
        const int j = k0 + jj;
        // every block reduces the candidates the same way: the same pivot row p (the order
        // of the reduction does not matter: "better" is a strict total order)
        if (wib == 0) {
            double bv = -1.0;
            int bi = INT_MAX;
            for (int b = lane; b < (int)gridDim.x; b += 32) {
                const double v = __ldcg(&cand_v[b]);
                const int i = __ldcg(&cand_i[b]);
                if (better(v, i, bv, bi)) { bv = v; bi = i; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
            }
            if (lane == 0) {
                s_p = bi;
                if (blockIdx.x == 0) {
                    piv[j] = bi;
                    if (!(bv > 0.0)) *singular = 1;
                }
            }
        }
        __syncthreads();
        const int p = s_p;
        for (int c = threadIdx.x; c < kb; c += blockDim.x) {
            prow[c] = __ldcg(&M[(size_t)p * n + k0 + c]);
            jrow[c] = __ldcg(&M[(size_t)j * n + k0 + c]);
        }
        __syncthreads();
        grid.sync();                       // rows j and p read by everyone before writes
        const double d = prow[jj];
        const double inv = (d != 0.0) ? 1.0 / d : 0.0;
        double v = -1.0;
        int idx = INT_MAX;
        for (int i = k0 + gw; i < n; i += W) {
            if (i < j) continue;
            double* row = M + (size_t)i * n + k0;
            const int c0 = lane, c1 = lane + 32;
            if (i == j) {
                if (c0 < kb) row[c0] = prow[c0];
                if (c1 < kb) row[c1] = prow[c1];
                continue;
            }
            double r0 = 0.0, r1 = 0.0;
            if (i == p) {
                r0 = c0 < kb ? jrow[c0] : 0.0;
                r1 = c1 < kb ? jrow[c1] : 0.0;
            } else {
                r0 = c0 < kb ? row[c0] : 0.0;
                r1 = c1 < kb ? row[c1] : 0.0;
            }
            // multiplier l = a_ij * (1/a_jj), then a_ic -= l * a_pc for c > j
            const double aij = __shfl_sync(0xffffffffu, jj < 32 ? r0 : r1, jj & 31);
            const double l = __dmul_rn(aij, inv);
            if (c0 < kb) {
                if (c0 == jj) r0 = l;
                else if (c0 > jj) r0 = __dsub_rn(r0, __dmul_rn(l, prow[c0]));
                row[c0] = r0;
            }
            if (c1 < kb) {
                if (c1 == jj) r1 = l;
                else if (c1 > jj) r1 = __dsub_rn(r1, __dmul_rn(l, prow[c1]));
                row[c1] = r1;
            }
            // candidate for the next column (j + 1) from the updated row
            if (jj + 1 < kb) {
                const int nc = jj + 1;
                const double a = fabs(__shfl_sync(0xffffffffu, nc < 32 ? r0 : r1, nc & 31));
                if (better(a, i, v, idx)) { v = a; idx = i; }
            }
        }
        if (jj + 1 < kb) block_candidate(v, idx);
        grid.sync();
    }
}

__global__ void k_abs_max(long long count, const double* __restrict__ a, unsigned long long* out) {
    double m = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(a[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    // non-negative doubles order like their bit patterns
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// Apply the panel's interchanges (rows k0 + jj <-> piv[k0 + jj], in order) to the columns
// outside the panel.
__global__ void k_lu_swap(int n, int k0, int kb, double* M, const int* __restrict__ piv) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        if (c >= k0 && c < k0 + kb) continue;
        for (int jj = 0; jj < kb; ++jj) {
            const int j = k0 + jj, p = piv[j];
            if (p == j) continue;
            const double t = M[(size_t)j * n + c];
            M[(size_t)j * n + c] = M[(size_t)p * n + c];
            M[(size_t)p * n + c] = t;
        }
    }
}

// B[r][c] for r in [k0, k0+kb): B := L11^-1 B (unit lower L11 = L[k0.., k0..]), columns
// [c0, c1) of B, one thread per column.  L and B may be the same matrix.
__global__ void k_trsm_lower_unit(int n, int k0, int kb, const double* __restrict__ L, int ldl,
                                  double* B, int ldb, int c0, int c1) {
    __shared__ double sl[kNb][kNb];
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
        const int r = t / kb, q = t - r * kb;
        sl[r][q] = L[(size_t)(k0 + r) * ldl + k0 + q];
    }
    __syncthreads();
    for (int c = c0 + blockIdx.x * blockDim.x + threadIdx.x; c < c1; c += gridDim.x * blockDim.x) {
        for (int r = 1; r < kb; ++r) {
            double acc = B[(size_t)(k0 + r) * ldb + c];
            for (int q = 0; q < r; ++q)
                acc = __dsub_rn(acc, __dmul_rn(sl[r][q], B[(size_t)(k0 + q) * ldb + c]));
            B[(size_t)(k0 + r) * ldb + c] = acc;
        }
    }
}

// Inverses of the factors of a kb x kb diagonal block held in shared memory `a` (L unit
// lower below the diagonal, U on and above it), by 256 threads: a pair of threads per
// column of Li = L^-1 (threads 0..127) and of Ui = U^-1 (threads 128..255).  The pair walks
// the column in the factor's row order (substitution), splits each row's sum by the parity
// of its terms and adds the halves with a shuffle; U's diagonal enters by its reciprocal.
// Each thread writes every entry of its column, so it only reads back its own writes.
// Results go to shared memory, then to Li / Ui (row-major, ld kNb).
__device__ void block_inverses_smem(int kb, const double (*a)[kNb + 1], double (*li)[kNb + 1],
                                    double (*ui)[kNb + 1], double* Li, double* Ui) {
    __shared__ double rdiag[kNb];
    const int t = threadIdx.x;
    if (t < kb) rdiag[t] = 1.0 / a[t][t];
    __syncthreads();
    if (t < 4 * kNb) {
        const bool upper = t >= 2 * kNb;
        const int u = t & (2 * kNb - 1);
        const int c = u >> 1, h = u & 1;
        const unsigned pm = 3u << ((t & 31) & ~1);              // the pair's two lanes
        if (c < kb) {
            if (!upper) {                                     // L x = e_c
                for (int r = 0; r < c; ++r) li[r][c] = 0.0;
                li[c][c] = 1.0;
                for (int r = c + 1; r < kb; ++r) {
                    double s = 0.0;
                    for (int q = c + h; q < r; q += 2) s = __dadd_rn(s, __dmul_rn(a[r][q], li[q][c]));
                    s = __dadd_rn(s, __shfl_xor_sync(pm, s, 1));
                    li[r][c] = -s;
                }
            } else {                                          // U x = e_c
                for (int r = c + 1; r < kb; ++r) ui[r][c] = 0.0;
                for (int r = c; r >= 0; --r) {
                    double s = 0.0;
                    for (int q = r + 1 + h; q <= c; q += 2) s = __dadd_rn(s, __dmul_rn(a[r][q], ui[q][c]));
                    s = __dadd_rn(s, __shfl_xor_sync(pm, s, 1));
                    ui[r][c] = __dmul_rn(__dsub_rn(r == c ? 1.0 : 0.0, s), rdiag[r]);
                }
            }
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
        const int r = e / kb, c = e - r * kb;
        Li[r * kNb + c] = li[r][c];
        Ui[r * kNb + c] = ui[r][c];
    }
}

constexpr size_t kDiagSmem = 3 * sizeof(double) * kNb * (kNb + 1);

// Inverses of the factors of diagonal block b0 + blockIdx.x (k0 = b * kNb): Li = L11^-1
// and Ui = U11^-1 at inv + 2 * b * kNb * kNb.  4 * kNb threads; dynamic shared memory:
// kDiagSmem.
__global__ void k_block_inverses(int n, int b0, const double* __restrict__ M, double* inv) {
    extern __shared__ double dsm[];
    auto a = reinterpret_cast<double (*)[kNb + 1]>(dsm);
    auto li = a + kNb;
    auto ui = li + kNb;
    const int b = b0 + blockIdx.x;
    const int k0 = b * kNb, kb = min(kNb, n - k0);
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
        const int r = t / kb, c = t - r * kb;
        a[r][c] = M[(size_t)(k0 + r) * n + k0 + c];
    }
    __syncthreads();
    double* Li = inv + 2LL * b * kNb * kNb;
    block_inverses_smem(kb, a, li, ui, Li, Li + kNb * kNb);
}

// ------------------------------------------------------------ without pivoting
// The no-interchange step for diagonal block k0 in one kernel: factor A11 = L11 U11 (the
// arithmetic of the column-by-column elimination: l = a_rj * (1/a_jj), a_rc -= l * a_jc,
// then the column scaled), flag a pivot below `floor`, write the factors back, and form
// Li, Ui (block_inverses_smem).  256 threads as 16 x 16, each holding its 4 x 4 elements
// (rows ty + 16i, columns tx + 16q) in registers; per column j only column j and row j go
// through shared memory, with two barriers.  Dynamic shared memory: kDiagSmem.
__global__ void __launch_bounds__(256) k_lu_diag_inv(int n, int k0, int kb, double* M, double floor,
                                                     int* tiny, double* inv) {
    extern __shared__ double dsm[];
    auto a = reinterpret_cast<double (*)[kNb + 1]>(dsm);
    auto li = a + kNb;
    auto ui = li + kNb;
    __shared__ double colj[kNb], rowj[kNb];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double e[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = ty + 16 * i, c = tx + 16 * q;
            e[i][q] = (r < kb && c < kb) ? M[(size_t)(k0 + r) * n + k0 + c] : 0.0;
        }
    for (int j = 0; j < kb; ++j) {
        const int jq = j >> 4, jm = j & 15;
        // (compile-time register indices: the block of column / row j is selected by q == jq)
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (tx == jm && q == jq) colj[ty + 16 * i] = e[i][q];   // column j (unscaled)
                if (ty == jm && i == jq) rowj[tx + 16 * q] = e[i][q];   // row j
            }
        __syncthreads();
        const double d = rowj[j];
        if (threadIdx.x == 0 && !(fabs(d) > floor)) *tiny = 1;
        const double inv_d = (d != 0.0) ? 1.0 / d : 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = ty + 16 * i;
            if (r <= j || r >= kb) continue;
            const double l = __dmul_rn(colj[r], inv_d);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int c = tx + 16 * q;
                if (c > j && c < kb) e[i][q] = __dsub_rn(e[i][q], __dmul_rn(l, rowj[c]));
            }
        }
        if (tx == jm)                                             // the multipliers of column j
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int r = ty + 16 * i;
                    if (q == jq && r > j && r < kb) e[i][q] = __dmul_rn(e[i][q], inv_d);
                }
        __syncthreads();                                          // colj / rowj reused
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = ty + 16 * i, c = tx + 16 * q;
            if (r < kb && c < kb) {
                a[r][c] = e[i][q];
                M[(size_t)(k0 + r) * n + k0 + c] = e[i][q];
            }
        }
    __syncthreads();
    double* Li = inv + 2LL * (k0 / kNb) * kNb * kNb;
    block_inverses_smem(kb, a, li, ui, Li, Li + kNb * kNb);
}

// dst (rows x cols, ld ldd) = src (ld lds), row-major.
__global__ void k_copy_block(int rows, int cols, const double* __restrict__ src, int lds, double* dst,
                             int ldd) {
    const long long total = (long long)rows * cols;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t / cols), c = (int)(t - (long long)r * cols);
        dst[(size_t)r * ldd + c] = src[(size_t)r * lds + c];
    }
}

// X = P I: the identity with the factorisation's row interchanges applied in order.
__global__ void k_perm_identity(int n, const int* __restrict__ piv, double* X) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        for (int r = 0; r < n; ++r) X[(size_t)r * n + c] = (r == c) ? 1.0 : 0.0;
        for (int j = 0; j < n; ++j) {
            const int p = piv[j];
            if (p == j) continue;
            const double t = X[(size_t)j * n + c];
            X[(size_t)j * n + c] = X[(size_t)p * n + c];
            X[(size_t)p * n + c] = t;
        }
    }
}

// ------------------------------------------------------------------------ DGEMM
// C (m x p, ldc) = alpha * A (m x k, lda) * B (k x p, ldb) + beta * C, all row-major FP64,
// on the FP64 tensor cores (mma.sync m8n8k4 .f64 -- the FP64 matrix path of sm_100a;
// tcgen05 has no FP64 kind).  A CTA computes a 128 x 64 tile with 8 warps of 32 x 32
// (4 x 4 MMA tiles each); K advances in steps of 16 staged in shared memory, the next
// step's tile loaded into registers while the current one is multiplied.  Row strides
// of the staged tiles (20 and 68 doubles) keep each half-warp's fragment loads on distinct
// banks.  Edges are zero-filled, so any m, p, k works.
constexpr int kGBM = 128, kGBN = 64, kGBK = 16, kGThreads = 256;
constexpr int kGAS = kGBK + 4;       // A tile row stride (doubles)
constexpr int kGBS = kGBN + 4;       // B tile row stride

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1]) : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kGThreads) k_dgemm(int m, int p, int k, double alpha,
                                                     const double* __restrict__ A, int lda,
                                                     const double* __restrict__ B, int ldb, double beta,
                                                     double* __restrict__ C, int ldc) {
    __shared__ double As[kGBM * kGAS];
    __shared__ double Bs[kGBK * kGBS];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;                 // 4 x 2 warps of 32 x 32
    const int bm = blockIdx.y * kGBM, bn = blockIdx.x * kGBN;
    const int fr = lane >> 2, fk = lane & 3;                 // fragment row / k (A), k / col (B)
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    double ra[(kGBM * kGBK) / kGThreads], rb[(kGBK * kGBN) / kGThreads];
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < (kGBM * kGBK) / kGThreads; ++q) {
            const int e = tid + kGThreads * q, r = e / kGBK, c = e % kGBK;
            const int gr = bm + r, gc = k0 + c;
            ra[q] = (gr < m && gc < k) ? A[(size_t)gr * lda + gc] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < (kGBK * kGBN) / kGThreads; ++q) {
            const int e = tid + kGThreads * q, r = e / kGBN, c = e % kGBN;
            const int gr = k0 + r, gc = bn + c;
            rb[q] = (gr < k && gc < p) ? B[(size_t)gr * ldb + gc] : 0.0;
        }
    };
    auto store = [&]() {
#pragma unroll
        for (int q = 0; q < (kGBM * kGBK) / kGThreads; ++q) {
            const int e = tid + kGThreads * q;
            As[(e / kGBK) * kGAS + e % kGBK] = ra[q];
        }
#pragma unroll
        for (int q = 0; q < (kGBK * kGBN) / kGThreads; ++q) {
            const int e = tid + kGThreads * q;
            Bs[(e / kGBN) * kGBS + e % kGBN] = rb[q];
        }
    };
    const int nk = (k + kGBK - 1) / kGBK;
    if (nk > 0) {
        load(0);
        store();
    }
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
        if (kt + 1 < nk) load((kt + 1) * kGBK);
#pragma unroll
        for (int ks = 0; ks < kGBK; ks += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = As[(wm * 32 + i * 8 + fr) * kGAS + ks + fk];
#pragma unroll
            for (int j = 0; j < 4; ++j) bf[j] = Bs[(ks + fk) * kGBS + wn * 32 + j * 8 + fr];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j], af[i], bf[j]);
        }
        __syncthreads();
        if (kt + 1 < nk) {
            store();
            __syncthreads();
        }
    }
    // accumulator element h of tile (i, j): row fr, column 2 * fk + h of the 8 x 8 tile
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = bm + wm * 32 + i * 8 + fr, c = bn + wn * 32 + j * 8 + 2 * fk + h;
                if (r < m && c < p) {
                    double* cp = C + (size_t)r * ldc + c;
                    const double v = alpha * acc[i][j][h];
                    *cp = beta != 0.0 ? v + beta * *cp : v;
                }
            }
}

// (st: the stream to launch on; nullptr = the context's stream)
void dgemm(Ctx& ctx, int m, int p, int k, double alpha, const double* A, int lda, const double* B, int ldb,
           double beta, double* C, int ldc, cudaStream_t st = nullptr) {
    if (m <= 0 || p <= 0) return;
    const dim3 grid(ceil_div(p, kGBN), ceil_div(m, kGBM));
    k_dgemm<<<grid, kGThreads, 0, st ? st : ctx.lane.stream>>>(m, p, k, alpha, A, lda, B, ldb, beta, C, ldc);
    HAMLSS_LAUNCH_CHECK();
}

// Row-major C (m x p, ld n) -= A (m x k, ld n) * B (k x p, ld n).
void gemm_sub(Ctx& ctx, int n, int m, int p, int k, const double* A, const double* B, double* C,
              cudaStream_t st = nullptr) {
    if (m <= 0 || p <= 0 || k <= 0) return;
    dgemm(ctx, m, p, k, -1.0, A, n, B, n, 1.0, C, n, st);
}

// Row-major C (m x p, ldc) = A (m x k, lda) * B (k x p, ldb).
void gemm_set(Ctx& ctx, int m, int p, int k, const double* A, int lda, const double* B, int ldb,
              double* C, int ldc, cudaStream_t st = nullptr) {
    if (m <= 0 || p <= 0 || k <= 0) return;
    dgemm(ctx, m, p, k, 1.0, A, lda, B, ldb, 0.0, C, ldc, st);
}

int copy_grid(Ctx& ctx, long long count) {
    return (int)std::max<long long>(1, std::min<long long>((count + 255) / 256, ctx.sm_count * 8LL));
}

int col_grid(Ctx& ctx, int cols) {
    return std::max(1, std::min(ceil_div(cols, 128), ctx.sm_count * 4));
}


__global__ void k_iota(int n, int* piv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) piv[i] = i;
}

// Blocked LU without row interchanges; false when a pivot falls below `floor`.
// L21 = A21 U11^-1 and U12 = L11^-1 A12 are GEMMs with the diagonal block's inverses
// (k_block_inverses) through the scratch T (n x kNb doubles).
//
// With look-ahead: step k's update of block column and block row k + 1 runs first, on a
// second stream, followed there by step k + 1's diagonal block and panels, while the rest of
// step k's trailing update runs on the context's stream.  The regions never overlap: the
// look-ahead writes block column / row k + 1, the trailing update the part beyond it; the
// second stream waits for trailing update k - 1 (the last writer of block k + 1) and the
// context's stream for panel k (the operands of trailing update k).
bool factor_nopivot(Ctx& ctx, int n, double* M, double floor, double* inv, double* T) {
    cudaStream_t s = ctx.lane.stream;
    DBuf<int> tiny(1);
    tiny.zero(s);
    const int nb = (n + kNb - 1) / kNb;
    cudaStream_t pst = nullptr;
    {
        // the look-ahead stream at the highest priority: its small launches take SMs as the
        // trailing update's tiles drain instead of queueing behind them
        int lo = 0, hi = 0;
        HAMLSS_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        HAMLSS_CUDA(cudaStreamCreateWithPriority(&pst, cudaStreamNonBlocking, hi));
    }
    std::vector<cudaEvent_t> panel_ev(nb, nullptr), trail_ev(nb, nullptr);
    cudaEvent_t start_ev = nullptr, done_ev = nullptr;
    auto cleanup = [&]() {
        for (auto e : panel_ev) if (e) cudaEventDestroy(e);
        for (auto e : trail_ev) if (e) cudaEventDestroy(e);
        if (start_ev) cudaEventDestroy(start_ev);
        if (done_ev) cudaEventDestroy(done_ev);
        if (pst) cudaStreamDestroy(pst);
    };
    try {
        for (int k = 0; k < nb; ++k) {
            HAMLSS_CUDA(cudaEventCreateWithFlags(&panel_ev[k], cudaEventDisableTiming));
            HAMLSS_CUDA(cudaEventCreateWithFlags(&trail_ev[k], cudaEventDisableTiming));
        }
        HAMLSS_CUDA(cudaEventCreateWithFlags(&start_ev, cudaEventDisableTiming));
        HAMLSS_CUDA(cudaEventCreateWithFlags(&done_ev, cudaEventDisableTiming));
        HAMLSS_CUDA(cudaEventRecord(start_ev, s));                  // M and tiny are ready
        HAMLSS_CUDA(cudaStreamWaitEvent(pst, start_ev, 0));
        // diagonal block k and its two panels, on the look-ahead stream
        auto panel = [&](int k) {
            const int k0 = k * kNb, kb = std::min(kNb, n - k0), rest = n - k0 - kb;
            k_lu_diag_inv<<<1, 256, kDiagSmem, pst>>>(n, k0, kb, M, floor, tiny.p, inv);
            HAMLSS_LAUNCH_CHECK();
            if (rest > 0) {
                const double* Li = inv + 2LL * k * kNb * kNb;
                const double* Ui = Li + kNb * kNb;
                double* A21 = M + (size_t)(k0 + kb) * n + k0;
                double* A12 = M + (size_t)k0 * n + k0 + kb;
                gemm_set(ctx, rest, kb, kb, A21, n, Ui, kNb, T, kNb, pst);
                k_copy_block<<<copy_grid(ctx, (long long)rest * kb), 256, 0, pst>>>(rest, kb, T, kNb, A21, n);
                HAMLSS_LAUNCH_CHECK();
                gemm_set(ctx, kb, rest, kb, Li, kNb, A12, n, T, rest, pst);
                k_copy_block<<<copy_grid(ctx, (long long)rest * kb), 256, 0, pst>>>(kb, rest, T, rest, A12, n);
                HAMLSS_LAUNCH_CHECK();
            }
            HAMLSS_CUDA(cudaEventRecord(panel_ev[k], pst));
        };
        panel(0);
        for (int k = 0; k < nb; ++k) {
            const int k0 = k * kNb, kb = std::min(kNb, n - k0), rest = n - k0 - kb;
            if (rest <= 0) break;
            const int kb1 = std::min(kNb, rest);                   // block k + 1
            const double* A21 = M + (size_t)(k0 + kb) * n + k0;      // rest x kb (L of step k)
            const double* A12 = M + (size_t)k0 * n + k0 + kb;        // kb x rest (U of step k)
            double* A22 = M + (size_t)(k0 + kb) * n + k0 + kb;
            // the rest of trailing update k: beyond block k + 1
            HAMLSS_CUDA(cudaStreamWaitEvent(s, panel_ev[k], 0));
            gemm_sub(ctx, n, rest - kb1, rest - kb1, kb, A21 + (size_t)kb1 * n, A12 + kb1,
                     A22 + (size_t)kb1 * n + kb1, s);
            HAMLSS_CUDA(cudaEventRecord(trail_ev[k], s));
            // look-ahead: block column and row k + 1 of update k, then panel k + 1
            if (k > 0) HAMLSS_CUDA(cudaStreamWaitEvent(pst, trail_ev[k - 1], 0));
            gemm_sub(ctx, n, rest, kb1, kb, A21, A12, A22, pst);                        // column
            gemm_sub(ctx, n, kb1, rest - kb1, kb, A21, A12 + kb1, A22 + kb1, pst);      // row
            panel(k + 1);
        }
        HAMLSS_CUDA(cudaEventRecord(done_ev, pst));
        HAMLSS_CUDA(cudaStreamWaitEvent(s, done_ev, 0));
    } catch (...) {
        cudaStreamSynchronize(pst);
        cleanup();
        throw;
    }
    int t = 0;
    tiny.download(&t, 1, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    cleanup();
    return t == 0;
}

// Blocked LU with partial pivoting (cooperative panels).
void factor_pivot(Ctx& ctx, int n, double* M, int* piv) {
    cudaStream_t s = ctx.lane.stream;
    DBuf<double> cand_v(ctx.sm_count);
    DBuf<int> cand_i(ctx.sm_count), singular(1);
    singular.zero(s);
    const int pblocks = ctx.sm_count;               // one block per SM: few candidates
    const int cg_ = col_grid(ctx, n);
    for (int k0 = 0; k0 < n; k0 += kNb) {
        const int kb = std::min(kNb, n - k0);
        int nn = n, kk0 = k0, kkb = kb;
        double* Mp = M;
        int* pp = piv;
        double* cv = cand_v.p;
        int* ci = cand_i.p;
        int* sg = singular.p;
        void* args[] = {&nn, &kk0, &kkb, &Mp, &pp, &cv, &ci, &sg};
        HAMLSS_CUDA(cudaLaunchCooperativeKernel((const void*)k_lu_panel, dim3(pblocks), dim3(kPanelThreads),
                                                args, 0, s));
        k_lu_swap<<<cg_, 128, 0, s>>>(n, k0, kb, M, piv);
        HAMLSS_LAUNCH_CHECK();
        const int rest = n - k0 - kb;
        if (rest > 0) {
            k_trsm_lower_unit<<<col_grid(ctx, rest), 128, 0, s>>>(n, k0, kb, M, n, M, n, k0 + kb, n);
            HAMLSS_LAUNCH_CHECK();
            gemm_sub(ctx, n, rest, rest, kb, M + (size_t)(k0 + kb) * n + k0, M + (size_t)k0 * n + k0 + kb,
                     M + (size_t)(k0 + kb) * n + k0 + kb);
        }
    }
    int sing = 0;
    singular.download(&sing, 1, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    if (sing) fail(HAMLSS_ERR_ZERO_PIVOT, "coarsest AMG level is singular (zero pivot in its dense LU)");
}

// ---------------------------------------------------------------- Gram matrix
constexpr int kGramRows = 128;
constexpr int kGramMaxC = 33;

// pair index q -> (a, b), a <= b, pairs listed row by row of the upper triangle
__device__ void gram_pair(int c, int q, int* a, int* b) {
    int r = 0;
    while (q >= c - r) { q -= c - r; ++r; }
    *a = r;
    *b = r + q;
}

__global__ void __launch_bounds__(256) k_gram_partial(int n, int c, const double* __restrict__ Y,
                                                      long long ld, double* part) {
    __shared__ double tile[kGramRows][kGramMaxC + 1];
    const int np = c * (c + 1) / 2;
    int pa[3], pb[3];
    double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int u = 0; u < 3; ++u) {
        const int q = threadIdx.x + 256 * u;
        pa[u] = pb[u] = 0;
        if (q < np) gram_pair(c, q, &pa[u], &pb[u]);
    }
    for (int r0 = blockIdx.x * kGramRows; r0 < n; r0 += gridDim.x * kGramRows) {
        for (int e = threadIdx.x; e < kGramRows * c; e += blockDim.x) {
            const int j = e / kGramRows, r = e - j * kGramRows;
            tile[r][j] = (r0 + r < n) ? Y[(size_t)j * ld + r0 + r] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 3; ++u)
            if (threadIdx.x + 256 * u < np)
                for (int r = 0; r < kGramRows; ++r) acc[u] += tile[r][pa[u]] * tile[r][pb[u]];
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 3; ++u) {
        const int q = threadIdx.x + 256 * u;
        if (q < np) part[(size_t)blockIdx.x * np + q] = acc[u];
    }
}

// Short columns (n <= kGramSeqRows): one thread per pair sums y_a[i] * y_b[i] over i in
// order with separate multiply and add -- the sequential dot product of the reference's
// Vector::dot on one thread, bit for bit.  The s-step iteration amplifies rounding
// differences in G, so small systems keep the reference's summation order.
constexpr int kGramSeqRows = 1 << 15;

__global__ void k_gram_seq(int n, int c, const double* __restrict__ Y, long long ld, double* G) {
    const int np = c * (c + 1) / 2;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
        int a, b;
        gram_pair(c, q, &a, &b);
        const double* ya = Y + (size_t)a * ld;
        const double* yb = Y + (size_t)b * ld;
        double s = 0.0;
        for (int i = 0; i < n; ++i) s = __dadd_rn(s, __dmul_rn(ya[i], yb[i]));
        G[a * c + b] = s;
        G[b * c + a] = s;
    }
}

// G[a][b] = G[b][a] = the blocks' partial sums of pair (a, b), added in block order
__global__ void k_gram_reduce(int c, int nblocks, const double* __restrict__ part, double* G) {
    const int np = c * (c + 1) / 2;
    for (int q = threadIdx.x; q < np; q += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * np + q];
        int a, bb;
        gram_pair(c, q, &a, &bb);
        G[a * c + bb] = s;
        G[bb * c + a] = s;
    }
}

}  // namespace

void dense_lu_inverse(Ctx& ctx, int n, double* M, double* Minv, int* piv) {
    cudaStream_t s = ctx.lane.stream;
    if (n <= 0) return;
    const int cg_ = col_grid(ctx, n);
    HAMLSS_CUDA(cudaFuncSetAttribute(k_lu_diag_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiagSmem));
    HAMLSS_CUDA(cudaFuncSetAttribute(k_block_inverses, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiagSmem));
    const size_t bytes = sizeof(double) * (size_t)n * n;
    // First without interchanges (the coarse operators here are symmetric positive definite
    // or close to diagonally dominant, where that is stable); if a pivot falls below
    // 1e-10 of the largest entry, start over with partial pivoting.
    DBuf<unsigned long long> amax(1);
    amax.zero(s);
    k_abs_max<<<col_grid(ctx, (int)std::min<size_t>((size_t)n * n / 8 + 1, 1u << 30)), 128, 0, s>>>(
        (long long)n * n, M, amax.p);
    HAMLSS_LAUNCH_CHECK();
    unsigned long long bits = 0;
    amax.download(&bits, 1, s);
    HAMLSS_CUDA(cudaMemcpyAsync(Minv, M, bytes, cudaMemcpyDeviceToDevice, s));   // backup
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    double big = 0.0;
    std::memcpy(&big, &bits, sizeof big);
    const int nblk = (n + kNb - 1) / kNb;
    DBuf<double> inv(2LL * nblk * kNb * kNb), T((size_t)n * kNb);
    const bool nopiv = factor_nopivot(ctx, n, M, 1e-10 * big, inv.p, T.p);
    if (nopiv) {
        k_iota<<<cg_, 128, 0, s>>>(n, piv);
        HAMLSS_LAUNCH_CHECK();
    } else {
        HAMLSS_CUDA(cudaMemcpyAsync(M, Minv, bytes, cudaMemcpyDeviceToDevice, s));
        factor_pivot(ctx, n, M, piv);
        k_block_inverses<<<nblk, 4 * kNb, kDiagSmem, s>>>(n, 0, M, inv.p);
        HAMLSS_LAUNCH_CHECK();
    }
    // X = P I; L Y = X (forward, unit lower); U X = Y (backward).  The diagonal blocks are
    // applied as GEMMs with their inverses, the off-diagonal blocks as GEMM updates.
    k_perm_identity<<<cg_, 128, 0, s>>>(n, piv, Minv);
    HAMLSS_LAUNCH_CHECK();
    DBuf<double> W((size_t)kNb * n);
    // Without interchanges X = I, so Y = L^-1 is lower triangular: block row k0 of Y has
    // nonzeros only in columns < k0 + kb, and the forward sweep touches only those
    // (n^3 / 3 multiply-adds instead of n^3).
    for (int k0 = 0; k0 < n; k0 += kNb) {
        const int kb = std::min(kNb, n - k0);
        const int w = nopiv ? k0 + kb : n;
        const double* Li = inv.p + 2LL * (k0 / kNb) * kNb * kNb;
        gemm_set(ctx, kb, w, kb, Li, kNb, Minv + (size_t)k0 * n, n, W.p, n);
        k_copy_block<<<copy_grid(ctx, (long long)kb * w), 256, 0, s>>>(kb, w, W.p, n, Minv + (size_t)k0 * n, n);
        HAMLSS_LAUNCH_CHECK();
        const int rest = n - k0 - kb;
        gemm_sub(ctx, n, rest, w, kb, M + (size_t)(k0 + kb) * n + k0, Minv + (size_t)k0 * n,
                 Minv + (size_t)(k0 + kb) * n);
    }
    const int last = ((n - 1) / kNb) * kNb;
    for (int k0 = last; k0 >= 0; k0 -= kNb) {
        const int kb = std::min(kNb, n - k0);
        const double* Ui = inv.p + 2LL * (k0 / kNb) * kNb * kNb + kNb * kNb;
        gemm_set(ctx, kb, n, kb, Ui, kNb, Minv + (size_t)k0 * n, n, W.p, n);
        k_copy_block<<<copy_grid(ctx, (long long)kb * n), 256, 0, s>>>(kb, n, W.p, n, Minv + (size_t)k0 * n, n);
        HAMLSS_LAUNCH_CHECK();
        gemm_sub(ctx, n, k0, n, kb, M + k0, Minv + (size_t)k0 * n, Minv);
    }
    HAMLSS_CUDA(cudaStreamSynchronize(s));
}

int gram_partials(Ctx& ctx, int c) { return ctx.sm_count * 4 * (c * (c + 1) / 2); }

void gram_matrix(Ctx& ctx, int n, int c, const double* Y, long long ld, double* G, double* part) {
    if (c < 1 || c > kGramMaxC) fail(HAMLSS_ERR_INVALID, "Gram matrix of more than 33 columns");
    if (n <= kGramSeqRows) {
        const int np = c * (c + 1) / 2;
        k_gram_seq<<<ceil_div(np, 64), 64, 0, ctx.lane.stream>>>(n, c, Y, ld, G);
        HAMLSS_LAUNCH_CHECK();
        return;
    }
    const int blocks = std::max(1, std::min(ceil_div(n, kGramRows), ctx.sm_count * 4));
    k_gram_partial<<<blocks, 256, 0, ctx.lane.stream>>>(n, c, Y, ld, part);
    HAMLSS_LAUNCH_CHECK();
    k_gram_reduce<<<1, 256, 0, ctx.lane.stream>>>(c, blocks, part, G);
    HAMLSS_LAUNCH_CHECK();
}

}  // namespace hamlss
