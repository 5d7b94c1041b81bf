// amg.cu -- smoothed-aggregation AMG on the device (AMGPreconditioner, amg.cpp).
//
// Setup (amg.cpp:183-237), every step a device kernel:
//   aggregate   greedy aggregation of amg.cpp:30-67, bit for bit.  The sequential pass
//               makes node i a seed iff no earlier seed s < i holds i as a strong, still
//               unassigned neighbour, where strong means |a_si| >= theta * max_{l != s}|a_sl|.
//               Every node before s is assigned when s is visited, so this is exactly:
//                 seed(i)  <=>  no seed in IN(i) = { s < i : s -> i strong }
//                 agg(i)    =  number of seeds before i            (seed)
//                           =  agg(min seed in IN(i))              (otherwise)
//               IN(i) only holds lower indices, so one cooperative kernel decides the
//               nodes in index order, warp by warp, each node as soon as its IN nodes are
//               decided (no grid barriers), then a scan numbers the seeds.
//   prolong     Jacobi-smoothed tentative prolongation (amg.cpp:101-178) computed
//               sparsely: row i starts at e_agg(i) and subtracts (omega/a_ii) a_ij at column
//               agg(j) in row order, then drops |v| <= 1e-14.  Same operations in the same
//               order as the reference's dense buffer, so P is identical bit for bit.
//   transpose   R = P^T with rows in increasing fine index (sparse_matrix.cpp:138-165).
//   Galerkin    A_c = R (A P) by a row-wise k-way merge SpGEMM: each output column sums
//               its products in the order of the left row, starting from 0.0, and drops
//               |v| <= eps^2 (sparse_matrix.cpp:171-237) -- bit for bit again.
//   coarsest    dense LU with partial pivoting, factored once (amg.cpp:260-291 redoes it
//               every cycle; the pivots and multipliers are the same).
// V-cycle (amg.cpp:296-343), FP64 (bit-exact with the reference) or FP32 (mixed
// precision): the first pre-smoothing sweep on x = 0 is the elementwise x = w D^-1 b and is
// fused into the restriction that produces b; every other sweep, the residual, the
// restriction and the prolongation+correction are single fused SpMV passes.
#include <cooperative_groups.h>

#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "krylov.cuh"
#include "dense_lu.cuh"
#include "scan.cuh"

namespace cg = cooperative_groups;

namespace hamlss {

namespace {

constexpr double kEps = 2.220446049250313e-16;
constexpr int kLongRow = 32;            // rows longer than this are given a whole block
constexpr int kSortMax = 8192;          // largest shared-memory sort (u64 keys)
constexpr int kBlockedCoarse = 1024;    // coarsest levels above this use the blocked LU
constexpr int kStallDenseMax = 8192;    // largest level the stall rule makes the coarsest
constexpr int kMaxLevels = 64;          // hierarchy depth cap (amg_levels above it is clamped)

// Rows that the block-per-row kernels (smoothed P, transpose sort) take.
__host__ __device__ __forceinline__ bool smooth_row_on_block(int len) {
    return len > kLongRow && len + 1 <= kSortMax;
}

struct DCsr {
    int n = 0, m = 0, nnz = 0;
    DBuf<int> rp, ci;
    DBuf<double> v;
    DBuf<float> v32;
    Csr<double> f64() const { return Csr<double>{n, m, nnz, rp.p, ci.p, v.p}; }
    Csr<float> f32() const { return Csr<float>{n, m, nnz, rp.p, ci.p, v32.p}; }
};

inline int grid_for(Ctx& ctx, long long n) {
    return std::max(1, std::min(ceil_div(n, 256), ctx.sm_count * 8));
}

// ------------------------------------------------------------------ aggregation
__global__ void k_rowmax(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                         const double* __restrict__ v, double* rmax) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double m = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] != i) m = fmax(m, fabs(v[k]));
        rmax[i] = m;
    }
}

// in_cnt[j] = |IN(j)|
__global__ void k_in_count(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ v, const double* __restrict__ rmax,
                           double theta, int* in_cnt) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const double th = theta * rmax[s];
        for (int k = rp[s]; k < rp[s + 1]; ++k) {
            int j = ci[k];
            if (j > s && fabs(v[k]) >= th) atomicAdd(&in_cnt[j], 1);
        }
    }
}

__global__ void k_in_fill(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                          const double* __restrict__ v, const double* __restrict__ rmax,
                          double theta, int* fillpos, int* in_src) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const double th = theta * rmax[s];
        for (int k = rp[s]; k < rp[s + 1]; ++k) {
            int j = ci[k];
            if (j > s && fabs(v[k]) >= th) in_src[atomicAdd(&fillpos[j], 1)] = s;
        }
    }
}

// The same three passes with a warp per row (lanes stride the row), for levels whose rows
// are long (the dense coarse operators): a thread per row there leaves most of the GPU
// idle.  The IN lists' order does not matter (they are used as sets).
__global__ void k_rowmax_w(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ v, double* rmax) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        double m = 0.0;
        for (int k = rp[i] + lane; k < rp[i + 1]; k += 32)
            if (ci[k] != i) m = fmax(m, fabs(v[k]));
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) rmax[i] = m;
    }
}

__global__ void k_in_count_w(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ v, const double* __restrict__ rmax,
                             double theta, int* in_cnt) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < n; s += nw) {
        const double th = theta * rmax[s];
        for (int k = rp[s] + lane; k < rp[s + 1]; k += 32) {
            const int j = ci[k];
            if (j > s && fabs(v[k]) >= th) atomicAdd(&in_cnt[j], 1);
        }
    }
}

__global__ void k_in_fill_w(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                            const double* __restrict__ v, const double* __restrict__ rmax,
                            double theta, int* fillpos, int* in_src) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < n; s += nw) {
        const double th = theta * rmax[s];
        for (int k = rp[s] + lane; k < rp[s + 1]; k += 32) {
            const int j = ci[k];
            if (j > s && fabs(v[k]) >= th) in_src[atomicAdd(&fillpos[j], 1)] = s;
        }
    }
}

// Decide seed / non-seed for every node: seed(i) <=> no seed in IN(i).  IN(i) holds only
// lower indices, so node i can be decided as soon as its IN nodes are.  Persistent warps
// claim chunks of 32 consecutive nodes in increasing order (atomic ticket).  For a chunk,
// each lane first reads, for its own node, the status of every IN node outside the chunk
// in one sweep (the loads do not wait on one another; one seed among them settles the
// node), waits only if none is a seed and some are undecided, and notes which IN nodes lie
// inside the chunk; the warp then decides the 32 nodes in order from registers alone and
// publishes them with one store.  The statuses are the only data exchanged, so the store
// needs no fence.  Every claimed chunk belongs to a running warp (cooperative launch: all
// blocks resident) and a chunk only waits on earlier chunks, so the waits end.  Each wait
// is bounded (about a second): past that the kernel records *err and moves on, and the host
// reports HAMLSS_ERR_TIMEOUT.
// status: 0 undecided (zeroed before the launch), 1 seed, 2 non-seed.
constexpr long long kWaitCycles = 2000000000LL;

__device__ __forceinline__ int wait_status(const int* status, int src, int* err) {
    const volatile int* vs = status + src;
    int st = *vs;
    if (st == 0) {
        const long long t0 = clock64();
        while ((st = *vs) == 0) {
            if (clock64() - t0 > kWaitCycles) {
                atomicExch(err, 1);
                return 2;
            }
            __nanosleep(32);                 // poll gently: the producer needs the memory system
        }
    }
    return st;
}

__global__ void k_aggregate_wave(int n, const int* __restrict__ in_rp, const int* __restrict__ in_src,
                                 int* status, int* ticket, int* err) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(ticket, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const int cnt = min(32, n - base);
        // pass 1, lane q for node base + q: whether an IN node outside the chunk is a seed
        // (bit q of `outside`) and which IN nodes lie inside the chunk (`inmask`)
        unsigned inmask = 0u;
        bool cap = false;
        if (lane < cnt) {
            const int i = base + lane;
            const int s0 = in_rp[i], s1 = in_rp[i + 1];
            bool pending = false;
            for (int k = s0; k < s1; ++k) {
                const int src = in_src[k];
                if (src >= base) {
                    inmask |= 1u << (src - base);
                } else {
                    const int st = *(const volatile int*)(status + src);
                    cap |= st == 1;
                    pending |= st == 0;
                }
            }
            if (!cap && pending)
                for (int k = s0; k < s1 && !cap; ++k) {
                    const int src = in_src[k];
                    if (src < base) cap = wait_status(status, src, err) == 1;
                }
        }
        const unsigned outside = __ballot_sync(0xffffffffu, cap);
        // pass 2: decide in order (seeds: bit q of `seeds`), registers only
        unsigned seeds = 0u;
#pragma unroll
        for (int q = 0; q < 32; ++q) {
            const unsigned mq = __shfl_sync(0xffffffffu, inmask, q);
            const bool captured = q >= cnt || ((outside >> q) & 1u) || (mq & seeds);
            seeds |= captured ? 0u : 1u << q;
        }
        if (lane < cnt) *(volatile int*)(status + base + lane) = ((seeds >> lane) & 1u) ? 1 : 2;
    }
}

__global__ void k_seed_flags(int n, const int* __restrict__ status, int* flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        flag[i] = status[i] == 1 ? 1 : 0;
}

// flag holds the exclusive seed count; assign every node
__global__ void k_assign(int n, const int* __restrict__ status, const int* __restrict__ seedno,
                         const int* __restrict__ in_rp, const int* __restrict__ in_src, int* agg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (status[i] == 1) { agg[i] = seedno[i]; continue; }
        int best = INT_MAX;
        for (int k = in_rp[i]; k < in_rp[i + 1]; ++k) {
            int s = in_src[k];
            if (status[s] == 1 && s < best) best = s;
        }
        agg[i] = (best == INT_MAX) ? -1 : seedno[best];
    }
}

// ------------------------------------------------------- smoothed prolongation
// Row i of P: candidates in first-occurrence order: agg(i), then agg(j) for off-diagonal
// j in row order.  Values computed exactly as amg.cpp:139-154 would for column c.
__device__ double p_value(int i, int c, int s, int e, const int* __restrict__ ci,
                          const double* __restrict__ v, const int* __restrict__ agg, double id,
                          bool raw) {
    double val = (c == agg[i]) ? 1.0 : 0.0;
    if (raw) return val;
    for (int k = s; k < e; ++k) {
        int j = ci[k];
        if (j == i) continue;
        if (agg[j] == c) val = __dsub_rn(val, __dmul_rn(id, v[k]));
    }
    return val;
}

// Rows of lo_len + 1 to W entries (lo_len >= -1), W lanes per row (W = 8, 16 or 32; lane a
// of the row's group holds entry a).  Candidate agg(i) first, then the off-diagonal
// entries' aggregates at their first occurrence (match.any); each candidate's value is
// formed by its lane walking the row's entries in order through shuffles, with p_value's
// operations: val = [c == agg(i)], then val -= (omega / a_ii) * a_ij for every off-diagonal
// j of aggregate c, in row order.  Survivors (|val| > 1e-14) are written in column order
// (rank = survivors with a smaller column) at prp[i], their count to pcnt[i].  Same entries,
// values and order as the thread-per-row kernel below.
template <int W>
__global__ void k_smooth_p_sub(int n, int lo_len, const int* __restrict__ rp, const int* __restrict__ ci,
                               const double* __restrict__ v, const int* __restrict__ agg, double omega,
                               int* pcnt, const int* __restrict__ prp, int* pci, double* pv) {
    static_assert(W == 8 || W == 16 || W == 32, "lanes a row");
    const int lane = threadIdx.x & 31, sl = lane & (W - 1), sub = lane / W;
    const unsigned smask = W == 32 ? 0xffffffffu : ((1u << W) - 1u) << (sub * W);
    const int ngroups = (gridDim.x * blockDim.x) / W;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) / W; i < n; i += ngroups) {
        const int s = rp[i], len = rp[i + 1] - s;
        if (len > W || len <= lo_len) continue;          // another kernel takes it
        const bool have = sl < len;
        const int j = have ? ci[s + sl] : -1;
        const double va = have ? v[s + sl] : 0.0;
        const bool diag = have && j == i;
        const unsigned dmask = __ballot_sync(smask, diag) & smask;
        double id = 0.0;
        if (dmask) {
            const double dv = __shfl_sync(smask, va, (__ffs(dmask) - 1) & (W - 1), W);
            id = (fabs(dv) > kEps) ? omega / dv : 0.0;
        }
        const bool raw = fabs(id) < kEps;
        const int ai = agg[i];
        const int c = (have && !diag) ? agg[j] : -1;     // this entry's aggregate
        const unsigned same = __match_any_sync(smask, c);
        const bool cand = !raw && c >= 0 && c != ai && (__ffs(same) - 1) == lane;
        double val = 0.0, val0 = 1.0;                    // own candidate / agg(i)
        if (!raw) {
            for (int l = 0; l < len; ++l) {
                const int cl = __shfl_sync(smask, c, l, W);
                const double vl = __shfl_sync(smask, va, l, W);
                if (cl < 0) continue;
                if (cand && cl == c) val = __dsub_rn(val, __dmul_rn(id, vl));
                if (cl == ai) val0 = __dsub_rn(val0, __dmul_rn(id, vl));
            }
        }
        const bool keep = cand && fabs(val) > 1e-14;
        const bool keep0 = fabs(val0) > 1e-14;
        const unsigned kmask = __ballot_sync(smask, keep) & smask;
        if (pcnt && sl == 0) pcnt[i] = __popc(kmask) + (keep0 ? 1 : 0);
        // ranks by column among the survivors
        const int myc = keep ? c : INT_MAX;
        int rank = (keep0 && ai < myc) ? 1 : 0, rank0 = 0;
        for (int l = 0; l < W; ++l) {
            const int cl = __shfl_sync(smask, myc, l, W);
            if (cl < myc) ++rank;
            if (cl < ai) ++rank0;
        }
        const int o = prp[i];
        if (keep) {
            pci[o + rank] = c;
            pv[o + rank] = val;
        }
        if (keep0 && sl == 0) {
            pci[o + rank0] = ai;
            pv[o + rank0] = val0;
        }
    }
}

// Slot of row i in a scratch of (entries of A + rows) slots: room for every candidate.
__global__ void k_slot_offsets(int n, const int* __restrict__ rp, int* off) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) off[i] = rp[i] + i;
}

// Rows the warp and block kernels leave (kSortMax entries or more), one thread per row.
template <bool FILL>
__global__ void k_smooth_p(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ v, const int* __restrict__ agg, double omega,
                           int* pcnt, const int* __restrict__ prp, int* pci, double* pv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = rp[i], e = rp[i + 1];
        if (e - s <= kLongRow || smooth_row_on_block(e - s)) continue;   // warp / block kernels
        double id = 0.0;
        for (int k = s; k < e; ++k)
            if (ci[k] == i) { id = (fabs(v[k]) > kEps) ? omega / v[k] : 0.0; break; }
        const bool raw = fabs(id) < kEps;
        // candidate list: index -1 = agg(i), then off-diagonal entries
        int count = 0;
        for (int a = -1; a < e - s; ++a) {
            int c;
            if (a < 0) c = agg[i];
            else { int j = ci[s + a]; if (j == i || raw) continue; c = agg[j]; }
            // first occurrence?
            bool first = (a < 0) || (c != agg[i]);
            if (first && a >= 0)
                for (int b = 0; b < a; ++b) {
                    int jb = ci[s + b];
                    if (jb != i && agg[jb] == c) { first = false; break; }
                }
            if (!first) continue;
            double val = p_value(i, c, s, e, ci, v, agg, id, raw);
            if (!(fabs(val) > 1e-14)) continue;
            if (FILL) {
                // rank among surviving candidates with a smaller column
                int rank = 0;
                for (int a2 = -1; a2 < e - s; ++a2) {
                    int c2;
                    if (a2 < 0) c2 = agg[i];
                    else { int j2 = ci[s + a2]; if (j2 == i || raw) continue; c2 = agg[j2]; }
                    if (c2 >= c) continue;
                    bool f2 = (a2 < 0) || (c2 != agg[i]);
                    if (f2 && a2 >= 0)
                        for (int b = 0; b < a2; ++b) {
                            int jb = ci[s + b];
                            if (jb != i && agg[jb] == c2) { f2 = false; break; }
                        }
                    if (!f2) continue;
                    if (fabs(p_value(i, c2, s, e, ci, v, agg, id, raw)) > 1e-14) ++rank;
                }
                pci[prp[i] + rank] = c;
                pv[prp[i] + rank] = val;
            }
            ++count;
        }
        if (pcnt) pcnt[i] = count;
    }
}

// ------------------------------------------------------------------- transpose
__global__ void k_t_count(int n, const int* __restrict__ rp, const int* __restrict__ ci, int* cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; ++k) atomicAdd(&cnt[ci[k]], 1);
}

__global__ void k_t_fill(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                         const double* __restrict__ v, int* fillpos, int* tci, double* tv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            int p = atomicAdd(&fillpos[ci[k]], 1);
            tci[p] = i;
            tv[p] = v[k];
        }
}

// rows of the transpose hold distinct source rows: sort each by index
__global__ void k_t_sort(int m, const int* __restrict__ trp, int* tci, double* tv) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < m; r += gridDim.x * blockDim.x) {
        const int s = trp[r], e = trp[r + 1];
        if (smooth_row_on_block(e - s)) continue;       // k_t_sort_rows takes it
        for (int a = s + 1; a < e; ++a) {
            int c = tci[a];
            double x = tv[a];
            int b = a - 1;
            while (b >= s && tci[b] > c) { tci[b + 1] = tci[b]; tv[b + 1] = tv[b]; --b; }
            tci[b + 1] = c;
            tv[b + 1] = x;
        }
    }
}

// -------------------------------------------------------------------- SpGEMM
// Row i of C = A B by a k-way merge of the rows of B selected by row i of A.  Each output
// column is the sum, starting at 0.0, of a_ij * b_jl in the order of row i of A, with
// separate multiply and add: mat_mat_product's dense accumulator (sparse_matrix.cpp:196-212)
// value for value.  Rows of A longer than kHeads keep their merge heads in `heads`
// (3 ints per nonzero of A at 3 * rp[i]).
constexpr int kHeads = 24;

// Capacity of row i of C = A B: min(products of the row, columns of B, the span from the
// smallest first column to the largest last column of the selected rows of B).
__global__ void k_spgemm_bound(int m, const int* __restrict__ arp, const int* __restrict__ aci,
                               const int* __restrict__ brp, const int* __restrict__ bci, int bcols,
                               int* cap) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        long long u = 0;
        int lo = INT_MAX, hi = -1;
        for (int t = arp[i]; t < arp[i + 1]; ++t) {
            const int j = aci[t];
            const int p0 = brp[j], p1 = brp[j + 1];
            u += p1 - p0;
            if (p1 > p0) {
                lo = min(lo, bci[p0]);
                hi = max(hi, bci[p1 - 1]);
            }
        }
        long long c = u < bcols ? u : bcols;
        const long long span = hi >= lo ? (long long)hi - lo + 1 : 0;
        cap[i] = (int)(c < span ? c : span);
    }
}

// Move row i's cnt[i] entries from its capacity slot (at off[i]) to its CSR place; one warp
// per row.
__global__ void k_spgemm_compact(int m, const int* __restrict__ off, const int* __restrict__ cnt,
                                 const int* __restrict__ wci, const double* __restrict__ wv,
                                 const int* __restrict__ crp, int* cci, double* cv) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < m; i += nw) {
        const int src = off[i], dst = crp[i], c = cnt[i];
        for (int t = lane; t < c; t += 32) {
            cci[dst + t] = wci[src + t];
            cv[dst + t] = wv[src + t];
        }
    }
}

template <bool FILL>
__global__ void k_spgemm(int m, const int* __restrict__ arp, const int* __restrict__ aci,
                         const double* __restrict__ av, const int* __restrict__ brp,
                         const int* __restrict__ bci, const double* __restrict__ bv, int* ccnt,
                         const int* __restrict__ crp, int* cci, double* cv, int* heads,
                         const int* __restrict__ cls) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (cls[i]) continue;                           // k_spgemm_rows takes it
        const int s = arp[i], k = arp[i + 1] - s;
        int lpos[kHeads], lend[kHeads], lcur[kHeads];
        int* pos = k <= kHeads ? lpos : heads + 3LL * s;
        int* end = k <= kHeads ? lend : heads + 3LL * s + k;
        int* cur = k <= kHeads ? lcur : heads + 3LL * s + 2 * k;
        for (int t = 0; t < k; ++t) {
            int j = aci[s + t];
            pos[t] = brp[j];
            end[t] = brp[j + 1];
            cur[t] = pos[t] < end[t] ? bci[pos[t]] : INT_MAX;
        }
        int o = FILL ? crp[i] : 0;
        for (;;) {
            int cmin = INT_MAX;
            for (int t = 0; t < k; ++t) cmin = min(cmin, cur[t]);
            if (cmin == INT_MAX) break;
            double sum = 0.0;
            for (int t = 0; t < k; ++t) {
                if (cur[t] != cmin) continue;
                sum = __dadd_rn(sum, __dmul_rn(av[s + t], bv[pos[t]]));
                ++pos[t];
                cur[t] = pos[t] < end[t] ? bci[pos[t]] : INT_MAX;
            }
            if (fabs(sum) > kEps * kEps) {
                if (FILL) { cci[o] = cmin; cv[o] = sum; }
                ++o;
            }
        }
        if (ccnt) ccnt[i] = FILL ? o - crp[i] : o;
    }
}

// ------------------------------------------------- block-per-row setup kernels
// Coarse AMG levels grow long rows (hundreds of entries); one thread per row is then
// quadratic or worse.  These kernels give such a row a whole block and sort in shared
// memory.  They produce exactly the same entries, values and order as the thread-per-row
// kernels above: every value is still accumulated by one thread, in the same order.
constexpr int kRowBlock = 256;
constexpr unsigned long long kNoKey = ~0ull;

// Ascending bitonic sort of N (a power of two) keys in shared memory by the whole block.
__device__ void block_bitonic(unsigned long long* a, int N) {
    __syncthreads();
    for (int k = 2; k <= N; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < N; t += blockDim.x) {
                const int p = t ^ j;
                if (p > t) {
                    const unsigned long long x = a[t], y = a[p];
                    if ((x > y) == ((t & k) == 0)) { a[t] = y; a[p] = x; }
                }
            }
            __syncthreads();
        }
}

__device__ __forceinline__ int pow2_at_least(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Rows [0, n) with kLongRow < len and len + 1 <= kSortMax, appended to `list`.
// count[1] receives the longest listed row.
// The same rows in three length buckets for the smoothed prolongation: len < 128 (sort of
// <= 128 keys), < 512 and the rest; list + b * n holds bucket b, count[b] its size and
// count[3 + b] its longest row.
__global__ void k_long_rows3(int n, const int* __restrict__ rp, int* list, int* count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int len = rp[i + 1] - rp[i];
        if (smooth_row_on_block(len)) {
            const int b = len < 128 ? 0 : len < 512 ? 1 : 2;
            list[(size_t)b * n + atomicAdd(count + b, 1)] = i;
            atomicMax(count + 3 + b, len);
        }
    }
}

__global__ void k_long_rows(int n, const int* __restrict__ rp, int* list, int* count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int len = rp[i + 1] - rp[i];
        if (smooth_row_on_block(len)) {
            list[atomicAdd(count, 1)] = i;
            atomicMax(count + 1, len);
        }
    }
}

// Smoothed prolongation of the listed rows (amg.cpp:101-178), one block per row.  The
// row's (agg(j), position) pairs are sorted, so each candidate column's contributions sit
// together in row order; the first thread of each group computes the value with the same
// operations as p_value().  Shared memory: pow2(len + 1) keys + as many doubles.
template <bool FILL>
__global__ void k_smooth_p_rows(const int* __restrict__ rows, int nrows, const int* __restrict__ rp,
                                const int* __restrict__ ci, const double* __restrict__ v,
                                const int* __restrict__ agg, double omega, int* pcnt,
                                const int* __restrict__ prp, int* pci, double* pv) {
    extern __shared__ unsigned long long sm_keys[];
    __shared__ double s_id;
    __shared__ int s_warp[kRowBlock / 32];
    for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
        const int i = rows[r];
        const int s = rp[i], e = rp[i + 1], len = e - s;
        const int N = pow2_at_least(len + 1);
        double* val = reinterpret_cast<double*>(sm_keys + N);
        if (threadIdx.x == 0) {
            double id = 0.0;
            for (int k = s; k < e; ++k)
                if (ci[k] == i) { id = (fabs(v[k]) > kEps) ? omega / v[k] : 0.0; break; }
            s_id = id;
        }
        __syncthreads();
        const double id = s_id;
        const bool raw = fabs(id) < kEps;
        const unsigned ai = (unsigned)agg[i];
        for (int t = threadIdx.x; t < N; t += blockDim.x) {
            unsigned long long key = kNoKey;
            if (t == 0) key = (unsigned long long)ai << 32;             // the row's own aggregate
            else if (t <= len && !raw) {
                const int j = ci[s + t - 1];
                if (j != i) key = ((unsigned long long)(unsigned)agg[j] << 32) | (unsigned)t;
            }
            sm_keys[t] = key;
        }
        block_bitonic(sm_keys, N);
        // group leaders compute their candidate's value; survivors are flagged in val[]
        int keep = 0;
        for (int t = threadIdx.x; t < N; t += blockDim.x) {
            const unsigned long long key = sm_keys[t];
            bool lead = key != kNoKey && (t == 0 || (sm_keys[t - 1] >> 32) != (key >> 32));
            double x = 0.0;
            if (lead) {
                const unsigned c = (unsigned)(key >> 32);
                x = (c == ai) ? 1.0 : 0.0;
                for (int u = t; u < N && (sm_keys[u] >> 32) == c && sm_keys[u] != kNoKey; ++u) {
                    const int pos = (int)(sm_keys[u] & 0xffffffffu);
                    if (pos == 0) continue;
                    x = __dsub_rn(x, __dmul_rn(id, v[s + pos - 1]));
                }
                if (!(fabs(x) > 1e-14)) lead = false;
            }
            val[t] = lead ? x : __longlong_as_double(0x7ff8dead00000000ll);  // NaN marks "none"
            keep += lead;
        }
        // block count of survivors
        int w = keep;
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = w;
        __syncthreads();
        if (pcnt && threadIdx.x == 0) {
            int tot = 0;
            for (int q = 0; q < (int)blockDim.x / 32; ++q) tot += s_warp[q];
            pcnt[i] = tot;
        }
        if (FILL && threadIdx.x == 0) {
            // survivors in ascending column order: one thread walks the sorted groups
            int o = prp[i];
            for (int t = 0; t < N; ++t) {
                const double x = val[t];
                if (x == x) {
                    pci[o] = (int)(sm_keys[t] >> 32);
                    pv[o] = x;
                    ++o;
                }
            }
        }
        __syncthreads();
    }
}

// SpGEMM row classes: 0 thread-per-row merge (short rows, or rows too long for the rest),
// 1 block-per-row hash accumulation, 2 block-per-row dense accumulation (the right operand
// has at most kDenseCols columns), 3 warp-per-row merge (left rows of kHeads+1 to
// kWarpHeads entries), 4 block-per-row dense accumulation over the row's column window,
// 5 / 6 ordered warp accumulation, 32 products / one left entry a step (rows of more than
// 32 products over a window of at most kDenseCols columns; see k_spgemm_classify).
// count[0] / list: class-1 rows, count[1] the widest class-1 table, count[2] / list + m:
// class-2 rows, count[3] / list + 2m: class-3 rows, count[4] their longest left row,
// count[5 + b] / list + (3 + b) m: class-4 rows of window bucket b (span <= 4096, <= 8192,
// <= kDenseCols), count[8 + b] the bucket's widest window, count[11] / list + 6m and
// count[13] / list + 7m: class-5 and class-6 rows, count[12] and count[14] their widest
// windows.
constexpr int kHashMax = 4096;          // distinct output columns a shared table may hold
constexpr int kDenseCols = 16384;       // columns a shared dense accumulator may hold
constexpr int kWarpHeads = 2048;        // merge heads a warp keeps in shared memory
constexpr int kWarpMergeK = 512;        // long rows with at most this many left entries merge
constexpr int kMergeWarps = 4;          // warps (rows) per block of k_spgemm_warp

// Ordered-accumulation SpGEMM (k_spgemm_seq below): output columns of a pass's
// accumulator, rows (warps) a block.  It takes rows whose right rows average at most
// kSeqRight entries; longer right rows keep a whole block busy a step in k_spgemm_window.
constexpr int kSeqCols = 512;
constexpr int kSeqWarps = 8;
constexpr int kSeqShort = 12;
constexpr int kSeqRight = 64;
constexpr int kSeqSteps = 96;

__global__ void k_spgemm_classify(int m, const int* __restrict__ arp, const int* __restrict__ aci,
                                  const int* __restrict__ brp, const int* __restrict__ bci, int bcols,
                                  int* cls, int* list, int* count, int* wlo, int* wspan) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const int s = arp[i], k = arp[i + 1] - s;
        long long u = 0;
        int lo = INT_MAX, hi = -1;
        for (int t = 0; t < k; ++t) {
            const int j = aci[s + t];
            const int p0 = brp[j], p1 = brp[j + 1];
            u += p1 - p0;
            if (p1 > p0) {
                lo = min(lo, bci[p0]);
                hi = max(hi, bci[p1 - 1]);
            }
        }
        const long long span = hi >= lo ? (long long)hi - lo + 1 : 0;
        const long long h = u < bcols ? u : bcols;
        const bool lng = k > kHeads || u > 512;
        // dense accumulation pays one barrier per left entry: worth it when the right rows
        // are long (>= 32 products a step); over the window of columns the row can reach it
        // also scans only that window.  The warp merge pays per output column
        const bool dense_ok = bcols <= kDenseCols && h > kHashMax / 4;
        // the ordered warp accumulation takes the rows of more than 32 products and a window
        // that fits its bitmap: 32 products a step where right rows are short (at most
        // kSeqShort entries on average), one left entry a step up to kSeqRight entries and
        // kSeqSteps left entries
        const bool seq = u > 32 && span > 0 && span <= kDenseCols;
        int c = 0;
        if (seq && u <= (long long)kSeqShort * k) c = 5;
        else if (seq && u <= (long long)kSeqRight * k && k <= kSeqSteps) c = 6;
        else if (lng && span <= kDenseCols && u >= 32LL * k && h > kHashMax / 4) c = 4;
        else if (lng && k <= kWarpMergeK) c = 3;
        else if (lng && dense_ok) c = 2;
        else if (lng && h <= kHashMax) c = 1;
        else if (k > kHeads && k <= kWarpHeads) c = 3;
        cls[i] = c;
        // the class's counter in `count`, its list at lbase, the maximum it tracks
        int ctr = -1, mxi = -1, mx = 0;
        long long lbase = 0;
        if (c == 1) {
            ctr = 0;
            mxi = 1;
            mx = (int)h;
        } else if (c == 2) {
            ctr = 2;
            lbase = m;
        } else if (c == 3) {
            ctr = 3;
            lbase = 2LL * m;
            mxi = 4;
            mx = k;
        } else if (c == 4) {
            // by window width, so narrow windows take less shared memory a block
            const int b = span <= 4096 ? 0 : span <= 8192 ? 1 : 2;
            ctr = 5 + b;
            lbase = (3LL + b) * m;
            mxi = 8 + b;
            mx = (int)span;
        } else if (c >= 5) {
            ctr = c == 5 ? 11 : 13;
            lbase = (1LL + c) * m;
            mxi = ctr + 1;
            mx = (int)span;
        }
        if (c >= 4) {
            wlo[i] = lo;
            wspan[i] = (int)span;
        }
        // one atomic per class and warp: most rows share a class
        const unsigned act = __activemask();
        const unsigned grp = __match_any_sync(act, ctr);
        const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
        const int gmx = __reduce_max_sync(grp, mx);
        int pos = 0;
        if (ctr >= 0 && lane == leader) {
            pos = atomicAdd(count + ctr, __popc(grp));
            if (mxi >= 0) atomicMax(count + mxi, gmx);
        }
        pos = __shfl_sync(grp, pos, leader) + __popc(grp & ((1u << lane) - 1u));
        if (ctr >= 0) list[lbase + pos] = i;
    }
}

// Row i of C = A B for the listed rows, one warp per row: a k-way merge of the selected
// rows of B with the k merge heads in shared memory (lane l owns heads l, l+32, ...).  Each
// output column is the warp-wide minimum of the heads; its products are added in the
// order of the left row (groups of 32 in turn, lanes in order within a group) from 0.0 with
// separate multiply and add -- the arithmetic of k_spgemm.  Shared memory: 3 * KH ints per
// warp (KH >= the longest listed left row).
template <bool FILL>
__global__ void k_spgemm_warp(const int* __restrict__ rows, int nrows, int KH,
                              const int* __restrict__ arp, const int* __restrict__ aci,
                              const double* __restrict__ av, const int* __restrict__ brp,
                              const int* __restrict__ bci, const double* __restrict__ bv,
                              int* ccnt, const int* __restrict__ crp, int* cci, double* cv) {
    extern __shared__ int sm_heads[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int* pos = sm_heads + (size_t)wid * 3 * KH;
    int* end = pos + KH;
    int* cur = end + KH;
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    for (int r = blockIdx.x * (blockDim.x >> 5) + wid; r < nrows; r += nwarps) {
        const int i = rows[r];
        const int s = arp[i], k = arp[i + 1] - s;
        // lane-local minimum over the lane's own heads (t = lane, lane + 32, ...)
        int lmin = INT_MAX;
        for (int t = lane; t < k; t += 32) {
            const int j = aci[s + t];
            const int p0 = brp[j], p1 = brp[j + 1];
            pos[t] = p0;
            end[t] = p1;
            const int c = p0 < p1 ? bci[p0] : INT_MAX;
            cur[t] = c;
            lmin = min(lmin, c);
        }
        int o = FILL ? crp[i] : 0;
        const int groups = (k + 31) >> 5;
        for (;;) {
            int m = lmin;
            for (int q = 16; q > 0; q >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, q));
            if (m == INT_MAX) break;
            // groups (t / 32) that hold a head at column m: every group when there are few,
            // else only those some lane finds (only lanes whose minimum is m look)
            unsigned long long gm;
            if (groups <= 4) {
                gm = (1ull << groups) - 1ull;
            } else {
                unsigned long long mine = 0ull;
                if (lmin == m)
                    for (int t = lane, g = 0; t < k; t += 32, ++g)
                        if (cur[t] == m) mine |= 1ull << g;
                unsigned lo = (unsigned)mine, hi = (unsigned)(mine >> 32);
                for (int q = 16; q > 0; q >>= 1) lo |= __shfl_xor_sync(0xffffffffu, lo, q);
                if (groups > 32)
                    for (int q = 16; q > 0; q >>= 1) hi |= __shfl_xor_sync(0xffffffffu, hi, q);
                gm = ((unsigned long long)hi << 32) | lo;
            }
            // products in the order of the left row: groups in turn, lanes in order inside
            double sum = 0.0;
            while (gm) {
                const int g = __ffsll((long long)gm) - 1;
                gm &= gm - 1;
                const int t = (g << 5) + lane;
                const bool hit = t < k && lmin == m && cur[t] == m;
                double prod = 0.0;
                if (hit) {
                    const int p = pos[t];
                    prod = __dmul_rn(av[s + t], bv[p]);
                    pos[t] = p + 1;
                    cur[t] = p + 1 < end[t] ? bci[p + 1] : INT_MAX;
                }
                unsigned mask = __ballot_sync(0xffffffffu, hit);
                while (mask) {
                    const int l = __ffs(mask) - 1;
                    sum = __dadd_rn(sum, __shfl_sync(0xffffffffu, prod, l));
                    mask &= mask - 1;
                }
            }
            if (lmin == m) {
                lmin = INT_MAX;
                for (int t = lane; t < k; t += 32) lmin = min(lmin, cur[t]);
            }
            if (fabs(sum) > kEps * kEps) {
                if (FILL && lane == 0) {
                    cci[o] = m;
                    cv[o] = sum;
                }
                ++o;
            }
        }
        if (ccnt && lane == 0) ccnt[i] = FILL ? o - crp[i] : o;
        __syncwarp();
    }
}

// Row i of C = A B for the listed rows, one block per row, with a dense accumulator of
// all B.m columns in shared memory: the products of left entry t are added one t at a time
// (barrier between t's), so each column sums over t in row order from 0.0 with separate
// multiply and add -- the arithmetic of k_spgemm.  Survivors (|v| > eps^2) come out in
// column order from a chunked block scan, which also clears the accumulator for the next
// row.  Shared memory: B.m doubles + B.m flag bytes.
template <bool FILL>
__global__ void k_spgemm_dense(const int* __restrict__ rows, int nrows, int bcols,
                               const int* __restrict__ arp, const int* __restrict__ aci,
                               const double* __restrict__ av, const int* __restrict__ brp,
                               const int* __restrict__ bci, const double* __restrict__ bv,
                               int* ccnt, const int* __restrict__ crp, int* cci, double* cv) {
    extern __shared__ double acc[];
    unsigned char* hit = reinterpret_cast<unsigned char*>(acc + bcols);
    __shared__ int s_warp[kRowBlock / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int chunk = (bcols + blockDim.x - 1) / blockDim.x;
    const int c0 = threadIdx.x * chunk, c1 = min(bcols, c0 + chunk);
    for (int c = c0; c < c1; ++c) {
        acc[c] = 0.0;
        hit[c] = 0;
    }
    __syncthreads();
    for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
        const int i = rows[r];
        const int s = arp[i], k = arp[i + 1] - s;
        for (int t = 0; t < k; ++t) {
            const int j = aci[s + t];
            const double a = av[s + t];
            const int e1 = brp[j + 1];
            for (int e = brp[j] + threadIdx.x; e < e1; e += blockDim.x) {
                const int col = bci[e];
                acc[col] = __dadd_rn(acc[col], __dmul_rn(a, bv[e]));
                hit[col] = 1;
            }
            __syncthreads();
        }
        // survivors of this thread's column chunk
        int mine = 0;
        for (int c = c0; c < c1; ++c) mine += (hit[c] && fabs(acc[c]) > kEps * kEps) ? 1 : 0;
        // block exclusive scan of `mine`
        int incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_warp[wid] = incl;
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < nw; ++w) {
            if (w < wid) before += s_warp[w];
            total += s_warp[w];
        }
        before += incl - mine;
        if (ccnt && threadIdx.x == 0) ccnt[i] = total;
        if (FILL) {
            int o = crp[i] + before;
            for (int c = c0; c < c1; ++c)
                if (hit[c] && fabs(acc[c]) > kEps * kEps) {
                    cci[o] = c;
                    cv[o] = acc[c];
                    ++o;
                }
        }
        for (int c = c0; c < c1; ++c) {
            acc[c] = 0.0;
            hit[c] = 0;
        }
        __syncthreads();
    }
}

// Row i of C = A B for the listed rows, one block per row, with a dense accumulator over the
// row's column window [lo_i, lo_i + span_i) (the span of the selected rows of B, at most
// W columns): the arithmetic and output order of k_spgemm_dense, for right operands with
// more columns than fit in shared memory.
// The left entries are added one at a time with a block barrier between them (so every
// column sums in left-row order), which makes each step's loads the critical path: the
// block first stages the row's (a_t, row bounds of B) for up to kWinLeft entries in shared
// memory, and every thread keeps its first product of the next kWinAhead steps in flight
// in registers, so a step costs a barrier and the adds rather than a chain of dependent
// global loads.  Shared memory: W doubles + W flag bytes (rounded up to 16) + kWinLeft
// staged entries of 16 bytes.
constexpr int kWinLeft = 512;
constexpr int kWinAhead = 4;

inline size_t window_smem(int W) { return ((9 * (size_t)std::max(W, 1) + 15) & ~(size_t)15) + 16 * (size_t)kWinLeft; }

template <bool FILL>
__global__ void k_spgemm_window(const int* __restrict__ rows, int nrows, int W,
                                const int* __restrict__ wlo, const int* __restrict__ wspan,
                                const int* __restrict__ arp, const int* __restrict__ aci,
                                const double* __restrict__ av, const int* __restrict__ brp,
                                const int* __restrict__ bci, const double* __restrict__ bv,
                                int* ccnt, const int* __restrict__ crp, int* cci, double* cv) {
    extern __shared__ double acc[];
    unsigned char* hit = reinterpret_cast<unsigned char*>(acc + W);
    double* sa = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(acc) +
                                           ((9 * (size_t)W + 15) & ~(size_t)15));
    int* sb0 = reinterpret_cast<int*>(sa + kWinLeft);
    int* sb1 = sb0 + kWinLeft;
    __shared__ int s_warp[kRowBlock / 32];
    const int tid = threadIdx.x, bdim = blockDim.x;
    const int lane = tid & 31, wid = tid >> 5, nw = bdim >> 5;
    for (int c = tid; c < W; c += bdim) {
        acc[c] = 0.0;
        hit[c] = 0;
    }
    __syncthreads();
    for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
        const int i = rows[r];
        const int s = arp[i], k = arp[i + 1] - s;
        const int lo = wlo[i], span = wspan[i];
        const int kk = min(k, kWinLeft);
        for (int t = tid; t < kk; t += bdim) {
            const int j = aci[s + t];
            sa[t] = av[s + t];
            sb0[t] = brp[j];
            sb1[t] = brp[j + 1];
        }
        __syncthreads();
        // first product of staged step t for this thread: column (window-relative) and value
        int pc[kWinAhead];
        double pv[kWinAhead];
#pragma unroll
        for (int q = 0; q < kWinAhead; ++q) {
            pc[q] = -1;
            pv[q] = 0.0;
            if (q < kk) {
                const int e = sb0[q] + tid;
                if (e < sb1[q]) { pc[q] = bci[e] - lo; pv[q] = bv[e]; }
            }
        }
        for (int t0 = 0; t0 < k; t0 += kWinAhead) {
#pragma unroll
            for (int q = 0; q < kWinAhead; ++q) {
                const int t = t0 + q;
                if (t < k) {
                    double a;
                    int b0, b1, e;
                    if (t < kk) {
                        a = sa[t];
                        b0 = sb0[t];
                        b1 = sb1[t];
                        if (pc[q] >= 0) {
                            acc[pc[q]] = __dadd_rn(acc[pc[q]], __dmul_rn(a, pv[q]));
                            hit[pc[q]] = 1;
                        }
                        e = b0 + tid + bdim;          // the staged first product is done
                    } else {
                        const int j = aci[s + t];
                        a = av[s + t];
                        b0 = brp[j];
                        b1 = brp[j + 1];
                        e = b0 + tid;
                    }
                    for (; e < b1; e += bdim) {
                        const int c = bci[e] - lo;
                        acc[c] = __dadd_rn(acc[c], __dmul_rn(a, bv[e]));
                        hit[c] = 1;
                    }
                    // refill slot q with step t + kWinAhead
                    const int tn = t + kWinAhead;
                    pc[q] = -1;
                    if (tn < kk) {
                        const int en = sb0[tn] + tid;
                        if (en < sb1[tn]) { pc[q] = bci[en] - lo; pv[q] = bv[en]; }
                    }
                    __syncthreads();
                }
            }
        }
        const int chunk = (span + bdim - 1) / bdim;
        const int c0 = min(span, tid * chunk), c1 = min(span, c0 + chunk);
        int mine = 0;
        for (int c = c0; c < c1; ++c) mine += (hit[c] && fabs(acc[c]) > kEps * kEps) ? 1 : 0;
        int incl = mine;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_warp[wid] = incl;
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < nw; ++w) {
            if (w < wid) before += s_warp[w];
            total += s_warp[w];
        }
        before += incl - mine;
        if (ccnt && tid == 0) ccnt[i] = total;
        if (FILL) {
            int o = crp[i] + before;
            for (int c = c0; c < c1; ++c)
                if (hit[c] && fabs(acc[c]) > kEps * kEps) {
                    cci[o] = lo + c;
                    cv[o] = acc[c];
                    ++o;
                }
        }
        for (int c = c0; c < c1; ++c) {
            acc[c] = 0.0;
            hit[c] = 0;
        }
        __syncthreads();
    }
}

// Row i of C = A B for the listed rows, one warp per row, every output column the sum of
// its products in the order of the left row, from 0.0, with separate multiply and add (the
// arithmetic of k_spgemm), into an accumulator indexed by the column's rank among the
// row's output columns:
//   mark   every product's column in a bitmap of the row's window [lo_i, lo_i + span_i);
//          the popcounts of the words and their prefix rank the columns in increasing order
//   add    STEP = false (short right rows): the products 32 at a time in row order (left
//          entries 32 at a time, their right rows flattened: product q belongs to the last
//          left entry whose exclusive prefix is <= q, found by a binary search over the lanes
//          with shuffles).  Lanes whose products share a column form a group (match.any);
//          its lowest lane adds the group's products to acc[rank] in lane order, which is
//          row order, and a warp barrier separates one 32 from the next.
//          STEP = true (longer right rows): one left entry at a time (seq_add_steps)
//   write  the sums with |v| > eps^2 in rank (= column) order
// A row with more output columns than the accumulator holds (CMAX) is added in passes over
// rank ranges.  Shared memory a warp: CMAX doubles + CMAX u16 columns + 2 ints a bitmap word.
__host__ __device__ constexpr size_t seq_warp_bytes(int cmax, int nwords) {
    return ((size_t)cmax * 10 + (size_t)nwords * 8 + 15) & ~(size_t)15;
}

__device__ __forceinline__ int seq_rank(const unsigned* bmp, const int* wpre, int c) {
    const int w = c >> 5;
    return wpre[w] + __popc(bmp[w] & ((1u << (c & 31)) - 1u));
}

// Lane holding left entry pos of the group for flattened product q (excl: lane's prefix).
__device__ __forceinline__ int seq_owner(int excl, int q) {
    int pos = 0;
#pragma unroll
    for (int st = 16; st >= 1; st >>= 1) {
        const int ex = __shfl_sync(0xffffffffu, excl, pos + st);
        if (ex <= q) pos += st;
    }
    return pos;
}

// Left entries g .. g+31 of row (s, k): lane q's right row bounds and value, its exclusive
// product prefix; returns the group's product count.
__device__ __forceinline__ int seq_group(int s, int k, int g, int lane, const int* __restrict__ aci,
                                         const double* __restrict__ av, const int* __restrict__ brp,
                                         int& b0, int& len, int& excl, double& a) {
    len = 0;
    b0 = 0;
    a = 0.0;
    if (g + lane < k) {
        const int j = aci[s + g + lane];
        b0 = brp[j];
        len = brp[j + 1] - b0;
        a = av[s + g + lane];
    }
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    excl = incl - len;
    return __shfl_sync(0xffffffffu, incl, 31);
}

constexpr int kSeqBatch = 4;            // 32-product batches loaded together
constexpr int kSeqAhead = 4;            // STEP: left entries whose first 32 products are loaded ahead

// STEP: add left entries 0 .. gc-1 of the group one at a time, lanes over the entry's right
// row (its columns are distinct, so no two lanes meet), the first 32 products of the next
// kSeqAhead entries already in registers.
__device__ __forceinline__ void seq_add_steps(int gc, int lane, int b0, int len, double a, int lo, int c0,
                                              int cn, const int* __restrict__ bci,
                                              const double* __restrict__ bv, const unsigned* bmp,
                                              const int* wpre, double* acc) {
    int pc[kSeqAhead];
    double pv[kSeqAhead];
#pragma unroll
    for (int d = 0; d < kSeqAhead; ++d) {
        pc[d] = -1;
        pv[d] = 0.0;
        if (d < gc) {
            const int L = __shfl_sync(0xffffffffu, len, d), B = __shfl_sync(0xffffffffu, b0, d);
            if (lane < L) {
                pc[d] = bci[B + lane];
                pv[d] = bv[B + lane];
            }
        }
    }
    for (int t0 = 0; t0 < gc; t0 += kSeqAhead) {
#pragma unroll
        for (int d = 0; d < kSeqAhead; ++d) {
            const int tt = t0 + d;
            if (tt < gc) {
                const double A = __shfl_sync(0xffffffffu, a, tt);
                const int L = __shfl_sync(0xffffffffu, len, tt), B = __shfl_sync(0xffffffffu, b0, tt);
                if (pc[d] >= 0) {
                    const int r = seq_rank(bmp, wpre, pc[d] - lo) - c0;
                    if ((unsigned)r < (unsigned)cn) acc[r] = __dadd_rn(acc[r], __dmul_rn(A, pv[d]));
                }
                for (int jj = lane + 32; jj < L; jj += 32) {
                    const int r = seq_rank(bmp, wpre, bci[B + jj] - lo) - c0;
                    if ((unsigned)r < (unsigned)cn) acc[r] = __dadd_rn(acc[r], __dmul_rn(A, bv[B + jj]));
                }
                __syncwarp();
                const int tn = tt + kSeqAhead;
                pc[d] = -1;
                if (tn < gc) {
                    const int Ln = __shfl_sync(0xffffffffu, len, tn), Bn = __shfl_sync(0xffffffffu, b0, tn);
                    if (lane < Ln) {
                        pc[d] = bci[Bn + lane];
                        pv[d] = bv[Bn + lane];
                    }
                }
            }
        }
    }
}

template <bool FILL, int CMAX, bool STEP>
__global__ void __launch_bounds__(32 * kSeqWarps, 3)
k_spgemm_seq(const int* __restrict__ rows, int nrows, int NW, const int* __restrict__ wlo,
             const int* __restrict__ wspan, const int* __restrict__ arp, const int* __restrict__ aci,
             const double* __restrict__ av, const int* __restrict__ brp, const int* __restrict__ bci,
             const double* __restrict__ bv, int* ccnt, const int* __restrict__ crp, int* cci, double* cv) {
    extern __shared__ __align__(16) unsigned char sm_seq[];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* base = sm_seq + (size_t)wid * seq_warp_bytes(CMAX, NW);
    double* acc = reinterpret_cast<double*>(base);                     // CMAX sums
    unsigned* bmp = reinterpret_cast<unsigned*>(acc + CMAX);           // NW bitmap words
    int* wpre = reinterpret_cast<int*>(bmp + NW);                      // NW ranks of the words
    unsigned short* colof = reinterpret_cast<unsigned short*>(wpre + NW);   // CMAX columns
    const unsigned lt = (1u << lane) - 1u;
    for (int q = lane; q < NW; q += 32) bmp[q] = 0u;
    __syncwarp();
    const int nwarps = gridDim.x * kSeqWarps;
    for (int rr = blockIdx.x * kSeqWarps + wid; rr < nrows; rr += nwarps) {
        const int i = rows[rr];
        const int s = arp[i], k = arp[i + 1] - s;
        const int lo = wlo[i], nwords = (wspan[i] + 31) >> 5;
        // mark; the lanes of a warp that mark one bitmap word merge their bits first
        for (int g = 0; g < k; g += 32) {
            int b0, len, excl;
            double a;
            const int gu = seq_group(s, k, g, lane, aci, av, brp, b0, len, excl, a);
            for (int qb = 0; qb < gu; qb += kSeqBatch * 32) {
                int ca[kSeqBatch];
#pragma unroll
                for (int d = 0; d < kSeqBatch; ++d) {
                    const int q = qb + d * 32 + lane;
                    const int pos = seq_owner(excl, q);
                    const int e = __shfl_sync(0xffffffffu, b0, pos) + q - __shfl_sync(0xffffffffu, excl, pos);
                    ca[d] = q < gu ? bci[e] : -1;
                }
#pragma unroll
                for (int d = 0; d < kSeqBatch; ++d) {
                    const bool ok = ca[d] >= 0;
                    const int c = ca[d] - lo;
                    const int w = ok ? c >> 5 : -1;
                    const unsigned grp = __match_any_sync(0xffffffffu, w);
                    const unsigned bits = __reduce_or_sync(grp, ok ? 1u << (c & 31) : 0u);
                    if (ok && lane == __ffs(grp) - 1) atomicOr(&bmp[w], bits);
                }
            }
        }
        __syncwarp();
        int ncols = 0;
        for (int wb = 0; wb < nwords; wb += 32) {
            const int w = wb + lane;
            const int x = w < nwords ? __popc(bmp[w]) : 0;
            int in = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, in, o);
                if (lane >= o) in += y;
            }
            if (w < nwords) wpre[w] = ncols + in - x;
            ncols += __shfl_sync(0xffffffffu, in, 31);
        }
        __syncwarp();
        int out = FILL ? crp[i] : 0, kept = 0;
        for (int c0 = 0; c0 < ncols; c0 += CMAX) {
            const int cn = min(CMAX, ncols - c0);
            for (int q = lane; q < cn; q += 32) acc[q] = 0.0;
            for (int w = lane; w < nwords; w += 32) {       // columns of ranks [c0, c0 + cn)
                unsigned m = bmp[w];
                int rk = wpre[w];
                if (rk >= c0 + cn || rk + __popc(m) <= c0) continue;
                while (m) {
                    const int b = __ffs(m) - 1;
                    m &= m - 1u;
                    if (rk >= c0 && rk < c0 + cn) colof[rk - c0] = (unsigned short)(w * 32 + b);
                    ++rk;
                }
            }
            __syncwarp();
            for (int g = 0; g < k; g += 32) {
                int b0, len, excl;
                double a;
                const int gu = seq_group(s, k, g, lane, aci, av, brp, b0, len, excl, a);
                if constexpr (STEP) {
                    seq_add_steps(min(32, k - g), lane, b0, len, a, lo, c0, cn, bci, bv, bmp, wpre, acc);
                } else {
                    for (int qb = 0; qb < gu; qb += kSeqBatch * 32) {
                        int ca[kSeqBatch];
                        double pa[kSeqBatch];
#pragma unroll
                        for (int d = 0; d < kSeqBatch; ++d) {
                            const int q = qb + d * 32 + lane;
                            const int pos = seq_owner(excl, q);
                            const int e = __shfl_sync(0xffffffffu, b0, pos) + q - __shfl_sync(0xffffffffu, excl, pos);
                            const double at = __shfl_sync(0xffffffffu, a, pos);
                            ca[d] = -1;
                            pa[d] = 0.0;
                            if (q < gu) {
                                ca[d] = bci[e];
                                pa[d] = __dmul_rn(at, bv[e]);
                            }
                        }
#pragma unroll
                        for (int d = 0; d < kSeqBatch; ++d) {
                            if (qb + d * 32 < gu) {                     // warp-uniform
                                const int r = ca[d] >= 0 ? seq_rank(bmp, wpre, ca[d] - lo) - c0 : -1;
                                const bool in = (unsigned)r < (unsigned)cn;
                                const unsigned grp = __match_any_sync(0xffffffffu, in ? r : -1 - lane);
                                if (in) {
                                    const int leader = __ffs(grp) - 1;
                                    double sum = lane == leader ? acc[r] : 0.0;
                                    unsigned rest = grp;
                                    while (rest) {                      // the group in lane order
                                        const int l = __ffs(rest) - 1;
                                        rest &= rest - 1u;
                                        const double v = __shfl_sync(grp, pa[d], l);
                                        if (lane == leader) sum = __dadd_rn(sum, v);
                                    }
                                    if (lane == leader) acc[r] = sum;
                                }
                                __syncwarp();
                            }
                        }
                    }
                }
            }
            for (int qb = 0; qb < cn; qb += 32) {
                const int q = qb + lane;
                const double v = q < cn ? acc[q] : 0.0;
                const bool keep = q < cn && fabs(v) > kEps * kEps;
                const unsigned bal = __ballot_sync(0xffffffffu, keep);
                if (FILL && keep) {
                    const int o = out + __popc(bal & lt);
                    cci[o] = lo + colof[q];
                    cv[o] = v;
                }
                out += __popc(bal);
                kept += __popc(bal);
            }
            __syncwarp();
        }
        if (ccnt && lane == 0) ccnt[i] = kept;
        for (int w = lane; w < nwords; w += 32) bmp[w] = 0u;
        __syncwarp();
    }
}

// Row i of C = A B for the listed rows, one block per row.  The products of left entry t
// are added into a shared hash table (slot per output column) one t at a time, with a
// barrier between t's, so every column's sum runs over t in row order from 0.0 with
// separate multiply and add -- the same arithmetic as k_spgemm.  Survivors (|v| > eps^2)
// are then sorted by column.  Shared memory: S ints + S doubles + S u64 (S = table size).
template <bool FILL>
__global__ void k_spgemm_rows(const int* __restrict__ rows, int nrows, int S,
                              const int* __restrict__ arp, const int* __restrict__ aci,
                              const double* __restrict__ av, const int* __restrict__ brp,
                              const int* __restrict__ bci, const double* __restrict__ bv,
                              int* ccnt, const int* __restrict__ crp, int* cci, double* cv) {
    extern __shared__ unsigned long long sm_keys[];
    double* vals = reinterpret_cast<double*>(sm_keys + S);
    int* cols = reinterpret_cast<int*>(vals + S);
    __shared__ int s_n;
    for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
        const int i = rows[r];
        const int s = arp[i], k = arp[i + 1] - s;
        for (int t = threadIdx.x; t < S; t += blockDim.x) {
            cols[t] = -1;
            vals[t] = 0.0;
        }
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
        for (int t = 0; t < k; ++t) {
            const int j = aci[s + t];
            const double a = av[s + t];
            const int e1 = brp[j + 1];
            for (int e = brp[j] + threadIdx.x; e < e1; e += blockDim.x) {
                const int col = bci[e];
                unsigned h = ((unsigned)col * 2654435761u) & (unsigned)(S - 1);
                for (;;) {
                    const int old = atomicCAS(&cols[h], -1, col);
                    if (old == -1 || old == col) break;
                    h = (h + 1) & (unsigned)(S - 1);
                }
                vals[h] = __dadd_rn(vals[h], __dmul_rn(a, bv[e]));
            }
            __syncthreads();
        }
        // compact the survivors (any order), then sort them by column
        for (int t = threadIdx.x; t < S; t += blockDim.x)
            if (cols[t] >= 0 && fabs(vals[t]) > kEps * kEps)
                sm_keys[atomicAdd(&s_n, 1)] = ((unsigned long long)(unsigned)cols[t] << 32) | (unsigned)t;
        __syncthreads();
        const int cnt = s_n;
        if (ccnt && threadIdx.x == 0) ccnt[i] = cnt;
        if (FILL) {
            const int N = pow2_at_least(cnt > 0 ? cnt : 1);
            for (int t = cnt + threadIdx.x; t < N; t += blockDim.x) sm_keys[t] = kNoKey;
            block_bitonic(sm_keys, N);
            const int o = crp[i];
            for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
                const unsigned long long key = sm_keys[t];
                cci[o + t] = (int)(key >> 32);
                cv[o + t] = vals[key & 0xffffffffu];
            }
        }
        __syncthreads();
    }
}

// Sort the listed rows of a transpose (distinct columns per row) by column, one block per
// row; the values move with their columns.  Shared memory: pow2(len) keys + len doubles.
__global__ void k_t_sort_rows(const int* __restrict__ rows, int nrows, const int* __restrict__ trp,
                              int* tci, double* tv) {
    extern __shared__ unsigned long long sm_keys[];
    for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
        const int row = rows[r];
        const int s = trp[row], len = trp[row + 1] - s;
        const int N = pow2_at_least(len);
        double* val = reinterpret_cast<double*>(sm_keys + N);
        for (int t = threadIdx.x; t < N; t += blockDim.x) {
            if (t < len) {
                sm_keys[t] = ((unsigned long long)(unsigned)tci[s + t] << 32) | (unsigned)t;
                val[t] = tv[s + t];
            } else {
                sm_keys[t] = kNoKey;
            }
        }
        block_bitonic(sm_keys, N);
        for (int t = threadIdx.x; t < len; t += blockDim.x) {
            const unsigned long long key = sm_keys[t];
            tci[s + t] = (int)(key >> 32);
            tv[s + t] = val[key & 0xffffffffu];
        }
        __syncthreads();
    }
}

__global__ void k_inv_diag(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ v, double* dinv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) { d = v[k]; break; }
        dinv[i] = (fabs(d) > kEps) ? 1.0 / d : 0.0;     // amg.cpp:192-195
    }
}

__global__ void k_d2f(const double* __restrict__ a, float* b, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// ------------------------------------------------------------- coarsest level
// Dense Gaussian elimination with partial pivoting (amg.cpp:260-291), one block, on the
// n x n matrix M (row-major).  Stores the multipliers below the diagonal, the pivot row
// of each column and whether the column was skipped (|pivot| < 1e-14).
__global__ void k_dense_factor(int n, double* M, int* piv, int* skip) {
    __shared__ int sp;
    for (int col = 0; col < n; ++col) {
        if (threadIdx.x == 0) {
            int p = col;
            for (int r = col + 1; r < n; ++r)
                if (fabs(M[(size_t)r * n + col]) > fabs(M[(size_t)p * n + col])) p = r;
            piv[col] = p;
            sp = p;
        }
        __syncthreads();
        const int p = sp;
        // columns < col hold multipliers that belong to the row position at their step
        if (p != col)
            for (int c = col + threadIdx.x; c < n; c += blockDim.x) {
                double t = M[(size_t)col * n + c];
                M[(size_t)col * n + c] = M[(size_t)p * n + c];
                M[(size_t)p * n + c] = t;
            }
        __syncthreads();
        const double d = M[(size_t)col * n + col];
        const bool sk = fabs(d) < 1e-14;
        if (threadIdx.x == 0) skip[col] = sk;
        if (!sk) {
            const double inv = 1.0 / d;
            for (int r = col + 1 + threadIdx.x; r < n; r += blockDim.x) {
                double f = __dmul_rn(M[(size_t)r * n + col], inv);
                for (int c = col + 1; c < n; ++c)
                    M[(size_t)r * n + c] = __dsub_rn(M[(size_t)r * n + c], __dmul_rn(f, M[(size_t)col * n + c]));
                M[(size_t)r * n + col] = f;       // multiplier (the reference's entry becomes 0)
            }
        }
        __syncthreads();
    }
}

// x = A^-1 b with the stored factors, one warp, the reference's operation order.
template <typename T>
__global__ void k_dense_solve(int n, const double* __restrict__ M, const int* __restrict__ piv,
                              const int* __restrict__ skip, const T* __restrict__ b, T* x,
                              double* work, const int* gate) {
    if (gate && *(volatile const int*)gate) return;
    double* y = work;
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = (double)b[i];
    __syncwarp();
    for (int col = 0; col < n; ++col) {
        const int p = piv[col];
        if (p != col && threadIdx.x == 0) { double t = y[col]; y[col] = y[p]; y[p] = t; }
        __syncwarp();
        if (!skip[col]) {
            const double yc = y[col];
            for (int r = col + 1 + threadIdx.x; r < n; r += blockDim.x)
                y[r] = __dsub_rn(y[r], __dmul_rn(M[(size_t)r * n + col], yc));
        }
        __syncwarp();
    }
    if (threadIdx.x == 0) {
        for (int i = n - 1; i >= 0; --i) {
            double s = y[i];
            for (int j = i + 1; j < n; ++j) s = __dsub_rn(s, __dmul_rn(M[(size_t)i * n + j], y[n + j]));
            double d = M[(size_t)i * n + i];
            y[n + i] = (fabs(d) > 1e-14) ? s / d : 0.0;
        }
    }
    __syncwarp();
    for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = (T)y[n + i];
}

// Columns of the inverse, one warp per unit right-hand side e_k: Minv[r][k].
__global__ void k_dense_inverse(int n, const double* __restrict__ M, const int* __restrict__ piv,
                                const int* __restrict__ skip, double* work, double* Minv) {
    const int k = blockIdx.x;
    double* y = work + (size_t)k * 2 * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) y[i] = (i == k) ? 1.0 : 0.0;
    __syncwarp();
    for (int col = 0; col < n; ++col) {
        const int p = piv[col];
        if (p != col && threadIdx.x == 0) { double t = y[col]; y[col] = y[p]; y[p] = t; }
        __syncwarp();
        if (!skip[col]) {
            const double yc = y[col];
            for (int r = col + 1 + threadIdx.x; r < n; r += blockDim.x)
                y[r] = __dsub_rn(y[r], __dmul_rn(M[(size_t)r * n + col], yc));
        }
        __syncwarp();
    }
    if (threadIdx.x == 0) {
        for (int i = n - 1; i >= 0; --i) {
            double t = y[i];
            for (int j = i + 1; j < n; ++j) t = __dsub_rn(t, __dmul_rn(M[(size_t)i * n + j], y[n + j]));
            double d = M[(size_t)i * n + i];
            y[n + i] = (fabs(d) > 1e-14) ? t / d : 0.0;
        }
    }
    __syncwarp();
    for (int i = threadIdx.x; i < n; i += blockDim.x) Minv[(size_t)i * n + k] = y[n + i];
}

// Explicit inverse applied as a dense matrix-vector product (large coarsest levels); the
// FP32 V-cycle reads an FP32 copy of the inverse (half the bytes; it fits L2).
// FP32: a block per row, each thread four columns' loads in flight at a time (a warp per
// row left each warp ~140 dependent steps along a 4,592-column row).
__global__ void __launch_bounds__(256) k_dense_gemv_rows(int n, const float* __restrict__ Minv,
                                                         const float* __restrict__ b, float* x, const int* gate) {
    __shared__ double part[8];
    if (gate && *(volatile const int*)gate) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int r = blockIdx.x; r < n; r += gridDim.x) {
        const float* row = Minv + (size_t)r * n;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int c = threadIdx.x;
        for (; c + 768 < n; c += 1024) {
            const float m0 = row[c], m1 = row[c + 256], m2 = row[c + 512], m3 = row[c + 768];
            const float b0 = b[c], b1 = b[c + 256], b2 = b[c + 512], b3 = b[c + 768];
            s0 += (double)m0 * (double)b0;
            s1 += (double)m1 * (double)b1;
            s2 += (double)m2 * (double)b2;
            s3 += (double)m3 * (double)b3;
        }
        for (; c < n; c += 256) s0 += (double)row[c] * (double)b[c];
        double s = warp_sum((s0 + s1) + (s2 + s3));
        if (lane == 0) part[wid] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < 8; ++w) t += part[w];
            x[r] = (float)t;
        }
        __syncthreads();
    }
}

template <typename T, typename TM>
__global__ void k_dense_gemv(int n, const TM* __restrict__ Minv, const T* __restrict__ b, T* x,
                             const int* gate) {
    if (gate && *(volatile const int*)gate) return;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = warp; r < n; r += nw) {
        double s = 0.0;
        for (int c = lane; c < n; c += 32) s += (double)Minv[(size_t)r * n + c] * (double)b[c];
        s = warp_sum(s);
        if (lane == 0) x[r] = (T)s;
    }
}

// one warp per row (the coarsest operators are dense: rows of thousands of entries)
__global__ void k_csr_to_dense(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                               const double* __restrict__ v, double* M) {
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw)
        for (int k = rp[i] + lane; k < rp[i + 1]; k += 32) M[(size_t)i * n + ci[k]] = v[k];
}

// ------------------------------------------------------------ V-cycle operators
template <typename T>
struct LevelVecs {
    T* b;     // right-hand side on this level
    T* x;     // iterate
    T* x2;    // second buffer for Jacobi sweeps
    T* r;     // residual
    const T* dinv;
};

// x_new = x + (w dinv) (b - A x)        (amg.cpp:250-252)
template <typename T>
struct EpiSmooth {
    const T* b;
    const T* x;
    T* xn;
    const T* dinv;
    T omega;
    HAMLSS_NO_LOAD
    __device__ __forceinline__ void prefetch(int r0, int r1) const {
        l2_prefetch_rows(b, r0, r1);
        l2_prefetch_rows(x, r0, r1);
        l2_prefetch_rows(dinv, r0, r1);
    }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&)[NV]) const {
        if constexpr (sizeof(T) == 8) {
            double t = __dmul_rn((double)omega, (double)dinv[i]);
            xn[i] = __dadd_rn((double)x[i], __dmul_rn(t, __dsub_rn((double)b[i], ax)));
        } else {
            xn[i] = (T)((double)x[i] + (double)(omega * dinv[i]) * ((double)b[i] - ax));
        }
    }
    // the same update with b[i], x[i], dinv[i] loaded ahead (bulk-copy SpMV)
    struct Pre {
        T b, x, d;
    };
    __device__ __forceinline__ Pre pre(int i) const { return Pre{b[i], x[i], dinv[i]}; }
    __device__ __forceinline__ T value(double ax, const Pre& p) const {
        if constexpr (sizeof(T) == 8) {
            double t = __dmul_rn((double)omega, (double)p.d);
            return __dadd_rn((double)p.x, __dmul_rn(t, __dsub_rn((double)p.b, ax)));
        } else {
            return (T)((double)p.x + (double)(omega * p.d) * ((double)p.b - ax));
        }
    }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&)[NV], const Pre& p) const {
        xn[i] = value(ax, p);
    }
};

// last post-smoothing sweep on level 0 inside PCG: also r.z for the CG scalar
template <typename T>
struct EpiSmoothDot {
    EpiSmooth<T> s;
    HAMLSS_NO_LOAD
    __device__ __forceinline__ void prefetch(int r0, int r1) const { s.prefetch(r0, r1); }
    using Pre = typename EpiSmooth<T>::Pre;
    __device__ __forceinline__ Pre pre(int i) const { return s.pre(i); }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV], const Pre& p) const {
        const T xv = s.value(ax, p);
        s.xn[i] = xv;
        acc[0] += (double)p.b * (double)xv;
    }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        s(i, ax, acc);
        acc[0] += (double)s.b[i] * (double)s.xn[i];
    }
};

// r = b - A x
template <typename T>
struct EpiResid {
    const T* b;
    T* r;
    HAMLSS_NO_LOAD
    __device__ __forceinline__ void prefetch(int r0, int r1) const { l2_prefetch_rows(b, r0, r1); }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&)[NV]) const {
        if constexpr (sizeof(T) == 8) r[i] = __dsub_rn((double)b[i], ax);
        else r[i] = (T)((double)b[i] - ax);
    }
    struct Pre {
        T b;
    };
    __device__ __forceinline__ Pre pre(int i) const { return Pre{b[i]}; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&)[NV], const Pre& p) const {
        if constexpr (sizeof(T) == 8) r[i] = __dsub_rn((double)p.b, ax);
        else r[i] = (T)((double)p.b - ax);
    }
};

// b_c = R r ; first coarse pre-smoothing sweep from x_c = 0: x_c = (w dinv_c) b_c
template <typename T>
struct EpiRestrict {
    T* bc;
    T* xc;
    const T* dinvc;
    T omega;
    bool smooth;     // false when the coarse level is the direct-solve level
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&)[NV]) const {
        T bi = (T)ax;
        bc[i] = bi;
        if (smooth) {
            if constexpr (sizeof(T) == 8) xc[i] = __dmul_rn(__dmul_rn((double)omega, (double)dinvc[i]), (double)bi);
            else xc[i] = (T)((double)(omega * dinvc[i]) * (double)bi);
        }
    }
    struct Pre {
        T d;
    };
    __device__ __forceinline__ Pre pre(int i) const { return Pre{smooth ? dinvc[i] : T(0)}; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&)[NV], const Pre& p) const {
        T bi = (T)ax;
        bc[i] = bi;
        if (smooth) {
            if constexpr (sizeof(T) == 8) xc[i] = __dmul_rn(__dmul_rn((double)omega, (double)p.d), (double)bi);
            else xc[i] = (T)((double)(omega * p.d) * (double)bi);
        }
    }
};

// x += P e_c
template <typename T>
struct EpiProlong {
    T* x;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&)[NV]) const {
        if constexpr (sizeof(T) == 8) x[i] = __dadd_rn((double)x[i], ax);
        else x[i] = (T)((double)x[i] + ax);
    }
};

// x_out = x_in + P e (prolongation and correction into the other Jacobi buffer)
template <typename T>
struct EpiProlongTo {
    const T* xin;
    T* xout;
    HAMLSS_NO_LOAD
    __device__ __forceinline__ void prefetch(int r0, int r1) const { l2_prefetch_rows(xin, r0, r1); }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&)[NV]) const {
        if constexpr (sizeof(T) == 8) xout[i] = __dadd_rn((double)xin[i], ax);
        else xout[i] = (T)((double)xin[i] + ax);
    }
    struct Pre {
        T x;
    };
    __device__ __forceinline__ Pre pre(int i) const { return Pre{xin[i]}; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&)[NV], const Pre& p) const {
        if constexpr (sizeof(T) == 8) xout[i] = __dadd_rn((double)p.x, ax);
        else xout[i] = (T)((double)p.x + ax);
    }
};

template <typename T>
struct BodyFirstSmooth {
    const T* b;
    T* x;
    const T* dinv;
    T omega;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const {
        if constexpr (sizeof(T) == 8) x[i] = __dmul_rn(__dmul_rn((double)omega, (double)dinv[i]), (double)b[i]);
        else x[i] = (T)((double)(omega * dinv[i]) * (double)b[i]);
    }
};

template <typename T>
struct BodyCopy {
    const T* a;
    T* b;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const { b[i] = a[i]; }
};

}  // namespace

// ----------------------------------------------------------------- the object
struct AmgLevel {
    DCsr A;          // level >= 1 (level 0 uses the user's matrix)
    DCsr P, R;
    DBuf<double> dinv;
    DBuf<float> dinv32;
    DBuf<double> b, x, x2, r;
    DBuf<float> b32, x32, x232, r32;
    int n = 0;
};

struct AmgPrec : Prec {
    hamlss_mat* A0 = nullptr;
    std::vector<std::unique_ptr<AmgLevel>> lev;
    double omega = 0.67;
    int pre = 2, post = 2;
    // coarsest dense data
    int nc = 0;
    bool coarse_inverse = false;
    DBuf<double> Md, Minv, cwork;
    DBuf<float> Minv32;                 // FP32 copy of Minv for the FP32 V-cycle
    DBuf<int> piv, skip;
    bool f32_ready = false;

    int levels() const { return (int)lev.size(); }

    Csr<double> Aview64(int l) const { return l == 0 ? A0->A.f64() : lev[l]->A.f64(); }
    Csr<float> Aview32(Ctx& ctx, int l) const {
        return l == 0 ? A0->A.f32(ctx.lane.stream) : lev[l]->A.f32();
    }

    template <typename T>
    LevelVecs<T> vecs(int l);

    template <typename T>
    Csr<T> Amat(Ctx& ctx, int l);
    template <typename T>
    Csr<T> Pmat(int l);
    template <typename T>
    Csr<T> Rmat(int l);

    template <typename T>
    void coarse_solve(Ctx& ctx, const Lane& L, const T* b, T* x, const int* gate) {
        if (coarse_inverse) {
            ProfScope ps(L, "amg_coarse", (double)sizeof(T) * nc * nc);
            const int g = std::max(1, std::min(ceil_div(nc, 8), ctx.sm_count * 4));
            if constexpr (sizeof(T) == 4)
                k_dense_gemv_rows<<<std::min(nc, ctx.sm_count * 8), 256, 0, L.stream>>>(nc, Minv32.p, b, x, gate);
            else
                k_dense_gemv<T, double><<<g, 256, 0, L.stream>>>(nc, Minv.p, b, x, gate);
        } else {
            ProfScope ps(L, "amg_coarse", 8.0 * nc * nc);
            k_dense_solve<T><<<1, 32, 0, L.stream>>>(nc, Md.p, piv.p, skip.p, b, x, cwork.p, gate);
        }
        HAMLSS_LAUNCH_CHECK();
    }

    // One V-cycle: z = M^-1 r (z starts at 0).  rz: when non-null, the last level-0 sweep
    // also accumulates r.z and hands the sum to `fin`.
    template <typename T, typename Fin>
    void vcycle(Ctx& ctx, const Lane& L, const T* rhs0, T* z, const int* gate, bool with_dot,
                const Fin& fin) {
        const int sm = ctx.sm_count;
        const int nl = levels();
        const T om = (T)omega;
        const double w = sizeof(T);
        if (nl == 1) {
            coarse_solve<T>(ctx, L, rhs0, z, gate);
            return;
        }
        // Jacobi sweeps alternate between a level's x and x2 buffers (no copies); cur[l] is
        // the buffer that holds level l's iterate.  With the usual pre = post = 2 every level
        // ends in its own x, else one copy puts level 0's result in z.
        T* cur[kMaxLevels];
        for (int l = 0; l < nl - 1; ++l) {
            LevelVecs<T> V = vecs<T>(l);
            const T* b = l == 0 ? rhs0 : V.b;
            T* x = l == 0 ? z : V.x;
            const int n = lev[l]->n;
            Csr<T> A = Amat<T>(ctx, l);
            int done_sweeps = 0;
            if (pre >= 1) {
                if (l == 0) launch_vec<0>(sm, L, n, BodyFirstSmooth<T>{b, x, V.dinv, om}, NoFin{}, gate,
                                          "amg_smooth", 3.0 * w * n);
                done_sweeps = 1;   // levels >= 1 had it fused into the restriction
            } else if (l == 0) {
                HAMLSS_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * n, L.stream));
            }
            T* c = x;
            for (int s = done_sweeps; s < pre; ++s) {
                T* o = (c == x) ? V.x2 : x;
                launch_spmv<T, 0>(sm, L, A, XVec<T>{c}, EpiSmooth<T>{b, c, o, V.dinv, om}, NoFin{}, gate,
                                  "amg_smooth", 4.0 * w * n);
                c = o;
            }
            cur[l] = c;
            launch_spmv<T, 0>(sm, L, A, XVec<T>{c}, EpiResid<T>{b, V.r}, NoFin{}, gate, "amg_resid",
                              3.0 * w * n);
            LevelVecs<T> C = vecs<T>(l + 1);
            const bool coarse_smooth = (l + 1 < nl - 1) && pre >= 1;
            launch_spmv<T, 0>(sm, L, Rmat<T>(l), XVec<T>{V.r}, EpiRestrict<T>{C.b, C.x, C.dinv, om, coarse_smooth},
                              NoFin{}, gate, "amg_restrict", w * n + (coarse_smooth ? 3.0 : 1.0) * w * lev[l + 1]->n);
            if (!coarse_smooth && l + 1 < nl - 1)
                HAMLSS_CUDA(cudaMemsetAsync(C.x, 0, sizeof(T) * lev[l + 1]->n, L.stream));
        }
        {
            LevelVecs<T> C = vecs<T>(nl - 1);
            coarse_solve<T>(ctx, L, C.b, C.x, gate);
            cur[nl - 1] = C.x;
        }
        for (int l = nl - 2; l >= 0; --l) {
            LevelVecs<T> V = vecs<T>(l);
            const T* b = l == 0 ? rhs0 : V.b;
            T* x = l == 0 ? z : V.x;
            const int n = lev[l]->n;
            Csr<T> A = Amat<T>(ctx, l);
            T* c = cur[l];
            T* o = (c == x) ? V.x2 : x;
            // prolongation + correction into the other buffer: o = c + P e
            launch_spmv<T, 0>(sm, L, Pmat<T>(l), XVec<T>{cur[l + 1]}, EpiProlongTo<T>{c, o}, NoFin{}, gate,
                              "amg_prolong", w * lev[l + 1]->n + 2.0 * w * n);
            c = o;
            for (int s = 0; s < post; ++s) {
                const bool last = (l == 0 && s == post - 1);
                o = (c == x) ? V.x2 : x;
                if (last && with_dot) {
                    launch_spmv<T, 1>(sm, L, A, XVec<T>{c}, EpiSmoothDot<T>{EpiSmooth<T>{b, c, o, V.dinv, om}},
                                      fin, gate, "amg_smooth", 4.0 * w * n);
                } else {
                    launch_spmv<T, 0>(sm, L, A, XVec<T>{c}, EpiSmooth<T>{b, c, o, V.dinv, om}, NoFin{}, gate,
                                      "amg_smooth", 4.0 * w * n);
                }
                c = o;
            }
            if (c != x && l == 0)
                launch_vec<0>(sm, L, n, BodyCopy<T>{c, x}, NoFin{}, gate, "vec", 2.0 * w * n);
            cur[l] = c;
        }
    }

    void apply(Ctx& ctx, const Lane& L, const double* r, double* z, const int* gate) override {
        vcycle<double>(ctx, L, r, z, gate, false, NoFin{});
    }
    void prepare32(Ctx& ctx) override;
    void apply32(Ctx& ctx, const Lane& L, const float* r, float* z, const int* gate) override {
        prepare32(ctx);
        vcycle<float>(ctx, L, r, z, gate, false, NoFin{});
    }
    bool has32() const override { return true; }
};

template <>
LevelVecs<double> AmgPrec::vecs<double>(int l) {
    AmgLevel& v = *lev[l];
    return LevelVecs<double>{v.b.p, v.x.p, v.x2.p, v.r.p, v.dinv.p};
}
template <>
LevelVecs<float> AmgPrec::vecs<float>(int l) {
    AmgLevel& v = *lev[l];
    return LevelVecs<float>{v.b32.p, v.x32.p, v.x232.p, v.r32.p, v.dinv32.p};
}
template <>
Csr<double> AmgPrec::Amat<double>(Ctx&, int l) { return Aview64(l); }
template <>
Csr<float> AmgPrec::Amat<float>(Ctx& ctx, int l) { return Aview32(ctx, l); }
template <>
Csr<double> AmgPrec::Pmat<double>(int l) { return lev[l]->P.f64(); }
template <>
Csr<float> AmgPrec::Pmat<float>(int l) { return lev[l]->P.f32(); }
template <>
Csr<double> AmgPrec::Rmat<double>(int l) { return lev[l]->R.f64(); }
template <>
Csr<float> AmgPrec::Rmat<float>(int l) { return lev[l]->R.f32(); }

void AmgPrec::prepare32(Ctx& ctx) {
    if (f32_ready) return;
    cudaStream_t s = ctx.lane.stream;
    AllocScope scope(s);                 // FP32 copies from the stream-ordered pool
    auto conv = [&](const DBuf<double>& a, DBuf<float>& b, long long n) {
        b.ensure(n);
        if (n) k_d2f<<<grid_for(ctx, n), 256, 0, s>>>(a.p, b.p, n);
    };
    for (int l = 0; l < levels(); ++l) {
        AmgLevel& L = *lev[l];
        if (l > 0) conv(L.A.v, L.A.v32, L.A.nnz);
        if (L.P.nnz) { conv(L.P.v, L.P.v32, L.P.nnz); conv(L.R.v, L.R.v32, L.R.nnz); }
        conv(L.dinv, L.dinv32, L.n);
        L.b32.ensure(L.n); L.x32.ensure(L.n); L.x232.ensure(L.n); L.r32.ensure(L.n);
    }
    if (coarse_inverse) conv(Minv, Minv32, (long long)nc * nc);
    HAMLSS_LAUNCH_CHECK();
    f32_ready = true;
}

// ------------------------------------------------------------------- building
namespace {

// Aggregation of one operator; returns the aggregate count (seeds).
int aggregate_device(Ctx& ctx, const Csr<double>& A, double theta, DBuf<int>& agg) {
    const int n = A.n;
    cudaStream_t s = ctx.lane.stream;
    const int g = grid_for(ctx, n);
    agg.ensure(n);
    if (n == 0) return 0;
    ProfScope ps(ctx.lane, "setup", 0.0);
    DBuf<double> rmax(n);
    DBuf<int> in_rp(n + 1), fill(n), status(n), cnt(2), flag(n + 1);
    // long rows (the dense coarse levels): a warp per row
    const bool wide = n > 0 && (long long)A.nnz >= 32LL * n;
    const int gwr = std::max(1, std::min(ceil_div(n, 8), ctx.sm_count * 8));
    if (wide) k_rowmax_w<<<gwr, 256, 0, s>>>(n, A.rp, A.ci, A.v, rmax.p);
    else k_rowmax<<<g, 256, 0, s>>>(n, A.rp, A.ci, A.v, rmax.p);
    HAMLSS_CUDA(cudaMemsetAsync(in_rp.p, 0, sizeof(int) * (n + 1), s));
    if (wide) k_in_count_w<<<gwr, 256, 0, s>>>(n, A.rp, A.ci, A.v, rmax.p, theta, in_rp.p);
    else k_in_count<<<g, 256, 0, s>>>(n, A.rp, A.ci, A.v, rmax.p, theta, in_rp.p);
    HAMLSS_LAUNCH_CHECK();
    long long tot = exclusive_scan(ctx, in_rp.p, n + 1);
    DBuf<int> in_src(std::max<long long>(tot, 1));
    HAMLSS_CUDA(cudaMemcpyAsync(fill.p, in_rp.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    if (wide) k_in_fill_w<<<gwr, 256, 0, s>>>(n, A.rp, A.ci, A.v, rmax.p, theta, fill.p, in_src.p);
    else k_in_fill<<<g, 256, 0, s>>>(n, A.rp, A.ci, A.v, rmax.p, theta, fill.p, in_src.p);
    HAMLSS_LAUNCH_CHECK();
    HAMLSS_CUDA(cudaMemsetAsync(status.p, 0, sizeof(int) * n, s));
    HAMLSS_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * 2, s));
    {
        // a few warps per SM: enough chunks in flight for the wavefront, few spinning loads
        // (operators of short rows have short dependency chains: there more chunks in flight
        // pay, measured 3.9 -> 2.8 ms on the 5-point level; longer chains do not gain)
        const int per_sm = (long long)A.nnz <= 8LL * n ? 4 : 2;
        int blocks = std::max(1, std::min(per_sm * ctx.sm_count, ceil_div(n, 128)));
        const int* irp = in_rp.p;
        const int* isrc = in_src.p;
        int* st = status.p;
        int* tk = cnt.p;
        int* er = cnt.p + 1;
        int nn = n;
        void* args[] = {&nn, &irp, &isrc, &st, &tk, &er};
        HAMLSS_CUDA(cudaLaunchCooperativeKernel((const void*)k_aggregate_wave, dim3(blocks), dim3(128),
                                                args, 0, s));
    }
    k_seed_flags<<<g, 256, 0, s>>>(n, status.p, flag.p);
    HAMLSS_CUDA(cudaMemsetAsync(flag.p + n, 0, sizeof(int), s));
    long long nseed = exclusive_scan(ctx, flag.p, n + 1);
    k_assign<<<g, 256, 0, s>>>(n, status.p, flag.p, in_rp.p, in_src.p, agg.p);
    HAMLSS_LAUNCH_CHECK();
    int err = 0;
    HAMLSS_CUDA(cudaMemcpyAsync(&err, cnt.p + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    if (err) fail(HAMLSS_ERR_TIMEOUT, "AMG aggregation: a bounded wait ran out");
    return (int)nseed;
}

void build_csr_counts(Ctx& ctx, DCsr& C, int rows, int cols, DBuf<int>& cnt) {
    C.n = rows;
    C.m = cols;
    C.rp.ensure(rows + 1);
    HAMLSS_CUDA(cudaMemcpyAsync(C.rp.p, cnt.p, sizeof(int) * rows, cudaMemcpyDeviceToDevice, ctx.lane.stream));
    HAMLSS_CUDA(cudaMemsetAsync(C.rp.p + rows, 0, sizeof(int), ctx.lane.stream));
    long long nnz = exclusive_scan(ctx, C.rp.p, rows + 1);
    if (nnz > INT_MAX) fail(HAMLSS_ERR_NOMEM, "AMG operator exceeds 2^31 nonzeros");
    C.nnz = (int)nnz;
    C.ci.ensure(std::max(C.nnz, 1));
    C.v.ensure(std::max(C.nnz, 1));
}

// Rows of a CSR that a block-per-row kernel takes (smooth_row_on_block); returns their
// count, the list in `list` and the shared memory the longest one needs, 16 bytes per slot
// of its sort (synchronises).
int long_rows(Ctx& ctx, int n, const int* rp, DBuf<int>& list, size_t* smem) {
    cudaStream_t s = ctx.lane.stream;
    list.ensure(std::max(n, 1));
    DBuf<int> cnt(2);
    cnt.zero(s);
    if (n) k_long_rows<<<grid_for(ctx, n), 256, 0, s>>>(n, rp, list.p, cnt.p);
    HAMLSS_LAUNCH_CHECK();
    int h[2] = {0, 0};
    cnt.download(h, 2, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    size_t N = 1;
    while (N < (size_t)h[1] + 1) N <<= 1;
    *smem = 16 * N;
    return h[0];
}

// Grid of a block-per-row kernel for `smem` dynamic shared bytes per block.  The kernel's
// dynamic shared-memory limit is raised once, to the largest any launch of it asks for
// (kMaxRowSmem), and never lowered: contexts on other threads launch it concurrently.
constexpr size_t kMaxRowSmem = 20 * (size_t)kSortMax;   // hash table of kSortMax slots
static_assert(kMaxRowSmem >= 9 * (size_t)kDenseCols + 16 + 16 * (size_t)kWinLeft &&
                  kMaxRowSmem >= 16 * (size_t)kSortMax &&
                  kMaxRowSmem >= 12 * (size_t)kWarpHeads * kMergeWarps,
              "row kernels' shared memory");

template <typename K>
void raise_smem_limit(K kernel) {
    HAMLSS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxRowSmem));
}

bool raise_row_kernel_limits() {
    raise_smem_limit(k_smooth_p_rows<true>);
    raise_smem_limit(k_spgemm_rows<false>);
    raise_smem_limit(k_spgemm_rows<true>);
    raise_smem_limit(k_spgemm_dense<false>);
    raise_smem_limit(k_spgemm_dense<true>);
    raise_smem_limit(k_t_sort_rows);
    raise_smem_limit(k_spgemm_warp<false>);
    raise_smem_limit(k_spgemm_warp<true>);
    raise_smem_limit(k_spgemm_window<false>);
    raise_smem_limit(k_spgemm_window<true>);
    return true;
}

// Grid of k_spgemm_warp (kMergeWarps rows per block).
template <typename K>
int merge_grid(Ctx& ctx, K kernel, size_t smem, int nrows) {
    static DeviceOnce raised;
    raised(ctx.device, raise_row_kernel_limits);
    int per = 0;
    HAMLSS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 32 * kMergeWarps, smem));
    return std::max(1, std::min(ceil_div(nrows, kMergeWarps), ctx.sm_count * std::max(per, 1)));
}

// Grid of a block-per-row kernel launched with `threads` threads a block.
template <typename K>
int rows_grid(Ctx& ctx, K kernel, int threads, size_t smem, int nrows) {
    static DeviceOnce raised;
    raised(ctx.device, raise_row_kernel_limits);
    int per = 0;
    HAMLSS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem));
    return std::max(1, std::min(nrows, ctx.sm_count * std::max(per, 1)));
}

template <typename K>
int row_grid(Ctx& ctx, K kernel, size_t smem, int nrows) {
    static DeviceOnce raised;
    raised(ctx.device, raise_row_kernel_limits);
    int per = 0;
    HAMLSS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kRowBlock, smem));
    return std::max(1, std::min(nrows, ctx.sm_count * std::max(per, 1)));
}

void smooth_prolongation(Ctx& ctx, const Csr<double>& A, const DBuf<int>& agg, int nc, double omega,
                         DCsr& P) {
    const int n = A.n;
    cudaStream_t s = ctx.lane.stream;
    const int g = grid_for(ctx, n);
    DBuf<int> cnt(n), list(3LL * std::max(n, 1)), bk(6);
    // rows longer than kLongRow by length bucket: a block of 64 / 128 / 256 threads a row
    // (shorter rows sort fewer keys, so smaller blocks keep more rows in flight)
    bk.zero(s);
    if (n) k_long_rows3<<<g, 256, 0, s>>>(n, A.rp, list.p, bk.p);
    HAMLSS_LAUNCH_CHECK();
    int hb[6] = {0, 0, 0, 0, 0, 0};
    bk.download(hb, 6, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    const int threads[3] = {64, 128, kRowBlock};
    // one pass into per-row slots (room for every candidate: entries + 1), then the counts
    // give P's rows and the survivors move to their places
    DBuf<int> off(n + 1);
    k_slot_offsets<<<g, 256, 0, s>>>(n, A.rp, off.p);
    HAMLSS_LAUNCH_CHECK();
    const long long slots = (long long)A.nnz + n;
    if ((size_t)slots > ctx.gemm_ci.n || (size_t)slots > ctx.gemm_v.n) {
        AllocScope plain(nullptr);              // long-lived: plain device memory, not the pool
        ctx.gemm_ci.ensure(std::max(slots, 1LL) + (1 << 20));
        ctx.gemm_v.ensure(std::max(slots, 1LL) + (1 << 20));
    }
    int* wci = ctx.gemm_ci.p;
    double* wv = ctx.gemm_v.p;
    // rows of up to 8 / 16 / kLongRow entries: 8 / 16 / 32 lanes a row
    const int g8 = std::max(1, std::min(ceil_div(n, 32), ctx.sm_count * 8));     // 32 rows a block
    const int g16 = std::max(1, std::min(ceil_div(n, 16), ctx.sm_count * 8));
    const int g32 = std::max(1, std::min(ceil_div(n, 8), ctx.sm_count * 8));
    k_smooth_p_sub<8><<<g8, 256, 0, s>>>(n, -1, A.rp, A.ci, A.v, agg.p, omega, cnt.p, off.p, wci, wv);
    k_smooth_p_sub<16><<<g16, 256, 0, s>>>(n, 8, A.rp, A.ci, A.v, agg.p, omega, cnt.p, off.p, wci, wv);
    k_smooth_p_sub<kLongRow><<<g32, 256, 0, s>>>(n, 16, A.rp, A.ci, A.v, agg.p, omega, cnt.p, off.p, wci, wv);
    k_smooth_p<true><<<g, 256, 0, s>>>(n, A.rp, A.ci, A.v, agg.p, omega, cnt.p, off.p, wci, wv);
    HAMLSS_LAUNCH_CHECK();
    for (int b = 0; b < 3; ++b) {
        if (!hb[b]) continue;
        int N = 1;
        while (N < hb[3 + b] + 1) N <<= 1;
        const size_t smem = 16 * (size_t)N;
        const int* lst = list.p + (size_t)b * n;
        const int gb = rows_grid(ctx, k_smooth_p_rows<true>, threads[b], smem, hb[b]);
        k_smooth_p_rows<true><<<gb, threads[b], smem, s>>>(lst, hb[b], A.rp, A.ci, A.v, agg.p, omega, cnt.p,
                                                           off.p, wci, wv);
        HAMLSS_LAUNCH_CHECK();
    }
    build_csr_counts(ctx, P, n, nc, cnt);
    if (n)
        k_spgemm_compact<<<std::max(1, std::min(ceil_div(n, 8), ctx.sm_count * 16)), 256, 0, s>>>(
            n, off.p, cnt.p, wci, wv, P.rp.p, P.ci.p, P.v.p);
    HAMLSS_LAUNCH_CHECK();
}

void transpose(Ctx& ctx, const DCsr& P, DCsr& R) {
    cudaStream_t s = ctx.lane.stream;
    R.n = P.m;
    R.m = P.n;
    R.nnz = P.nnz;
    R.rp.ensure(R.n + 1);
    R.ci.ensure(std::max(R.nnz, 1));
    R.v.ensure(std::max(R.nnz, 1));
    HAMLSS_CUDA(cudaMemsetAsync(R.rp.p, 0, sizeof(int) * (R.n + 1), s));
    k_t_count<<<grid_for(ctx, P.n), 256, 0, s>>>(P.n, P.rp.p, P.ci.p, R.rp.p);
    HAMLSS_LAUNCH_CHECK();
    exclusive_scan(ctx, R.rp.p, R.n + 1);
    DBuf<int> fill(std::max(R.n, 1));
    HAMLSS_CUDA(cudaMemcpyAsync(fill.p, R.rp.p, sizeof(int) * R.n, cudaMemcpyDeviceToDevice, s));
    k_t_fill<<<grid_for(ctx, P.n), 256, 0, s>>>(P.n, P.rp.p, P.ci.p, P.v.p, fill.p, R.ci.p, R.v.p);
    k_t_sort<<<grid_for(ctx, R.n), 256, 0, s>>>(R.n, R.rp.p, R.ci.p, R.v.p);
    HAMLSS_LAUNCH_CHECK();
    DBuf<int> list;
    size_t smem = 0;
    const int nlong = long_rows(ctx, R.n, R.rp.p, list, &smem);
    if (nlong) {
        const int gb = row_grid(ctx, k_t_sort_rows, smem, nlong);
        k_t_sort_rows<<<gb, kRowBlock, smem, s>>>(list.p, nlong, R.rp.p, R.ci.p, R.v.p);
        HAMLSS_LAUNCH_CHECK();
    }
}

// k_spgemm_seq over its listed rows, shared memory sized to their widest window.
template <int CMAX, bool STEP>
void seq_rows(Ctx& ctx, bool fill, const int* rows, int nrows, int span, const int* wlo, const int* wspan,
              const Csr<double>& A, const Csr<double>& B, int* ccnt, const int* crp, int* cci, double* cv) {
    if (!nrows) return;
    cudaStream_t s = ctx.lane.stream;
    const int nw = std::max(1, (span + 31) / 32);
    const size_t smem = kSeqWarps * seq_warp_bytes(CMAX, nw);
    static DeviceOnce raised;
    raised(ctx.device, [] {
        constexpr int lim = (int)(kSeqWarps * seq_warp_bytes(CMAX, kDenseCols / 32));
        HAMLSS_CUDA(cudaFuncSetAttribute(k_spgemm_seq<false, CMAX, STEP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         lim));
        HAMLSS_CUDA(cudaFuncSetAttribute(k_spgemm_seq<true, CMAX, STEP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         lim));
    });
    auto kern = fill ? k_spgemm_seq<true, CMAX, STEP> : k_spgemm_seq<false, CMAX, STEP>;
    int per = 0;
    HAMLSS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 32 * kSeqWarps, smem));
    const int gb = std::max(1, std::min(ceil_div(nrows, kSeqWarps), ctx.sm_count * std::max(per, 1)));
    kern<<<gb, 32 * kSeqWarps, smem, s>>>(rows, nrows, nw, wlo, wspan, A.rp, A.ci, A.v, B.rp, B.ci, B.v, ccnt, crp,
                                          cci, cv);
    HAMLSS_LAUNCH_CHECK();
}

void spgemm(Ctx& ctx, const Csr<double>& A, const Csr<double>& B, DCsr& C) {
    cudaStream_t s = ctx.lane.stream;
    const int g = grid_for(ctx, A.n);
    DBuf<int> heads(3LL * std::max(A.nnz, 1));
    DBuf<int> cnt(std::max(A.n, 1)), cls(std::max(A.n, 1)), list(8LL * std::max(A.n, 1)), meta(15);
    DBuf<int> wlo(std::max(A.n, 1)), wspan(std::max(A.n, 1));
    meta.zero(s);
    if (A.n)
        k_spgemm_classify<<<g, 256, 0, s>>>(A.n, A.rp, A.ci, B.rp, B.ci, B.m, cls.p, list.p, meta.p, wlo.p,
                                            wspan.p);
    HAMLSS_LAUNCH_CHECK();
    int hm[15] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    meta.download(hm, 15, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    const int nlong = hm[0], ndense = hm[2], nwarp = hm[3];
    // class-4 windows by width bucket: each launch sizes its shared memory to its widest row
    auto windows = [&](bool fill, int* ccnt, const int* crp, int* cci, double* cv) {
        for (int b = 0; b < 3; ++b) {
            const int nw = hm[5 + b];
            if (!nw) continue;
            const int W = hm[8 + b];
            const size_t wsm = window_smem(W);       // window accumulator + hit flags + left row
            const int* wl = list.p + (3LL + b) * A.n;
            if (fill) {
                const int gb = row_grid(ctx, k_spgemm_window<true>, wsm, nw);
                k_spgemm_window<true><<<gb, kRowBlock, wsm, s>>>(wl, nw, W, wlo.p, wspan.p, A.rp, A.ci, A.v,
                                                                 B.rp, B.ci, B.v, ccnt, crp, cci, cv);
            } else {
                const int gb = row_grid(ctx, k_spgemm_window<false>, wsm, nw);
                k_spgemm_window<false><<<gb, kRowBlock, wsm, s>>>(wl, nw, W, wlo.p, wspan.p, A.rp, A.ci, A.v,
                                                                  B.rp, B.ci, B.v, ccnt, crp, cci, cv);
            }
            HAMLSS_LAUNCH_CHECK();
        }
    };
    // classes 5 and 6: ordered warp accumulation, 32 products / one left entry a step
    auto ordered = [&](bool fill, int* ccnt, const int* crp, int* cci, double* cv) {
        seq_rows<kSeqCols, false>(ctx, fill, list.p + 6LL * A.n, hm[11], hm[12], wlo.p, wspan.p, A, B, ccnt, crp,
                                  cci, cv);
        seq_rows<kSeqCols, true>(ctx, fill, list.p + 7LL * A.n, hm[13], hm[14], wlo.p, wspan.p, A, B, ccnt, crp,
                                 cci, cv);
    };
    int KH = 32;
    while (KH < hm[4]) KH <<= 1;
    const size_t wsmem = sizeof(int) * 3 * (size_t)KH * kMergeWarps;
    const int* wlist = list.p + 2LL * A.n;
    int S = 64;
    while (S < 2 * hm[1]) S <<= 1;
    const size_t smem = 20 * (size_t)S;                 // u64 keys + doubles + ints per slot
    const size_t dsmem = 9 * (size_t)std::max(B.m, 1);   // dense accumulator + hit flags
    const int* dlist = list.p + A.n;
    // One numeric pass into per-row capacity slots (min(products, B.m) each), then a
    // compaction into the CSR -- when the slots fit (below 2^31 entries and 8 GB); else the
    // counting pass below followed by the numeric pass in place.
    {
        DBuf<int> off(A.n + 1);
        HAMLSS_CUDA(cudaMemsetAsync(off.p + A.n, 0, sizeof(int), s));
        if (A.n) k_spgemm_bound<<<g, 256, 0, s>>>(A.n, A.rp, A.ci, B.rp, B.ci, std::max(B.m, 1), off.p);
        HAMLSS_LAUNCH_CHECK();
        const long long total = exclusive_scan(ctx, off.p, A.n + 1);
        if (total <= INT_MAX && total * 12 <= (8LL << 30)) {
            if ((size_t)total > ctx.gemm_ci.n || (size_t)total > ctx.gemm_v.n) {
                AllocScope plain(nullptr);          // long-lived: plain device memory, not the pool
                ctx.gemm_ci.ensure(std::max(total, 1LL) + (1 << 20));
                ctx.gemm_v.ensure(std::max(total, 1LL) + (1 << 20));
            }
            DBuf<int>& wci = ctx.gemm_ci;
            DBuf<double>& wv = ctx.gemm_v;
            k_spgemm<true><<<g, 256, 0, s>>>(A.n, A.rp, A.ci, A.v, B.rp, B.ci, B.v, cnt.p, off.p, wci.p,
                                             wv.p, heads.p, cls.p);
            HAMLSS_LAUNCH_CHECK();
            if (nlong) {
                const int gb = row_grid(ctx, k_spgemm_rows<true>, smem, nlong);
                k_spgemm_rows<true><<<gb, kRowBlock, smem, s>>>(list.p, nlong, S, A.rp, A.ci, A.v, B.rp, B.ci,
                                                                B.v, cnt.p, off.p, wci.p, wv.p);
                HAMLSS_LAUNCH_CHECK();
            }
            if (nwarp) {
                const int gb = merge_grid(ctx, k_spgemm_warp<true>, wsmem, nwarp);
                k_spgemm_warp<true><<<gb, 32 * kMergeWarps, wsmem, s>>>(wlist, nwarp, KH, A.rp, A.ci, A.v,
                                                                         B.rp, B.ci, B.v, cnt.p, off.p,
                                                                         wci.p, wv.p);
                HAMLSS_LAUNCH_CHECK();
            }
            if (ndense) {
                const int gb = row_grid(ctx, k_spgemm_dense<true>, dsmem, ndense);
                k_spgemm_dense<true><<<gb, kRowBlock, dsmem, s>>>(dlist, ndense, B.m, A.rp, A.ci, A.v, B.rp,
                                                                  B.ci, B.v, cnt.p, off.p, wci.p, wv.p);
                HAMLSS_LAUNCH_CHECK();
            }
            windows(true, cnt.p, off.p, wci.p, wv.p);
            ordered(true, cnt.p, off.p, wci.p, wv.p);
            build_csr_counts(ctx, C, A.n, B.m, cnt);
            if (A.n)
                k_spgemm_compact<<<std::max(1, std::min(ceil_div(A.n, 8), ctx.sm_count * 16)), 256, 0, s>>>(
                    A.n, off.p, cnt.p, wci.p, wv.p, C.rp.p, C.ci.p, C.v.p);
            HAMLSS_LAUNCH_CHECK();
            return;
        }
    }
    k_spgemm<false><<<g, 256, 0, s>>>(A.n, A.rp, A.ci, A.v, B.rp, B.ci, B.v, cnt.p, nullptr, nullptr,
                                      nullptr, heads.p, cls.p);
    HAMLSS_LAUNCH_CHECK();
    if (nlong) {
        const int gb = row_grid(ctx, k_spgemm_rows<false>, smem, nlong);
        k_spgemm_rows<false><<<gb, kRowBlock, smem, s>>>(list.p, nlong, S, A.rp, A.ci, A.v, B.rp, B.ci, B.v,
                                                         cnt.p, nullptr, nullptr, nullptr);
        HAMLSS_LAUNCH_CHECK();
    }
    if (nwarp) {
        const int gb = merge_grid(ctx, k_spgemm_warp<false>, wsmem, nwarp);
        k_spgemm_warp<false><<<gb, 32 * kMergeWarps, wsmem, s>>>(wlist, nwarp, KH, A.rp, A.ci, A.v, B.rp,
                                                                  B.ci, B.v, cnt.p, nullptr, nullptr, nullptr);
        HAMLSS_LAUNCH_CHECK();
    }
    if (ndense) {
        const int gb = row_grid(ctx, k_spgemm_dense<false>, dsmem, ndense);
        k_spgemm_dense<false><<<gb, kRowBlock, dsmem, s>>>(dlist, ndense, B.m, A.rp, A.ci, A.v, B.rp, B.ci,
                                                           B.v, cnt.p, nullptr, nullptr, nullptr);
        HAMLSS_LAUNCH_CHECK();
    }
    windows(false, cnt.p, nullptr, nullptr, nullptr);
    ordered(false, cnt.p, nullptr, nullptr, nullptr);
    build_csr_counts(ctx, C, A.n, B.m, cnt);
    k_spgemm<true><<<g, 256, 0, s>>>(A.n, A.rp, A.ci, A.v, B.rp, B.ci, B.v, nullptr, C.rp.p, C.ci.p,
                                     C.v.p, heads.p, cls.p);
    HAMLSS_LAUNCH_CHECK();
    if (nlong) {
        const int gb = row_grid(ctx, k_spgemm_rows<true>, smem, nlong);
        k_spgemm_rows<true><<<gb, kRowBlock, smem, s>>>(list.p, nlong, S, A.rp, A.ci, A.v, B.rp, B.ci, B.v,
                                                        nullptr, C.rp.p, C.ci.p, C.v.p);
        HAMLSS_LAUNCH_CHECK();
    }
    if (nwarp) {
        const int gb = merge_grid(ctx, k_spgemm_warp<true>, wsmem, nwarp);
        k_spgemm_warp<true><<<gb, 32 * kMergeWarps, wsmem, s>>>(wlist, nwarp, KH, A.rp, A.ci, A.v, B.rp,
                                                                 B.ci, B.v, nullptr, C.rp.p, C.ci.p, C.v.p);
        HAMLSS_LAUNCH_CHECK();
    }
    if (ndense) {
        const int gb = row_grid(ctx, k_spgemm_dense<true>, dsmem, ndense);
        k_spgemm_dense<true><<<gb, kRowBlock, dsmem, s>>>(dlist, ndense, B.m, A.rp, A.ci, A.v, B.rp, B.ci,
                                                          B.v, nullptr, C.rp.p, C.ci.p, C.v.p);
        HAMLSS_LAUNCH_CHECK();
    }
    windows(true, nullptr, C.rp.p, C.ci.p, C.v.p);
    ordered(true, nullptr, C.rp.p, C.ci.p, C.v.p);
}

}  // namespace

std::unique_ptr<Prec> make_amg(Ctx& ctx, hamlss_mat* A, const hamlss_params& p) {
    if (A->A.n != A->A.m) fail(HAMLSS_ERR_SIZE, "AMG needs a square matrix");
    auto M = std::make_unique<AmgPrec>();
    M->kind = HAMLSS_PREC_AMG;
    M->A0 = A;
    M->n = A->A.n;
    M->omega = p.amg_omega;
    M->pre = p.amg_smooth_pre;
    M->post = p.amg_smooth_post;
    cudaStream_t s = ctx.lane.stream;
    ProfScope ps(ctx.lane, "setup", 0.0);
    AllocScope scope(s);                 // setup buffers from the stream-ordered pool
    const int max_levels = std::min(kMaxLevels, std::max(1, p.amg_levels));
    {
        auto L0 = std::make_unique<AmgLevel>();
        L0->n = A->A.n;
        L0->dinv.ensure(L0->n);
        if (L0->n) k_inv_diag<<<grid_for(ctx, L0->n), 256, 0, s>>>(L0->n, A->A.rp.p, A->A.ci.p, A->A.v.p, L0->dinv.p);
        HAMLSS_LAUNCH_CHECK();
        M->lev.push_back(std::move(L0));
    }
    // verbose >= 2: per-phase wall times of every level on stderr (SolverParams::verbose)
    const bool trace = p.verbose >= 2;
    auto tick = std::chrono::steady_clock::now();
    long long alloc0 = alloc_ns().load();
    auto phase = [&](int lv, const char* what) {
        if (!trace) return;
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        auto now = std::chrono::steady_clock::now();
        const long long a = alloc_ns().load();
        std::fprintf(stderr, "[hamlss amg] level %d %-10s %9.3f ms (alloc/free %7.3f ms)\n", lv, what,
                     std::chrono::duration<double, std::milli>(now - tick).count(), (a - alloc0) * 1e-6);
        tick = now;
        alloc0 = a;
    };
    for (int lv = 0; lv < max_levels - 1; ++lv) {
        AmgLevel& F = *M->lev.back();
        Csr<double> Af = M->Aview64(M->levels() - 1);
        if (Af.n <= p.amg_coarse_limit) break;
        DBuf<int> agg;
        int nc = aggregate_device(ctx, Af, p.amg_strong, agg);
        phase(lv, "aggregate");
        if (nc >= Af.n) break;
        // engine option: a level that barely coarsens becomes the (dense) coarsest one,
        // when it is small enough for the dense factorisation
        if (p.amg_stall_ratio > 0.0 && (double)nc > p.amg_stall_ratio * (double)Af.n &&
            Af.n <= kStallDenseMax)
            break;
        smooth_prolongation(ctx, Af, agg, nc, M->omega, F.P);
        phase(lv, "prolong");
        transpose(ctx, F.P, F.R);
        phase(lv, "transpose");
        DCsr AP;
        spgemm(ctx, Af, F.P.f64(), AP);
        phase(lv, "A*P");
        auto C = std::make_unique<AmgLevel>();
        spgemm(ctx, F.R.f64(), AP.f64(), C->A);
        phase(lv, "R*(AP)");
        if (trace)
            std::fprintf(stderr, "[hamlss amg] level %d n=%d nnz=%d -> n_c=%d nnz_c=%d nnz_P=%d\n", lv,
                         Af.n, Af.nnz, C->A.n, C->A.nnz, F.P.nnz);
        C->n = C->A.n;
        C->dinv.ensure(std::max(C->n, 1));
        if (C->n) k_inv_diag<<<grid_for(ctx, C->n), 256, 0, s>>>(C->n, C->A.rp.p, C->A.ci.p, C->A.v.p, C->dinv.p);
        HAMLSS_LAUNCH_CHECK();
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        M->lev.push_back(std::move(C));
    }
    // work vectors (FP64)
    for (int l = 0; l < M->levels(); ++l) {
        AmgLevel& L = *M->lev[l];
        int n = std::max(L.n, 1);
        L.b.ensure(n); L.x.ensure(n); L.x2.ensure(n); L.r.ensure(n);
    }
    // coarsest level: dense factorisation (or explicit inverse for the large ones)
    {
        const int l = M->levels() - 1;
        Csr<double> C = M->Aview64(l);
        const int nc = C.n;
        M->nc = nc;
        if ((long long)nc * nc > (1LL << 28)) fail(HAMLSS_ERR_NOMEM, "coarsest AMG level too large for a dense solve");
        M->Md.ensure((size_t)std::max(nc, 1) * std::max(nc, 1));
        M->piv.ensure(std::max(nc, 1));
        M->skip.ensure(std::max(nc, 1));
        M->cwork.ensure(2 * std::max(nc, 1));
        HAMLSS_CUDA(cudaMemsetAsync(M->Md.p, 0, sizeof(double) * (size_t)nc * nc, s));
        if (nc) {
            k_csr_to_dense<<<std::max(1, std::min(ceil_div(nc, 8), ctx.sm_count * 8)), 256, 0, s>>>(
                nc, C.rp, C.ci, C.v, M->Md.p);
            HAMLSS_LAUNCH_CHECK();
        }
        if (nc > kBlockedCoarse) {
            // large coarsest level: blocked LU with partial pivoting + explicit inverse
            M->coarse_inverse = true;
            M->Minv.ensure((size_t)nc * nc);
            dense_lu_inverse(ctx, nc, M->Md.p, M->Minv.p, M->piv.p);
            M->Md.release();
            phase(M->levels() - 1, "blocked LU");
            return M;
        }
        if (nc) {
            k_dense_factor<<<1, 256, 0, s>>>(nc, M->Md.p, M->piv.p, M->skip.p);
            HAMLSS_LAUNCH_CHECK();
        }
        phase(M->levels() - 1, "coarse LU");
        M->coarse_inverse = nc > 96;
        if (M->coarse_inverse) {
            M->Minv.ensure((size_t)nc * nc);
            DBuf<double> work((size_t)nc * 2 * nc);
            k_dense_inverse<<<nc, 32, 0, s>>>(nc, M->Md.p, M->piv.p, M->skip.p, work.p, M->Minv.p);
            HAMLSS_LAUNCH_CHECK();
            HAMLSS_CUDA(cudaStreamSynchronize(s));
        }
    }
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    phase(M->levels() - 1, "coarse inv");
    return M;
}

// ---------------------------------------------------------------- inspection
int amg_num_levels(const Prec* P, int* levels) {
    auto* M = dynamic_cast<const AmgPrec*>(P);
    if (!M) return HAMLSS_ERR_INVALID;
    *levels = M->levels();
    return HAMLSS_OK;
}

int amg_level_matrix(const Prec* P, int level, int which, int* rows, int* cols, int* nnz, int* rp,
                     int* ci, double* v, cudaStream_t s) {
    auto* M = dynamic_cast<const AmgPrec*>(P);
    if (!M || level < 0 || level >= M->levels() || which < 0 || which > 2) return HAMLSS_ERR_INVALID;
    Csr<double> C;
    if (which == 0) C = M->Aview64(level);
    else {
        if (level == M->levels() - 1) return HAMLSS_ERR_INVALID;
        C = which == 1 ? M->lev[level]->P.f64() : M->lev[level]->R.f64();
    }
    if (rows) *rows = C.n;
    if (cols) *cols = C.m;
    if (nnz) *nnz = C.nnz;
    if (rp) HAMLSS_CUDA(cudaMemcpyAsync(rp, C.rp, sizeof(int) * (C.n + 1), cudaMemcpyDeviceToHost, s));
    if (ci && C.nnz) HAMLSS_CUDA(cudaMemcpyAsync(ci, C.ci, sizeof(int) * C.nnz, cudaMemcpyDeviceToHost, s));
    if (v && C.nnz) HAMLSS_CUDA(cudaMemcpyAsync(v, C.v, sizeof(double) * C.nnz, cudaMemcpyDeviceToHost, s));
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    return HAMLSS_OK;
}

int amg_aggregate_matrix(Ctx& ctx, hamlss_mat* A, double theta, int* agg_host, int* n_agg) {
    DBuf<int> agg;
    int nc = aggregate_device(ctx, A->A.f64(), theta, agg);
    if (A->A.n) agg.download(agg_host, A->A.n, ctx.lane.stream);
    HAMLSS_CUDA(cudaStreamSynchronize(ctx.lane.stream));
    *n_agg = nc;
    return HAMLSS_OK;
}

}  // namespace hamlss
