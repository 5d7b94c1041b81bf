// spmv_stream.cuh -- CSR SpMV whose matrix stream is staged by bulk asynchronous copies.
//
// For operators with short rows (the 5-point fine level, the ~20-entry first coarse
// level) the plain kernel (spmv.cuh) is latency-bound: each warp has only a few cache
// lines of col_idx / values in flight, then waits on the x gathers that depend on them.
// Here every CTA owns a ring of S shared-memory stages, each with a `full` mbarrier (its
// copies landed) and an `empty` one (all eight warps are done with it), so warps do not
// wait for one another between tiles.  One thread per CTA is the producer: for row tile g (rows [g*TR, g*TR + TR)) it reads the tile's entry range from
// row_ptr and issues three cp.async.bulk copies into a stage -- the tile's row_ptr slice,
// col_idx slice and values slice -- that complete on the stage's mbarrier, plus L2
// prefetches (cp.async.bulk.prefetch.L2) of the vectors the tile's epilogue and x
// gathers will read.  It keeps S - 1 tiles in flight ahead of the one being consumed, so
// a CTA has tens of KB of the matrix stream in flight instead of a few lines per warp.
//
// Consumers: G lanes per row (TR = 256 / G rows per tile).  G = 1 sums each row in column
// order with the reference's separate multiply and add (sparse_matrix.cpp:80-86), so
// FP64 results are bit-identical to the plain kernel; G > 1 (FP32 operands only) strides
// the row's entries and adds the lanes' partial sums with shuffles.  Entries that do not
// fit a stage (a tile with more than K entries) are read from global memory by the same
// loop, so any matrix is handled; the launcher picks G so that tiles normally fit.
//
// Rows longer than skip_len (a skewed matrix's few very long rows) are left to
// k_spmv_rows_seq: the kernel neither sums them nor applies their epilogue.
//
// Waits are bounded: a stage whose copies have not landed after ~1 s is read from
// global memory instead (the results stay right) and the lane's error word is set; the
// host reports it as HAMLSS_ERR_TIMEOUT.  No cluster launch, no multicast: single-GPU
// bulk copies into the CTA's own shared memory.
#pragma once

#include <type_traits>

#include "spmv.cuh"

namespace hamlss {

constexpr int kStreamThreads = 256;
constexpr int kStreamWarps = kStreamThreads / 32;

// Optional hooks of XOp / Epi functors: prefetch(r0, r1) issues L2 prefetches for the
// vector ranges a row tile [r0, r1) will read.
template <typename F, typename = void>
struct has_prefetch : std::false_type {};
template <typename F>
struct has_prefetch<F, std::void_t<decltype(std::declval<const F&>().prefetch(0, 0))>> : std::true_type {};

// Optional hook of Epi functors: pre(i) loads the row's own epilogue operands (a struct
// Pre) and operator()(i, ax, acc, pre) applies them.  The kernel calls pre before the
// row's x gathers, so the epilogue's loads are in flight together with them instead of
// after the sum.
template <typename F, typename = void>
struct has_pre : std::false_type {};
template <typename F>
struct has_pre<F, std::void_t<decltype(std::declval<const F&>().pre(0))>> : std::true_type {};

struct NoPre {};

template <typename Epi>
__device__ __forceinline__ auto epi_pre(const Epi& e, int row) {
    if constexpr (has_pre<Epi>::value) return e.pre(row);
    else return NoPre{};
}

template <typename Epi, typename P, int NV>
__device__ __forceinline__ void epi_apply(const Epi& e, int row, double sum, double (&acc)[NV], const P& p) {
    if constexpr (has_pre<Epi>::value) e(row, sum, acc, p);
    else e(row, sum, acc);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return done != 0;
}

// Wait for the phase of `bar` with the given parity; false after ~1 s (2^31 SM clocks)
// without completion.  try_wait may itself suspend the thread for a while, so the bound
// is on elapsed clocks, not on polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > (1ll << 31)) return false;
    return true;
}

// Bulk copy global -> this CTA's shared memory, completing on `bar`.  Both addresses
// 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

// Stage capacity in entries (a multiple of 4) and stages per CTA, by value type: FP32
// 21.5 KB x 2 stages (five CTAs per SM), FP64 19.5 KB x 3 stages (three per SM).  Measured
// on the 2048^2 hierarchy (V-cycle SpMVs, GB/s): 1536 entries x 3 stages at five CTAs
// 2456; 3072 x 2 at four 3007; 2560 x 2 at five 3218; 4096 x 2 at three 2800; 3072 x 3 at
// two 2007 -- FP32 tiles of ~2,500 entries (half the lanes a row of the 1536-entry shape,
// so each lane has more gathers in flight) in two stages, with as many CTAs as fit.
template <typename T>
struct StreamShape {
    static constexpr int K = sizeof(T) == 8 ? 1536 : 2560;
    static constexpr int S = sizeof(T) == 8 ? 3 : 2;
    static constexpr int kMinBlocks = sizeof(T) == 8 ? 3 : 5;   // CTAs per SM the smem allows
    static constexpr int kTrMax = kStreamThreads;            // rows per tile with G = 1
    static constexpr size_t rp_bytes = (kTrMax + 4) * 4;
    static constexpr size_t ci_bytes = (K + 4) * 4;
    static constexpr size_t v_bytes = (K + 4) * sizeof(T);
    static constexpr size_t stage_bytes = rp_bytes + ci_bytes + v_bytes;
    static constexpr size_t smem_bytes = S * stage_bytes;
};

template <typename T>
__device__ __forceinline__ int* stage_rp(unsigned char* smem, int s) {
    return reinterpret_cast<int*>(smem + s * StreamShape<T>::stage_bytes);
}
template <typename T>
__device__ __forceinline__ int* stage_ci(unsigned char* smem, int s) {
    return reinterpret_cast<int*>(smem + s * StreamShape<T>::stage_bytes + StreamShape<T>::rp_bytes);
}
template <typename T>
__device__ __forceinline__ T* stage_v(unsigned char* smem, int s) {
    return reinterpret_cast<T*>(smem + s * StreamShape<T>::stage_bytes + StreamShape<T>::rp_bytes +
                                StreamShape<T>::ci_bytes);
}

// Producer step: rows [r0, r1) into stage s -- the row_ptr slice, and the entries from
// row_ptr[r0] (aligned down to 4) up to K of them -- completing on bar; records the staged
// entry range in base / end.
template <typename T>
__device__ __forceinline__ void stream_issue(unsigned char* smem, int s, uint64_t* bar, int r0, int r1,
                                             const int* __restrict__ rp, const int* __restrict__ ci,
                                             const T* __restrict__ v, int* base_out, int* end_out) {
    constexpr int K = StreamShape<T>::K;
    const int e0 = __ldg(&rp[r0]), e1 = __ldg(&rp[r1]);
    const int base = e0 & ~3;
    const int end = min(e1, base + K);
    const int cnt = ((end - base) + 3) & ~3;          // <= K (K % 4 == 0); at most 3 past e1
    const unsigned rp_cnt = (unsigned)(((r1 - r0 + 1) + 3) & ~3);
    *base_out = base;
    *end_out = end;
    const unsigned bytes = rp_cnt * 4u + (unsigned)cnt * (4u + (unsigned)sizeof(T));
    mbar_arrive_tx(bar, bytes);
    bulk_load(stage_rp<T>(smem, s), rp + r0, rp_cnt * 4u, bar);
    if (cnt > 0) {
        bulk_load(stage_ci<T>(smem, s), ci + base, (unsigned)cnt * 4u, bar);
        bulk_load(stage_v<T>(smem, s), v + base, (unsigned)cnt * (unsigned)sizeof(T), bar);
    }
}

template <typename T, int NRED, typename XOp, typename Epi, typename Fin, int G>
__global__ void __launch_bounds__(kStreamThreads, StreamShape<T>::kMinBlocks)
k_spmv_stream(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ v,
              XOp xop, Epi epi, Reducer red, Fin fin, const int* gate, int* err, int skip_len) {
    constexpr int S = StreamShape<T>::S;
    constexpr int TR = kStreamThreads / G;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t full[S];      // the stage's copies have landed (one arrival + bytes)
    __shared__ uint64_t empty[S];     // every warp is done with the stage (one arrival a warp)
    __shared__ int s_base[S], s_end[S];
    __shared__ int s_staged;          // tiles of this CTA issued so far
    __shared__ int s_stop;            // a wait ran out: no more copies are issued
    __shared__ double rsh[kStreamWarps * (NRED > 0 ? NRED : 1)];
    if (gate && *(volatile const int*)gate) return;
    XOp xop_l = xop;
    Epi epi_l = epi;
    xop_l.load();
    epi_l.load();
    const int tid = threadIdx.x, lane = tid & 31;
    const int ntiles = (n + TR - 1) / TR;
    const int G0 = (int)blockIdx.x, GS = (int)gridDim.x;
    // tiles of this CTA: G0 + u * GS for u < mine
    const int mine = G0 < ntiles ? (ntiles - 1 - G0) / GS + 1 : 0;
    volatile int* staged = &s_staged;
    volatile int* stop = &s_stop;
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kStreamWarps);
        }
        mbar_fence_init();
        int u = 0;
        for (; u < S - 1 && u < mine; ++u) {
            const int r0 = (G0 + u * GS) * TR;
            stream_issue<T>(smem, u, &full[u], r0, min(n, r0 + TR), rp, ci, v, &s_base[u], &s_end[u]);
            if constexpr (has_prefetch<XOp>::value) xop_l.prefetch(r0, min(n, r0 + TR));
            if constexpr (has_prefetch<Epi>::value) epi_l.prefetch(r0, min(n, r0 + TR));
        }
        s_staged = u;
        s_stop = 0;
    }
    __syncthreads();

    double acc[NRED > 0 ? NRED : 1];
#pragma unroll
    for (int k = 0; k < (NRED > 0 ? NRED : 1); ++k) acc[k] = 0.0;
    const int sub = tid / G, gl = tid - sub * G;
    // Warps do not wait for one another between tiles: a warp that is done with a stage
    // arrives on its `empty` barrier, and the producer (thread 0) waits for all eight
    // arrivals before it refills the stage.
    for (int u = 0; u < mine; ++u) {
        const int s = u % S;
        if (tid == 0 && u + S - 1 < mine && !*stop) {
            const int w = u + S - 1, sw = w % S, use = w / S;
            // stage sw last held tile w - S (use - 1), which every warp has to be done with
            if (use == 0 || mbar_wait_bounded(&empty[sw], (unsigned)((use - 1) & 1))) {
                const int r0 = (G0 + w * GS) * TR, r1 = min(n, r0 + TR);
                stream_issue<T>(smem, sw, &full[sw], r0, r1, rp, ci, v, &s_base[sw], &s_end[sw]);
                if constexpr (has_prefetch<XOp>::value) xop_l.prefetch(r0, r1);
                if constexpr (has_prefetch<Epi>::value) epi_l.prefetch(r0, r1);
                *staged = w + 1;
            } else {
                if (err) atomicExch(err, 1);
                *stop = 1;
            }
        }
        // a warp may run ahead of the producer: wait (bounded) until tile u is issued or
        // the producer has stopped
        if (u >= *staged && !*stop) {
            const long long t0 = clock64();
            while (u >= *staged && !*stop) {
                if (clock64() - t0 > (1ll << 31)) {
                    if (err) atomicExch(err, 1);
                    *stop = 1;
                    break;
                }
                __nanosleep(64);
            }
        }
        const int r0 = (G0 + u * GS) * TR, r1 = min(n, r0 + TR);
        bool landed = u < *staged;        // tile u was issued
        if (landed) {                     // phase u / S of stage s; bounded (~1 s)
            landed = mbar_wait_bounded(&full[s], (unsigned)((u / S) & 1));
            if (!landed) {
                if (err) atomicExch(err, 1);
                *stop = 1;
            }
        }
        const int row = r0 + sub;
        decltype(epi_pre(epi_l, 0)) pre{};
        if (row < r1 && gl == 0) pre = epi_pre(epi_l, row);
        double sum = 0.0;
        bool own = row < r1;
        if (own) {
            const int base = landed ? s_base[s] : 0;
            const int lim = landed ? s_end[s] : 0;        // entries below lim are staged
            const int* srp = stage_rp<T>(smem, s);
            const int rs = landed ? srp[sub] : __ldg(&rp[row]);
            int re = landed ? srp[sub + 1] : __ldg(&rp[row + 1]);
            own = re - rs <= skip_len;                    // longer rows: k_spmv_rows_seq
            if (!own) re = rs;
            const int* sci = stage_ci<T>(smem, s);
            const T* sv = stage_v<T>(smem, s);
            // four entries at a time: their x gathers are issued together, then added in
            // order (the row's summation order is unchanged)
            auto entry = [&](int k, T& a, int& c) {
                if (k < lim) {
                    a = sv[k - base];
                    c = sci[k - base];
                } else {
                    a = __ldg(&v[k]);
                    c = __ldg(&ci[k]);
                }
            };
            int k = rs + gl;
            for (; k + 3 * G < re; k += 4 * G) {
                T a0, a1, a2, a3;
                int c0, c1, c2, c3;
                entry(k, a0, c0);
                entry(k + G, a1, c1);
                entry(k + 2 * G, a2, c2);
                entry(k + 3 * G, a3, c3);
                const double x0 = xop_l(c0), x1 = xop_l(c1), x2 = xop_l(c2), x3 = xop_l(c3);
                sum = mul_add<T>(sum, a0, x0);
                sum = mul_add<T>(sum, a1, x1);
                sum = mul_add<T>(sum, a2, x2);
                sum = mul_add<T>(sum, a3, x3);
            }
            for (; k < re; k += G) {
                T a;
                int c;
                entry(k, a, c);
                sum = mul_add<T>(sum, a, xop_l(c));
            }
        }
        if constexpr (G > 1) {
#pragma unroll
            for (int o = G >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        }
        if (own && gl == 0) epi_apply(epi_l, row, sum, acc, pre);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);           // this warp is done with stage s
    }
    __syncthreads();
    if (tid == 0 && *stop) {
        // a wait ran out: give each stage's last issued copies a bounded chance to land
        // before the CTA's shared memory is released
        const int issued = *staged;
        for (int s = 0; s < S && s < issued; ++s) {
            const int last = s + S * ((issued - 1 - s) / S);     // last tile issued into s
            mbar_wait_bounded(&full[s], (unsigned)((last / S) & 1));
        }
    }
    if constexpr (NRED > 0) {
        double tot[NRED];
        if (grid_reduce<NRED>(red, acc, rsh, tot)) fin(tot);
    }
}

}  // namespace hamlss
