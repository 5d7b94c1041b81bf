// engine.cuh -- context, device matrices and launch helpers shared by all solvers.
#pragma once

#include <memory>
#include <mutex>

#include "common.cuh"
#include "spmv.cuh"
#include "spmv_stream.cuh"

namespace hamlss {

// Optional per-launch timing: when enabled, each engine launch is bracketed by a pair of
// CUDA events on its own stream and tagged with its kernel family and the algorithmic
// bytes it must move.  Used by bench.py for the live roofline figure.
struct Profiler {
    bool on = false;
    int depth = 0;            // open ProfScopes on the lane
    std::vector<cudaEvent_t> ev;
    size_t next = 0;
    struct Mark { const char* name; double bytes; size_t e0; };
    std::vector<Mark> marks;
    void reserve(size_t pairs) {
        while (ev.size() < 2 * pairs) {
            cudaEvent_t e;
            HAMLSS_CUDA(cudaEventCreate(&e));
            ev.push_back(e);
        }
    }
    // returns the slot of the start event, or -1 when off / out of events
    long begin(cudaStream_t s) {
        if (!on || next + 2 > ev.size()) return -1;
        HAMLSS_CUDA(cudaEventRecord(ev[next], s));
        return (long)next;
    }
    void end(cudaStream_t s, long slot, const char* name, double bytes) {
        if (slot < 0) return;
        HAMLSS_CUDA(cudaEventRecord(ev[slot + 1], s));
        marks.push_back(Mark{name, bytes, (size_t)slot});
        next = slot + 2;
    }
    // Position of the next mark: a solver notes it around each iteration it issues, so it
    // can find that iteration's launches once it knows where the device stopped.
    size_t pos() const { return marks.size(); }
    // Marks [from, to) are launches that their gate turned into no-ops (issued ahead of
    // the device's stop test): they moved no bytes, and are reported as "gated".
    void gated(size_t from, size_t to) {
        for (size_t k = from; k < to && k < marks.size(); ++k) {
            marks[k].name = "gated";
            marks[k].bytes = 0.0;
        }
    }
};

inline size_t prof_pos(const Profiler* p) { return p ? p->pos() : 0; }
inline void prof_gated(Profiler* p, size_t from, size_t to) {
    if (p && from < to) p->gated(from, to);
}

// A stream plus the scratch its reductions use.  Kernels on one lane run in order, so
// one reducer (partials + ticket) per lane is enough.
struct Lane {
    cudaStream_t stream = nullptr;
    DBuf<double> partials;
    DBuf<unsigned> ticket;
    size_t red_cap = 0;       // entries of `partials`
    DBuf<int> err;            // set by a bulk-copy SpMV whose wait ran out (zero otherwise)
    Profiler* prof = nullptr;
    Reducer red() const { return Reducer{partials.p, ticket.p}; }
    // a grid of `blocks` blocks, each storing `nred` partial sums, must fit `partials`
    void red_check(int blocks, int nred) const {
        if ((size_t)blocks * (size_t)(nred > 0 ? nred : 1) > red_cap)
            fail(HAMLSS_ERR_INVALID, "reduction grid exceeds the lane's partial-sum buffer");
    }
};

// Only the outermost scope on a lane is recorded: a setup phase that launches many
// kernels (or calls helpers with scopes of their own) counts once, under its own name.
struct ProfScope {
    const Lane& L;
    long slot;
    const char* name;
    double bytes;
    ProfScope(const Lane& l, const char* nm, double b)
        : L(l), slot(l.prof && l.prof->depth++ == 0 ? l.prof->begin(l.stream) : -1), name(nm), bytes(b) {}
    ~ProfScope() {
        if (!L.prof) return;
        L.prof->end(L.stream, slot, name, bytes);
        --L.prof->depth;
    }
};

struct Ctx {
    int device = 0;
    int sm_count = 148;
    Lane lane;
    Profiler prof;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    HBuf<char> host_poll;      // pinned landing zone for polled device state
    // SpGEMM capacity slots (AMG setup), grown on demand and kept: setups of similar
    // matrices then allocate nothing large (fresh pool memory of GBs maps slowly)
    DBuf<int> gemm_ci;
    DBuf<double> gemm_v;
    std::mutex mu;
};

// Max co-resident blocks of a kernel (cached per kernel instantiation by the caller).
template <typename K>
int occupancy_blocks(K kernel, int threads, size_t dyn_smem = 0) {
    int b = 0;
    HAMLSS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, dyn_smem));
    return b > 0 ? b : 1;
}

constexpr int kMaxBlocksPerSm = 8;
constexpr int kMaxRed = 72;   // widest reduction (multi-dot of an FGMRES basis + 2)

void lane_init(Lane& L, int sm_count);
void lane_destroy(Lane& L);
// Whether a bulk-copy SpMV on the lane gave up waiting for its copies since the last call
// (it then read the matrix from global memory, so its results stand); clears the word.
bool lane_take_timeout(const Lane& L);
// The matrix's row-length profile for hamlss_spmv: when its longest row has more than
// kSkewRow entries and more than kSkewRatio times the average, the rows above
// max(kSkewRow, kSkewRatio x average) are listed (once per matrix; the pattern is fixed).
constexpr int kSkewRow = 1024;
constexpr double kSkewRatio = 32.0;
void ensure_row_profile(Ctx& ctx, hamlss_mat* M);

// Device view of a CSR matrix.
template <typename T>
struct Csr {
    int n = 0, m = 0, nnz = 0;
    const int* rp = nullptr;
    const int* ci = nullptr;
    const T* v = nullptr;
};

// Owning device CSR (structure + FP64 values, FP32 values on demand).
struct DevMat {
    int n = 0, m = 0, nnz = 0;
    DBuf<int> rp, ci;
    DBuf<double> v;
    DBuf<float> v32;
    bool v32_valid = false;
    Csr<double> f64() const { return Csr<double>{n, m, nnz, rp.p, ci.p, v.p}; }
    Csr<float> f32(cudaStream_t s);
};

// Algorithmic bytes of one CSR SpMV pass: row_ptr + (index + value) per nonzero; the
// vector traffic is added by the caller (vec_bytes; default: read x once, write y).
template <typename T>
double csr_bytes(const Csr<T>& A) {
    return 4.0 * (A.n + 1) + (4.0 + sizeof(T)) * (double)A.nnz;
}

// Lanes per row of an SpMV: 1 (the 32-row tiles, the reference's summation order) for FP64
// operands and for short rows; for FP32 operands a group sized to the average row length
// (the mixed-precision inner solves and V-cycles carry no bit-exactness requirement).
template <typename T>
int spmv_group_size(const Csr<T>& A) {
    if (sizeof(T) != sizeof(float) || A.n == 0) return 1;
    // measured on B200 (FP32 Jacobi sweep, banded rows of W entries, cold L2): one lane per
    // row is best up to W ~ 20, four lanes at W ~ 50, eight from W ~ 150
    const double avg = (double)A.nnz / A.n;
    if (avg < 32.0) return 1;
    if (avg < 100.0) return 4;
    return 8;
}

// Lanes per row of the bulk-copy kernel (spmv_stream.cuh), or 0 for the plain kernel.  A
// tile of 256 / G rows should fit one stage (2560 FP32 entries), so G grows with the
// average row length; FP64 keeps G = 1 (each row summed in column order, bit-exact) and so
// takes only the short-row operators.  Small operators (< 32768 rows) stay on the plain
// kernel.
template <typename T>
int stream_group(const Csr<T>& A) {
    if (A.n < 32768) return 0;
    const double avg = (double)A.nnz / A.n;
    if (avg <= 5.5) return 1;
    if (sizeof(T) == 8) return 0;
    if (avg <= 11.0) return 1;
    if (avg <= 22.0) return 2;
    if (avg <= 44.0) return 4;
    if (avg <= 88.0) return 8;
    if (avg <= 176.0) return 16;
    return 0;
}

// FP32 operators with rows longer than the bulk-copy kernel stages (or too few rows for
// it) and at least 48 entries a row on average: a warp per row (k_spmv_long).
template <typename T>
bool long_rows_warp(const Csr<T>& A) {
    return sizeof(T) == 4 && A.n > 0 && (double)A.nnz / A.n >= 48.0;
}

// Max co-resident CTAs of a bulk-copy SpMV instantiation (its dynamic shared memory
// raised above the 48 KB default once).
template <typename K>
int stream_per_sm(K kernel, size_t smem) {
    HAMLSS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return std::min(occupancy_blocks(kernel, kStreamThreads, smem), kMaxBlocksPerSm);
}

template <typename T, int NRED, typename XOp, typename Epi, typename Fin, int G>
void launch_spmv_stream(int sm_count, const Lane& L, const Csr<T>& A, const XOp& xop, const Epi& epi,
                        const Fin& fin, const int* gate, int skip_len) {
    auto kern = k_spmv_stream<T, NRED, XOp, Epi, Fin, G>;
    constexpr size_t smem = StreamShape<T>::smem_bytes;
    static const int per_sm = stream_per_sm(kern, smem);
    const int tiles = ceil_div(A.n, kStreamThreads / G);
    const int blocks = std::max(1, std::min(tiles, sm_count * per_sm));
    if (NRED > 0) L.red_check(blocks, NRED);
    kern<<<blocks, kStreamThreads, smem, L.stream>>>(A.n, A.rp, A.ci, A.v, xop, epi, L.red(), fin, gate,
                                                     L.err.p, skip_len);
    HAMLSS_LAUNCH_CHECK();
}

template <typename T, int NRED, typename XOp, typename Epi, typename Fin = NoFin>
void launch_spmv(int sm_count, const Lane& L, const Csr<T>& A, const XOp& xop, const Epi& epi,
                 const Fin& fin = Fin{}, const int* gate = nullptr, const char* name = "spmv",
                 double vec_bytes = -1.0, int skip_len = INT_MAX) {
    ProfScope ps(L, name, csr_bytes(A) + (vec_bytes >= 0 ? vec_bytes : 2.0 * sizeof(T) * A.n));
    switch (stream_group(A)) {
        case 1: return launch_spmv_stream<T, NRED, XOp, Epi, Fin, 1>(sm_count, L, A, xop, epi, fin, gate, skip_len);
        case 2:
            if constexpr (sizeof(T) == 4)
                return launch_spmv_stream<T, NRED, XOp, Epi, Fin, 2>(sm_count, L, A, xop, epi, fin, gate, skip_len);
            break;
        case 4:
            if constexpr (sizeof(T) == 4)
                return launch_spmv_stream<T, NRED, XOp, Epi, Fin, 4>(sm_count, L, A, xop, epi, fin, gate, skip_len);
            break;
        case 8:
            if constexpr (sizeof(T) == 4)
                return launch_spmv_stream<T, NRED, XOp, Epi, Fin, 8>(sm_count, L, A, xop, epi, fin, gate, skip_len);
            break;
        case 16:
            if constexpr (sizeof(T) == 4)
                return launch_spmv_stream<T, NRED, XOp, Epi, Fin, 16>(sm_count, L, A, xop, epi, fin, gate, skip_len);
            break;
        default: break;
    }
    if constexpr (sizeof(T) == 4) {
        if (long_rows_warp(A)) {
            auto kl = k_spmv_long<T, NRED, XOp, Epi, Fin, 32>;
            static const int per_sm_l = std::min(occupancy_blocks(kl, 256), kMaxBlocksPerSm);
            const int blocks = std::max(1, std::min(ceil_div(A.n, 8), sm_count * per_sm_l));
            if (NRED > 0) L.red_check(blocks, NRED);
            // (FP32 only; the skewed-row split of hamlss_spmv is FP64)
            if (skip_len != INT_MAX) fail(HAMLSS_ERR_INVALID, "long-row split on an FP32 long-row operator");
            kl<<<blocks, 256, 0, L.stream>>>(A.n, A.rp, A.ci, A.v, xop, epi, L.red(), fin, gate);
            HAMLSS_LAUNCH_CHECK();
            return;
        }
    }
    auto kern = k_spmv<T, NRED, XOp, Epi, Fin>;
    // thread-safe one-time initialisation (contexts may be driven from several threads)
    static const int per_sm = std::min(occupancy_blocks(kern, kSpmvThreads), kMaxBlocksPerSm);
    const int gsz = spmv_group_size(A);
    const int rows_per_warp = gsz > 1 ? 32 / gsz : 32;
    const int nwork = ceil_div(A.n, rows_per_warp);
    int blocks = std::max(1, std::min(ceil_div(nwork, kSpmvWarps), sm_count * per_sm));
    if (NRED > 0) L.red_check(blocks, NRED);
    kern<<<blocks, kSpmvThreads, 0, L.stream>>>(A.n, A.rp, A.ci, A.v, xop, epi, L.red(), fin, gate, gsz,
                                                skip_len);
    HAMLSS_LAUNCH_CHECK();
}

template <int NRED, typename Body, typename Fin = NoFin>
void launch_vec(int sm_count, const Lane& L, int n, const Body& body, const Fin& fin = Fin{},
                const int* gate = nullptr, const char* name = "vec", double bytes = 0.0) {
    ProfScope ps(L, name, bytes);
    int blocks = std::max(1, std::min(ceil_div(n, 256), sm_count * kMaxBlocksPerSm));
    if (NRED > 0) L.red_check(blocks, NRED);
    k_vec<NRED, Body, Fin><<<blocks, 256, 0, L.stream>>>(n, body, L.red(), fin, gate);
    HAMLSS_LAUNCH_CHECK();
}

// Buffers a solve needs, cached on the matrix (allocated once per size and kind; the
// solve loops themselves allocate nothing).
struct Workspace {
    DBuf<double> d[8];
    DBuf<float> f[8];
    DBuf<double> basis;     // FGMRES V (m+1) x n and Z m x n
    DBuf<double> small;     // Hessenberg, Givens, scalars
    DBuf<char> state;
};

// Validate a CSR already on the device: row_ptr monotone from 0 to nnz, columns in
// [0, m), strictly increasing within a row.  Returns HAMLSS_OK or HAMLSS_ERR_MALFORMED.
int validate_csr(Ctx& ctx, const Csr<double>& A);

}  // namespace hamlss

// Opaque ABI types.
struct hamlss_ctx {
    hamlss::Ctx c;
};

struct hamlss_mat {
    hamlss_ctx* ctx = nullptr;
    hamlss::DevMat A;
    hamlss::DBuf<double> diag;      // a_ii (0 where the row has no diagonal entry)
    bool diag_valid = false;
    // row-length profile (hamlss::ensure_row_profile): rows longer than long_len, listed in
    // long_rows, are summed by a warp each apart from the rest; n_long < 0: not built yet
    hamlss::DBuf<int> long_rows;
    int n_long = -1;
    int long_len = INT_MAX;
    uint64_t version = 0;           // bumped by hamlss_mat_update_values
    hamlss::Workspace ws;
};
