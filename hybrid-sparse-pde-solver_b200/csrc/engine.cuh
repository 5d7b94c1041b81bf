// engine.cuh -- context, device matrices and launch helpers shared by all solvers.
#pragma once

#include <memory>
#include <mutex>

#include "common.cuh"
#include "spmv.cuh"

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
};

// A stream plus the scratch its reductions use.  Kernels on one lane run in order, so
// one reducer (partials + ticket) per lane is enough.
struct Lane {
    cudaStream_t stream = nullptr;
    DBuf<double> partials;
    DBuf<unsigned> ticket;
    Profiler* prof = nullptr;
    Reducer red() const { return Reducer{partials.p, ticket.p}; }
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
    void* blas = nullptr;      // cuBLAS handle, created on first use (dense coarse LU)
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
constexpr int kPartialCap = 148 * kMaxBlocksPerSm * kMaxRed;

void lane_init(Lane& L, int sm_count);
void lane_destroy(Lane& L);

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

template <typename T, int NRED, typename XOp, typename Epi, typename Fin = NoFin>
void launch_spmv(int sm_count, const Lane& L, const Csr<T>& A, const XOp& xop, const Epi& epi,
                 const Fin& fin = Fin{}, const int* gate = nullptr, const char* name = "spmv",
                 double vec_bytes = -1.0) {
    ProfScope ps(L, name, csr_bytes(A) + (vec_bytes >= 0 ? vec_bytes : 2.0 * sizeof(T) * A.n));
    auto kern = k_spmv<T, NRED, XOp, Epi, Fin>;
    // thread-safe one-time initialisation (contexts may be driven from several threads)
    static const int per_sm = std::min(occupancy_blocks(kern, kSpmvThreads), kMaxBlocksPerSm);
    const int gsz = spmv_group_size(A);
    const int rows_per_warp = gsz > 1 ? 32 / gsz : 32;
    const int nwork = ceil_div(A.n, rows_per_warp);
    int blocks = std::max(1, std::min(ceil_div(nwork, kSpmvWarps), sm_count * per_sm));
    kern<<<blocks, kSpmvThreads, 0, L.stream>>>(A.n, A.rp, A.ci, A.v, xop, epi, L.red(), fin, gate, gsz);
    HAMLSS_LAUNCH_CHECK();
}

template <int NRED, typename Body, typename Fin = NoFin>
void launch_vec(int sm_count, const Lane& L, int n, const Body& body, const Fin& fin = Fin{},
                const int* gate = nullptr, const char* name = "vec", double bytes = 0.0) {
    ProfScope ps(L, name, bytes);
    int blocks = std::max(1, std::min(ceil_div(n, 256), sm_count * kMaxBlocksPerSm));
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
    uint64_t version = 0;           // bumped by hamlss_mat_update_values
    hamlss::Workspace ws;
};
