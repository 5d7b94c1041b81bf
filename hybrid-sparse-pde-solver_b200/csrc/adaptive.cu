// adaptive.cu -- AdaptiveSelector on the device (adaptive_selector.cpp:37-394).
//
// Features: one pass over the rows gathers every row statistic the selector uses
// (Frobenius norm, diagonal dominance, bandwidth, nnz variance, diagonal sign / presence,
// Gershgorin radius, lower/upper counts, zero diagonals, strong-connection count, and the
// sampled symmetry checks); 30 Lanczos steps run as fused SpMV + dot kernels with the
// alpha/beta recurrence on the device.  The host only assembles the 24-entry vector and
// applies select_initial_state (:225-233).
// Ladder: features -> initial state -> attempts CG+Jacobi / FGMRES+ILU(0) / FGMRES+AMG
// with warm starts, escalating when an attempt fails (the reference) or, with
// ladder_mode = 1, as soon as the device-side stall / budget / divergence test fires.
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>

#include "krylov.cuh"

namespace hamlss {

namespace {

constexpr double kEps = 2.220446049250313e-16;

// binary search for a_ji (SparseMatrix::get, sparse_matrix.cpp:40-53)
__device__ double get_entry(const int* rp, const int* ci, const double* v, int i, int j) {
    int lo = rp[i], hi = rp[i + 1];
    while (lo < hi) {
        int mid = lo + (hi - lo) / 2;
        if (ci[mid] < j) lo = mid + 1; else hi = mid;
    }
    return (lo < rp[i + 1] && ci[lo] == j) ? v[lo] : 0.0;
}

// Row statistics.  Sums (Frobenius, nnz variance, strong count) go through the
// deterministic grid reduction; extrema use integer atomics on the bit patterns of
// non-negative doubles.
struct Extrema {
    unsigned long long min_dd;     // bits of min dd (>= 0, +inf when none)
    unsigned long long max_rowsum; // bits of max row |.| sum
    unsigned long long max_asym;   // bits of max |a_ij - a_ji| over the first 200 rows
    unsigned long long min_posdiag;// bits of min diagonal > eps (+inf when none)
    int bandwidth;
    int diag_pos, diag_count, zero_diag;
    long long lo, hi;
    int sym_fail, nonpos_diag;
};

__global__ void k_features(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ v, double mean, int stride, Extrema* ex,
                           Reducer red, double* sums) {
    __shared__ double rsh[8 * 3];
    double acc[3] = {0.0, 0.0, 0.0};
    int bw = 0, dpos = 0, dcnt = 0, zd = 0;
    unsigned symf = 0, npd = 0;
    long long lo = 0, hi = 0;
    double mdd = INFINITY, mrs = 0.0, masym = 0.0, mpd = INFINITY;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = rp[i], e = rp[i + 1];
        double da = 0.0, off = 0.0, rs = 0.0, rmax = 0.0;
        bool has_d = false;
        double dval = 0.0;
        for (int k = s; k < e; ++k) {
            const int j = ci[k];
            const double a = v[k];
            acc[0] += a * a;
            rs += fabs(a);
            int d = abs(i - j);
            bw = max(bw, d);
            if (j == i) { da = fabs(a); if (!has_d) { has_d = true; dval = a; } }
            else { off += fabs(a); rmax = fmax(rmax, fabs(a)); }
            if (j < i) ++lo;
            if (j > i) ++hi;
        }
        double dd = (off > kEps) ? (da / off) : INFINITY;
        mdd = fmin(mdd, dd);
        mrs = fmax(mrs, rs);
        double dl = (double)(e - s) - mean;
        acc[1] += dl * dl;
        if (has_d) {
            ++dcnt;
            if (dval > 0.0) ++dpos;
            if (fabs(dval) <= 1e-15) ++zd;
            if (dval > kEps) mpd = fmin(mpd, dval);
            if (dval <= 0.0) ++npd;
        } else {
            ++zd;
        }
        for (int k = s; k < e; ++k)
            if (ci[k] != i && fabs(v[k]) >= 0.25 * rmax) acc[2] += 1.0;
        const bool first200 = i < 200;
        const bool sampled = (i % stride) == 0;
        if (first200 || sampled) {
            for (int k = s; k < e; ++k) {
                const int j = ci[k];
                if (j == i) continue;
                const double aij = v[k], aji = get_entry(rp, ci, v, j, i);
                if (first200) masym = fmax(masym, fabs(aij - aji));
                if (sampled && fabs(aij - aji) > 1e-6 * (1.0 + fabs(aij))) symf = 1;
            }
        }
    }
    // warp-level pre-reduction, then one set of atomics per warp
    unsigned long long b_mdd = (unsigned long long)__double_as_longlong(mdd);
    unsigned long long b_mrs = (unsigned long long)__double_as_longlong(mrs);
    unsigned long long b_mas = (unsigned long long)__double_as_longlong(masym);
    unsigned long long b_mpd = (unsigned long long)__double_as_longlong(mpd);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        b_mdd = min(b_mdd, __shfl_xor_sync(0xffffffffu, b_mdd, o));
        b_mrs = max(b_mrs, __shfl_xor_sync(0xffffffffu, b_mrs, o));
        b_mas = max(b_mas, __shfl_xor_sync(0xffffffffu, b_mas, o));
        b_mpd = min(b_mpd, __shfl_xor_sync(0xffffffffu, b_mpd, o));
        lo += __shfl_xor_sync(0xffffffffu, lo, o);
        hi += __shfl_xor_sync(0xffffffffu, hi, o);
    }
    bw = __reduce_max_sync(0xffffffffu, bw);
    dpos = __reduce_add_sync(0xffffffffu, dpos);
    dcnt = __reduce_add_sync(0xffffffffu, dcnt);
    zd = __reduce_add_sync(0xffffffffu, zd);
    symf = __reduce_or_sync(0xffffffffu, symf);
    npd = __reduce_or_sync(0xffffffffu, npd);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&ex->min_dd, b_mdd);
        atomicMax(&ex->max_rowsum, b_mrs);
        atomicMax(&ex->max_asym, b_mas);
        atomicMin(&ex->min_posdiag, b_mpd);
        atomicMax(&ex->bandwidth, bw);
        atomicAdd(&ex->diag_pos, dpos);
        atomicAdd(&ex->diag_count, dcnt);
        atomicAdd(&ex->zero_diag, zd);
        atomicAdd((unsigned long long*)&ex->lo, (unsigned long long)lo);
        atomicAdd((unsigned long long*)&ex->hi, (unsigned long long)hi);
        if (symf) atomicOr(&ex->sym_fail, 1);
        if (npd) atomicOr(&ex->nonpos_diag, 1);
    }
    double tot[3];
    if (grid_reduce<3>(red, acc, rsh, tot)) { sums[0] = tot[0]; sums[1] = tot[1]; sums[2] = tot[2]; }
}

// ----------------------------------------------------------------------- Lanczos
struct LzState {
    double alpha[32], beta[32];
    double beta_prev;    // beta_j of the recurrence
    int na, nb, halt;
};

struct EpiLz {
    const double* q;
    double* Aq;
    double* terms;     // set: store the terms for an in-order sum (k_lz_seq_sum)
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        Aq[i] = ax;
        const double t = __dmul_rn(q[i], ax);
        if (terms) terms[i] = t;
        else acc[0] += t;
    }
};

struct FinAlpha {
    LzState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const { s->alpha[s->na++] = t[0]; }
};

// Aq -= alpha q + beta q_prev ; ||Aq||^2       (adaptive_selector.cpp:80-82)
struct BodyLzUpd {
    double* Aq;
    const double* q;
    const double* qp;
    const LzState* s;
    double a, b;
    double* terms;
    __device__ __forceinline__ void load() { a = s->alpha[s->na - 1]; b = s->beta_prev; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&acc)[NV]) const {
        const double t = __dsub_rn(Aq[i], __dadd_rn(__dmul_rn(a, q[i]), __dmul_rn(b, qp[i])));
        Aq[i] = t;
        const double tt = __dmul_rn(t, t);
        if (terms) terms[i] = tt;
        else acc[0] += tt;
    }
};

// Systems of at most kLzSeqRows rows: the stored terms added in row order by one thread
// (the reference's sequential dot / norm), then the finaliser.
constexpr int kLzSeqRows = 1 << 15;

template <typename Fin>
__global__ void k_lz_seq_sum(int n, const double* __restrict__ terms, Fin fin, const int* gate) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || *(volatile const int*)gate) return;
    double acc = 0.0;
    for (int i = 0; i < n; ++i) acc = __dadd_rn(acc, terms[i]);
    const double t[1] = {acc};
    fin(t);
}

struct FinBeta {
    LzState* s;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const {
        double bj = sqrt(t[0]);
        s->beta_prev = bj;
        if (bj < kEps * 1e6) { s->halt = 1; return; }
        s->beta[s->nb++] = bj;
    }
};

// q_prev = q ; q = Aq / beta
struct BodyLzShift {
    double* q;
    double* qp;
    const double* Aq;
    const LzState* s;
    double inv;
    __device__ __forceinline__ void load() { inv = 1.0 / s->beta_prev; }
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const {
        qp[i] = q[i];
        q[i] = Aq[i] * inv;
    }
};

struct BodyInit {
    double* q;
    double* qp;
    double val;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const { q[i] = val; qp[i] = 0.0; }
};

double bits_to_double(unsigned long long b) {
    double d;
    std::memcpy(&d, &b, sizeof(d));
    return d;
}

// K Lanczos steps from the uniform vector (the recurrence of adaptive_selector.cpp:66-89
// and sparse_matrix.cpp:451-468, as fused SpMV + dot kernels), then the Gershgorin bounds
// of the tridiagonal T (adaptive_selector.cpp:91-101, sparse_matrix.cpp:469-478).
void lanczos_bounds(Ctx& ctx, hamlss_mat* A, int K, double* tmin_out, double* tmax_out) {
    const int n = A->A.n;
    const Lane& L = ctx.lane;
    cudaStream_t st = L.stream;
    Workspace& ws = A->ws;
    double* q = (ws.d[0].ensure(n), ws.d[0].p);
    double* qp = (ws.d[1].ensure(n), ws.d[1].p);
    double* Aq = (ws.d[2].ensure(n), ws.d[2].p);
    DBuf<char> lzb(sizeof(LzState));
    LzState* lz = reinterpret_cast<LzState*>(lzb.p);
    HAMLSS_CUDA(cudaMemsetAsync(lz, 0, sizeof(LzState), st));
    launch_vec<0>(ctx.sm_count, L, n, BodyInit{q, qp, 1.0 / std::sqrt((double)n)});
    DBuf<double> term_buf;
    double* terms = nullptr;
    if (n <= kLzSeqRows) {
        term_buf.ensure((size_t)std::max(n, 1));
        terms = term_buf.p;
    }
    // with terms, the launches' own grid sums are unused (NoFin) and k_lz_seq_sum finishes
    for (int j = 0; j < K; ++j) {
        if (terms) {
            launch_spmv<double, 1>(ctx.sm_count, L, A->A.f64(), XVec<double>{q}, EpiLz{q, Aq, terms}, NoFin{},
                                   &lz->halt, "features_spmv", 24.0 * n);
            k_lz_seq_sum<<<1, 32, 0, st>>>(n, terms, FinAlpha{lz}, &lz->halt);
            HAMLSS_LAUNCH_CHECK();
            launch_vec<1>(ctx.sm_count, L, n, BodyLzUpd{Aq, q, qp, lz, 0.0, 0.0, terms}, NoFin{}, &lz->halt,
                          "features", 32.0 * n);
            k_lz_seq_sum<<<1, 32, 0, st>>>(n, terms, FinBeta{lz}, &lz->halt);
            HAMLSS_LAUNCH_CHECK();
        } else {
            launch_spmv<double, 1>(ctx.sm_count, L, A->A.f64(), XVec<double>{q}, EpiLz{q, Aq, nullptr},
                                   FinAlpha{lz}, &lz->halt, "features_spmv", 24.0 * n);
            launch_vec<1>(ctx.sm_count, L, n, BodyLzUpd{Aq, q, qp, lz, 0.0, 0.0, nullptr}, FinBeta{lz},
                          &lz->halt, "features", 32.0 * n);
        }
        launch_vec<0>(ctx.sm_count, L, n, BodyLzShift{q, qp, Aq, lz, 0.0}, NoFin{}, &lz->halt,
                      "features", 32.0 * n);
    }
    LzState hl;
    HAMLSS_CUDA(cudaMemcpyAsync(&hl, lz, sizeof(hl), cudaMemcpyDeviceToHost, st));
    HAMLSS_CUDA(cudaStreamSynchronize(st));
    int sz = hl.na;
    double tmin = hl.alpha[0], tmax = hl.alpha[0];
    for (int i = 0; i < sz; ++i) {
        double r = 0.0;
        if (i > 0) r += std::fabs(hl.beta[i - 1]);
        if (i < sz - 1) r += std::fabs(hl.beta[i]);
        tmin = std::min(tmin, hl.alpha[i] - r);
        tmax = std::max(tmax, hl.alpha[i] + r);
    }
    *tmin_out = tmin;
    *tmax_out = tmax;
}

}  // namespace

void spectral_interval(Ctx& ctx, hamlss_mat* A, int steps, double* lo, double* hi) {
    lanczos_bounds(ctx, A, std::min(A->A.n, steps), lo, hi);
}

int extract_features(Ctx& ctx, hamlss_mat* A, double feat[24], int* initial_state) {
    const int n = A->A.n;
    const int nnz = A->A.nnz;
    if (n == 0) fail(HAMLSS_ERR_INVALID, "features of an empty matrix");
    const Lane& L = ctx.lane;
    cudaStream_t st = L.stream;
    ProfScope ps(L, "features", 0.0);
    // ---- row statistics
    DBuf<char> exbuf(sizeof(Extrema));
    Extrema h0{};
    h0.min_dd = 0x7ff0000000000000ULL;       // +inf
    h0.min_posdiag = 0x7ff0000000000000ULL;
    HAMLSS_CUDA(cudaMemcpyAsync(exbuf.p, &h0, sizeof(h0), cudaMemcpyHostToDevice, st));
    DBuf<double> sums(4);
    const int sample_rows = std::min(200, n);
    const int stride = std::max(1, n / sample_rows);
    const double mean = (double)nnz / n;
    int blocks = std::max(1, std::min(ceil_div(n, 256), ctx.sm_count * 8));
    L.red_check(blocks, 3);
    k_features<<<blocks, 256, 0, st>>>(n, A->A.rp.p, A->A.ci.p, A->A.v.p, mean, stride,
                                       reinterpret_cast<Extrema*>(exbuf.p), L.red(), sums.p);
    HAMLSS_LAUNCH_CHECK();
    double tmin = 0.0, tmax = 0.0;
    lanczos_bounds(ctx, A, std::min(n, 30), &tmin, &tmax);     // adaptive_selector.cpp:66-101
    Extrema ex;
    double hs[3];
    HAMLSS_CUDA(cudaMemcpyAsync(&ex, exbuf.p, sizeof(ex), cudaMemcpyDeviceToHost, st));
    HAMLSS_CUDA(cudaMemcpyAsync(hs, sums.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
    HAMLSS_CUDA(cudaStreamSynchronize(st));
    // ---- assemble (adaptive_selector.cpp:37-220)
    const double fro = std::sqrt(hs[0]);
    double min_dd = bits_to_double(ex.min_dd);
    const double diag_dom = std::isinf(min_dd) ? 1.0 : min_dd;
    double lam_max = std::max(tmax, kEps);
    double lam_min = tmin;
    if (lam_min <= kEps) {
        double mpd = bits_to_double(ex.min_posdiag);
        if (std::isinf(mpd)) mpd = kEps;
        lam_min = mpd * 0.5;
    }
    lam_min = std::max(lam_min, kEps);
    const double cond = lam_max / lam_min;
    const double avg = (double)nnz / n;
    const double var = hs[1] / n;
    const double dsf = (double)ex.diag_pos / std::max(n, 1);
    const double masym = bits_to_double(ex.max_asym);
    const double ods = (fro > kEps) ? masym / fro : 0.0;
    const double grad = bits_to_double(ex.max_rowsum);
    const double dfrac = nnz == 0 ? 0.0 : (double)ex.diag_count / nnz;
    const double lur = ex.hi > 0 ? (double)ex.lo / (double)ex.hi : 1.0;
    const double coarsen = 1.0 / (1.0 + hs[2] / n);
    int depth = (int)std::log2((double)n / 50.0);
    if (depth < 1) depth = 1;
    const double af = 2e-10, am = 5e-9;
    const double it_easy = std::min(std::sqrt(cond) * 0.5, 5000.0);
    const double it_hard = std::min(std::log(cond + 1.0) * 5.0, 200.0);
    const bool spd = !ex.sym_fail && !ex.nonpos_diag;
    double f[24] = {(double)n, (double)nnz, (double)nnz / ((double)n * n), diag_dom, ods, fro, cond,
                    spd ? 1.0 : 0.0, (double)ex.bandwidth, avg, var, dsf, ods, lam_max,
                    std::max(lam_min, kEps), grad, dfrac, lur, (double)ex.zero_diag, 1.0, coarsen,
                    (double)depth, it_easy * (af * 2.0 * nnz + am * 2.0 * n * 8),
                    it_hard * (af * 2.0 * nnz + am * 2.0 * n * 8)};
    std::memcpy(feat, f, sizeof(f));
    int s;
    if (spd && cond < 1e6 && diag_dom >= 0.8) s = HAMLSS_STATE_EASY;
    else if (cond >= 1e6 || diag_dom < 0.3) s = HAMLSS_STATE_HARD;
    else s = HAMLSS_STATE_MODERATE;
    if (initial_state) *initial_state = s;
    return HAMLSS_OK;
}

}  // namespace hamlss
