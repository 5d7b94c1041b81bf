// capi.cu -- the extern "C" boundary (include/hamlss.h).  Every entry point catches
// engine errors and returns a HAMLSS_ERR_* code; hamlss_last_error() explains it.
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "batch.cuh"
#include "dense_lu.cuh"
#include "krylov.cuh"
#include "nvml_energy.cuh"

using namespace hamlss;

namespace {

thread_local std::string g_err;

int set_err(int code, const std::string& m) {
    g_err = m;
    return code;
}

template <typename F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const Error& e) {
        return set_err(e.code, e.what());
    } catch (const std::bad_alloc&) {
        return set_err(HAMLSS_ERR_NOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        return set_err(HAMLSS_ERR_INVALID, e.what());
    }
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// flop_model (energy_monitor.hpp:163-177)
long long spmv_flops(long long nz) { return 2LL * nz; }
long long spmv_bytes(long long n, long long nz) { return (n + 1 + nz) * 4 + nz * 8 + n * 16; }

void cg_cost(long long n, long long nz, const SolveResult& r, long long* flops, long long* bytes) {
    long long trips = r.iterations, partial = 0;
    if (r.converged && trips > 0) { partial = 1; trips -= 1; }
    long long restart_trips = std::min<long long>(r.restarts, trips);
    trips -= restart_trips;
    long long f_full = spmv_flops(nz) + 2 * n + 2 * (2 * n) + 2 * n + 2 * n;
    long long b_full = spmv_bytes(n, nz) + 16 * n + 2 * (24 * n) + 16 * n + 24 * n;
    long long f_part = spmv_flops(nz) + 2 * n + 2 * (2 * n);
    long long b_part = spmv_bytes(n, nz) + 16 * n + 2 * (24 * n);
    long long f_rs = spmv_flops(nz) + 2 * n, b_rs = spmv_bytes(n, nz) + 16 * n;
    *flops = trips * f_full + partial * f_part + restart_trips * f_rs;
    *bytes = trips * b_full + partial * b_part + restart_trips * b_rs;
}

void fgmres_cost(long long n, long long nz, const SolveResult& r, long long* flops, long long* bytes) {
    *flops = (long long)r.iterations * (spmv_flops(nz) + 4 * n);
    *bytes = (long long)r.iterations * (spmv_bytes(n, nz) + 4 * n * 8);
}

}  // namespace

namespace hamlss {
int set_last_error(int code, const std::string& msg) { return set_err(code, msg); }
}  // namespace hamlss

extern "C" {

const char* hamlss_version(void) { return "hamlss-b200 0.1 (sm_100a)"; }
const char* hamlss_last_error(void) { return g_err.c_str(); }

void hamlss_params_default(hamlss_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->tol = 1e-8;
    p->max_iter = 2000;
    p->restart_size = 50;
    p->drop_tol = 1e-4;
    p->amg_levels = 10;
    p->amg_strength = 0.25;
    p->amg_strong = 0.25;
    p->amg_smooth_pre = 2;
    p->amg_smooth_post = 2;
    p->stall_window = 15;
    p->stall_threshold = 0.95;
    p->print_every = 25;
    p->sstep_k = 1;
    p->sstep_cond_tol = 1e12;
    p->async_max_stale = 3;
    p->block_size = 1;
    p->precision = HAMLSS_FP64;
    p->ir_inner_tol = 1e-5;
    p->ir_max_outer = 30;
    p->amg_omega = 0.67;
    p->amg_coarse_limit = 50;
    p->jacobi_omega = 1.0;
    p->ladder_mode = 0;
    p->check_every = 8;
    p->ir_update = 1e-2;
}

// ------------------------------------------------------------------------ context
int hamlss_ctx_create(int device, hamlss_ctx** out) {
    return guarded([&]() -> int {
        if (!out) return set_err(HAMLSS_ERR_INVALID, "out is null");
        int count = 0;
        HAMLSS_CUDA(cudaGetDeviceCount(&count));
        if (device < 0 || device >= count) return set_err(HAMLSS_ERR_INVALID, "no such device");
        HAMLSS_CUDA(cudaSetDevice(device));
        auto* c = new hamlss_ctx();
        c->c.device = device;
        HAMLSS_CUDA(cudaDeviceGetAttribute(&c->c.sm_count, cudaDevAttrMultiProcessorCount, device));
        pool_keep_memory(device);
        lane_init(c->c.lane, c->c.sm_count);
        c->c.lane.prof = &c->c.prof;
        HAMLSS_CUDA(cudaEventCreate(&c->c.ev0));
        HAMLSS_CUDA(cudaEventCreate(&c->c.ev1));
        c->c.host_poll.alloc(4096);
        *out = c;
        return HAMLSS_OK;
    });
}

int hamlss_ctx_destroy(hamlss_ctx* ctx) {
    return guarded([&]() -> int {
        if (!ctx) return HAMLSS_OK;
        cudaSetDevice(ctx->c.device);
        lane_destroy(ctx->c.lane);
        for (auto e : ctx->c.prof.ev) cudaEventDestroy(e);
        if (ctx->c.ev0) cudaEventDestroy(ctx->c.ev0);
        if (ctx->c.ev1) cudaEventDestroy(ctx->c.ev1);
        delete ctx;
        return HAMLSS_OK;
    });
}

int hamlss_ctx_synchronize(hamlss_ctx* ctx) {
    return guarded([&]() -> int {
        if (!ctx) return set_err(HAMLSS_ERR_INVALID, "ctx is null");
        HAMLSS_CUDA(cudaStreamSynchronize(ctx->c.lane.stream));
        return HAMLSS_OK;
    });
}

int hamlss_ctx_stream(hamlss_ctx* ctx, void** stream) {
    if (!ctx || !stream) return set_err(HAMLSS_ERR_INVALID, "null argument");
    *stream = (void*)ctx->c.lane.stream;
    return HAMLSS_OK;
}

int hamlss_profile_enable(hamlss_ctx* ctx, int enable, int32_t max_launches) {
    return guarded([&]() -> int {
        if (!ctx) return set_err(HAMLSS_ERR_INVALID, "null context");
        Profiler& P = ctx->c.prof;
        HAMLSS_CUDA(cudaStreamSynchronize(ctx->c.lane.stream));
        P.marks.clear();
        P.next = 0;
        P.on = enable != 0;
        if (P.on) P.reserve(std::max(1, max_launches));
        return HAMLSS_OK;
    });
}

int hamlss_profile_read(hamlss_ctx* ctx, int32_t cap, char* names, int32_t* launches,
                        double* total_ms, double* total_bytes, int32_t* count) {
    return guarded([&]() -> int {
        if (!ctx || !count) return set_err(HAMLSS_ERR_INVALID, "null argument");
        Profiler& P = ctx->c.prof;
        HAMLSS_CUDA(cudaStreamSynchronize(ctx->c.lane.stream));
        std::vector<std::string> fam;
        std::vector<int> nl;
        std::vector<double> ms, by;
        for (auto& m : P.marks) {
            float t = 0.f;
            HAMLSS_CUDA(cudaEventElapsedTime(&t, P.ev[m.e0], P.ev[m.e0 + 1]));
            size_t k = 0;
            while (k < fam.size() && fam[k] != m.name) ++k;
            if (k == fam.size()) { fam.push_back(m.name); nl.push_back(0); ms.push_back(0); by.push_back(0); }
            nl[k] += 1;
            ms[k] += t;
            by[k] += m.bytes;
        }
        int32_t c = 0;
        for (size_t k = 0; k < fam.size() && c < cap; ++k, ++c) {
            if (names) { std::strncpy(names + 32 * c, fam[k].c_str(), 31); names[32 * c + 31] = 0; }
            if (launches) launches[c] = nl[k];
            if (total_ms) total_ms[c] = ms[k];
            if (total_bytes) total_bytes[c] = by[k];
        }
        *count = c;
        return HAMLSS_OK;
    });
}

int hamlss_energy_read(int device, double* joules) {
    return guarded([&]() -> int {
        if (!joules) return set_err(HAMLSS_ERR_INVALID, "null argument");
        *joules = 0.0;
        if (!nvml_energy_available(device))
            return set_err(HAMLSS_ERR_NOT_READY, "NVML energy counter not available for this device");
        *joules = nvml_energy_j(device);
        return HAMLSS_OK;
    });
}

// ------------------------------------------------------------------------- matrix
int hamlss_mat_upload(hamlss_ctx* ctx, int32_t rows, int32_t cols, int32_t nnz,
                      const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                      int where, hamlss_mat** out) {
    return guarded([&]() -> int {
        if (!ctx || !out || rows < 0 || cols < 0 || nnz < 0 || !row_ptr ||
            (nnz > 0 && (!col_idx || !values)))
            return set_err(HAMLSS_ERR_INVALID, "hamlss_mat_upload: bad arguments");
        HAMLSS_CUDA(cudaSetDevice(ctx->c.device));
        // the matrix, and the workspaces later cached on it, come from the device's
        // stream-ordered pool: a serving loop that uploads and releases a matrix per request
        // then reuses memory instead of mapping and unmapping it each time
        AllocScope scope(ctx->c.lane.stream);
        auto* M = new hamlss_mat();
        M->ctx = ctx;
        DevMat& A = M->A;
        A.n = rows;
        A.m = cols;
        A.nnz = nnz;
        cudaStream_t s = ctx->c.lane.stream;
        A.rp.ensure((size_t)rows + 1);
        A.ci.ensure(nnz);
        A.v.ensure(nnz);
        auto kind = where == HAMLSS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        HAMLSS_CUDA(cudaMemcpyAsync(A.rp.p, row_ptr, sizeof(int) * ((size_t)rows + 1), kind, s));
        if (nnz) {
            HAMLSS_CUDA(cudaMemcpyAsync(A.ci.p, col_idx, sizeof(int) * (size_t)nnz, kind, s));
            HAMLSS_CUDA(cudaMemcpyAsync(A.v.p, values, sizeof(double) * (size_t)nnz, kind, s));
        }
        int rc = validate_csr(ctx->c, A.f64());
        if (rc != HAMLSS_OK) {
            delete M;
            return set_err(rc, "hamlss_mat_upload: malformed CSR (row_ptr, column range or "
                               "unsorted/duplicate columns)");
        }
        *out = M;
        return HAMLSS_OK;
    });
}

int hamlss_mat_update_values(hamlss_mat* M, const double* values, int where) {
    return guarded([&]() -> int {
        if (!M || (M->A.nnz && !values)) return set_err(HAMLSS_ERR_INVALID, "null argument");
        auto kind = where == HAMLSS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        if (M->A.nnz)
            HAMLSS_CUDA(cudaMemcpyAsync(M->A.v.p, values, sizeof(double) * M->A.nnz, kind,
                                        M->ctx->c.lane.stream));
        M->A.v32_valid = false;
        M->diag_valid = false;
        M->version++;
        return HAMLSS_OK;
    });
}

int hamlss_mat_info(const hamlss_mat* M, int32_t* rows, int32_t* cols, int32_t* nnz) {
    if (!M) return set_err(HAMLSS_ERR_INVALID, "null matrix");
    if (rows) *rows = M->A.n;
    if (cols) *cols = M->A.m;
    if (nnz) *nnz = M->A.nnz;
    return HAMLSS_OK;
}

int hamlss_mat_download(const hamlss_mat* M, int32_t* row_ptr, int32_t* col_idx, double* values) {
    return guarded([&]() -> int {
        if (!M) return set_err(HAMLSS_ERR_INVALID, "null matrix");
        cudaStream_t s = M->ctx->c.lane.stream;
        if (row_ptr) M->A.rp.download(row_ptr, (size_t)M->A.n + 1, s);
        if (col_idx) M->A.ci.download(col_idx, M->A.nnz, s);
        if (values) M->A.v.download(values, M->A.nnz, s);
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        return HAMLSS_OK;
    });
}

int hamlss_mat_release(hamlss_mat* M) {
    return guarded([&]() -> int {
        if (!M) return HAMLSS_OK;
        cudaStreamSynchronize(M->ctx->c.lane.stream);
        AllocScope scope(M->ctx->c.lane.stream);     // pooled buffers go back on this stream
        delete M;
        return HAMLSS_OK;
    });
}

// ------------------------------------------------------------------ SpMV / BLAS-1
}  // extern "C"

namespace {
struct BodyDot {
    const double* x;
    const double* y;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&acc)[NV]) const { acc[0] += x[i] * y[i]; }
};
struct FinStore1 {
    double* out;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const { out[0] = t[0]; }
};
struct BodyAxpby {
    double a, b;
    const double* x;
    double* y;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const {
        // Vector::axpby (vector.cpp:82-89): y = a*x + b*y, no fused multiply-add
        y[i] = __dadd_rn(__dmul_rn(a, x[i]), __dmul_rn(b, y[i]));
    }
};
struct BodyAxpy {
    double a;
    const double* x;
    double* y;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const {
        y[i] = __dadd_rn(y[i], __dmul_rn(a, x[i]));   // vector.cpp:79
    }
};
struct BodyScale {
    double a;
    double* x;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&)[NV]) const { x[i] = __dmul_rn(x[i], a); }
};

int dot_impl(hamlss_ctx* ctx, int32_t n, const double* x, const double* y, double* result) {
    if (!ctx || n < 0 || !result || (n && (!x || !y))) return set_err(HAMLSS_ERR_INVALID, "bad arguments");
    Ctx& c = ctx->c;
    DBuf<double> out(1);
    out.zero(c.lane.stream);
    if (n) launch_vec<1>(c.sm_count, c.lane, n, BodyDot{x, y}, FinStore1{out.p});
    out.download(result, 1, c.lane.stream);
    HAMLSS_CUDA(cudaStreamSynchronize(c.lane.stream));
    return HAMLSS_OK;
}
}  // namespace

extern "C" {

int hamlss_spmv(hamlss_ctx* ctx, const hamlss_mat* A, const double* x, double* y, int where) {
    return guarded([&]() -> int {
        if (!ctx || !A || (A->A.n && (!x || !y))) return set_err(HAMLSS_ERR_INVALID, "null argument");
        Ctx& c = ctx->c;
        cudaStream_t s = c.lane.stream;
        auto* Am = const_cast<hamlss_mat*>(A);
        const double* dx = x;
        double* dy = y;
        Workspace& ws = Am->ws;
        if (where == HAMLSS_HOST) {
            ws.d[6].upload(x, A->A.m, s);
            ws.d[7].ensure(A->A.n);
            dx = ws.d[6].p;
            dy = ws.d[7].p;
        }
        if (A->A.n) {
            // a skewed row-length profile: the few very long rows by a warp each (still in
            // column order), the rest by the usual kernels, which skip them
            ensure_row_profile(c, Am);
            launch_spmv<double, 0>(c.sm_count, c.lane, A->A.f64(), XVec<double>{dx}, EpiStore<double>{dy},
                                   NoFin{}, nullptr, "spmv", -1.0, Am->long_len);
            if (Am->n_long > 0) {
                const int g = std::max(1, std::min(ceil_div(Am->n_long, kSeqRowWarps), c.sm_count * 8));
                k_spmv_rows_seq<double><<<g, 32 * kSeqRowWarps, 0, s>>>(Am->long_rows.p, Am->n_long, A->A.rp.p,
                                                                        A->A.ci.p, A->A.v.p, XVec<double>{dx},
                                                                        EpiStore<double>{dy});
                HAMLSS_LAUNCH_CHECK();
            }
        }
        if (where == HAMLSS_HOST) ws.d[7].download(y, A->A.n, s);
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        if (lane_take_timeout(c.lane))
            return set_err(HAMLSS_ERR_TIMEOUT, "an SpMV gave up waiting for its bulk copies");
        return HAMLSS_OK;
    });
}

int hamlss_dot(hamlss_ctx* ctx, int32_t n, const double* x, const double* y, double* result) {
    return guarded([&]() -> int { return dot_impl(ctx, n, x, y, result); });
}

int hamlss_norm2(hamlss_ctx* ctx, int32_t n, const double* x, double* result) {
    return guarded([&]() -> int {
        int rc = dot_impl(ctx, n, x, x, result);
        if (rc == HAMLSS_OK) *result = std::sqrt(*result);
        return rc;
    });
}

int hamlss_axpy(hamlss_ctx* ctx, int32_t n, double alpha, const double* x, double* y) {
    return guarded([&]() -> int {
        if (!ctx || n < 0 || (n && (!x || !y))) return set_err(HAMLSS_ERR_INVALID, "bad arguments");
        if (n) launch_vec<0>(ctx->c.sm_count, ctx->c.lane, n, BodyAxpy{alpha, x, y});
        HAMLSS_CUDA(cudaStreamSynchronize(ctx->c.lane.stream));
        return HAMLSS_OK;
    });
}

int hamlss_axpby(hamlss_ctx* ctx, int32_t n, double a, const double* x, double b, double* y) {
    return guarded([&]() -> int {
        if (!ctx || n < 0 || (n && (!x || !y))) return set_err(HAMLSS_ERR_INVALID, "bad arguments");
        if (n) launch_vec<0>(ctx->c.sm_count, ctx->c.lane, n, BodyAxpby{a, b, x, y});
        HAMLSS_CUDA(cudaStreamSynchronize(ctx->c.lane.stream));
        return HAMLSS_OK;
    });
}

int hamlss_scale(hamlss_ctx* ctx, int32_t n, double alpha, double* x) {
    return guarded([&]() -> int {
        if (!ctx || n < 0 || (n && !x)) return set_err(HAMLSS_ERR_INVALID, "bad arguments");
        if (n) launch_vec<0>(ctx->c.sm_count, ctx->c.lane, n, BodyScale{alpha, x});
        HAMLSS_CUDA(cudaStreamSynchronize(ctx->c.lane.stream));
        return HAMLSS_OK;
    });
}

// ---------------------------------------------------------------- preconditioners
int hamlss_precond_setup(hamlss_ctx* ctx, const hamlss_mat* A, int kind,
                         const hamlss_params* params, hamlss_prec** out, double* setup_time_s) {
    return guarded([&]() -> int {
        if (!ctx || !A || !out) return set_err(HAMLSS_ERR_INVALID, "null argument");
        hamlss_params p;
        if (params) p = *params; else hamlss_params_default(&p);
        *out = nullptr;
        AllocScope scope(ctx->c.lane.stream);
        double t0 = now_s();
        auto* Am = const_cast<hamlss_mat*>(A);
        std::unique_ptr<Prec> P;
        switch (kind) {
            case HAMLSS_PREC_NONE:
                if (setup_time_s) *setup_time_s = 0.0;
                return HAMLSS_OK;
            case HAMLSS_PREC_JACOBI:
                P = make_jacobi(ctx->c, Am, p.jacobi_omega);
                break;
            case HAMLSS_PREC_ILU:
                P = make_ilu(ctx->c, Am, p);
                break;
            case HAMLSS_PREC_AMG:
                P = make_amg(ctx->c, Am, p);
                break;
            default:
                return set_err(HAMLSS_ERR_INVALID, "SolverFactory: unknown PrecondType");
        }
        HAMLSS_CUDA(cudaStreamSynchronize(ctx->c.lane.stream));
        auto* h = new hamlss_prec();
        h->ctx = ctx;
        h->A = Am;
        h->p = std::move(P);
        *out = h;
        if (setup_time_s) *setup_time_s = now_s() - t0;
        return HAMLSS_OK;
    });
}

int hamlss_precond_apply(hamlss_ctx* ctx, const hamlss_prec* M, const double* r, double* z,
                         int where) {
    return guarded([&]() -> int {
        if (!ctx || !M || !r || !z) return set_err(HAMLSS_ERR_INVALID, "null argument");
        Ctx& c = ctx->c;
        cudaStream_t s = c.lane.stream;
        AllocScope scope(s);
        const int n = M->p->n;
        Workspace& ws = M->A->ws;
        const double* dr = r;
        double* dz = z;
        if (where == HAMLSS_HOST) {
            ws.d[6].upload(r, n, s);
            ws.d[7].ensure(n);
            dr = ws.d[6].p;
            dz = ws.d[7].p;
        }
        M->p->apply(c, c.lane, dr, dz, nullptr);
        if (where == HAMLSS_HOST) ws.d[7].download(z, n, s);
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        return HAMLSS_OK;
    });
}

int hamlss_precond_type(const hamlss_prec* M, int32_t* kind) {
    if (!M || !kind) return set_err(HAMLSS_ERR_INVALID, "null argument");
    *kind = M->p->kind;
    return HAMLSS_OK;
}

int hamlss_precond_release(hamlss_prec* M) {
    return guarded([&]() -> int {
        if (!M) return HAMLSS_OK;
        cudaStreamSynchronize(M->ctx->c.lane.stream);
        AllocScope scope(M->ctx->c.lane.stream);
        delete M;
        return HAMLSS_OK;
    });
}

int hamlss_amg_aggregate(hamlss_ctx* ctx, const hamlss_mat* A, double theta, int32_t* agg,
                         int32_t* n_agg) {
    return guarded([&]() -> int {
        if (!ctx || !A || !agg || !n_agg) return set_err(HAMLSS_ERR_INVALID, "null argument");
        return amg_aggregate_matrix(ctx->c, const_cast<hamlss_mat*>(A), theta, agg, n_agg);
    });
}

int hamlss_amg_num_levels(const hamlss_prec* M, int32_t* levels) {
    if (!M || !levels) return set_err(HAMLSS_ERR_INVALID, "null argument");
    int rc = amg_num_levels(M->p.get(), levels);
    return rc ? set_err(rc, "not an AMG preconditioner") : HAMLSS_OK;
}

int hamlss_amg_level_matrix(const hamlss_prec* M, int32_t level, int32_t which, int32_t* rows,
                            int32_t* cols, int32_t* nnz, int32_t* row_ptr, int32_t* col_idx,
                            double* values) {
    return guarded([&]() -> int {
        if (!M) return set_err(HAMLSS_ERR_INVALID, "null argument");
        int rc = amg_level_matrix(M->p.get(), level, which, rows, cols, nnz, row_ptr, col_idx, values,
                                  M->ctx->c.lane.stream);
        return rc ? set_err(rc, "no such AMG level / operator") : HAMLSS_OK;
    });
}

int hamlss_ilu_factors(const hamlss_prec* M, double* lu_values) {
    return guarded([&]() -> int {
        if (!M || !lu_values) return set_err(HAMLSS_ERR_INVALID, "null argument");
        return ilu_copy_factors(M->p.get(), lu_values, M->ctx->c.lane.stream);
    });
}

int hamlss_ilu_factor_csr(const hamlss_prec* M, int32_t* nnz, int32_t* row_ptr, int32_t* col_idx,
                          double* values) {
    return guarded([&]() -> int {
        if (!M || !nnz) return set_err(HAMLSS_ERR_INVALID, "null argument");
        const int rc = ilu_factor_csr(M->p.get(), nnz, row_ptr, col_idx, values, M->ctx->c.lane.stream);
        return rc ? set_err(rc, "not an ILU preconditioner") : HAMLSS_OK;
    });
}

int hamlss_ilu_levels(const hamlss_prec* M, int32_t which, int32_t* level, int32_t* n_levels) {
    return guarded([&]() -> int {
        if (!M || !level || !n_levels || (which != 0 && which != 1))
            return set_err(HAMLSS_ERR_INVALID, "bad arguments");
        return ilu_copy_levels(M->p.get(), which, level, n_levels, M->ctx->c.lane.stream);
    });
}

// -------------------------------------------------------------------------- solve
}  // extern "C"

namespace {

// One solve attempt with the given solver / preconditioner on device vectors.
SolveResult solve_core(Ctx& c, int solver, hamlss_mat* Am, Prec* P, const double* db, double* dx,
                       const hamlss_params& p, const LadderCfg* lad, int* outer) {
    *outer = 1;
    Workspace& ws = Am->ws;
    if (solver == HAMLSS_SOLVER_SSTEP_CG) return sstep_solve(c, Am, db, dx, p, ws);   // FP64 only
    if (p.precision == HAMLSS_MIXED) {
        const int inner = solver == HAMLSS_SOLVER_PIPELINED_FGMRES ? HAMLSS_SOLVER_FGMRES : solver;
        return mixed_solve(c, inner, Am, P, db, dx, p, ws, outer, lad);
    }
    if (solver == HAMLSS_SOLVER_PIPELINED_FGMRES)
        return fgmres_solve(c, Am, P, db, dx, p.tol, p.max_iter, p.restart_size, ws, lad, true);
    if (solver == HAMLSS_SOLVER_CG)
        return cg_solve<double>(c, Am, P, db, dx, p.tol, p.max_iter, p.check_every, ws, lad);
    return fgmres_solve(c, Am, P, db, dx, p.tol, p.max_iter, p.restart_size, ws, lad);
}

void fill_stats(Ctx& c, hamlss_mat* Am, int solver, const Prec* P, const SolveResult& r,
                double wall_s, int outer, double e0, double e1, const double* db, const double* dx,
                hamlss_stats* out) {
    hamlss_stats st;
    std::memset(&st, 0, sizeof(st));
    const long long n = Am->A.n, nnz = Am->A.nnz;
    st.iterations = r.iterations;
    st.initial_residual = r.initial_residual;
    st.final_residual = r.final_residual;
    st.converged = r.converged;
    st.solve_time_s = wall_s;
    // PipelinedFGMRESSolver reports FGMRES (pipelined_fgmres_solver.cpp:189)
    st.solver_used = solver == HAMLSS_SOLVER_PIPELINED_FGMRES ? HAMLSS_SOLVER_FGMRES : solver;
    st.precond_used = P ? P->kind : HAMLSS_PREC_NONE;
    st.state_used = HAMLSS_STATE_EASY;
    st.restarts = r.restarts;
    st.sstep_k = r.sstep_k;
    st.comm_bytes = r.comm_events;   // the reference counts one event per Gram reduction
    long long fl = 0, by = 0;
    if (r.flops >= 0) { fl = r.flops; by = r.bytes; }
    else if (solver == HAMLSS_SOLVER_CG) cg_cost(n, nnz, r, &fl, &by);
    else fgmres_cost(n, nnz, r, &fl, &by);
    st.flop_count = fl;
    st.mem_bytes = by;
    st.energy_joules = 2.0e-10 * (double)fl + 5.0e-9 * (double)by;
    st.energy_joules_hw = (e1 > e0) ? e1 - e0 : 0.0;
    st.rapl_start_j = e0;
    st.rapl_end_j = e1;
    st.outer_iterations = outer;
    st.status = r.status;
    st.device_time_s = r.device_time_s;
    st.true_residual = true_relative_residual(c, Am, db, dx, Am->ws);
    *out = st;
}

struct IoVecs {
    const double* b;
    double* x;
};

IoVecs stage_in(hamlss_mat* Am, const double* b, double* x, int where, cudaStream_t s) {
    if (where != HAMLSS_HOST) return IoVecs{b, x};
    Workspace& ws = Am->ws;
    const int n = Am->A.n;
    ws.d[6].upload(b, n, s);
    ws.d[7].upload(x, n, s);
    return IoVecs{ws.d[6].p, ws.d[7].p};
}

}  // namespace

extern "C" {

int hamlss_solve(hamlss_ctx* ctx, int solver, const hamlss_mat* A, const hamlss_prec* M,
                 const double* b, double* x, int where, const hamlss_params* params,
                 hamlss_stats* stats) {
    return guarded([&]() -> int {
        if (!ctx || !A || !b || !x) return set_err(HAMLSS_ERR_INVALID, "null argument");
        if (A->A.n != A->A.m) return set_err(HAMLSS_ERR_SIZE, "solve needs a square matrix");
        if (M && M->p->n != A->A.n)
            return set_err(HAMLSS_ERR_SIZE, "preconditioner size differs from the matrix");
        hamlss_params p;
        if (params) p = *params; else hamlss_params_default(&p);
        if (solver == HAMLSS_SOLVER_BICGSTAB) solver = HAMLSS_SOLVER_FGMRES;  // solver_factory.cpp:34-37
        if (solver != HAMLSS_SOLVER_CG && solver != HAMLSS_SOLVER_FGMRES &&
            solver != HAMLSS_SOLVER_SSTEP_CG && solver != HAMLSS_SOLVER_PIPELINED_FGMRES)
            return set_err(HAMLSS_ERR_INVALID, "solver type not provided by the engine");
        Ctx& c = ctx->c;
        HAMLSS_CUDA(cudaSetDevice(c.device));
        cudaStream_t s = c.lane.stream;
        AllocScope scope(s);
        auto* Am = const_cast<hamlss_mat*>(A);
        Prec* P = M ? M->p.get() : nullptr;
        IoVecs io = stage_in(Am, b, x, where, s);
        double e0 = p.record_hw_energy ? nvml_energy_j(c.device) : 0.0;
        double t0 = now_s();
        int outer = 1;
        SolveResult r = solve_core(c, solver, Am, P, io.b, io.x, p, nullptr, &outer);
        double t1 = now_s();
        double e1 = p.record_hw_energy ? nvml_energy_j(c.device) : 0.0;
        if (stats) fill_stats(c, Am, solver, P, r, t1 - t0, outer, e0, e1, io.b, io.x, stats);
        if (where == HAMLSS_HOST) Am->ws.d[7].download(x, A->A.n, s);
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        if (r.status != HAMLSS_OK)
            return set_err(r.status, "non-finite values met during the solve");
        if (lane_take_timeout(c.lane))
            return set_err(HAMLSS_ERR_TIMEOUT, "an SpMV gave up waiting for its bulk copies");
        return HAMLSS_OK;
    });
}

int hamlss_extract_features(hamlss_ctx* ctx, const hamlss_mat* A, double features[24],
                            int32_t* initial_state) {
    return guarded([&]() -> int {
        if (!ctx || !A || !features) return set_err(HAMLSS_ERR_INVALID, "null argument");
        int st = 0;
        int rc = extract_features(ctx->c, const_cast<hamlss_mat*>(A), features, &st);
        if (initial_state) *initial_state = st;
        return rc;
    });
}

// AdaptiveSelector::solve (adaptive_selector.cpp:298-394)
int hamlss_solve_adaptive(hamlss_ctx* ctx, const hamlss_mat* A, const double* b, double* x,
                          int where, const hamlss_params* params, hamlss_stats* stats,
                          hamlss_escalation* log, int32_t log_cap, int32_t* n_log,
                          int32_t* initial_state) {
    return guarded([&]() -> int {
        if (!ctx || !A || !b || !x) return set_err(HAMLSS_ERR_INVALID, "null argument");
        if (A->A.n != A->A.m) return set_err(HAMLSS_ERR_SIZE, "solve needs a square matrix");
        hamlss_params p;
        if (params) p = *params; else hamlss_params_default(&p);
        Ctx& c = ctx->c;
        HAMLSS_CUDA(cudaSetDevice(c.device));
        cudaStream_t s = c.lane.stream;
        AllocScope scope(s);
        auto* Am = const_cast<hamlss_mat*>(A);
        double feat[24];
        int state = 0;
        extract_features(c, Am, feat, &state);
        if (initial_state) *initial_state = state;
        IoVecs io = stage_in(Am, b, x, where, s);
        int nlog = 0;
        bool solved = false;
        hamlss_stats last;
        std::memset(&last, 0, sizeof(last));
        SolveResult r;
        for (;;) {
            const int kind = state == HAMLSS_STATE_EASY ? HAMLSS_PREC_JACOBI
                           : state == HAMLSS_STATE_MODERATE ? HAMLSS_PREC_ILU : HAMLSS_PREC_AMG;
            const int solver = state == HAMLSS_STATE_EASY ? HAMLSS_SOLVER_CG : HAMLSS_SOLVER_FGMRES;
            double t0 = now_s();
            std::unique_ptr<Prec> P;
            if (kind == HAMLSS_PREC_JACOBI) P = make_jacobi(c, Am, p.jacobi_omega);
            else if (kind == HAMLSS_PREC_ILU) {
                // the selector's ILU comes from SolverFactory::make_precond, which sets
                // drop_tol only (solver_factory.cpp:73-77): fill_per_row stays 0
                hamlss_params q = p;
                q.fill_per_row = 0;
                P = make_ilu(c, Am, q);
            } else P = make_amg(c, Am, p);
            HAMLSS_CUDA(cudaStreamSynchronize(s));
            double setup = now_s() - t0;
            LadderCfg lad;
            // mode 1: the device-side checks escalate the lower rungs; mode 2: they also end
            // the top rung early on a stall or divergence (its caller then decides)
            lad.on = (p.ladder_mode == 1 && state != HAMLSS_STATE_HARD) || p.ladder_mode >= 2;
            // mode 3: the CG rung escalates on the divergence and budget rules only
            lad.no_stall = p.ladder_mode == 3 && solver == HAMLSS_SOLVER_CG;
            lad.state = state;
            lad.window = p.stall_window;
            lad.threshold = p.stall_threshold;
            lad.max_iter = p.max_iter;
            double e0 = p.record_hw_energy ? nvml_energy_j(c.device) : 0.0;
            double t1 = now_s();
            int outer = 1;
            r = solve_core(c, solver, Am, P.get(), io.b, io.x, p, &lad, &outer);
            double t2 = now_s();
            double e1 = p.record_hw_energy ? nvml_energy_j(c.device) : 0.0;
            if (r.status != HAMLSS_OK) return set_err(r.status, "non-finite values met during the solve");
            fill_stats(c, Am, solver, P.get(), r, t2 - t1, outer, e0, e1, io.b, io.x, &last);
            last.setup_time_s = setup + setup;     // stats.setup_time_s counted twice (:350-351)
            last.state_used = state;
            solved = r.converged != 0;
            if (solved || state == HAMLSS_STATE_HARD) break;
            const int next = state + 1;
            if (log && nlog < log_cap) {
                log[nlog].at_iteration = r.iterations;
                log[nlog].from_state = state;
                log[nlog].to_state = next;
                log[nlog].residual_at_escalation = r.final_residual;
                log[nlog].reason = r.escalate;
            }
            ++nlog;
            state = next;
        }
        last.state_used = state;
        if (stats) *stats = last;
        if (n_log) *n_log = nlog;
        if (where == HAMLSS_HOST) Am->ws.d[7].download(x, A->A.n, s);
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        return HAMLSS_OK;
    });
}

// ------------------------------------------------------------------ batched solves
int hamlss_batch_create(hamlss_ctx* ctx, int32_t count, const int32_t* row_off,
                        const int32_t* row_ptr, const int32_t* col_idx, const double* values,
                        const int32_t* solver, const int32_t* precond, int where,
                        const hamlss_params* params, hamlss_batch** out) {
    return guarded([&]() -> int {
        if (!ctx || !out) return set_err(HAMLSS_ERR_INVALID, "null argument");
        hamlss_params p;
        if (params) p = *params;
        else hamlss_params_default(&p);
        std::lock_guard<std::mutex> g(ctx->c.mu);
        HAMLSS_CUDA(cudaSetDevice(ctx->c.device));
        auto* h = new hamlss_batch();
        h->ctx = ctx;
        try {
            h->b = batch_create(ctx->c, ctx, count, row_off, row_ptr, col_idx, values, solver, precond,
                                where, p);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
        return HAMLSS_OK;
    });
}

int hamlss_batch_solve(hamlss_ctx* ctx, hamlss_batch* B, const double* b, double* x, int where,
                       hamlss_batch_result* results, hamlss_stats* total) {
    return guarded([&]() -> int {
        if (!ctx || !B || !B->b || !b || !x) return set_err(HAMLSS_ERR_INVALID, "null argument");
        if (B->ctx != ctx) return set_err(HAMLSS_ERR_INVALID, "batch belongs to another context");
        std::lock_guard<std::mutex> g(ctx->c.mu);
        HAMLSS_CUDA(cudaSetDevice(ctx->c.device));
        Batch& Bt = *B->b;
        cudaStream_t s = ctx->c.lane.stream;
        const double t0 = now_s();
        const double* db = b;
        double* dx = x;
        if (where == HAMLSS_HOST) {
            Bt.bb.upload(b, Bt.N, s);
            Bt.xb.upload(x, Bt.N, s);
            db = Bt.bb.p;
            dx = Bt.xb.p;
        }
        const double ms = batch_run(ctx->c, Bt, db, dx, 0xFu);
        std::vector<hamlss_batch_result> res(Bt.count);
        Bt.out.download(res.data(), Bt.count, s);
        if (where == HAMLSS_HOST) Bt.xb.download(x, Bt.N, s);
        HAMLSS_CUDA(cudaStreamSynchronize(s));
        if (results) std::memcpy(results, res.data(), sizeof(hamlss_batch_result) * Bt.count);
        if (total) {
            hamlss_stats st;
            std::memset(&st, 0, sizeof(st));
            st.converged = 1;
            st.outer_iterations = 0;
            st.solver_used = -1;
            st.precond_used = -1;
            for (const auto& r : res) {
                st.iterations += r.iterations;
                st.outer_iterations = std::max(st.outer_iterations, r.outer_iterations);
                st.converged &= r.converged;
                st.final_residual = std::max(st.final_residual, r.final_residual);
                st.initial_residual = std::max(st.initial_residual, r.initial_residual);
                if (r.status != HAMLSS_OK && st.status == HAMLSS_OK) st.status = r.status;
            }
            st.true_residual = st.final_residual;
            st.device_time_s = ms * 1e-3;
            st.solve_time_s = now_s() - t0;
            *total = st;
        }
        return HAMLSS_OK;
    });
}

int hamlss_batch_set_widths(hamlss_batch* B, const int32_t widths[4]) {
    return guarded([&]() -> int {
        if (!B || !B->b || !widths) return set_err(HAMLSS_ERR_INVALID, "null argument");
        for (int c = 0; c < kBatchClasses; ++c) {
            bool ok = false;
            for (int w : kBatchWidths) ok |= w == widths[c];
            if (!ok) return set_err(HAMLSS_ERR_INVALID, "team width must be 32, 64, 128, 256 or 512");
        }
        for (int c = 0; c < kBatchClasses; ++c) B->b->width[c] = widths[c];
        return HAMLSS_OK;
    });
}

int hamlss_batch_get_widths(const hamlss_batch* B, int32_t widths[4]) {
    return guarded([&]() -> int {
        if (!B || !B->b || !widths) return set_err(HAMLSS_ERR_INVALID, "null argument");
        for (int c = 0; c < kBatchClasses; ++c) widths[c] = B->b->width[c];
        return HAMLSS_OK;
    });
}

int hamlss_batch_autotune(hamlss_ctx* ctx, hamlss_batch* B, const double* b, int where,
                          const char* cache_path, int32_t widths[4]) {
    return guarded([&]() -> int {
        if (!ctx || !B || !B->b || !b) return set_err(HAMLSS_ERR_INVALID, "null argument");
        std::lock_guard<std::mutex> g(ctx->c.mu);
        HAMLSS_CUDA(cudaSetDevice(ctx->c.device));
        Batch& Bt = *B->b;
        const double* db = b;
        if (where == HAMLSS_HOST) {
            Bt.bb.upload(b, Bt.N, ctx->c.lane.stream);
            db = Bt.bb.p;
        }
        int w[kBatchClasses];
        batch_autotune(ctx->c, Bt, db, cache_path, w);
        if (widths)
            for (int c = 0; c < kBatchClasses; ++c) widths[c] = w[c];
        return HAMLSS_OK;
    });
}

int hamlss_batch_release(hamlss_batch* B) {
    return guarded([&]() -> int {
        if (!B) return HAMLSS_OK;
        if (B->ctx) {
            HAMLSS_CUDA(cudaSetDevice(B->ctx->c.device));
            cudaStreamSynchronize(B->ctx->c.lane.stream);
        }
        delete B;
        return HAMLSS_OK;
    });
}

}  // extern "C"
