// engine.cu -- context / lane setup, device CSR helpers, Jacobi, residual check.
#include <mutex>
#include <cmath>
#include <cstring>

#include "krylov.cuh"

namespace hamlss {

void pool_keep_memory(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> g(mu);
    if (device < 0 || device >= 64 || done[device]) return;
    cudaMemPool_t pool;
    HAMLSS_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;
    HAMLSS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    done[device] = true;
}

void lane_init(Lane& L, int sm_count) {
    HAMLSS_CUDA(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
    // every reducing launch has at most sm_count * kMaxBlocksPerSm blocks of at most
    // kMaxRed sums each (red_check enforces it before the launch)
    L.red_cap = (size_t)std::max(sm_count, 1) * kMaxBlocksPerSm * kMaxRed;
    L.partials.alloc(L.red_cap);
    L.err.alloc(1);
    L.err.zero(L.stream);
    L.ticket.alloc(1);
    L.ticket.zero(L.stream);
}

bool lane_take_timeout(const Lane& L) {
    int e = 0;
    HAMLSS_CUDA(cudaMemcpyAsync(&e, L.err.p, sizeof(int), cudaMemcpyDeviceToHost, L.stream));
    HAMLSS_CUDA(cudaStreamSynchronize(L.stream));
    if (e) HAMLSS_CUDA(cudaMemsetAsync(L.err.p, 0, sizeof(int), L.stream));
    return e != 0;
}

void lane_destroy(Lane& L) {
    if (L.stream) {
        cudaStreamSynchronize(L.stream);
        cudaStreamDestroy(L.stream);
        L.stream = nullptr;
    }
    L.partials.release();
    L.ticket.release();
    L.err.release();
}

namespace {

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

// flags[0]: bad row_ptr, flags[1]: column out of range, flags[2]: unsorted/duplicate row
__global__ void k_validate(int n, int m, int nnz, const int* __restrict__ rp,
                           const int* __restrict__ ci, int* flags) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int s = rp[i], e = rp[i + 1];
        if (i == 0 && s != 0) flags[0] = 1;
        if (i == n - 1 && e != nnz) flags[0] = 1;
        if (e < s || s < 0 || e > nnz) { flags[0] = 1; continue; }
        int prev = -1;
        for (int k = s; k < e; ++k) {
            int c = ci[k];
            if (c < 0 || c >= m) flags[1] = 1;
            if (c <= prev) flags[2] = 1;
            prev = c;
        }
    }
}

__global__ void k_diag(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                       const double* __restrict__ v, double* __restrict__ d) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double di = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) { di = v[k]; break; }
        d[i] = di;
    }
}

// JacobiPreconditioner::setup (jacobi.cpp:23-31): first zero diagonal row -> error.
__global__ void k_jacobi_setup(int n, const double* __restrict__ d, double omega,
                               double* __restrict__ inv, int* bad_row) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double di = d[i];
        if (fabs(di) < 2.220446049250313e-16) { atomicMin(bad_row, i); inv[i] = 0.0; }
        else inv[i] = omega / di;
    }
}

template <typename T>
__global__ void k_jacobi_apply(int n, const T* __restrict__ inv, const T* __restrict__ r,
                               T* __restrict__ z, const int* gate) {
    if (gate && *(volatile const int*)gate) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        z[i] = (T)__dmul_rn((double)inv[i], (double)r[i]);
}

__global__ void k_row_len_max(int n, const int* __restrict__ rp, int* mx) {
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = max(m, rp[i + 1] - rp[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(mx, m);
}

__global__ void k_rows_longer(int n, const int* __restrict__ rp, int len, int* list, int* count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (rp[i + 1] - rp[i] > len) list[atomicAdd(count, 1)] = i;
}

}  // namespace

Csr<float> DevMat::f32(cudaStream_t s) {
    if (!v32_valid) {
        v32.ensure(nnz);
        if (nnz) {
            k_to_f32<<<std::min(ceil_div(nnz, 256), 148 * 16), 256, 0, s>>>(v.p, v32.p, nnz);
            HAMLSS_LAUNCH_CHECK();
        }
        v32_valid = true;
    }
    return Csr<float>{n, m, nnz, rp.p, ci.p, v32.p};
}

int validate_csr(Ctx& ctx, const Csr<double>& A) {
    if (A.n == 0) return HAMLSS_OK;
    DBuf<int> flags(3);
    flags.zero(ctx.lane.stream);
    k_validate<<<std::min(ceil_div(A.n, 256), ctx.sm_count * 8), 256, 0, ctx.lane.stream>>>(
        A.n, A.m, A.nnz, A.rp, A.ci, flags.p);
    HAMLSS_LAUNCH_CHECK();
    int h[3];
    flags.download(h, 3, ctx.lane.stream);
    HAMLSS_CUDA(cudaStreamSynchronize(ctx.lane.stream));
    return (h[0] || h[1] || h[2]) ? HAMLSS_ERR_MALFORMED : HAMLSS_OK;
}

void ensure_row_profile(Ctx& ctx, hamlss_mat* M) {
    if (M->n_long >= 0) return;
    const int n = M->A.n;
    M->n_long = 0;
    M->long_len = INT_MAX;
    if (n == 0) return;
    cudaStream_t s = ctx.lane.stream;
    DBuf<int> cnt(1);
    cnt.zero(s);
    const int g = std::min(ceil_div(n, 256), ctx.sm_count * 8);
    k_row_len_max<<<g, 256, 0, s>>>(n, M->A.rp.p, cnt.p);
    HAMLSS_LAUNCH_CHECK();
    int h = 0;
    cnt.download(&h, 1, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    const double avg = (double)M->A.nnz / n;
    if (h <= kSkewRow || h <= kSkewRatio * avg) return;
    const int len = std::max(kSkewRow, (int)std::ceil(kSkewRatio * avg));
    M->long_rows.ensure(n);
    cnt.zero(s);
    k_rows_longer<<<g, 256, 0, s>>>(n, M->A.rp.p, len, M->long_rows.p, cnt.p);
    HAMLSS_LAUNCH_CHECK();
    cnt.download(&h, 1, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    M->n_long = h;
    M->long_len = len;
}

void ensure_diag(Ctx& ctx, hamlss_mat* M) {
    if (M->diag_valid) return;
    M->diag.ensure(M->A.n);
    if (M->A.n) {
        ProfScope ps(ctx.lane, "setup", 16.0 * M->A.n + 12.0 * M->A.nnz);
        k_diag<<<std::min(ceil_div(M->A.n, 256), ctx.sm_count * 8), 256, 0, ctx.lane.stream>>>(
            M->A.n, M->A.rp.p, M->A.ci.p, M->A.v.p, M->diag.p);
        HAMLSS_LAUNCH_CHECK();
    }
    M->diag_valid = true;
}

// ---------------------------------------------------------------------------- Jacobi
void JacobiPrec::apply(Ctx& ctx, const Lane& L, const double* r, double* z, const int* gate) {
    if (!n) return;
    ProfScope ps(L, "jacobi", 24.0 * n);
    k_jacobi_apply<double><<<std::min(ceil_div(n, 256), ctx.sm_count * 8), 256, 0, L.stream>>>(
        n, inv.p, r, z, gate);
    HAMLSS_LAUNCH_CHECK();
}

void JacobiPrec::prepare32(Ctx& ctx) {
    if (inv32_valid) return;
    inv32.ensure(n);
    if (n) {
        k_to_f32<<<std::min(ceil_div(n, 256), 148 * 16), 256, 0, ctx.lane.stream>>>(inv.p, inv32.p, n);
        HAMLSS_LAUNCH_CHECK();
    }
    inv32_valid = true;
}

void JacobiPrec::apply32(Ctx& ctx, const Lane& L, const float* r, float* z, const int* gate) {
    prepare32(ctx);
    if (!n) return;
    ProfScope ps(L, "jacobi", 12.0 * n);
    k_jacobi_apply<float><<<std::min(ceil_div(n, 256), ctx.sm_count * 8), 256, 0, L.stream>>>(
        n, inv32.p, r, z, gate);
    HAMLSS_LAUNCH_CHECK();
}

std::unique_ptr<Prec> make_jacobi(Ctx& ctx, hamlss_mat* A, double omega) {
    ensure_diag(ctx, A);
    auto J = std::make_unique<JacobiPrec>();
    J->kind = HAMLSS_PREC_JACOBI;
    J->n = A->A.n;
    J->inv.ensure(J->n);
    DBuf<int> bad(1);
    int init = 0x7fffffff;
    bad.upload(&init, 1, ctx.lane.stream);
    if (J->n) {
        ProfScope ps(ctx.lane, "setup", 16.0 * J->n);
        k_jacobi_setup<<<std::min(ceil_div(J->n, 256), ctx.sm_count * 8), 256, 0, ctx.lane.stream>>>(
            J->n, A->diag.p, omega, J->inv.p, bad.p);
        HAMLSS_LAUNCH_CHECK();
    }
    int h = 0;
    bad.download(&h, 1, ctx.lane.stream);
    HAMLSS_CUDA(cudaStreamSynchronize(ctx.lane.stream));
    if (h != 0x7fffffff)
        fail(HAMLSS_ERR_ZERO_DIAG, "JacobiPreconditioner: zero diagonal at row " + std::to_string(h));
    return J;
}

// ------------------------------------------------------------------ true residual
namespace {
struct EpiRes2 {
    const double* b;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double ax, double (&acc)[NV]) const {
        double bi = b[i];
        double ri = __dsub_rn(bi, ax);
        acc[0] += bi * bi;
        acc[1] += ri * ri;
    }
};
struct FinStore2 {
    double* out;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const { out[0] = t[0]; out[1] = t[1]; }
};
}  // namespace

double true_relative_residual(Ctx& ctx, hamlss_mat* A, const double* b, const double* x,
                              Workspace& ws) {
    ws.small.ensure(4096);
    double* out = ws.small.p + 4000;
    launch_spmv<double, 2>(ctx.sm_count, ctx.lane, A->A.f64(), XVec<double>{x}, EpiRes2{b},
                           FinStore2{out});
    double h[2];
    HAMLSS_CUDA(cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, ctx.lane.stream));
    HAMLSS_CUDA(cudaStreamSynchronize(ctx.lane.stream));
    double bn = std::sqrt(h[0]), rn = std::sqrt(h[1]);
    return bn > 2.220446049250313e-16 ? rn / bn : rn;
}

}  // namespace hamlss
