// common.cuh -- shared pieces of the engine: errors, device buffers, reductions.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hamlss.h"

namespace hamlss {

// An engine failure: a HAMLSS_ERR_* code plus a message.  Thrown inside the engine and
// turned into the C status at the ABI boundary (capi.cu).
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

// Record the thread's hamlss_last_error() message; returns `code`.
int set_last_error(int code, const std::string& msg);

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        int code = (e == cudaErrorMemoryAllocation) ? HAMLSS_ERR_NOMEM : HAMLSS_ERR_CUDA;
        throw Error(code, std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" +
                              std::to_string(line) + ")");
    }
}
#define HAMLSS_CUDA(call) ::hamlss::cuda_check((call), #call, __FILE__, __LINE__)
#define HAMLSS_LAUNCH_CHECK() ::hamlss::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__)

// Owning device allocation (cudaMalloc at setup time; the solve loops allocate nothing).
template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    explicit DBuf(size_t count) { alloc(count); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DBuf() { release(); }
    void alloc(size_t count) {
        release();
        n = count;
        // pad to a 256-byte multiple plus one line: vector loads and bulk copies may touch
        // the tail of the last row tile
        size_t bytes = ((count * sizeof(T) + 255) / 256 + 1) * 256;
        HAMLSS_CUDA(cudaMalloc(&p, bytes));
    }
    void ensure(size_t count) { if (count > n || !p) alloc(count); }
    void release() { if (p) { cudaFree(p); p = nullptr; n = 0; } }
    void zero(cudaStream_t s) { if (p) HAMLSS_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
    void upload(const T* h, size_t count, cudaStream_t s) {
        ensure(count);
        if (count) HAMLSS_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void download(T* h, size_t count, cudaStream_t s) const {
        if (count) HAMLSS_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
};

// Pinned host staging (for the few scalars the host polls).
template <typename T>
struct HBuf {
    T* p = nullptr;
    size_t n = 0;
    HBuf() = default;
    explicit HBuf(size_t c) { alloc(c); }
    HBuf(const HBuf&) = delete;
    HBuf& operator=(const HBuf&) = delete;
    ~HBuf() { if (p) cudaFreeHost(p); }
    void alloc(size_t c) {
        if (p) cudaFreeHost(p);
        n = c;
        HAMLSS_CUDA(cudaMallocHost(&p, c * sizeof(T)));
    }
};

constexpr int kWarp = 32;

// ---------------------------------------------------------------- warp / block reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum of NV values per thread; result valid in thread 0.
// `sh` must hold (blockDim.x / 32) * NV doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[wid * NV + k] = v[k];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = (lane < nw) ? sh[lane * NV + k] : 0.0;
            v[k] = warp_sum(t);
        }
    }
}

// Two-stage deterministic grid reduction.  Each block writes its NV partial sums to
// partials[block * NV + k]; the block that finishes last (ticket counter) sums all of them
// in block order and returns true in thread 0 with the totals in `tot`.  The ticket is
// reset by that block, so the same Reducer can be reused by the next launch.
struct Reducer {
    double* partials;     // >= gridDim.x * NV
    unsigned* ticket;     // one counter, zero between launches
};

template <int NV>
__device__ __forceinline__ bool grid_reduce(const Reducer& R, double (&v)[NV], double* sh,
                                            double (&tot)[NV]) {
    block_sum<NV>(v, sh);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) R.partials[blockIdx.x * NV + k] = v[k];
        __threadfence();
        unsigned t = atomicAdd(R.ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += __ldcg(&R.partials[b * NV + k]);
    }
    block_sum<NV>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) tot[k] = acc[k];
        *R.ticket = 0u;
    }
    return threadIdx.x == 0;
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace hamlss
