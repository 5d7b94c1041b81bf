// common.cuh -- shared pieces of the engine: errors, device buffers, reductions.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <mutex>
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

// Nanoseconds spent in device allocation and release calls, process-wide (the setup trace
// at verbose >= 2 reports it per phase).
inline std::atomic<long long>& alloc_ns() {
    static std::atomic<long long> ns{0};
    return ns;
}
struct AllocTimer {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    ~AllocTimer() {
        alloc_ns() += std::chrono::duration_cast<std::chrono::nanoseconds>(
                          std::chrono::steady_clock::now() - t0).count();
    }
};

// Stream of the enclosing setup scope on this thread (null: none).  Inside a scope, device
// buffers come from the device's stream-ordered memory pool on that stream, so the many
// temporaries of a preconditioner setup neither map fresh memory nor synchronise the
// device when freed (cudaFree does both).
inline cudaStream_t& alloc_scope_stream() {
    static thread_local cudaStream_t s = nullptr;
    return s;
}
// Keep freed pool memory cached in the process (once per device).
void pool_keep_memory(int device);

// One-time work per device and process (function attributes are per device), thread-safe.
struct DeviceOnce {
    std::once_flag flag[64];
    template <typename F>
    void operator()(int device, F&& f) { std::call_once(flag[device & 63], std::forward<F>(f)); }
};

struct AllocScope {
    cudaStream_t prev;
    explicit AllocScope(cudaStream_t s) : prev(alloc_scope_stream()) { alloc_scope_stream() = s; }
    ~AllocScope() { alloc_scope_stream() = prev; }
    AllocScope(const AllocScope&) = delete;
    AllocScope& operator=(const AllocScope&) = delete;
};

// Owning device allocation (at setup time; the solve loops allocate nothing).  A buffer
// allocated inside an AllocScope is freed in stream order: on the scope's stream when
// released inside a scope (temporaries whose kernels may still be queued there), else on
// the legacy stream -- by then the engine has synchronised the stream that used it (every
// solve call and every release entry point synchronises its context's stream).
template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    bool pooled = false;
    DBuf() = default;
    explicit DBuf(size_t count) { alloc(count); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), pooled(o.pooled) { o.p = nullptr; o.n = 0; o.pooled = false; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p; n = o.n; pooled = o.pooled;
            o.p = nullptr; o.n = 0; o.pooled = false;
        }
        return *this;
    }
    ~DBuf() { release(); }
    void alloc(size_t count) {
        release();
        n = count;
        // pad to a 256-byte multiple plus one line: vector loads and bulk copies may touch
        // the tail of the last row tile
        size_t bytes = ((count * sizeof(T) + 255) / 256 + 1) * 256;
        AllocTimer at;
        cudaStream_t s = alloc_scope_stream();
        if (s) {
            HAMLSS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p), bytes, s));
            pooled = true;
        } else {
            HAMLSS_CUDA(cudaMalloc(&p, bytes));
            pooled = false;
        }
    }
    void ensure(size_t count) { if (count > n || !p) alloc(count); }
    void release() {
        if (p) {
            AllocTimer at;
            if (pooled) {
                cudaStream_t s = alloc_scope_stream();
                cudaFreeAsync(p, s ? s : cudaStreamLegacy);
            } else {
                cudaFree(p);
            }
            p = nullptr;
            n = 0;
            pooled = false;
        }
    }
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
