// dot_noalloc.cu -- hamlss_dot_noalloc: a dot product that allocates no memory.
//
// Some callers cannot let a library allocate device memory: an application that reserves
// the GPU's memory up front for its own pool (a library cudaMalloc then fails or breaks
// its accounting), or a latency-critical loop where cudaMalloc / cudaFree would stall on
// the whole device.  hamlss_dot (a context's stream and reduction buffers, plus a result
// buffer per call) is not usable there.  This entry point runs the same reduction kernel
// as hamlss_dot, but its scratch -- the per-block partial sums, the result slot and the
// last-block ticket -- lives in one fixed array compiled into the library.
//
// The array holds kMaxBlocks partial sums (16 KiB in all).  Every GPU that loads the
// library holds it until the process exits.  All calls on a device share it.
#include <mutex>
#include <string>

#include "engine.cuh"

namespace {

constexpr int kMaxBlocks = 2048;                  // partial-sum slots in the fixed scratch
constexpr int kMaxDevices = 64;

// [0, kMaxBlocks) partial sums | [kMaxBlocks] the result | [kMaxBlocks + 1] the ticket
static __device__ __align__(256) double g_dot_scratch[kMaxBlocks + 2];

// Same arithmetic as hamlss_dot's body and finaliser.
struct DotBody {
    const double* x;
    const double* y;
    HAMLSS_NO_LOAD
    template <int NV>
    __device__ __forceinline__ void operator()(int i, double (&acc)[NV]) const { acc[0] += x[i] * y[i]; }
};
struct StoreResult {
    double* out;
    template <int NV>
    __device__ void operator()(const double (&t)[NV]) const { out[0] = t[0]; }
};

// Per-device set-up: the device address of g_dot_scratch (in host code the symbol's name
// is only a host-side stand-in, never a usable device address) and the SM count.
struct DeviceScratch {
    std::mutex mu;
    bool ready = false;
    double* base = nullptr;
    int sm_count = 0;
};
DeviceScratch g_dev[kMaxDevices];

int fail(int code, const std::string& m) { return hamlss::set_last_error(code, m); }

// Look up the scratch of the current device (once per device; the address is kept for
// the life of the process, so it goes stale if the process resets the device).
int scratch_of_current_device(DeviceScratch** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(HAMLSS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(HAMLSS_ERR_INVALID, "device index out of range");
    DeviceScratch& d = g_dev[dev];
    std::lock_guard<std::mutex> g(d.mu);
    if (!d.ready) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_dot_scratch);
        if (e != cudaSuccess)
            return fail(HAMLSS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        e = cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess)
            return fail(HAMLSS_ERR_CUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
        d.base = static_cast<double*>(p);
        d.ready = true;
    }
    *out = &d;
    return HAMLSS_OK;
}

}  // namespace

extern "C" int hamlss_dot_noalloc(int32_t n, const double* x, const double* y, double* result,
                                  void* stream) {
    if (n < 0 || !result || (n > 0 && (!x || !y)))
        return fail(HAMLSS_ERR_INVALID, "hamlss_dot_noalloc: bad arguments");
    if (n == 0) {
        *result = 0.0;
        return HAMLSS_OK;
    }
    DeviceScratch* d = nullptr;
    int rc = scratch_of_current_device(&d);
    if (rc != HAMLSS_OK) return rc;
    // the same grid as hamlss_dot, so the partial sums and their order are the same
    const int blocks = std::max(1, std::min(hamlss::ceil_div(n, 256), d->sm_count * hamlss::kMaxBlocksPerSm));
    if (blocks > kMaxBlocks)
        return fail(HAMLSS_ERR_SIZE, "hamlss_dot_noalloc: this device needs " + std::to_string(blocks) +
                                         " partial sums, more than the fixed scratch holds (" +
                                         std::to_string(kMaxBlocks) + ")");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* partials = d->base;
    double* res = d->base + kMaxBlocks;
    unsigned* ticket = reinterpret_cast<unsigned*>(d->base + kMaxBlocks + 1);
    // the last-block ticket must start at zero (a launch resets it, but an interrupted one
    // would not)
    cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(unsigned), s);
    if (e == cudaSuccess) {
        hamlss::k_vec<1, DotBody, StoreResult><<<blocks, 256, 0, s>>>(
            n, DotBody{x, y}, hamlss::Reducer{partials, ticket}, StoreResult{res}, nullptr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(result, res, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return fail(HAMLSS_ERR_CUDA, std::string("hamlss_dot_noalloc: ") + cudaGetErrorString(e));
    return HAMLSS_OK;
}
