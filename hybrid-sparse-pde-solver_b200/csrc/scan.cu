// scan.cu -- see scan.cuh.
#include "scan.cuh"

namespace hamlss {

namespace {

constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;                       // elements per thread
constexpr int kScanTile = kScanBlock * kScanItems;  // elements per block

__device__ __forceinline__ int block_exclusive(int v, int* sh, int* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < (kScanBlock / 32) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        sh[lane] = s;   // inclusive warp sums
    }
    __syncthreads();
    int base = wid > 0 ? sh[wid - 1] : 0;
    if (total) *total = sh[kScanBlock / 32 - 1];
    return base + x - v;
}

__global__ void __launch_bounds__(kScanBlock) k_tile_sums(const int* __restrict__ a, int count, int* sums) {
    __shared__ int sh[32];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) s += (base + k < count) ? a[base + k] : 0;
    int tot;
    block_exclusive(s, sh, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_sums(int* sums, int nb, long long* total) {
    __shared__ int sh[32];
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nb; b0 += kScanBlock) {
        int i = b0 + threadIdx.x;
        int v = i < nb ? sums[i] : 0;
        int tot;
        int ex = block_exclusive(v, sh, &tot);
        if (i < nb) sums[i] = (int)(carry + ex);
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanBlock) k_tile_apply(int* a, int count, const int* __restrict__ sums) {
    __shared__ int sh[32];
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) { v[k] = (base + k < count) ? a[base + k] : 0; s += v[k]; }
    int ex = block_exclusive(s, sh, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < count) a[base + k] = ex;
        ex += v[k];
    }
}

}  // namespace

long long exclusive_scan(Ctx& ctx, int* data, int count) {
    if (count <= 0) return 0;
    cudaStream_t s = ctx.lane.stream;
    const int nb = ceil_div(count, kScanTile);
    DBuf<int> sums(nb);
    DBuf<long long> total(1);
    ProfScope ps(ctx.lane, "setup", 8.0 * count);
    k_tile_sums<<<nb, kScanBlock, 0, s>>>(data, count, sums.p);
    k_scan_sums<<<1, kScanBlock, 0, s>>>(sums.p, nb, total.p);
    k_tile_apply<<<nb, kScanBlock, 0, s>>>(data, count, sums.p);
    HAMLSS_LAUNCH_CHECK();
    long long h = 0;
    total.download(&h, 1, s);
    HAMLSS_CUDA(cudaStreamSynchronize(s));
    return h;
}

}  // namespace hamlss
