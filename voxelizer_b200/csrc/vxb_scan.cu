// Work-list scan kernels.
#include "vxb_common.cuh"
#include "vxb_device.cuh"
#include "vxb_kernels.cuh"

#include <cfloat>

namespace vxb {

using namespace detail;

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

// ---------------------------------------------------------------------------
// Exclusive scan of per-triangle counts (three kernels: tile scan, scan of
// tile sums, tile offsets).  Totals of 2^32 - 1 or more set *overflow: a
// tile whose own sum wraps 32 bits reports the saturated sum 2^32 - 1, so
// the 64-bit carry over the tile sums sees it.

__device__ __forceinline__ uint32_t blockExclusiveScan(uint32_t v, uint32_t* warpSums, uint32_t& blockTotal) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warpSums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t s = lane < nw ? warpSums[lane] : 0u;
        uint32_t si = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += t;
        }
        if (lane < nw) warpSums[lane] = si - s;
        if (lane == 31) warpSums[32] = si;
    }
    __syncthreads();
    uint32_t res = warpSums[warp] + incl - v;
    blockTotal = warpSums[32];
    __syncthreads();
    return res;
}

__global__ void scanTileKernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t n,
                               uint32_t* __restrict__ tileSums) {
    __shared__ uint32_t warpSums[33];
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    unsigned long long sum64 = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = (base + i < n) ? in[base + i] : 0u;
        sum64 += v[i];
    }
    const uint32_t sum = (uint32_t)sum64;
    uint32_t total;
    uint32_t ex = blockExclusiveScan(sum, warpSums, total);
    // A 32-bit prefix that passes 2^32 wraps at the thread whose items cross
    // it, so the tile's sum is exact unless some thread saw a wrap.
    const int wrapped = __syncthreads_or(sum64 > 0xFFFFFFFFull || ex + sum < ex);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = ex;
        ex += v[i];
    }
    if (threadIdx.x == 0) tileSums[blockIdx.x] = wrapped ? 0xFFFFFFFFu : total;
}

__global__ void scanSumsKernel(uint32_t* tileSums, uint32_t nTiles, uint32_t* total, uint32_t* overflow) {
    __shared__ uint32_t warpSums[33];
    unsigned long long carry = 0;
    int wrapped = 0;
    for (uint32_t start = 0; start < nTiles; start += blockDim.x) {
        uint32_t i = start + threadIdx.x;
        uint32_t v = i < nTiles ? tileSums[i] : 0u;
        uint32_t chunk;
        uint32_t ex = blockExclusiveScan(v, warpSums, chunk);
        wrapped |= __syncthreads_or(ex + v < ex);
        if (i < nTiles) tileSums[i] = (uint32_t)(carry + ex);
        carry += chunk;
    }
    if (threadIdx.x == 0) {
        *total = (uint32_t)carry;
        *overflow = (wrapped || carry >= 0xFFFFFFFFull) ? 1u : 0u;
    }
}

__global__ void scanAddKernel(uint32_t* out, uint32_t n, const uint32_t* tileSums, const uint32_t* total) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tileSums[i / kScanTile];
    if (i == 0) out[n] = *total;
}

}  // namespace

void launch_scan(const uint32_t* in, uint32_t* offsets, uint32_t n, uint32_t* blockSums, uint32_t* total,
                 uint32_t* overflow, cudaStream_t s, uint32_t* launches) {
    const uint32_t tiles = n == 0 ? 1 : (n + kScanTile - 1) / kScanTile;
    scanTileKernel<<<tiles, kScanThreads, 0, s>>>(in, offsets, n, blockSums);
    scanSumsKernel<<<1, kScanThreads, 0, s>>>(blockSums, tiles, total, overflow);
    scanAddKernel<<<(n + 1 + 255) / 256, 256, 0, s>>>(offsets, n, blockSums, total);
    *launches += 3;
}
}  // namespace vxb
