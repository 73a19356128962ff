// Mesh checks of vxb_create on the device: the largest index, the first
// out-of-range index, and the bounding box, from the mesh copy that the
// voxelizer uploads anyway (the reference computes the box on the host while
// it copies the mesh, src/host_side.cpp:72-99).
//
// The box must equal the host's sequential scan (boundingBox in
// vxb_plan.h): start from vertex 0 and replace a bound only by a strictly
// smaller (larger) coordinate.  That scan ends at the first occurrence of
// the extreme value among vertex 0 and the later non-NaN coordinates, with
// +0 and -0 equal.  Here every later coordinate that is not NaN becomes the
// key (order code of the value, vertex index); the smallest key names the
// first occurrence of the minimum, and the host compares that coordinate
// with vertex 0 as the scan would.

#include "vxb.h"
#include "vxb_host.h"
#include "vxb_kernels.cuh"

#include <algorithm>

namespace vxb {

namespace {

constexpr int kBlock = 256;

// Monotone code of a non-NaN float with +0 and -0 equal.
__device__ __forceinline__ uint32_t orderCode(float f) {
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7FFFFFFFu) == 0u) return 0x80000000u;
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ unsigned long long warpMin(unsigned long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xFFFFFFFFu, v, o);
        v = t < v ? t : v;
    }
    return v;
}

__device__ __forceinline__ uint32_t warpMax(uint32_t v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}

// out[0..2]: min keys per axis, out[3..5]: max keys (as minima of the
// complemented code), out[6]: largest index, out[7]: first index position
// holding an index >= nV.  The host sets out to (~0, ..., ~0, 0, ~0) first.
__global__ void __launch_bounds__(kBlock) meshCheckKernel(const float* __restrict__ V, uint32_t nV,
                                                          const uint32_t* __restrict__ I, uint64_t nIdx,
                                                          unsigned long long* out) {
    unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {~0ull, ~0ull, ~0ull};
    uint32_t maxIdx = 0;
    unsigned long long firstBad = ~0ull;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = 1 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nV; i += stride) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float f = __ldg(V + 3 * i + a);
            if (f != f) continue;   // NaN: the scan's comparisons are false
            const uint32_t c = orderCode(f);
            const unsigned long long kl = ((unsigned long long)c << 32) | i;
            const unsigned long long kh = ((unsigned long long)(~c) << 32) | i;
            lo[a] = kl < lo[a] ? kl : lo[a];
            hi[a] = kh < hi[a] ? kh : hi[a];
        }
    }
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nIdx; i += stride) {
        const uint32_t x = __ldg(I + i);
        maxIdx = max(maxIdx, x);
        if (x >= nV && i < firstBad) firstBad = i;
    }
    __shared__ unsigned long long part[kBlock / 32][8];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    unsigned long long r[8];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        r[a] = warpMin(lo[a]);
        r[3 + a] = warpMin(hi[a]);
    }
    r[6] = warpMax(maxIdx);
    r[7] = warpMin(firstBad);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 8; ++k) part[warp][k] = r[k];
    __syncthreads();
    if (threadIdx.x < 8) {
        const int k = threadIdx.x;
        unsigned long long v = part[0][k];
        for (int w = 1; w < kBlock / 32; ++w) {
            const unsigned long long t = part[w][k];
            v = k == 6 ? (t > v ? t : v) : (t < v ? t : v);
        }
        if (k == 6) atomicMax(out + 6, v);
        else atomicMin(out + k, v);
    }
}

}  // namespace

int meshCheck(const float* dV, uint32_t nV, const uint32_t* dI, uint64_t nIdx, unsigned long long* dOut,
              unsigned long long* hostOut, cudaStream_t s) {
    unsigned long long init[8] = {~0ull, ~0ull, ~0ull, ~0ull, ~0ull, ~0ull, 0ull, ~0ull};
    VXB_CUDA(cudaMemcpyAsync(dOut, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const uint64_t work = std::max<uint64_t>(nV, nIdx);
    const uint32_t grid = (uint32_t)std::min<uint64_t>((work + kBlock - 1) / kBlock, 148ull * 8ull);
    if (work) meshCheckKernel<<<grid ? grid : 1, kBlock, 0, s>>>(dV, nV, dI, nIdx, dOut);
    VXB_CUDA(cudaGetLastError());
    VXB_CUDA(cudaMemcpyAsync(hostOut, dOut, sizeof(init), cudaMemcpyDeviceToHost, s));
    VXB_CUDA(cudaStreamSynchronize(s));
    return 0;
}

}  // namespace vxb
