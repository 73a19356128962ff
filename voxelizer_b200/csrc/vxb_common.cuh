// Helpers shared by the kernel files.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vxb {
namespace detail {

struct D3 { double x, y, z; };
struct F3 { float x, y, z; };

__device__ __forceinline__ uint32_t laneMaskLt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Largest t with offsets[t] <= item (offsets: n + 1 non-decreasing entries).
__device__ __forceinline__ uint32_t findOwner(const uint32_t* __restrict__ offsets, uint32_t n, uint32_t item) {
    uint32_t lo = 0, hi = n;  // invariant: offsets[lo] <= item < offsets[hi]
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(offsets + mid) <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Unit of element x: the largest u < n with base[u] <= x (base[0] = 0).
template <class T>
__device__ __forceinline__ uint32_t unitOf(const T* __restrict__ base, uint32_t n, T x) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(base + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Largest t < n with off[t] <= item (off[n] > item), by a 32-way search of
// the whole warp: ceil(log32 n) dependent loads.
__device__ __forceinline__ uint32_t warpFindOwner(const uint32_t* __restrict__ off, uint32_t n, uint32_t item,
                                                  uint32_t lane) {
    uint32_t lo = 0, hi = n;  // off[lo] <= item < off[hi]
    while (hi - lo > 1) {
        const uint32_t step = (hi - lo + 31u) / 32u;
        const uint32_t p = lo + lane * step;
        const bool ok = p < hi && __ldg(off + p) <= item;
        const uint32_t m = __ballot_sync(0xffffffffu, ok);
        const uint32_t nlo = lo + (31u - (uint32_t)__clz(m)) * step;
        hi = min(nlo + step, hi);
        lo = nlo;
    }
    return lo;
}

// Blocks for `work` items at `threads` per block, capped (grid-stride loops).
inline uint32_t gridFor(uint64_t work, uint32_t threads, uint32_t cap = 148u * 32u) {
    uint64_t b = (work + threads - 1) / threads;
    if (b == 0) b = 1;
    return (uint32_t)(b < cap ? b : cap);
}

}  // namespace detail
}  // namespace vxb
