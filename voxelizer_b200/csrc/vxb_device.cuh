// Device-side building blocks shared by the vxb kernels: explicit-rounding
// arithmetic that reproduces the reference build's multiply-add contraction,
// node layouts and key encodings, and the boundary-id table.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vxb {

// ---------------------------------------------------------------------------
// Contraction sites.  The reference (hakarlss/Voxelizer) is compiled with
// nvcc's default --fmad=true, so a multiply feeding an add may be fused into
// one FMA; which ones were fused decides results at exact ties (vertices on
// voxel centres or cell faces).  Every expression of the reference's
// arithmetic is evaluated here with explicitly rounded intrinsics
// (__dmul_rn / __dadd_rn / __fma_rn never contract), in the form selected
// per site below.  The modes were fitted against the reference's own CUDA
// output on a B200; the CPU oracle evaluates the same sites identically.
//
//   p = i*d + m          P_*, PC_*    0: mul, add      1: fma(i, d, m)
//   a*b + c*d + e        E_*, OT_*    0: no fma  1: fma(a,b,c*d)+e  2: fma(c,d,a*b)+e  3: fma(a,b,fma(c,d,e))
//   -(a*b + c*d)         D_*, DE_*    0: no fma  1: -fma(a,b,c*d)   2: -fma(c,d,a*b)
//   a*b - c*d            CR*          0: no fma  1: fma(a,b,-(c*d)) 2: fma(-c,d,a*b)
//   a*b + c*d + e*f      B_*, TN, DT_* 0: no fma 1: fma(e,f,fma(a,b,c*d)) 2: fma(e,f,fma(c,d,a*b))
//                                      3: fma(a,b,c*d)+e*f  4: fma(e,f,a*b+c*d)  5: fma(c,d,a*b)+e*f
// The DE_* and OT_* sites hold one mode per triangle edge: bits 2i..2i+1
// for edge i.
namespace site {
#include "vxb_sites.inc"
}

// ---- FP64 forms ----
template <int M> __device__ __forceinline__ double sum2p1(double a, double b, double c, double d, double e) {
    if (M == 0) return __dadd_rn(__dadd_rn(__dmul_rn(a, b), __dmul_rn(c, d)), e);
    if (M == 1) return __dadd_rn(__fma_rn(a, b, __dmul_rn(c, d)), e);
    if (M == 2) return __dadd_rn(__fma_rn(c, d, __dmul_rn(a, b)), e);
    return __fma_rn(a, b, __fma_rn(c, d, e));
}
template <int M> __device__ __forceinline__ double sum2(double a, double b, double c, double d) {
    if (M == 0) return __dadd_rn(__dmul_rn(a, b), __dmul_rn(c, d));
    if (M == 1) return __fma_rn(a, b, __dmul_rn(c, d));
    return __fma_rn(c, d, __dmul_rn(a, b));
}
template <int M> __device__ __forceinline__ double diff2(double a, double b, double c, double d) {
    if (M == 0) return __dsub_rn(__dmul_rn(a, b), __dmul_rn(c, d));
    if (M == 1) return __fma_rn(a, b, -__dmul_rn(c, d));
    return __fma_rn(-c, d, __dmul_rn(a, b));
}
template <int M> __device__ __forceinline__ double sum3(double a, double b, double c, double d, double e, double f) {
    if (M == 0) return __dadd_rn(__dadd_rn(__dmul_rn(a, b), __dmul_rn(c, d)), __dmul_rn(e, f));
    if (M == 1) return __fma_rn(e, f, __fma_rn(a, b, __dmul_rn(c, d)));
    if (M == 2) return __fma_rn(e, f, __fma_rn(c, d, __dmul_rn(a, b)));
    if (M == 3) return __dadd_rn(__fma_rn(a, b, __dmul_rn(c, d)), __dmul_rn(e, f));
    if (M == 4) return __fma_rn(e, f, __dadd_rn(__dmul_rn(a, b), __dmul_rn(c, d)));
    return __dadd_rn(__fma_rn(c, d, __dmul_rn(a, b)), __dmul_rn(e, f));
}
template <int M> __device__ __forceinline__ double lin(double i, double d, double m) {
    return M ? __fma_rn(i, d, m) : __dadd_rn(__dmul_rn(i, d), m);
}

// ---- FP32 forms ----
template <int M> __device__ __forceinline__ float sum2p1f(float a, float b, float c, float d, float e) {
    if (M == 0) return __fadd_rn(__fadd_rn(__fmul_rn(a, b), __fmul_rn(c, d)), e);
    if (M == 1) return __fadd_rn(__fmaf_rn(a, b, __fmul_rn(c, d)), e);
    if (M == 2) return __fadd_rn(__fmaf_rn(c, d, __fmul_rn(a, b)), e);
    return __fmaf_rn(a, b, __fmaf_rn(c, d, e));
}
template <int M> __device__ __forceinline__ float sum2f(float a, float b, float c, float d) {
    if (M == 0) return __fadd_rn(__fmul_rn(a, b), __fmul_rn(c, d));
    if (M == 1) return __fmaf_rn(a, b, __fmul_rn(c, d));
    return __fmaf_rn(c, d, __fmul_rn(a, b));
}
template <int M> __device__ __forceinline__ float diff2f(float a, float b, float c, float d) {
    if (M == 0) return __fsub_rn(__fmul_rn(a, b), __fmul_rn(c, d));
    if (M == 1) return __fmaf_rn(a, b, -__fmul_rn(c, d));
    return __fmaf_rn(-c, d, __fmul_rn(a, b));
}
template <int M> __device__ __forceinline__ float sum3f(float a, float b, float c, float d, float e, float f) {
    if (M == 0) return __fadd_rn(__fadd_rn(__fmul_rn(a, b), __fmul_rn(c, d)), __fmul_rn(e, f));
    if (M == 1) return __fmaf_rn(e, f, __fmaf_rn(a, b, __fmul_rn(c, d)));
    if (M == 2) return __fmaf_rn(e, f, __fmaf_rn(c, d, __fmul_rn(a, b)));
    if (M == 3) return __fadd_rn(__fmaf_rn(a, b, __fmul_rn(c, d)), __fmul_rn(e, f));
    if (M == 4) return __fmaf_rn(e, f, __fadd_rn(__fmul_rn(a, b), __fmul_rn(c, d)));
    return __fadd_rn(__fmaf_rn(c, d, __fmul_rn(a, b)), __fmul_rn(e, f));
}
template <int M> __device__ __forceinline__ float linf(float a, float d, float m) {
    return M ? __fmaf_rn(a, d, m) : __fadd_rn(m, __fmul_rn(a, d));
}

// ---------------------------------------------------------------------------
// Node layouts (byte-identical to the reference's include/node_types.h) and
// the surface key each layout stores in its own slot while the surface pass
// runs.  A key orders the triangles that touched a node: triangle class
// (1D < 2D < 3D) first, then material; the largest key wins.
enum NodeKind { kShort = 0, kLong = 1, kPartial = 2, kShortFcc = 3, kLongFcc = 4 };

template <int K> struct NodeT;
template <> struct NodeT<kShort> {
    typedef uint8_t slot_t;
    static constexpr int bytes = 1;
    static constexpr bool fcc = false;
    __device__ static slot_t key(uint32_t cls, uint32_t mat, uint32_t) { return (slot_t)((cls << 3) | (mat & 7u)); }
    __device__ static uint32_t keyMat(uint64_t k) { return (uint32_t)k & 7u; }
    __device__ static uint64_t pack(uint32_t bid, uint32_t mat, float) { return (uint64_t)(((mat << 5) | (bid & 31u)) & 0xFFu); }
};
template <> struct NodeT<kLong> {
    typedef uint16_t slot_t;
    static constexpr int bytes = 2;
    static constexpr bool fcc = false;
    __device__ static slot_t key(uint32_t cls, uint32_t mat, uint32_t) { return (slot_t)((cls << 8) | (mat & 255u)); }
    __device__ static uint32_t keyMat(uint64_t k) { return (uint32_t)k & 255u; }
    __device__ static uint64_t pack(uint32_t bid, uint32_t mat, float) { return (uint64_t)((bid & 255u) | ((mat & 255u) << 8)); }
};
template <> struct NodeT<kPartial> {
    typedef unsigned long long slot_t;
    static constexpr int bytes = 8;
    static constexpr bool fcc = false;
    __device__ static slot_t key(uint32_t cls, uint32_t mat, uint32_t tri) {
        return ((slot_t)cls << 40) | ((slot_t)(mat & 255u) << 32) | (slot_t)tri;
    }
    __device__ static uint32_t keyMat(uint64_t k) { return (uint32_t)(k >> 32) & 255u; }
    __device__ static uint64_t pack(uint32_t bid, uint32_t mat, float r) {
        return (uint64_t)(bid & 255u) | ((uint64_t)(mat & 255u) << 8) | ((uint64_t)__float_as_uint(r) << 32);
    }
};
template <> struct NodeT<kShortFcc> {
    typedef uint16_t slot_t;
    static constexpr int bytes = 2;
    static constexpr bool fcc = true;
    __device__ static slot_t key(uint32_t cls, uint32_t mat, uint32_t) { return (slot_t)((cls << 4) | (mat & 15u)); }
    __device__ static uint32_t keyMat(uint64_t k) { return (uint32_t)k & 15u; }
    __device__ static uint64_t pack(uint32_t bid, uint32_t mat, float) { return (uint64_t)(((mat << 12) | (bid & 4095u)) & 0xFFFFu); }
};
template <> struct NodeT<kLongFcc> {
    typedef uint32_t slot_t;
    static constexpr int bytes = 4;
    static constexpr bool fcc = true;
    __device__ static slot_t key(uint32_t cls, uint32_t mat, uint32_t) { return (slot_t)((cls << 8) | (mat & 255u)); }
    __device__ static uint32_t keyMat(uint64_t k) { return (uint32_t)k & 255u; }
    __device__ static uint64_t pack(uint32_t bid, uint32_t mat, float) { return (uint64_t)((bid & 0xFFFFu) | ((mat & 255u) << 16)); }
};

// Atomic max of a node-sized key inside the 32-bit (or 64-bit) word that
// holds it.  Slots never straddle words: nodes are 1, 2, 4 or 8 bytes.
template <class S> __device__ __forceinline__ void slotMax(S* slot, S key);
template <> __device__ __forceinline__ void slotMax<unsigned long long>(unsigned long long* slot, unsigned long long key) {
    atomicMax(slot, key);
}
template <> __device__ __forceinline__ void slotMax<uint32_t>(uint32_t* slot, uint32_t key) { atomicMax(slot, key); }
template <class S> __device__ __forceinline__ void slotMax(S* slot, S key) {
    uintptr_t a = reinterpret_cast<uintptr_t>(slot);
    uint32_t* w = reinterpret_cast<uint32_t*>(a & ~uintptr_t(3));
    const uint32_t shift = (uint32_t)(a & 3u) * 8u;
    const uint32_t mask = (sizeof(S) == 1 ? 0xFFu : 0xFFFFu) << shift;
    uint32_t old = *reinterpret_cast<volatile uint32_t*>(w);
    for (;;) {
        uint32_t cur = (old & mask) >> shift;
        if ((uint32_t)key <= cur) return;
        uint32_t nv = (old & ~mask) | ((uint32_t)key << shift);
        uint32_t prev = atomicCAS(w, old, nv);
        if (prev == old) return;
        old = prev;
    }
}

// Boundary ids by 6-neighbour permutation (bits -x 1, +x 2, -y 4, +y 8,
// -z 16, +z 32), the numbering of the reference's getOrientation
// (src/voxelizer.cu:2142-2236, include/voxelizer.h:47-83).  Zero where an
// axis has no solid neighbour.
__device__ __constant__ static const uint8_t kOrientTable[64] = {
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
    0, 0, 0, 0, 0, 1, 2, 9, 0, 3, 4, 10, 0, 11, 12, 21,
    0, 0, 0, 0, 0, 5, 6, 13, 0, 7, 8, 14, 0, 15, 16, 26,
    0, 0, 0, 0, 0, 17, 18, 23, 0, 19, 20, 22, 0, 25, 24, 27,
};

}  // namespace vxb
