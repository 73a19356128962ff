// Test infrastructure (never linked into the product): evaluates, on the GPU,
// the reference's own PartialNode ratio arithmetic next to this project's.
//
// The reference's calculateVoxelPlaneIntersectionVolume (hakarlss/Voxelizer
// src/voxelizer.cu:4220-4807) is an inline __host__ __device__ function of
// src/voxelizer.cu, so this file includes that source file (from the
// reference tree, -I$(REF)/src; nothing is copied) and calls the function
// from a kernel, with processVoxel<PartialNode>'s final step
// |1 - V / d^3| (src/voxelizer.cu:3029-3032).  The same inputs go through
// vxb::ratio::cutVolume (voxelizer_b200/csrc/vxb_ratio.cuh).
//
// The plane normal the reference's class kernels pass is the cross product
// (v0 - v2) x (v1 - v0) with some multiply-add contraction; the probe
// evaluates both functions for three forms of it (per component a*b - c*d):
//   0: no fma   1: fma(a, b, -(c*d))   2: fma(-c, d, a*b)
// and 1D-class inputs (cls 1) get the zero normal the 1D kernel passes.

#include "voxelizer.cu"
#include "vxb_ratio.cuh"

namespace {

__device__ float crossComp(float a, float b, float c, float d, int mode) {
    if (mode == 0) return __fsub_rn(__fmul_rn(a, b), __fmul_rn(c, d));
    if (mode == 1) return __fmaf_rn(a, b, -__fmul_rn(c, d));
    return __fmaf_rn(-c, d, __fmul_rn(a, b));
}

__global__ void probeKernel(int n, const float* __restrict__ tris, const unsigned char* __restrict__ cls,
                            const int* __restrict__ xyz, float3 m, float d, float* __restrict__ refOut,
                            float* __restrict__ ourOut) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float3 t[3];
        for (int k = 0; k < 3; ++k) t[k] = make_float3(tris[9 * i + 3 * k], tris[9 * i + 3 * k + 1], tris[9 * i + 3 * k + 2]);
        const float3 a = make_float3(__fsub_rn(t[0].x, t[2].x), __fsub_rn(t[0].y, t[2].y), __fsub_rn(t[0].z, t[2].z));
        const float3 b = make_float3(__fsub_rn(t[1].x, t[0].x), __fsub_rn(t[1].y, t[0].y), __fsub_rn(t[1].z, t[0].z));
        const int3 v = make_int3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        for (int mode = 0; mode < 3; ++mode) {
            float3 nr = make_float3(0.0f, 0.0f, 0.0f);
            if (cls[i] >= 2)
                nr = make_float3(crossComp(a.y, b.z, a.z, b.y, mode), crossComp(a.z, b.x, a.x, b.z, mode),
                                 crossComp(a.x, b.y, a.y, b.x, mode));
            float3 tt[3] = {t[0], t[1], t[2]};
            const float rv = vox::calculateVoxelPlaneIntersectionVolume(tt, v, nr, m, d);
            refOut[(size_t)mode * n + i] = fabsf(1.0f - rv / (d * d * d));
            const float ov = vxb::ratio::cutVolume(vxb::detail::F3{t[0].x, t[0].y, t[0].z},
                                                   vxb::detail::F3{nr.x, nr.y, nr.z}, v.x, v.y, v.z,
                                                   vxb::detail::F3{m.x, m.y, m.z}, d);
            ourOut[(size_t)mode * n + i] = fabsf(1.0f - ov / (d * d * d));
        }
    }
}

}  // namespace

// n inputs: tris (9 floats each), cls (1..3), xyz (node coordinates, 3 ints
// each); outputs ref / ours hold 3 * n ratios (normal form major).
extern "C" int probe_ratios(int n, const float* tris, const unsigned char* cls, const int* xyz, const float* m,
                            float d, float* ref, float* ours) {
    float *dT = nullptr, *dR = nullptr, *dO = nullptr;
    unsigned char* dC = nullptr;
    int* dX = nullptr;
    const size_t nn = (size_t)(n > 0 ? n : 1);
    if (cudaMalloc(&dT, 9 * nn * sizeof(float)) || cudaMalloc(&dC, nn) || cudaMalloc(&dX, 3 * nn * sizeof(int)) ||
        cudaMalloc(&dR, 3 * nn * sizeof(float)) || cudaMalloc(&dO, 3 * nn * sizeof(float)))
        return -1;
    cudaMemcpy(dT, tris, 9 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(dC, cls, (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(dX, xyz, 3 * (size_t)n * sizeof(int), cudaMemcpyHostToDevice);
    if (n > 0) probeKernel<<<(n + 127) / 128, 128>>>(n, dT, dC, dX, make_float3(m[0], m[1], m[2]), d, dR, dO);
    int rc = cudaDeviceSynchronize() == cudaSuccess ? 0 : -2;
    cudaMemcpy(ref, dR, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(ours, dO, 3 * (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(dT);
    cudaFree(dC);
    cudaFree(dX);
    cudaFree(dR);
    cudaFree(dO);
    return rc;
}
