// PartialNode volume ratio (processVoxel<PartialNode> and
// calculateVoxelPlaneIntersectionVolume, hakarlss/Voxelizer
// src/voxelizer.cu:2996-3033, 4220-4807).
//
// The stored ratio of a surface node is |1 - V / d^3|, V the volume of the
// part of a voxel behind the plane of the node's triangle: the cut polygon
// and the three voxel faces reached from the corner nearest the plane are
// rotated flat and summed as pyramids with that corner as apex.  Facts of
// the reference the result depends on:
//  * the voxel is centred at minCorner + d * (node coordinates), the node
//    coordinates including the one-voxel padding, i.e. one voxel further
//    along x, y and z than the voxel that passed the overlap test;
//  * the normal is the class kernel's unnormalised cross product (zero for
//    1D-class triangles, which makes the ratio NaN);
//  * |n.x|, |n.y| or |n.z| exactly 1 takes the axis-parallel shortcut;
//  * a plane that misses the voxel leaves the cut polygon empty; the
//    reference then reads an unset array element for its pyramid, which is
//    taken here as an empty pyramid.
// The arithmetic is plain FP32 in the reference's operation order, compiled
// with nvcc's default contraction like the reference build, with IEEE
// division and square root and rsqrtf in the face normalisation as there.
#pragma once

#include "vxb_common.cuh"
#include "vxb_device.cuh"

namespace vxb {
namespace ratio {

using detail::F3;

__device__ __forceinline__ F3 add(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 sub(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 mul(float s, F3 a) { return F3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 rotX(F3 v, float s, float c) { return F3{v.x, v.y * c - v.z * s, v.y * s + v.z * c}; }
__device__ __forceinline__ F3 rotY(F3 v, float s, float c) { return F3{v.x * c + v.z * s, v.y, v.z * c - v.x * s}; }

struct Poly {
    F3 p[6];
    int n;
};
__device__ __forceinline__ void push(Poly& q, F3 v) {
    if (q.n < 6) q.p[q.n++] = v;
}

// Pyramid over `b` (already rotated into a plane z = const), apex `top`;
// surveyor's formula for the base area.
__device__ __forceinline__ float pyramid(const Poly& b, F3 top) {
    float area = 0.0f;
    for (int i = 0; i < b.n; i++) {
        const F3 u = b.p[i], w = b.p[(i + 1) % b.n];
        area += 0.5f * (u.x * w.y - w.x * u.y);
    }
    const float base0z = b.n ? b.p[0].z : 0.0f;
    return fabsf((1.0f / 3.0f) * area * (top.z - base0z));
}

// Rotates the polygon (in place) and the apex so that `rn` becomes the z
// axis: about x when rn.y != 0, then about y when the rotated rn.x != 0.
__device__ __forceinline__ float rotatedPyramid(Poly& q, F3 rn, F3 apex) {
    F3 top = apex;
    if (rn.y != 0.0f) {
        const float pl = sqrtf(rn.y * rn.y + rn.z * rn.z);
        const float sn = rn.y / pl, cs = rn.z / pl;
        top = rotX(top, sn, cs);
        for (int i = 0; i < q.n; i++) q.p[i] = rotX(q.p[i], sn, cs);
        rn = rotX(rn, sn, cs);
    }
    if (rn.x != 0.0f) {
        const float pl = sqrtf(rn.z * rn.z + rn.x * rn.x);
        const float sn = -rn.x / pl, cs = rn.z / pl;
        top = rotY(top, sn, cs);
        for (int i = 0; i < q.n; i++) q.p[i] = rotY(q.p[i], sn, cs);
    }
    return pyramid(q, top);
}

__device__ __forceinline__ float along(F3 n, F3 t0, F3 p, F3 q) { return dot(n, sub(t0, p)) / dot(n, sub(q, p)); }
__device__ __forceinline__ F3 point(F3 p, F3 q, float t) { return add(p, mul(t, sub(q, p))); }
// Both predicates are needed: a NaN t (an edge lying in the plane) is
// neither outside nor inside, and the reference tests the first two edges of
// a path for "outside" and the rest for "inside".
__device__ __forceinline__ bool inside(float t) { return t >= 0.0f && t <= 1.0f; }
__device__ __forceinline__ bool outside(float t) { return t < 0.0f || t > 1.0f; }

// Volume of voxel (x, y, z) (node coordinates) behind the plane through t0
// with normal n.
static __device__ __noinline__ float cutVolume(F3 t0, F3 n, int x, int y, int z, F3 m, float d) {
    const F3 vc = add(m, mul(d, F3{float(x), float(y), float(z)}));
    if (fabsf(n.x) == 1.0f) return (d * d) * ((d / 2.0f) + t0.x - vc.x);
    if (fabsf(n.y) == 1.0f) return (d * d) * ((d / 2.0f) + t0.y - vc.y);
    if (fabsf(n.z) == 1.0f) return (d * d) * ((d / 2.0f) + t0.z - vc.z);
    const bool sx = n.x > 0.0f, sy = n.y > 0.0f, sz = n.z > 0.0f;
    // Steps away from the corner on the normal's side; y and z steps trade
    // places when an odd number of components are positive (right-handed).
    const float ex = sx ? -d : d, ey = sy ? -d : d, ez = sz ? -d : d;
    const bool even = ((int)sx + (int)sy + (int)sz) % 2 == 0;
    const F3 dx{ex, 0.0f, 0.0f};
    const F3 dy = even ? F3{0.0f, ey, 0.0f} : F3{0.0f, 0.0f, ez};
    const F3 dz = even ? F3{0.0f, 0.0f, ez} : F3{0.0f, ey, 0.0f};
    const float h = d / 2.0f;
    F3 c[8];
    c[0] = add(vc, F3{sx ? h : -h, sy ? h : -h, sz ? h : -h});
    c[1] = add(c[0], dx);
    c[2] = add(c[0], dy);
    c[3] = add(c[0], dz);
    c[4] = add(c[1], dz);
    c[5] = add(c[2], dx);
    c[6] = add(c[3], dy);
    c[7] = add(c[4], dy);
    // Three corner paths 0 -> A -> B -> 7 with a side edge A -> S; path k
    // builds face k and closes the previous face where it turns at B.
    Poly cut, face[3];
    cut.n = face[0].n = face[1].n = face[2].n = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int A = k + 1, B = k + 4, S = k == 2 ? 4 : k + 5;
        Poly& own = face[k];
        Poly& prev = face[(k + 2) % 3];
        float t = along(n, t0, c[0], c[A]);
        if (outside(t)) {
            push(own, c[A]);
            t = along(n, t0, c[A], c[B]);
            if (outside(t)) {
                t = along(n, t0, c[B], c[7]);
                if (inside(t)) {
                    const F3 ip = point(c[B], c[7], t);
                    push(own, c[B]);
                    push(own, ip);
                    push(prev, ip);
                    push(prev, c[B]);
                    push(cut, ip);
                } else {
                    push(own, c[B]);
                    push(prev, c[B]);
                }
            } else {
                const F3 ip = point(c[A], c[B], t);
                push(own, ip);
                push(cut, ip);
            }
        } else {
            push(cut, point(c[0], c[A], t));
        }
        t = along(n, t0, c[A], c[S]);
        if (inside(t)) {
            const F3 ip = point(c[A], c[S], t);
            push(own, ip);
            push(cut, ip);
        }
    }
    float vol = rotatedPyramid(cut, n, c[0]);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        Poly& f = face[k];
        if (f.n <= 2) continue;
        const F3 e0 = sub(f.p[0], f.p[2]), e1 = sub(f.p[1], f.p[0]);
        const F3 fn = F3{e0.y * e1.z - e0.z * e1.y, e0.z * e1.x - e0.x * e1.z, e0.x * e1.y - e0.y * e1.x};
        const float inv = rsqrtf(dot(fn, fn));
        vol += rotatedPyramid(f, F3{fn.x * inv, fn.y * inv, fn.z * inv}, c[0]);
    }
    return vol;
}

// The ratio PartialNode stores for surface node (x, y, z) written by
// triangle `tri` of class `cls` (1D, 2D, 3D = 1, 2, 3).  The normal is the
// class kernel's cross product (v0 - v2) x (v1 - v0) with that kernel's
// contraction.  1D kernels pass a zero normal: every edge parameter is then
// 0 / 0 and the stored ratio is the NaN the reference's GPU build writes
// (0x7FFFFFFF after fabsf); it is returned directly, so cutVolume is only
// ever evaluated for a computed normal.
__device__ __forceinline__ float nodeRatio(const float* __restrict__ V, const uint32_t* __restrict__ I, uint32_t tri,
                                           uint32_t cls, int x, int y, int z, F3 m, float d) {
    if (cls < 2) return __int_as_float(0x7FFFFFFF);
    F3 v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const uint32_t a = __ldg(I + 3 * (size_t)tri + k);
        v[k] = F3{__ldg(V + 3 * (size_t)a), __ldg(V + 3 * (size_t)a + 1), __ldg(V + 3 * (size_t)a + 2)};
    }
    const F3 a{__fsub_rn(v[0].x, v[2].x), __fsub_rn(v[0].y, v[2].y), __fsub_rn(v[0].z, v[2].z)};
    const F3 b{__fsub_rn(v[1].x, v[0].x), __fsub_rn(v[1].y, v[0].y), __fsub_rn(v[1].z, v[0].z)};
    F3 n;
    if (cls == 2)
        n = F3{diff2f<site::CRF_2D>(a.y, b.z, a.z, b.y), diff2f<site::CRF_2D>(a.z, b.x, a.x, b.z),
               diff2f<site::CRF_2D>(a.x, b.y, a.y, b.x)};
    else
        n = F3{diff2f<site::CRF_3D>(a.y, b.z, a.z, b.y), diff2f<site::CRF_3D>(a.z, b.x, a.x, b.z),
               diff2f<site::CRF_3D>(a.x, b.y, a.y, b.x)};
    const float vol = cutVolume(v[0], n, x, y, z, m, d);
    return fabsf(1.0f - vol / (d * d * d));
}

}  // namespace ratio
}  // namespace vxb
