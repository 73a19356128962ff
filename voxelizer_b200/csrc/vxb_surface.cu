// Surface voxelization kernels (FP32): classifyTriangles / analyzeBoundingBox
// / encodeTriangleType (src/voxelizer.cu:3040-3221) and the 1D / 2D / 3D
// processing kernels (3306-3955) with processVoxel (2946-2989).
//
// Work is a flat list of (triangle, material subspace, column) items over an
// exclusive scan of per-triangle column counts, one thread per column (per
// voxel of a 1D line).  A block stages the triangles its 256 items belong to
// in shared memory first: vertices, class code, voxel box, normal and the
// edge functions of the three projections are computed once per triangle,
// not once per column.
//
// Hits set the voxel's bit in the surface grid and append (bit position,
// material key) to a hit list.  Once all surface bits exist, every surface
// voxel gets a rank (prefix popcount over the surface grid), and the list is
// max-merged into a compact key array indexed by rank; the emit kernels read
// materials from there.  The key orders triangles by class, then material
// (NodeT in vxb_device.cuh), so the merged key names the winning material.
// If the list overflows, a second traversal (mode 1) merges every hit
// directly.

#include "vxb_common.cuh"
#include "vxb_device.cuh"
#include "vxb_kernels.cuh"

namespace vxb {

using namespace detail;

namespace {

constexpr int kBlock = 256;
constexpr uint32_t kSlots = 144;  // staged triangles per block (27 KB of shared memory)

__device__ __forceinline__ void loadTriF(const float* __restrict__ V, const uint32_t* __restrict__ I, uint32_t t,
                                         F3* v) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        uint32_t a = __ldg(I + 3 * t + k);
        v[k] = F3{__ldg(V + 3 * a), __ldg(V + 3 * a + 1), __ldg(V + 3 * a + 2)};
    }
}

__device__ __forceinline__ F3 subF(F3 a, F3 b) { return F3{__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }

template <int M> __device__ __forceinline__ F3 crossF(F3 a, F3 b) {
    return F3{diff2f<M>(a.y, b.z, a.z, b.y), diff2f<M>(a.z, b.x, a.x, b.z), diff2f<M>(a.x, b.y, a.y, b.x)};
}

struct IBox { int lo[3], hi[3]; };

// getTriangleBounds (float3, src/voxelizer.cu:2366-2390) and
// getVoxelBoundsHalf (2471-2492).
__device__ __forceinline__ IBox voxBoundsHalf(const F3* v, const PassGeom& g) {
    F3 mn = v[0], mx = v[0];
#pragma unroll
    for (int i = 1; i < 3; ++i) {
        if (v[i].x < mn.x) mn.x = v[i].x;
        if (v[i].y < mn.y) mn.y = v[i].y;
        if (v[i].z < mn.z) mn.z = v[i].z;
        if (v[i].x > mx.x) mx.x = v[i].x;
        if (v[i].y > mx.y) mx.y = v[i].y;
        if (v[i].z > mx.z) mx.z = v[i].z;
    }
    const float d = g.df;
    IBox b;
    b.lo[0] = __float2int_rz(ceilf(__fsub_rn(__fdiv_rn(__fsub_rn(mn.x, g.mnf[0]), d), 0.5f)));
    b.lo[1] = __float2int_rz(ceilf(__fsub_rn(__fdiv_rn(__fsub_rn(mn.y, g.mnf[1]), d), 0.5f)));
    b.lo[2] = __float2int_rz(ceilf(__fsub_rn(__fdiv_rn(__fsub_rn(mn.z, g.mnf[2]), d), 0.5f)));
    b.hi[0] = __float2int_rz(floorf(__fadd_rn(__fdiv_rn(__fsub_rn(mx.x, g.mnf[0]), d), 0.5f)));
    b.hi[1] = __float2int_rz(floorf(__fadd_rn(__fdiv_rn(__fsub_rn(mx.y, g.mnf[1]), d), 0.5f)));
    b.hi[2] = __float2int_rz(floorf(__fadd_rn(__fdiv_rn(__fsub_rn(mx.z, g.mnf[2]), d), 0.5f)));
    return b;
}

__device__ __forceinline__ uint32_t classifyTri(const F3* v, const PassGeom& g) {
    const F3 n = crossF<site::CRF_CLS>(subF(v[0], v[2]), subF(v[1], v[0]));
    if (!(n.x != 0.0f || n.y != 0.0f || n.z != 0.0f)) return 0u;
    const IBox b = voxBoundsHalf(v, g);
    const int dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    uint32_t bb, axis, cols;
    if (dx == 0) {
        if (dy == 0) {
            if (dz == 0) { bb = 1; axis = 0; cols = 1; }
            else { bb = 1; axis = 2; cols = (uint32_t)dz; }
        } else if (dz == 0) { bb = 1; axis = 1; cols = (uint32_t)dy; }
        else { bb = 2; axis = 0; cols = (uint32_t)(dy * dz); }
    } else if (dy == 0) {
        if (dz == 0) { bb = 1; axis = 0; cols = (uint32_t)dx; }
        else { bb = 2; axis = 1; cols = (uint32_t)(dx * dz); }
    } else if (dz == 0) { bb = 2; axis = 2; cols = (uint32_t)(dx * dy); }
    else {
        bb = 3;
        const float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
        if (ax > ay && ax > az) axis = 0;
        else if (ay > ax && ay > az) axis = 1;
        else axis = 2;
        cols = axis == 0 ? (uint32_t)(dy * dz) : axis == 1 ? (uint32_t)(dx * dz) : (uint32_t)(dx * dy);
    }
    return cols | (axis << 28) | (bb << 30);
}

// adjustVoxelRange, src/voxelizer.cu:3963-3993.
__device__ __forceinline__ bool clampBox(IBox& b, const Split3& s) {
    const int lo[3] = {(int)s.x0, (int)s.y0, (int)s.z0};
    const int hi[3] = {(int)s.x1 - 1, (int)s.y1 - 1, (int)s.z1 - 1};
    if (lo[0] > b.hi[0] || lo[1] > b.hi[1] || lo[2] > b.hi[2]) return false;
    if (b.lo[0] > hi[0] || b.lo[1] > hi[1] || b.lo[2] > hi[2]) return false;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = max(b.lo[a], lo[a]);
        b.hi[a] = min(b.hi[a], hi[a]);
    }
    return true;
}

// Work units of one (triangle, material subspace): voxels along the axis for
// 1D boxes, columns of the dominant projection otherwise.
__device__ __forceinline__ uint32_t surfUnits(const IBox& b, uint32_t code) {
    const uint32_t bb = code >> 30, axis = (code >> 28) & 3u;
    const uint32_t ex = (uint32_t)(b.hi[0] - b.lo[0] + 1), ey = (uint32_t)(b.hi[1] - b.lo[1] + 1),
                   ez = (uint32_t)(b.hi[2] - b.lo[2] + 1);
    if (bb == 1) return axis == 0 ? ex : axis == 1 ? ey : ez;
    return axis == 0 ? ey * ez : axis == 1 ? ex * ez : ex * ey;
}

__global__ void surfaceCountKernel(const float* __restrict__ V, const uint32_t* __restrict__ I, uint32_t nT,
                                   PassGeom g, const Split3* __restrict__ splits, uint32_t nSplits,
                                   uint32_t* __restrict__ codes, uint32_t* __restrict__ counts) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nT; t += gridDim.x * blockDim.x) {
        F3 v[3];
        loadTriF(V, I, t, v);
        const uint32_t code = classifyTri(v, g);
        codes[t] = code;
        uint32_t c = 0;
        if ((code >> 30) != 0) {
            const IBox full = voxBoundsHalf(v, g);
            for (uint32_t s = 0; s < nSplits; ++s) {
                IBox b = full;
                if (!clampBox(b, splits[s])) continue;
                c += surfUnits(b, code);
            }
        }
        counts[t] = c;
    }
}

struct Overlap { float nx[3], ny[3], de[3]; };

// Per-edge contraction modes: the three edge expressions of a test are
// separate (unrolled) expressions in the reference, so a site's mode packs
// two bits per edge.
__device__ __forceinline__ float sum2fm(int m, float a, float b, float c, float d) {
    return m == 0 ? sum2f<0>(a, b, c, d) : m == 1 ? sum2f<1>(a, b, c, d) : sum2f<2>(a, b, c, d);
}
__device__ __forceinline__ float sum2p1fm(int m, float a, float b, float c, float d, float e) {
    return m == 0 ? sum2p1f<0>(a, b, c, d, e) : m == 1 ? sum2p1f<1>(a, b, c, d, e)
         : m == 2 ? sum2p1f<2>(a, b, c, d, e) : sum2p1f<3>(a, b, c, d, e);
}

// setupYZ / ZX / XYOverlapTest (src/voxelizer.cu:2675-2757).  A = 0: (y, z)
// oriented by n.x; A = 1: (z, x) by n.y; A = 2: (x, y) by n.z.
template <int A, int DE> __device__ __forceinline__ Overlap setupOverlap(const F3* t, F3 n, float d) {
    Overlap o;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const F3& p = t[i];
        const F3& q = t[(i + 1) % 3];
        float pa, pb, qa, qb, nn;
        if (A == 0) { pa = p.y; pb = p.z; qa = q.y; qb = q.z; nn = n.x; }
        else if (A == 1) { pa = p.z; pb = p.x; qa = q.z; qb = q.x; nn = n.y; }
        else { pa = p.x; pb = p.y; qa = q.x; qb = q.y; nn = n.z; }
        if (nn >= 0.0f) { o.nx[i] = __fsub_rn(pb, qb); o.ny[i] = __fsub_rn(qa, pa); }
        else { o.nx[i] = __fsub_rn(qb, pb); o.ny[i] = __fsub_rn(pa, qa); }
        const float s = sum2fm((DE >> (2 * i)) & 3, o.nx[i], pa, o.ny[i], pb);
        o.de[i] = __fadd_rn(__fadd_rn(-s, fmaxf(0.0f, __fmul_rn(d, o.nx[i]))), fmaxf(0.0f, __fmul_rn(d, o.ny[i])));
    }
    return o;
}

template <int OT> __device__ __forceinline__ bool overlapTest(const Overlap& o, float a, float b) {
    bool r = true;
#pragma unroll
    for (int i = 0; i < 3; ++i) r &= sum2p1fm((OT >> (2 * i)) & 3, o.nx[i], a, o.ny[i], b, o.de[i]) >= 0.0f;
    return r;
}

// getSingleVoxelBoundsComponent, src/voxelizer.cu:2575-2586.
template <int M> __device__ __forceinline__ float vbComp(int c, float m, float d) {
    return linf<M>(__fsub_rn((float)c, 0.5f), d, m);
}

// determineDepthRange{X,Y,Z} (src/voxelizer.cu:3994-4119) with
// intersectWithPlane* and boundsCheck.
template <int A, int DT> __device__ __forceinline__ void depthRange(const F3* t, F3 p, F3 n, const PassGeom& g,
                                                                    int& lo, int& hi) {
    const float d = g.df;
    F3 pmin, pmax;
    float a, b;
    if (A == 0) {
        const float sy = n.y > 0.0f ? 1.0f : 0.0f, sz = n.z > 0.0f ? 1.0f : 0.0f;
        pmin = F3{0.0f, __fadd_rn(p.y, __fmul_rn(sy, d)), __fadd_rn(p.z, __fmul_rn(sz, d))};
        pmax = F3{0.0f, __fadd_rn(p.y, __fmul_rn(1.0f - sy, d)), __fadd_rn(p.z, __fmul_rn(1.0f - sz, d))};
        const F3 u = subF(t[0], pmin), w = subF(t[0], pmax);
        a = __fdiv_rn(sum3f<DT>(u.x, n.x, u.y, n.y, u.z, n.z), n.x);
        b = __fdiv_rn(sum3f<DT>(w.x, n.x, w.y, n.y, w.z, n.z), n.x);
    } else if (A == 1) {
        const float sx = n.x > 0.0f ? 1.0f : 0.0f, sz = n.z > 0.0f ? 1.0f : 0.0f;
        pmin = F3{__fadd_rn(p.x, __fmul_rn(sx, d)), 0.0f, __fadd_rn(p.z, __fmul_rn(sz, d))};
        pmax = F3{__fadd_rn(p.x, __fmul_rn(1.0f - sx, d)), 0.0f, __fadd_rn(p.z, __fmul_rn(1.0f - sz, d))};
        const F3 u = subF(t[0], pmin), w = subF(t[0], pmax);
        a = __fdiv_rn(sum3f<DT>(u.x, n.x, u.y, n.y, u.z, n.z), n.y);
        b = __fdiv_rn(sum3f<DT>(w.x, n.x, w.y, n.y, w.z, n.z), n.y);
    } else {
        const float sx = n.x > 0.0f ? 1.0f : 0.0f, sy = n.y > 0.0f ? 1.0f : 0.0f;
        pmin = F3{__fadd_rn(p.x, __fmul_rn(sx, d)), __fadd_rn(p.y, __fmul_rn(sy, d)), 0.0f};
        pmax = F3{__fadd_rn(p.x, __fmul_rn(1.0f - sx, d)), __fadd_rn(p.y, __fmul_rn(1.0f - sy, d)), 0.0f};
        const F3 u = subF(t[0], pmin), w = subF(t[0], pmax);
        a = __fdiv_rn(sum3f<DT>(u.x, n.x, u.y, n.y, u.z, n.z), n.z);
        b = __fdiv_rn(sum3f<DT>(w.x, n.x, w.y, n.y, w.z, n.z), n.z);
    }
    if (a > b) { float tmp = a; a = b; b = tmp; }
    const float m = A == 0 ? g.mnf[0] : A == 1 ? g.mnf[1] : g.mnf[2];
    lo = __float2int_rz(ceilf(__fsub_rn(__fdiv_rn(__fsub_rn(a, m), d), 0.5f)));
    hi = __float2int_rz(floorf(__fadd_rn(__fdiv_rn(__fsub_rn(b, m), d), 0.5f)));
}

// Triangle setup shared by the columns of a block.
struct TriStage {
    F3 v[3];
    F3 n;
    IBox full;
    uint32_t code;
    uint32_t key;      // class << 8 | material (32-bit key types)
    uint32_t tri;
    Overlap o[3];
};

__device__ __forceinline__ void stageTriangle(TriStage& st, const float* V, const uint32_t* I, const uint8_t* M,
                                              const uint32_t* codes, uint32_t t, const PassGeom& g) {
    loadTriF(V, I, t, st.v);
    st.code = __ldg(codes + t);
    st.tri = t;
    st.full = voxBoundsHalf(st.v, g);
    const uint32_t bb = st.code >> 30;
    st.key = (bb << 8) | __ldg(M + t);
    const float d = g.df;
    if (bb == 2) {
        st.n = crossF<site::CRF_2D>(subF(st.v[0], st.v[2]), subF(st.v[1], st.v[0]));
        const uint32_t axis = (st.code >> 28) & 3u;
        if (axis == 0) st.o[0] = setupOverlap<0, site::DE_2D_YZ>(st.v, st.n, d);
        else if (axis == 1) st.o[1] = setupOverlap<1, site::DE_2D_ZX>(st.v, st.n, d);
        else st.o[2] = setupOverlap<2, site::DE_2D_XY>(st.v, st.n, d);
    } else if (bb == 3) {
        st.n = crossF<site::CRF_3D>(subF(st.v[0], st.v[2]), subF(st.v[1], st.v[0]));
        st.o[0] = setupOverlap<0, site::DE_3D_YZ>(st.v, st.n, d);
        st.o[1] = setupOverlap<1, site::DE_3D_ZX>(st.v, st.n, d);
        st.o[2] = setupOverlap<2, site::DE_3D_XY>(st.v, st.n, d);
    }
}

// processVoxel of the surface pass, coordinates with the 1-voxel padding.
// mode 0: set the bit and append (bit position << 24 | key) to the hit list;
// mode 1: merge the key at the voxel's rank (surface bits are complete).
struct Sink {
    uint32_t* bits;          // surface grid of this lattice
    uint64_t posBase;        // bit position of bits[0] in the rank space
    const uint32_t* wordRank;  // exclusive popcount prefix per word (mode 1)
    void* keys;              // compact key array (mode 1)
    unsigned long long* list;
    uint32_t* listCount;
    uint32_t listCap;
    int mode;
    int wide;                // 64-bit keys (PartialNode)
    PassGeom g;
    __device__ __forceinline__ void operator()(int xi, int yi, int zi, uint64_t key) const {
        const uint32_t x = (uint32_t)xi, y = (uint32_t)yi, z = (uint32_t)zi;
        const size_t w = ((size_t)z * g.AY + y) * g.ipx + (x >> 5);
        const uint32_t b = x & 31u;
        const uint32_t bit = 0x80000000u >> b;
        if (mode == 0) {
            atomicOr(bits + w, bit);
            const uint32_t active = __activemask();
            const uint32_t lane = threadIdx.x & 31u;
            const uint32_t leader = __ffs(active) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(listCount, (uint32_t)__popc(active));
            base = __shfl_sync(active, base, leader);
            const uint32_t at = base + __popc(active & laneMaskLt());
            if (at < listCap)
                list[at] = ((unsigned long long)(posBase + (uint64_t)w * 32 + b) << 24) | (key & 0xFFFFFFull);
        } else {
            const uint32_t word = __ldg(bits + w);
            const uint32_t r = __ldg(wordRank + (posBase >> 5) + w) + (b ? __popc(word >> (32 - b)) : 0u);
            if (wide) atomicMax(reinterpret_cast<unsigned long long*>(keys) + r, (unsigned long long)key);
            else atomicMax(reinterpret_cast<uint32_t*>(keys) + r, (uint32_t)key);
        }
    }
};

// Columns of one staged triangle (process1D/2D/3DTriangles).
__device__ __forceinline__ void surfaceColumn(const TriStage& st, const IBox& b, uint32_t u, const PassGeom& g,
                                              uint64_t key, const Sink& sink) {
    const uint32_t bb = st.code >> 30, axis = (st.code >> 28) & 3u;
    const float d = g.df;
    const uint32_t ex = (uint32_t)(b.hi[0] - b.lo[0] + 1), ey = (uint32_t)(b.hi[1] - b.lo[1] + 1);
    const F3* v = st.v;
    if (bb == 1) {
        // process1DTriangles (3306-3411): every voxel of the line, no test.
        if (axis == 0) sink(b.lo[0] + (int)u + 1, b.lo[1] + 1, b.lo[2] + 1, key);
        else if (axis == 1) sink(b.lo[0] + 1, b.lo[1] + (int)u + 1, b.lo[2] + 1, key);
        else sink(b.lo[0] + 1, b.lo[1] + 1, b.lo[2] + (int)u + 1, key);
        return;
    }
    if (bb == 2) {
        // process2DTriangles (3418-3596): the dominant projection only.
        if (axis == 0) {
            const int j = b.lo[1] + (int)(u % ey), k = b.lo[2] + (int)(u / ey);
            if (overlapTest<site::OT_2D_YZ>(st.o[0], vbComp<site::PC_2D>(j, g.mnf[1], d), vbComp<site::PC_2D>(k, g.mnf[2], d)))
                sink(b.lo[0] + 1, j + 1, k + 1, key);
        } else if (axis == 1) {
            const int i = b.lo[0] + (int)(u % ex), k = b.lo[2] + (int)(u / ex);
            if (overlapTest<site::OT_2D_ZX>(st.o[1], vbComp<site::PC_2D>(k, g.mnf[2], d), vbComp<site::PC_2D>(i, g.mnf[0], d)))
                sink(i + 1, b.lo[1] + 1, k + 1, key);
        } else {
            const int i = b.lo[0] + (int)(u % ex), j = b.lo[1] + (int)(u / ex);
            if (overlapTest<site::OT_2D_XY>(st.o[2], vbComp<site::PC_2D>(i, g.mnf[0], d), vbComp<site::PC_2D>(j, g.mnf[1], d)))
                sink(i + 1, j + 1, b.lo[2] + 1, key);
        }
        return;
    }
    // process3DTriangles (3603-3955): dominant projection, depth range from
    // the plane, then the other two projections per voxel unless the range
    // is a single voxel.
    const F3 n = st.n;
    if (axis == 0) {
        const int j = b.lo[1] + (int)(u % ey), k = b.lo[2] + (int)(u / ey);
        F3 p{0.0f, vbComp<site::PC_3D>(j, g.mnf[1], d), vbComp<site::PC_3D>(k, g.mnf[2], d)};
        if (!overlapTest<site::OT_3D_YZ>(st.o[0], p.y, p.z)) return;
        int r0, r1;
        depthRange<0, site::DT_3DX>(v, p, n, g, r0, r1);
        if (r0 > b.hi[0] || r1 < b.lo[0]) return;
        r0 = r0 < b.lo[0] ? b.lo[0] : r0;
        r1 = r1 > b.hi[0] ? b.hi[0] : r1;
        if (r0 == r1) { sink(r0 + 1, j + 1, k + 1, key); return; }
        for (int i = r0; i <= r1; ++i) {
            p.x = vbComp<site::PC_3DL>(i, g.mnf[0], d);
            if (overlapTest<site::OT_3DX_ZX>(st.o[1], p.z, p.x) && overlapTest<site::OT_3DX_XY>(st.o[2], p.x, p.y))
                sink(i + 1, j + 1, k + 1, key);
        }
    } else if (axis == 1) {
        const int i = b.lo[0] + (int)(u % ex), k = b.lo[2] + (int)(u / ex);
        F3 p{vbComp<site::PC_3D>(i, g.mnf[0], d), 0.0f, vbComp<site::PC_3D>(k, g.mnf[2], d)};
        if (!overlapTest<site::OT_3D_ZX>(st.o[1], p.z, p.x)) return;
        int r0, r1;
        depthRange<1, site::DT_3DY>(v, p, n, g, r0, r1);
        if (r0 > b.hi[1] || r1 < b.lo[1]) return;
        r0 = r0 < b.lo[1] ? b.lo[1] : r0;
        r1 = r1 > b.hi[1] ? b.hi[1] : r1;
        if (r0 == r1) { sink(i + 1, r0 + 1, k + 1, key); return; }
        for (int j = r0; j <= r1; ++j) {
            p.y = vbComp<site::PC_3DL>(j, g.mnf[1], d);
            if (overlapTest<site::OT_3DY_XY>(st.o[2], p.x, p.y) && overlapTest<site::OT_3DY_YZ>(st.o[0], p.y, p.z))
                sink(i + 1, j + 1, k + 1, key);
        }
    } else {
        const int i = b.lo[0] + (int)(u % ex), j = b.lo[1] + (int)(u / ex);
        F3 p{vbComp<site::PC_3D>(i, g.mnf[0], d), vbComp<site::PC_3D>(j, g.mnf[1], d), 0.0f};
        if (!overlapTest<site::OT_3D_XY>(st.o[2], p.x, p.y)) return;
        int r0, r1;
        depthRange<2, site::DT_3DZ>(v, p, n, g, r0, r1);
        if (r0 > b.hi[2] || r1 < b.lo[2]) return;
        r0 = r0 < b.lo[2] ? b.lo[2] : r0;
        r1 = r1 > b.hi[2] ? b.hi[2] : r1;
        if (r0 == r1) { sink(i + 1, j + 1, r0 + 1, key); return; }
        for (int k = r0; k <= r1; ++k) {
            p.z = vbComp<site::PC_3DL>(k, g.mnf[2], d);
            if (overlapTest<site::OT_3DZ_YZ>(st.o[0], p.y, p.z) && overlapTest<site::OT_3DZ_ZX>(st.o[1], p.z, p.x))
                sink(i + 1, j + 1, k + 1, key);
        }
    }
}

// The (split, column) of a staged triangle for its `local` work unit.
__device__ __forceinline__ IBox locateUnit(const TriStage& st, const Split3* __restrict__ splits, uint32_t nSplits,
                                           uint32_t& local) {
    IBox b = st.full;
    for (uint32_t s = 0; s < nSplits; ++s) {
        b = st.full;
        if (!clampBox(b, splits[s])) continue;
        const uint32_t n = surfUnits(b, st.code);
        if (local < n) break;
        local -= n;
    }
    return b;
}

__global__ void __launch_bounds__(kBlock) surfaceWorkKernel(
    Sink sink, const float* __restrict__ V, const uint32_t* __restrict__ I, const uint8_t* __restrict__ M, uint32_t nT,
    PassGeom g, const Split3* __restrict__ splits, uint32_t nSplits, const uint32_t* __restrict__ codes,
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ totalPtr) {
    __shared__ TriStage stage[kSlots];
    __shared__ uint32_t stOff[kSlots + 1];
    __shared__ uint32_t tFirst, nStage;
    const uint32_t total = *totalPtr;
    for (uint32_t base = blockIdx.x * kBlock; base < total; base += gridDim.x * kBlock) {
        const uint32_t last = min(base + kBlock, total) - 1;
        if (threadIdx.x == 0) {
            const uint32_t t0 = findOwner(offsets, nT, base);
            const uint32_t t1 = findOwner(offsets, nT, last);
            tFirst = t0;
            nStage = min(t1 - t0 + 1, kSlots);
        }
        __syncthreads();
        const uint32_t t0 = tFirst, ns = nStage;
        if (threadIdx.x < ns) {
            stageTriangle(stage[threadIdx.x], V, I, M, codes, t0 + threadIdx.x, g);
            stOff[threadIdx.x] = __ldg(offsets + t0 + threadIdx.x);
        }
        if (threadIdx.x == 0) stOff[ns] = __ldg(offsets + t0 + ns);
        __syncthreads();
        const uint32_t item = base + threadIdx.x;
        if (item <= last) {
            if (item < stOff[ns]) {
                uint32_t lo = 0, hi = ns;  // stOff[lo] <= item < stOff[hi]
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (stOff[mid] <= item) lo = mid;
                    else hi = mid;
                }
                const TriStage& st = stage[lo];
                uint32_t local = item - stOff[lo];
                const IBox b = locateUnit(st, splits, nSplits, local);
                const uint64_t key = sink.wide ? (((uint64_t)(st.code >> 30) << 40) |
                                                  ((uint64_t)(st.key & 255u) << 32) | st.tri)
                                               : (uint64_t)st.key;
                surfaceColumn(st, b, local, g, key, sink);
            } else {
                // More triangles than staging slots (runs of zero-unit
                // triangles): stage privately.
                const uint32_t t = findOwner(offsets, nT, item);
                TriStage st;
                stageTriangle(st, V, I, M, codes, t, g);
                uint32_t local = item - __ldg(offsets + t);
                const IBox b = locateUnit(st, splits, nSplits, local);
                const uint64_t key = sink.wide ? (((uint64_t)(st.code >> 30) << 40) |
                                                  ((uint64_t)(st.key & 255u) << 32) | st.tri)
                                               : (uint64_t)st.key;
                surfaceColumn(st, b, local, g, key, sink);
            }
        }
        __syncthreads();
    }
}

// Exclusive popcount prefix over the surface words (ranks of surface voxels).
constexpr int kRankItems = 8;
constexpr uint32_t kRankTile = kBlock * kRankItems;

__global__ void rankTileKernel(const uint32_t* __restrict__ words, uint64_t n, uint32_t* __restrict__ ranks,
                               uint32_t* __restrict__ tileSums) {
    __shared__ uint32_t warpSums[33];
    const uint64_t base = (uint64_t)blockIdx.x * kRankTile + (uint64_t)threadIdx.x * kRankItems;
    uint32_t c[kRankItems];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kRankItems; ++i) {
        c[i] = base + i < n ? (uint32_t)__popc(__ldg(words + base + i)) : 0u;
        sum += c[i];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warpSums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t s = lane < (kBlock / 32) ? warpSums[lane] : 0u;
        uint32_t si = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += t;
        }
        if (lane < kBlock / 32) warpSums[lane] = si - s;
        if (lane == 31) warpSums[32] = si;
    }
    __syncthreads();
    uint32_t ex = warpSums[warp] + incl - sum;
#pragma unroll
    for (int i = 0; i < kRankItems; ++i) {
        if (base + i < n) ranks[base + i] = ex;
        ex += c[i];
    }
    if (threadIdx.x == 0) tileSums[blockIdx.x] = warpSums[32];
}

__global__ void rankSumsKernel(uint32_t* tileSums, uint32_t nTiles, uint32_t* total) {
    __shared__ uint32_t warpSums[33];
    uint32_t carry = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t start = 0; start < nTiles; start += blockDim.x) {
        const uint32_t i = start + threadIdx.x;
        const uint32_t v = i < nTiles ? tileSums[i] : 0u;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warpSums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint32_t s = lane < (int)(blockDim.x >> 5) ? warpSums[lane] : 0u;
            uint32_t si = s;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, si, o);
                if (lane >= o) si += t;
            }
            if (lane < (int)(blockDim.x >> 5)) warpSums[lane] = si - s;
            if (lane == 31) warpSums[32] = si;
        }
        __syncthreads();
        if (i < nTiles) tileSums[i] = carry + warpSums[warp] + incl - v;
        carry += warpSums[32];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void rankAddKernel(uint32_t* ranks, uint64_t n, const uint32_t* __restrict__ tileSums) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        ranks[i] += tileSums[i / kRankTile];
}

__global__ void zeroKeysKernel(void* keys, const uint32_t* __restrict__ countPtr, int wide) {
    const uint32_t n = *countPtr;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (wide) reinterpret_cast<unsigned long long*>(keys)[i] = 0ull;
        else reinterpret_cast<uint32_t*>(keys)[i] = 0u;
    }
}

// Max-merges the hit list into the rank-indexed key array.
__global__ void mergeKeysKernel(const unsigned long long* __restrict__ list, const uint32_t* __restrict__ countPtr,
                                uint32_t cap, const uint32_t* __restrict__ bits, const uint32_t* __restrict__ ranks,
                                uint32_t* keys) {
    const uint32_t n = min(*countPtr, cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long e = list[i];
        const uint64_t pos = e >> 24;
        const uint64_t w = pos >> 5;
        const uint32_t b = (uint32_t)(pos & 31u);
        const uint32_t word = __ldg(bits + w);
        const uint32_t r = __ldg(ranks + w) + (b ? __popc(word >> (32 - b)) : 0u);
        atomicMax(keys + r, (uint32_t)(e & 0xFFFFFFull));
    }
}

}  // namespace

void launch_surface_count(const float* V, const uint32_t* I, uint32_t nT, PassGeom g, const Split3* splits,
                          uint32_t nSplits, uint32_t* codes, uint32_t* counts, cudaStream_t s, uint32_t* launches) {
    surfaceCountKernel<<<gridFor(nT, 256), 256, 0, s>>>(V, I, nT, g, splits, nSplits, codes, counts);
    *launches += 1;
}

void launch_surface_work(int mode, int wide, const float* V, const uint32_t* I, const uint8_t* M, uint32_t nT,
                         PassGeom g, const Split3* splits, uint32_t nSplits, const uint32_t* codes,
                         const uint32_t* offsets, const uint32_t* total, uint32_t* surfBits, uint64_t posBase,
                         const uint32_t* ranks, void* keys, unsigned long long* list, uint32_t* listCount,
                         uint32_t listCap, cudaStream_t s, uint32_t* launches) {
    Sink sink;
    sink.bits = surfBits;
    sink.posBase = posBase;
    sink.wordRank = ranks;
    sink.keys = keys;
    sink.list = list;
    sink.listCount = listCount;
    sink.listCap = listCap;
    sink.mode = mode;
    sink.wide = wide;
    sink.g = g;
    surfaceWorkKernel<<<148 * 4, kBlock, 0, s>>>(sink, V, I, M, nT, g, splits, nSplits, codes, offsets, total);
    *launches += 1;
}

void launch_surface_rank(const uint32_t* bits, uint64_t words, uint32_t* ranks, uint32_t* tileSums, uint32_t* total,
                         cudaStream_t s, uint32_t* launches) {
    const uint32_t tiles = (uint32_t)((words + kRankTile - 1) / kRankTile);
    rankTileKernel<<<tiles ? tiles : 1, kBlock, 0, s>>>(bits, words, ranks, tileSums);
    rankSumsKernel<<<1, 1024, 0, s>>>(tileSums, tiles, total);
    rankAddKernel<<<gridFor(words, 256, 148u * 32u), 256, 0, s>>>(ranks, words, tileSums);
    *launches += 3;
}

void launch_surface_keys_zero(void* keys, const uint32_t* count, int wide, cudaStream_t s, uint32_t* launches) {
    zeroKeysKernel<<<148 * 8, 256, 0, s>>>(keys, count, wide);
    *launches += 1;
}

void launch_surface_merge(const unsigned long long* list, const uint32_t* listCount, uint32_t listCap,
                          const uint32_t* bits, const uint32_t* ranks, uint32_t* keys, cudaStream_t s,
                          uint32_t* launches) {
    mergeKeysKernel<<<148 * 8, 256, 0, s>>>(list, listCount, listCap, bits, ranks, keys);
    *launches += 1;
}

}  // namespace vxb
