// Surface voxelization kernels (FP32): classifyTriangles / analyzeBoundingBox
// / encodeTriangleType (src/voxelizer.cu:3040-3221) and the 1D / 2D / 3D
// processing kernels (3306-3955) with processVoxel (2946-2989).
//
// Per pass: classify every triangle (class, dominant axis, voxel box clamped
// to the grid, work units), partition the triangles with work by (class,
// axis) as the reference's sort by triangle type does, write one set-up
// record per partitioned triangle (box, normal, the edge functions of the
// projections it tests), scan the unit counts and run the work list: one
// thread per column of the dominant projection (per voxel of a 1D line).
// Warps find the triangle of each of their 32 items with one coalesced load
// of 32 offsets, so the work kernel has no block-wide barrier.
//
// The reference runs the surface kernels once per material subspace on
// boxes clamped to it.  Subspaces tile the grid, so the columns of the
// grid-clamped box are the union of the subspaces' columns; along the depth
// axis a column still visits each subspace's slice separately, because the
// single-voxel shortcut (no further tests when the clamped depth range is
// one voxel) depends on the slice.
//
// Hits set the voxel's bit in the surface grid and append (bit position,
// material key) to a hit list.  Once all surface bits exist, every surface
// voxel gets a rank (prefix popcount over the surface grid), and the list is
// max-merged into a compact key array indexed by rank; the emit kernels read
// materials from there.  The key orders triangles by class, then material
// (NodeT in vxb_device.cuh), so the merged key names the winning material.
// If the list overflows, a second traversal (mode 1) merges every hit
// directly.  The same second traversal is the whole merge where no list is
// kept (64-bit PartialNode keys, or when the launch-shape tuner measured it
// faster): the first traversal then sets surface bits only (mode 2).

#include "vxb_common.cuh"
#include "vxb_device.cuh"
#include "vxb_kernels.cuh"

#include <algorithm>

namespace vxb {

using namespace detail;

namespace {

constexpr int kBlock = 256;
constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kNone = 0xFFu;

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

// Class (bits 30-31: 0 degenerate, 1 / 2 / 3 for 1D / 2D / 3D boxes) and
// axis (bits 28-29: the line's axis for 1D, the flat axis for 2D, the
// dominant normal axis for 3D) of a triangle, from its unclamped box.
__device__ __forceinline__ uint32_t classifyTri(const F3* v, const IBox& b) {
    const F3 n = crossF<site::CRF_CLS>(subF(v[0], v[2]), subF(v[1], v[0]));
    if (!(n.x != 0.0f || n.y != 0.0f || n.z != 0.0f)) return 0u;
    const int dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    uint32_t bb, axis;
    if (dx == 0) {
        if (dy == 0) { bb = 1; axis = dz == 0 ? 0 : 2; }
        else if (dz == 0) { bb = 1; axis = 1; }
        else { bb = 2; axis = 0; }
    } else if (dy == 0) {
        if (dz == 0) { bb = 1; axis = 0; }
        else { bb = 2; axis = 1; }
    } else if (dz == 0) { bb = 2; axis = 2; }
    else {
        bb = 3;
        const float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
        if (ax > ay && ax > az) axis = 0;
        else if (ay > ax && ay > az) axis = 1;
        else axis = 2;
    }
    return (axis << 28) | (bb << 30);
}

// The box clamped to the grid, i.e. to the union of the material subspaces
// (adjustVoxelRange, src/voxelizer.cu:3963-3993, over all of them).
__device__ __forceinline__ IBox gridClamp(IBox b, const PassGeom& g) {
    const int hi[3] = {(int)g.X - 1, (int)g.resY - 1, (int)g.resZ - 1};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = max(b.lo[a], 0);
        b.hi[a] = min(b.hi[a], hi[a]);
    }
    return b;
}

// Work units: voxels along the axis for 1D boxes, columns of the dominant
// projection otherwise; 0 for an empty (fully outside) box.
__device__ __forceinline__ uint32_t surfUnits(const IBox& b, uint32_t code) {
    if (b.lo[0] > b.hi[0] || b.lo[1] > b.hi[1] || b.lo[2] > b.hi[2]) return 0u;
    const uint32_t bb = code >> 30, axis = (code >> 28) & 3u;
    const uint32_t ex = (uint32_t)(b.hi[0] - b.lo[0] + 1), ey = (uint32_t)(b.hi[1] - b.lo[1] + 1),
                   ez = (uint32_t)(b.hi[2] - b.lo[2] + 1);
    if (bb == 0) return 0u;
    if (bb == 1) return axis == 0 ? ex : axis == 1 ? ey : ez;
    return axis == 0 ? ey * ez : axis == 1 ? ex * ez : ex * ey;
}

__device__ __forceinline__ uint32_t bucketOf(uint32_t code, uint32_t units) {
    return units ? ((code >> 30) - 1u) * 3u + ((code >> 28) & 3u) : kNone;
}

// The unit and mesh triangle of work triangle wt.
__device__ __forceinline__ uint32_t workUnit(const Batch& b, uint32_t wt, uint32_t* t) {
    const uint32_t u = unitOf(b.workBase, b.nUnits, wt);
    *t = wt - __ldg(b.workBase + u);
    return u;
}

// Pass 1 (work-triangle order): code and units per triangle, triangles per
// bucket.  Units without materials have no surface pass.
__global__ void surfaceClassifyKernel(Batch b, uint32_t nWork, uint32_t* __restrict__ codes,
                                      uint32_t* __restrict__ units, uint32_t* __restrict__ bucketCount) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < nWork; base += stride) {
        const uint32_t wt = base + lane;
        uint32_t code = 0, u = 0;
        if (wt < nWork) {
            uint32_t t;
            const Unit& U = b.units[workUnit(b, wt, &t)];
            if (U.materials) {
                const PassGeom g = U.g;
                F3 v[3];
                loadTriF(U.V, U.I, t, v);
                const IBox full = voxBoundsHalf(v, g);
                code = classifyTri(v, full);
                u = surfUnits(gridClamp(full, g), code);
            }
            codes[wt] = code;
            units[wt] = u;
        }
        const uint32_t bk = bucketOf(code, u);
        const uint32_t peers = __match_any_sync(kFull, bk);
        if (bk != kNone && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(bucketCount + bk, (uint32_t)__popc(peers));
    }
}

struct Overlap { float nx[3], ny[3], de[3]; };

// Set-up record of one partitioned triangle (64 bytes) and its projection
// edge functions (o[axis] for 2D boxes, all three for 3D boxes).
struct __align__(16) SurfRec {
    int lo[3], hi[3];   // voxel box clamped to the grid
    uint32_t code;      // class << 30 | axis << 28
    uint32_t key;       // class << 8 | material
    uint32_t tri;       // mesh index (PartialNode keys)
    float v0[3];        // first vertex (3D depth range)
    float n[3];         // normal (3D depth range)
    uint32_t unit;      // unit of the batch
};
struct __align__(16) SurfOvl {
    Overlap o[3];
    uint32_t pad;
};
static_assert(sizeof(SurfRec) == kSurfRecBytes, "record size");
static_assert(sizeof(SurfOvl) == kSurfOvlBytes, "record size");

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

// The set-up record of work triangle wt at partitioned position pos.
__device__ __forceinline__ void setupRecord(const Batch& b, uint32_t wt, uint32_t code, uint32_t pos,
                                            SurfRec* __restrict__ recs, SurfOvl* __restrict__ ovl) {
    uint32_t t;
    const uint32_t unit = workUnit(b, wt, &t);
    const Unit& U = b.units[unit];
    const PassGeom g = U.g;
    F3 v[3];
    loadTriF(U.V, U.I, t, v);
    const uint32_t bb = code >> 30, axis = (code >> 28) & 3u;
    const IBox box = gridClamp(voxBoundsHalf(v, g), g);
    SurfRec r;
#pragma unroll
    for (int a = 0; a < 3; ++a) { r.lo[a] = box.lo[a]; r.hi[a] = box.hi[a]; }
    r.code = code;
    r.key = (bb << 8) | (U.M ? __ldg(U.M + t) : 0u);
    r.tri = t;
    r.v0[0] = v[0].x; r.v0[1] = v[0].y; r.v0[2] = v[0].z;
    r.n[0] = r.n[1] = r.n[2] = 0.0f;
    r.unit = unit;
    const float d = g.df;
    if (bb == 2) {
        const F3 n = crossF<site::CRF_2D>(subF(v[0], v[2]), subF(v[1], v[0]));
        r.n[0] = n.x; r.n[1] = n.y; r.n[2] = n.z;
        if (axis == 0) ovl[pos].o[0] = setupOverlap<0, site::DE_2D_YZ>(v, n, d);
        else if (axis == 1) ovl[pos].o[1] = setupOverlap<1, site::DE_2D_ZX>(v, n, d);
        else ovl[pos].o[2] = setupOverlap<2, site::DE_2D_XY>(v, n, d);
    } else if (bb == 3) {
        const F3 n = crossF<site::CRF_3D>(subF(v[0], v[2]), subF(v[1], v[0]));
        r.n[0] = n.x; r.n[1] = n.y; r.n[2] = n.z;
        SurfOvl o;
        o.o[0] = setupOverlap<0, site::DE_3D_YZ>(v, n, d);
        o.o[1] = setupOverlap<1, site::DE_3D_ZX>(v, n, d);
        o.o[2] = setupOverlap<2, site::DE_3D_XY>(v, n, d);
        o.pad = 0;
        ovl[pos] = o;
    }
    recs[pos] = r;
}

// Pass 2 (work-triangle order): the position of every triangle with work in
// the partitioned order, its units there (unitsP, zero past the end) and its
// set-up record.
__global__ void surfacePartitionKernel(Batch bt, const uint32_t* __restrict__ codes,
                                       const uint32_t* __restrict__ units, uint32_t nT,
                                       const uint32_t* __restrict__ bucketCount, uint32_t* __restrict__ bucketCursor,
                                       uint32_t* __restrict__ unitsP, SurfRec* __restrict__ recs,
                                       SurfOvl* __restrict__ ovl) {
    __shared__ uint32_t bucketBase[kSurfaceBuckets];
    if (threadIdx.x < kSurfaceBuckets) {
        uint32_t s = 0;
        for (uint32_t k = 0; k < threadIdx.x; ++k) s += bucketCount[k];
        bucketBase[threadIdx.x] = s;
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < nT; base += stride) {
        const uint32_t t = base + lane;
        const uint32_t u = t < nT ? __ldg(units + t) : 0u;
        const uint32_t code = t < nT ? __ldg(codes + t) : 0u;
        const uint32_t b = t < nT ? bucketOf(code, u) : kNone;
        const uint32_t peers = __match_any_sync(kFull, b);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t start = 0;
        if (b != kNone && lane == leader) start = atomicAdd(bucketCursor + b, (uint32_t)__popc(peers));
        start = __shfl_sync(kFull, start, leader);
        if (b != kNone) {
            const uint32_t pos = bucketBase[b] + start + __popc(peers & laneMaskLt());
            unitsP[pos] = u;
            setupRecord(bt, t, code, pos, recs, ovl);
        }
    }
}

// getSingleVoxelBoundsComponent, src/voxelizer.cu:2575-2586.
template <int M> __device__ __forceinline__ float vbComp(int c, float m, float d) {
    return linf<M>(__fsub_rn((float)c, 0.5f), d, m);
}

// determineDepthRange{X,Y,Z} (src/voxelizer.cu:3994-4119) with
// intersectWithPlane* and boundsCheck; t0 is the triangle's first vertex.
template <int A, int DT> __device__ __forceinline__ void depthRange(F3 t0, F3 p, F3 n, const PassGeom& g, int& lo,
                                                                    int& hi) {
    const float d = g.df;
    F3 pmin, pmax;
    float a, b;
    if (A == 0) {
        const float sy = n.y > 0.0f ? 1.0f : 0.0f, sz = n.z > 0.0f ? 1.0f : 0.0f;
        pmin = F3{0.0f, __fadd_rn(p.y, __fmul_rn(sy, d)), __fadd_rn(p.z, __fmul_rn(sz, d))};
        pmax = F3{0.0f, __fadd_rn(p.y, __fmul_rn(1.0f - sy, d)), __fadd_rn(p.z, __fmul_rn(1.0f - sz, d))};
        const F3 u = subF(t0, pmin), w = subF(t0, pmax);
        a = __fdiv_rn(sum3f<DT>(u.x, n.x, u.y, n.y, u.z, n.z), n.x);
        b = __fdiv_rn(sum3f<DT>(w.x, n.x, w.y, n.y, w.z, n.z), n.x);
    } else if (A == 1) {
        const float sx = n.x > 0.0f ? 1.0f : 0.0f, sz = n.z > 0.0f ? 1.0f : 0.0f;
        pmin = F3{__fadd_rn(p.x, __fmul_rn(sx, d)), 0.0f, __fadd_rn(p.z, __fmul_rn(sz, d))};
        pmax = F3{__fadd_rn(p.x, __fmul_rn(1.0f - sx, d)), 0.0f, __fadd_rn(p.z, __fmul_rn(1.0f - sz, d))};
        const F3 u = subF(t0, pmin), w = subF(t0, pmax);
        a = __fdiv_rn(sum3f<DT>(u.x, n.x, u.y, n.y, u.z, n.z), n.y);
        b = __fdiv_rn(sum3f<DT>(w.x, n.x, w.y, n.y, w.z, n.z), n.y);
    } else {
        const float sx = n.x > 0.0f ? 1.0f : 0.0f, sy = n.y > 0.0f ? 1.0f : 0.0f;
        pmin = F3{__fadd_rn(p.x, __fmul_rn(sx, d)), __fadd_rn(p.y, __fmul_rn(sy, d)), 0.0f};
        pmax = F3{__fadd_rn(p.x, __fmul_rn(1.0f - sx, d)), __fadd_rn(p.y, __fmul_rn(1.0f - sy, d)), 0.0f};
        const F3 u = subF(t0, pmin), w = subF(t0, pmax);
        a = __fdiv_rn(sum3f<DT>(u.x, n.x, u.y, n.y, u.z, n.z), n.z);
        b = __fdiv_rn(sum3f<DT>(w.x, n.x, w.y, n.y, w.z, n.z), n.z);
    }
    if (a > b) { float tmp = a; a = b; b = tmp; }
    const float m = A == 0 ? g.mnf[0] : A == 1 ? g.mnf[1] : g.mnf[2];
    lo = __float2int_rz(ceilf(__fsub_rn(__fdiv_rn(__fsub_rn(a, m), d), 0.5f)));
    hi = __float2int_rz(floorf(__fadd_rn(__fdiv_rn(__fsub_rn(b, m), d), 0.5f)));
}

// Hits of one warp staged in shared memory before they go to the global
// hit list, so that the list takes one atomic per flush instead of one per
// hit.
constexpr uint32_t kStageHits = 256;
constexpr uint32_t kFlushAt = kStageHits - 96;
struct WarpStage {
    unsigned long long* buf;
    uint32_t* count;
};

// Where a unit's surface bits live.
struct UnitGrid {
    uint64_t wordBase;   // first word of the unit in the surface arena
    uint32_t AY, ipx, padY, padZ;
};

// processVoxel of the surface pass.
// mode 0: set the bit and append (bit position << 24 | key) to the hit list;
// mode 1: merge the key at the voxel's rank (surface bits are complete);
// mode 2: set the bit only (a mode-1 traversal merges the keys).
struct Sink {
    uint32_t* bits;            // surface arena
    const WordRank* wordRank;  // complete surface words with their ranks (mode 1)
    void* keys;                // compact key array (mode 1)
    uint32_t keysCap;          // keys at ranks past it are dropped
    unsigned long long* list;
    uint32_t* listCount;
    uint32_t listCap;
    int mode;
    int wide;                  // 64-bit keys (PartialNode)
    // (xi, yi, zi): voxel of the unit's voxelized box; the allocation holds
    // it one column further along x and padY / padZ rows further along y / z.
    __device__ __forceinline__ void operator()(int xi, int yi, int zi, uint64_t key, const UnitGrid& ug,
                                               const WarpStage& ws) const {
        const uint32_t x = (uint32_t)xi + 1u, y = (uint32_t)yi + ug.padY, z = (uint32_t)zi + ug.padZ;
        const uint64_t w = ug.wordBase + ((uint64_t)z * ug.AY + y) * ug.ipx + (x >> 5);
        const uint32_t b = x & 31u;
        const uint32_t bit = 0x80000000u >> b;
        if (mode == 2) {
            atomicOr(bits + w, bit);
        } else if (mode == 0) {
            atomicOr(bits + w, bit);
            const unsigned long long e = ((unsigned long long)(w * 32 + b) << 24) | (key & 0xFFFFFFull);
            const uint32_t at = atomicAdd(ws.count, 1u);
            if (at < kStageHits) {
                ws.buf[at] = e;
            } else {
                const uint32_t gat = atomicAdd(listCount, 1u);
                if (gat < listCap) list[gat] = e;
            }
        } else {
            const WordRank wr = wordRank[w];
            const uint32_t r = wr.rank + (b ? __popc(wr.bits >> (32 - b)) : 0u);
            if (r >= keysCap) return;
            if (wide) atomicMax(reinterpret_cast<unsigned long long*>(keys) + r, (unsigned long long)key);
            else atomicMax(reinterpret_cast<uint32_t*>(keys) + r, (uint32_t)key);
        }
    }
    // Moves the warp's staged hits to the global list (whole warp, converged).
    __device__ __forceinline__ void flush(const WarpStage& ws, uint32_t lane) const {
        __syncwarp();
        const uint32_t n = min(*ws.count, kStageHits);
        uint32_t base = 0;
        if (lane == 0 && n) base = atomicAdd(listCount, n);
        base = __shfl_sync(kFull, base, 0);
        for (uint32_t i = lane; i < n; i += 32u)
            if (base + i < listCap) list[base + i] = ws.buf[i];
        __syncwarp();
        if (lane == 0) *ws.count = 0;
        __syncwarp();
    }
};

// The loop of the reference over [lo, hi] along one axis runs inside one
// material subspace (adjustVoxelRange, src/voxelizer.cu:3963-3993): clamps
// [lo, hi] to the subspace slice (sl: nSl (lo, hi) pairs) that holds c.
__device__ __forceinline__ void subspaceRange(const uint32_t* sl, uint32_t nSl, int c, int& lo, int& hi) {
    for (uint32_t s = 0; s < nSl; ++s) {
        const int a = (int)__ldg(sl + 2 * s), b = (int)__ldg(sl + 2 * s + 1) - 1;
        if (c >= a && c <= b) {
            lo = max(lo, a);
            hi = min(hi, b);
            return;
        }
    }
}

// Whether iteration `pos` of a loop of n iterations falls in the prolog of a
// loop the reference build unrolled U times (the prolog runs the first
// n mod U iterations; vxb_sites.inc).
template <int U> __device__ __forceinline__ bool inProlog(int pos, int n) { return U > 1 && pos < n % U; }

template <int M, int P> __device__ __forceinline__ bool overlapAt(bool prolog, const Overlap& o, float a, float b) {
    return prolog ? overlapTest<P>(o, a, b) : overlapTest<M>(o, a, b);
}

// One column (one voxel for 1D boxes) of a partitioned triangle
// (process1D/2D/3DTriangles, instantiated per node type K as the reference
// instantiates them).  xr / yr / zr: the material subspace slices along each
// axis ((lo, hi) pairs).
template <int K>
__device__ __forceinline__ void surfaceItem(uint32_t bb, uint32_t axis, const SurfRec& r, const Overlap& od,
                                            const SurfOvl* __restrict__ ov, uint32_t u, const PassGeom& g,
                                            const uint32_t* __restrict__ slices, const uint32_t* sliceOff,
                                            const uint32_t* sliceN, uint64_t key, const Sink& sink,
                                            const UnitGrid& ug, const WarpStage& ws) {
    const float d = g.df;
    const uint32_t ex = (uint32_t)(r.hi[0] - r.lo[0] + 1), ey = (uint32_t)(r.hi[1] - r.lo[1] + 1);
    if (bb == 1) {
        // process1DTriangles (3306-3411): every voxel of the line, no test.
        if (axis == 0) sink(r.lo[0] + (int)u, r.lo[1], r.lo[2], key, ug, ws);
        else if (axis == 1) sink(r.lo[0], r.lo[1] + (int)u, r.lo[2], key, ug, ws);
        else sink(r.lo[0], r.lo[1], r.lo[2] + (int)u, key, ug, ws);
        return;
    }
    if (bb == 2) {
        // process2DTriangles (3418-3596): the dominant projection only; the
        // inner loop (z for the x and y axes, y for the z axis) evaluates its
        // prolog iterations in their own forms.
        constexpr int U = site::UNR_2D[K];
        if (axis == 0) {
            const int j = r.lo[1] + (int)(u % ey), k = r.lo[2] + (int)(u / ey);
            int lo = r.lo[2], hi = r.hi[2];
            if (U > 1) subspaceRange(slices + 2 * sliceOff[2], sliceN[2], k, lo, hi);
            if (overlapAt<site::OT_2D_YZ, site::OT_2DP_YZ>(inProlog<U>(k - lo, hi - lo + 1), od,
                                                           vbComp<site::PC_2D>(j, g.mnf[1], d),
                                                           vbComp<site::PC_2D>(k, g.mnf[2], d)))
                sink(r.lo[0], j, k, key, ug, ws);
        } else if (axis == 1) {
            const int i = r.lo[0] + (int)(u % ex), k = r.lo[2] + (int)(u / ex);
            int lo = r.lo[2], hi = r.hi[2];
            if (U > 1) subspaceRange(slices + 2 * sliceOff[2], sliceN[2], k, lo, hi);
            if (overlapAt<site::OT_2D_ZX, site::OT_2DP_ZX>(inProlog<U>(k - lo, hi - lo + 1), od,
                                                           vbComp<site::PC_2D>(k, g.mnf[2], d),
                                                           vbComp<site::PC_2D>(i, g.mnf[0], d)))
                sink(i, r.lo[1], k, key, ug, ws);
        } else {
            const int i = r.lo[0] + (int)(u % ex), j = r.lo[1] + (int)(u / ex);
            int lo = r.lo[1], hi = r.hi[1];
            if (U > 1) subspaceRange(slices + 2 * sliceOff[1], sliceN[1], j, lo, hi);
            if (overlapAt<site::OT_2D_XY, site::OT_2DP_XY>(inProlog<U>(j - lo, hi - lo + 1), od,
                                                           vbComp<site::PC_2D>(i, g.mnf[0], d),
                                                           vbComp<site::PC_2D>(j, g.mnf[1], d)))
                sink(i, j, r.lo[2], key, ug, ws);
        }
        return;
    }
    // process3DTriangles (3603-3955): dominant projection, depth range from
    // the plane, then per subspace slice of the depth axis either the single
    // voxel or the other two projections per voxel (the depth loop's prolog
    // iterations in their own forms).
    constexpr int UL = site::UNR_3DL[K];
    const F3 n{r.n[0], r.n[1], r.n[2]};
    const F3 t0{r.v0[0], r.v0[1], r.v0[2]};
    if (axis == 0) {
        const int j = r.lo[1] + (int)(u % ey), k = r.lo[2] + (int)(u / ey);
        F3 p{0.0f, vbComp<site::PC_3D>(j, g.mnf[1], d), vbComp<site::PC_3D>(k, g.mnf[2], d)};
        if (!overlapTest<site::OT_3D_YZ>(od, p.y, p.z)) return;
        int d0, d1;
        depthRange<0, site::DT_3DX[K]>(t0, p, n, g, d0, d1);
        const uint32_t* sl = slices + 2 * sliceOff[0];
        for (uint32_t s = 0; s < sliceN[0]; ++s) {
            const int lo = max(r.lo[0], (int)__ldg(sl + 2 * s)), hi = min(r.hi[0], (int)__ldg(sl + 2 * s + 1) - 1);
            if (lo > hi || d0 > hi || d1 < lo) continue;
            const int a = d0 < lo ? lo : d0, c = d1 > hi ? hi : d1;
            if (a == c) { sink(a, j, k, key, ug, ws); continue; }
            for (int i = a; i <= c; ++i) {
                p.x = vbComp<site::PC_3DL>(i, g.mnf[0], d);
                const bool pro = inProlog<UL>(i - a, c - a + 1);
                if (overlapAt<site::OT_3DX_ZX, site::OT_3DXP_ZX[K]>(pro, ov->o[1], p.z, p.x) &&
                    overlapAt<site::OT_3DX_XY, site::OT_3DXP_XY>(pro, ov->o[2], p.x, p.y))
                    sink(i, j, k, key, ug, ws);
            }
        }
    } else if (axis == 1) {
        const int i = r.lo[0] + (int)(u % ex), k = r.lo[2] + (int)(u / ex);
        F3 p{vbComp<site::PC_3D>(i, g.mnf[0], d), 0.0f, vbComp<site::PC_3D>(k, g.mnf[2], d)};
        if (!overlapTest<site::OT_3D_ZX>(od, p.z, p.x)) return;
        int d0, d1;
        depthRange<1, site::DT_3DY>(t0, p, n, g, d0, d1);
        const uint32_t* sl = slices + 2 * sliceOff[1];
        for (uint32_t s = 0; s < sliceN[1]; ++s) {
            const int lo = max(r.lo[1], (int)__ldg(sl + 2 * s)), hi = min(r.hi[1], (int)__ldg(sl + 2 * s + 1) - 1);
            if (lo > hi || d0 > hi || d1 < lo) continue;
            const int a = d0 < lo ? lo : d0, c = d1 > hi ? hi : d1;
            if (a == c) { sink(i, a, k, key, ug, ws); continue; }
            for (int j = a; j <= c; ++j) {
                p.y = vbComp<site::PC_3DL>(j, g.mnf[1], d);
                const bool pro = inProlog<UL>(j - a, c - a + 1);
                if (overlapAt<site::OT_3DY_XY, site::OT_3DYP_XY>(pro, ov->o[2], p.x, p.y) &&
                    overlapAt<site::OT_3DY_YZ, site::OT_3DYP_YZ>(pro, ov->o[0], p.y, p.z))
                    sink(i, j, k, key, ug, ws);
            }
        }
    } else {
        const int i = r.lo[0] + (int)(u % ex), j = r.lo[1] + (int)(u / ex);
        F3 p{vbComp<site::PC_3D>(i, g.mnf[0], d), vbComp<site::PC_3D>(j, g.mnf[1], d), 0.0f};
        if (!overlapTest<site::OT_3D_XY>(od, p.x, p.y)) return;
        int d0, d1;
        depthRange<2, site::DT_3DZ>(t0, p, n, g, d0, d1);
        const uint32_t* sl = slices + 2 * sliceOff[2];
        for (uint32_t s = 0; s < sliceN[2]; ++s) {
            const int lo = max(r.lo[2], (int)__ldg(sl + 2 * s)), hi = min(r.hi[2], (int)__ldg(sl + 2 * s + 1) - 1);
            if (lo > hi || d0 > hi || d1 < lo) continue;
            const int a = d0 < lo ? lo : d0, c = d1 > hi ? hi : d1;
            if (a == c) { sink(i, j, a, key, ug, ws); continue; }
            for (int k = a; k <= c; ++k) {
                p.z = vbComp<site::PC_3DL>(k, g.mnf[2], d);
                const bool pro = inProlog<UL>(k - a, c - a + 1);
                if (overlapAt<site::OT_3DZ_YZ, site::OT_3DZP_YZ>(pro, ov->o[0], p.y, p.z) &&
                    overlapAt<site::OT_3DZ_ZX, site::OT_3DZP_ZX>(pro, ov->o[1], p.z, p.x))
                    sink(i, j, k, key, ug, ws);
            }
        }
    }
}

// Pass 4: the work list.  Warps take batches of kBatch (8, 16 or 32, the
// launch shape) consecutive 32-item
// chunks; within a batch the owner of each chunk's first item follows from
// the previous chunk.  Every partitioned triangle has at least one unit, so
// a chunk's 32 items belong to at most 32 consecutive triangles: lane l
// loads off[t0 + l] and a bit mask of the triangle starts inside the chunk
// gives every lane its owner.  The class and axis of a position follow from
// the bucket bounds, so the projection edge functions load together with
// the record.
template <uint32_t kBatch, int K>
__global__ void __launch_bounds__(kBlock) surfaceWorkKernel(Sink sink, Batch b, const SurfRec* __restrict__ recs,
                                                            const SurfOvl* __restrict__ ovl,
                                                            const uint32_t* __restrict__ off, uint32_t n,
                                                            const uint32_t* __restrict__ totalPtr,
                                                            const uint32_t* __restrict__ bucketCount,
                                                            uint32_t* queue) {
    __shared__ unsigned long long stageBuf[kBlock / 32][kStageHits];
    __shared__ uint32_t stageCount[kBlock / 32];
    __shared__ uint32_t bucketEnd[kSurfaceBuckets];
    const uint32_t total = *totalPtr;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t wib = threadIdx.x >> 5;
    const WarpStage ws{stageBuf[wib], stageCount + wib};
    if (lane == 0) stageCount[wib] = 0;
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (uint32_t k = 0; k < kSurfaceBuckets; ++k) {
            acc += __ldg(bucketCount + k);
            bucketEnd[k] = acc;
        }
    }
    __syncthreads();
    const uint32_t chunks = (total + 31u) / 32u;
    const uint32_t batches = (chunks + kBatch - 1) / kBatch;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nWarps = (gridDim.x * blockDim.x) >> 5;
    // Batches in a fixed grid-stride order, or (queue != NULL) taken from a
    // device work queue, one atomic per batch, so that warps that drew cheap
    // batches keep working while others finish expensive ones.
    auto nextBatch = [&](uint32_t cur) {
        if (!queue) return cur + nWarps;
        uint32_t v = 0;
        if (lane == 0) v = atomicAdd(queue, 1u);
        return __shfl_sync(kFull, v, 0);
    };
    for (uint32_t bt = queue ? nextBatch(0) : warp; bt < batches; bt = nextBatch(bt)) {
        const uint32_t c1 = min((bt + 1) * kBatch, chunks);
        uint32_t t0 = warpFindOwner(off, n, bt * kBatch * 32u, lane);
        for (uint32_t c = bt * kBatch; c < c1; ++c) {
            const uint32_t base = c * 32u;
            const uint32_t ol = t0 + lane <= n ? __ldg(off + t0 + lane) : 0xFFFFFFFFu;
            const uint32_t o32 = t0 + 32u <= n ? __ldg(off + t0 + 32u) : 0xFFFFFFFFu;
            const uint32_t starts = __reduce_or_sync(kFull, (lane >= 1u && ol < base + 32u) ? 1u << (ol - base) : 0u);
            const uint32_t k = __popc(starts & ((2u << lane) - 1u));
            const uint32_t ok = __shfl_sync(kFull, ol, k);
            const uint32_t k31 = __popc(starts);
            const uint32_t next = __shfl_sync(kFull, ol, (k31 + 1u) & 31u);
            const uint32_t nextOff = k31 < 31u ? next : o32;
            const uint32_t item = base + lane;
            if (item < total) {
                const uint32_t pos = t0 + k;
                uint32_t bucket = 0;
#pragma unroll
                for (uint32_t q = 0; q + 1 < kSurfaceBuckets; ++q) bucket += pos >= bucketEnd[q] ? 1u : 0u;
                const uint32_t bb = bucket / 3u + 1u, axis = bucket % 3u;
                Overlap od;
                if (bb >= 2) od = ovl[pos].o[axis];
                const SurfRec r = recs[pos];
                const uint64_t key = sink.wide ? (((uint64_t)bb << 40) | ((uint64_t)(r.key & 255u) << 32) | r.tri)
                                               : (uint64_t)r.key;
                const Unit& U = b.units[r.unit];
                const PassGeom g = U.g;
                const UnitGrid ug{U.wordBase, g.AY, g.ipx, g.padY, g.padZ};
                const uint32_t sliceOff[3] = {U.sliceBase, U.sliceBase + U.sliceN[0],
                                              U.sliceBase + U.sliceN[0] + U.sliceN[1]};
                const uint32_t sliceN[3] = {U.sliceN[0], U.sliceN[1], U.sliceN[2]};
                surfaceItem<K>(bb, axis, r, od, ovl + pos, item - ok, g, b.slices, sliceOff, sliceN, key, sink,
                               ug, ws);
            }
            __syncwarp();
            if (sink.mode == 0 && *ws.count >= kFlushAt) sink.flush(ws, lane);
            t0 += k31 + (nextOff == base + 32u ? 1u : 0u);
        }
    }
    if (sink.mode == 0) sink.flush(ws, lane);
}

// Exclusive popcount prefix over the surface words (ranks of surface voxels).
constexpr int kRankItems = 8;
constexpr uint32_t kRankTile = kBlock * kRankItems;

// Two passes over the surface words, the second after the tile sums are
// scanned: kApply false writes each tile's popcount sum, kApply true writes
// the ranks (tile offset plus the block's exclusive scan).  The words were
// just written by the surface pass and are read from L2 where they stay.
template <bool kApply>
__global__ void rankTileKernel(const uint32_t* __restrict__ words, uint64_t n, WordRank* __restrict__ ranks,
                               uint32_t* __restrict__ tileSums) {
    __shared__ uint32_t warpSums[33];
    const uint64_t base = (uint64_t)blockIdx.x * kRankTile + (uint64_t)threadIdx.x * kRankItems;
    const bool whole = base + kRankItems <= n;   // 32-byte aligned: kRankItems words per thread
    uint32_t x[kRankItems], c[kRankItems];
    if (whole) {
        const uint4 a = __ldg(reinterpret_cast<const uint4*>(words + base));
        const uint4 b = __ldg(reinterpret_cast<const uint4*>(words + base) + 1);
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
        x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
    } else {
#pragma unroll
        for (int i = 0; i < kRankItems; ++i) x[i] = base + i < n ? __ldg(words + base + i) : 0u;
    }
#pragma unroll
    for (int i = 0; i < kRankItems; ++i) c[i] = (uint32_t)__popc(x[i]);
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kRankItems; ++i) sum += c[i];
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
    if (!kApply) {
        if (threadIdx.x == 0) tileSums[blockIdx.x] = warpSums[32];
        return;
    }
    uint32_t r[kRankItems];
    uint32_t ex = __ldg(tileSums + blockIdx.x) + warpSums[warp] + incl - sum;
#pragma unroll
    for (int i = 0; i < kRankItems; ++i) {
        r[i] = ex;
        ex += c[i];
    }
    if (whole) {
        uint4* out = reinterpret_cast<uint4*>(ranks + base);
#pragma unroll
        for (int i = 0; i < kRankItems; i += 2) out[i / 2] = make_uint4(x[i], r[i], x[i + 1], r[i + 1]);
    } else {
#pragma unroll
        for (int i = 0; i < kRankItems; ++i)
            if (base + i < n) ranks[base + i] = WordRank{x[i], r[i]};
    }
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

__global__ void zeroKeysKernel(void* keys, const uint32_t* __restrict__ countPtr, uint32_t cap, int wide) {
    const uint32_t n = min(*countPtr, cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (wide) reinterpret_cast<unsigned long long*>(keys)[i] = 0ull;
        else reinterpret_cast<uint32_t*>(keys)[i] = 0u;
    }
}

// Max-merges the hit list into the rank-indexed key array.  Each thread
// takes two pairs of consecutive entries (16-byte loads) per iteration, so
// the scattered word / rank loads of four entries overlap; one 8-byte load
// gives an entry's surface word and rank.
__global__ void mergeKeysKernel(const unsigned long long* __restrict__ list, const uint32_t* __restrict__ countPtr,
                                uint32_t cap, const WordRank* __restrict__ ranks, uint32_t* keys, uint32_t keysCap) {
    constexpr int U = 2;   // entry pairs per thread and iteration
    const uint32_t n = min(*countPtr, cap);
    const uint32_t pairs = (n + 1) / 2;
    const uint32_t stride = gridDim.x * blockDim.x;
    const ulonglong2* list2 = reinterpret_cast<const ulonglong2*>(list);
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < pairs; i0 += U * stride) {
        unsigned long long e[2 * U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t i = i0 + u * stride;
            ulonglong2 q = make_ulonglong2(~0ull, ~0ull);
            if (i < pairs) q = list2[i];
            e[2 * u] = q.x;
            e[2 * u + 1] = 2 * i + 1 < n ? q.y : ~0ull;
        }
        WordRank wr[2 * U];
#pragma unroll
        for (int u = 0; u < 2 * U; ++u)
            if (e[u] != ~0ull) wr[u] = ranks[(e[u] >> 24) >> 5];
#pragma unroll
        for (int u = 0; u < 2 * U; ++u) {
            if (e[u] == ~0ull) continue;
            const uint32_t b = (uint32_t)((e[u] >> 24) & 31u);
            const uint32_t r = wr[u].rank + (b ? __popc(wr[u].bits >> (32 - b)) : 0u);
            if (r < keysCap) atomicMax(keys + r, (uint32_t)(e[u] & 0xFFFFFFull));
        }
    }
}

}  // namespace

void launch_surface_prepare(const Batch& b, uint32_t nWork, uint32_t* codes, uint32_t* units, uint32_t* buckets,
                            uint32_t* unitsP, void* recs, void* ovl, cudaStream_t s,
                            uint32_t* launches) {
    const uint32_t grid = gridFor(nWork, 256);
    surfaceClassifyKernel<<<grid, 256, 0, s>>>(b, nWork, codes, units, buckets);
    surfacePartitionKernel<<<grid, 256, 0, s>>>(b, codes, units, nWork, buckets, buckets + kSurfaceBuckets, unitsP,
                                                static_cast<SurfRec*>(recs), static_cast<SurfOvl*>(ovl));
    *launches += 2;
}

template <int K>
static void launchSurfaceWorkKind(uint32_t batch, uint32_t grid, const Sink& sink, const Batch& b, const SurfRec* R,
                                  const SurfOvl* O, const uint32_t* offsets, uint32_t nWork, const uint32_t* total,
                                  const uint32_t* buckets, uint32_t* queue, cudaStream_t s) {
    if (batch == 8)
        surfaceWorkKernel<8, K><<<grid, kBlock, 0, s>>>(sink, b, R, O, offsets, nWork, total, buckets, queue);
    else if (batch == 32)
        surfaceWorkKernel<32, K><<<grid, kBlock, 0, s>>>(sink, b, R, O, offsets, nWork, total, buckets, queue);
    else surfaceWorkKernel<16, K><<<grid, kBlock, 0, s>>>(sink, b, R, O, offsets, nWork, total, buckets, queue);
}

void launch_surface_work(int kind, int mode, int wide, const Batch& b, const void* recs, const void* ovl,
                         const uint32_t* offsets, uint32_t nWork, const uint32_t* total, const uint32_t* buckets,
                         uint32_t* surf, const WordRank* ranks, void* keys, uint32_t keysCap,
                         unsigned long long* list, uint32_t* listCount, uint32_t listCap, uint32_t blocksPerSm,
                         uint32_t batch, uint32_t* queue, cudaStream_t s, uint32_t* launches) {
    if (queue) cudaMemsetAsync(queue, 0, sizeof(uint32_t), s);
    Sink sink;
    sink.bits = surf;
    sink.wordRank = ranks;
    sink.keys = keys;
    sink.keysCap = keysCap;
    sink.list = list;
    sink.listCount = listCount;
    sink.listCap = listCap;
    sink.mode = mode;
    sink.wide = wide;
    const uint32_t grid = 148u * blocksPerSm;
    const SurfRec* R = static_cast<const SurfRec*>(recs);
    const SurfOvl* O = static_cast<const SurfOvl*>(ovl);
    switch (kind) {
    case kShort: launchSurfaceWorkKind<kShort>(batch, grid, sink, b, R, O, offsets, nWork, total, buckets, queue, s); break;
    case kLong: launchSurfaceWorkKind<kLong>(batch, grid, sink, b, R, O, offsets, nWork, total, buckets, queue, s); break;
    case kPartial:
        launchSurfaceWorkKind<kPartial>(batch, grid, sink, b, R, O, offsets, nWork, total, buckets, queue, s);
        break;
    case kShortFcc:
        launchSurfaceWorkKind<kShortFcc>(batch, grid, sink, b, R, O, offsets, nWork, total, buckets, queue, s);
        break;
    default:
        launchSurfaceWorkKind<kLongFcc>(batch, grid, sink, b, R, O, offsets, nWork, total, buckets, queue, s);
        break;
    }
    *launches += 1;
}

void launch_surface_rank(const uint32_t* bits, uint64_t words, WordRank* ranks, uint32_t* tileSums, uint32_t* total,
                         cudaStream_t s, uint32_t* launches) {
    const uint32_t tiles = (uint32_t)((words + kRankTile - 1) / kRankTile);
    rankTileKernel<false><<<tiles ? tiles : 1, kBlock, 0, s>>>(bits, words, ranks, tileSums);
    rankSumsKernel<<<1, 1024, 0, s>>>(tileSums, tiles, total);
    rankTileKernel<true><<<tiles ? tiles : 1, kBlock, 0, s>>>(bits, words, ranks, tileSums);
    *launches += 3;
}

void launch_surface_keys_zero(void* keys, const uint32_t* count, uint32_t cap, int wide, cudaStream_t s,
                              uint32_t* launches) {
    zeroKeysKernel<<<148 * 8, 256, 0, s>>>(keys, count, cap, wide);
    *launches += 1;
}

void launch_surface_merge(const unsigned long long* list, const uint32_t* listCount, uint32_t listCap,
                          const WordRank* ranks, uint32_t* keys, uint32_t keysCap,
                          uint32_t blocksPerSm, uint32_t entries, cudaStream_t s, uint32_t* launches) {
    // blocksPerSm 0: a block per 1,024 of the expected entries, so that blocks
    // retire as they finish and other streams' blocks get room (blocks past
    // the count exit at once; entries past the grid are taken by its
    // grid-stride loop).
    const uint32_t grid = blocksPerSm ? 148u * blocksPerSm : std::max(1u, (entries / 2 + 511) / 512);
    mergeKeysKernel<<<grid, 256, 0, s>>>(list, listCount, listCap, ranks, keys, keysCap);
    *launches += 1;
}

}  // namespace vxb
