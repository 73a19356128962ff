// CUDA kernels of the B200 voxelizer (sm_100a).
//
// The reference (hakarlss/Voxelizer, src/voxelizer.cu) bins triangles into a
// sorted (tile, triangle) work queue, voxelizes one tile per block with
// global atomicXor flushes, voxelizes surfaces with one thread per triangle
// and classifies nodes with repeated full passes over a node array.  This
// design keeps the reference's arithmetic bit for bit but restructures the
// work for the B200:
//
//  * work lists are flat (triangle, candidate) expansions over an exclusive
//    scan of per-triangle counts, so a 1M-voxel wall triangle and a 2-voxel
//    sliver cost one thread per candidate tile/column each; no sort is
//    needed because parity toggles commute (XOR) and surface keys merge by
//    max;
//  * solid voxels are produced as a toggle grid (one bit per voxel, L2
//    resident: 54 MB at 1088x771x515) and turned into solid runs by a
//    warp-per-row prefix XOR (in-word log-step XOR + ballot carry);
//  * pruning works on packed bits (32 nodes per word per thread);
//  * the node grid, the only large output, is written once by an emit
//    kernel with 16-byte vector stores.

#include "vxb_device.cuh"
#include "vxb_kernels.cuh"

#include <cfloat>

namespace vxb {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;
constexpr double kDblMin = 2.2250738585072014e-308;  // DBL_MIN, src/voxelizer.cu:1443

struct D3 { double x, y, z; };
struct F3 { float x, y, z; };

__device__ __forceinline__ uint32_t laneMaskLt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---------------------------------------------------------------------------
// Exclusive scan of per-triangle counts (three kernels: tile scan, scan of
// tile sums, tile offsets).  Totals above 2^32 set *overflow.

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
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = (base + i < n) ? in[base + i] : 0u;
        sum += v[i];
    }
    uint32_t total;
    uint32_t ex = blockExclusiveScan(sum, warpSums, total);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = ex;
        ex += v[i];
    }
    if (threadIdx.x == 0) tileSums[blockIdx.x] = total;
}

__global__ void scanSumsKernel(uint32_t* tileSums, uint32_t nTiles, uint32_t* total, uint32_t* overflow) {
    __shared__ uint32_t warpSums[33];
    unsigned long long carry = 0;
    for (uint32_t start = 0; start < nTiles; start += blockDim.x) {
        uint32_t i = start + threadIdx.x;
        uint32_t v = i < nTiles ? tileSums[i] : 0u;
        uint32_t chunk;
        uint32_t ex = blockExclusiveScan(v, warpSums, chunk);
        if (i < nTiles) tileSums[i] = (uint32_t)(carry + ex);
        carry += chunk;
    }
    if (threadIdx.x == 0) {
        *total = (uint32_t)carry;
        *overflow = carry > 0xFFFFFFFFull ? 1u : 0u;
    }
}

__global__ void scanAddKernel(uint32_t* out, uint32_t n, const uint32_t* tileSums, const uint32_t* total) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tileSums[i / kScanTile];
    if (i == 0) out[n] = *total;
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

// ---------------------------------------------------------------------------
// Solid voxelization.

__device__ __forceinline__ void loadTriD(const float* __restrict__ V, const uint32_t* __restrict__ I, uint32_t t,
                                         D3* v) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        uint32_t a = __ldg(I + 3 * t + k);
        v[k] = D3{(double)__ldg(V + 3 * a), (double)__ldg(V + 3 * a + 1), (double)__ldg(V + 3 * a + 2)};
    }
}

// Per-triangle binning setup: calculateTileOverlap / constructWorkQueue,
// src/voxelizer.cu:861-945 and 1086-1144 (getTriangleBounds 2397-2418,
// getVoxelBoundsDouble 2446-2458, tN 882-884).
struct BinTri {
    D3 v[3];
    int vlo[2], vhi[2];
    double tN;
};

__device__ __forceinline__ void binSetup(const float* V, const uint32_t* I, uint32_t t, const PassGeom& g, BinTri& b) {
    loadTriD(V, I, t, b.v);
    double ymin = b.v[0].y, zmin = b.v[0].z, ymax = ymin, zmax = zmin;
#pragma unroll
    for (int i = 1; i < 3; ++i) {
        ymin = b.v[i].y < ymin ? b.v[i].y : ymin;
        zmin = b.v[i].z < zmin ? b.v[i].z : zmin;
        ymax = b.v[i].y > ymax ? b.v[i].y : ymax;
        zmax = b.v[i].z > zmax ? b.v[i].z : zmax;
    }
    const double d = g.d;
    double a0 = __ddiv_rn(__dsub_rn(ymin, g.mn[1]), d), a1 = __ddiv_rn(__dsub_rn(zmin, g.mn[2]), d);
    double b0 = __ddiv_rn(__dsub_rn(ymax, g.mn[1]), d), b1 = __ddiv_rn(__dsub_rn(zmax, g.mn[2]), d);
    b.vlo[0] = __double2int_rz(ceil(a0));
    b.vlo[1] = __double2int_rz(ceil(a1));
    b.vhi[0] = __double2int_rz(__dadd_rn(floor(b0), 1.0));
    b.vhi[1] = __double2int_rz(__dadd_rn(floor(b1), 1.0));
    const D3* v = b.v;
    b.tN = __dsub_rn(sum3<site::TN>(v[0].y, v[1].z, v[2].y, v[0].z, v[2].z, v[1].y),
                     sum3<site::TN>(v[2].y, v[1].z, v[0].z, v[1].y, v[2].z, v[0].y));
}

__device__ __forceinline__ bool binRejected(const BinTri& b) {
    return b.tN == 0.0 || b.vlo[0] >= b.vhi[0] || b.vlo[1] >= b.vhi[1];
}

// commonSpace of a triangle and one yz subspace (src/voxelizer.cu:893-926).
__device__ __forceinline__ bool commonSpace(const BinTri& b, const SplitYZ& sp, uint32_t* csLo, uint32_t* csHi) {
    if (b.vhi[0] <= (int)sp.y0 || b.vhi[1] <= (int)sp.z0) return false;
    if (b.vlo[0] >= (int)sp.y1 || b.vlo[1] >= (int)sp.z1) return false;
    csLo[0] = (uint32_t)max((int)sp.y0, b.vlo[0]);
    csLo[1] = (uint32_t)max((int)sp.z0, b.vlo[1]);
    csHi[0] = min(sp.y1, (uint32_t)b.vhi[0]);
    csHi[1] = min(sp.z1, (uint32_t)b.vhi[1]);
    return true;
}

__global__ void solidCountKernel(const float* __restrict__ V, const uint32_t* __restrict__ I, uint32_t nT, PassGeom g,
                                 const SplitYZ* __restrict__ splits, uint32_t nSplits, uint32_t* __restrict__ counts) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nT; t += gridDim.x * blockDim.x) {
        BinTri b;
        binSetup(V, I, t, g, b);
        uint32_t c = 0;
        if (!binRejected(b)) {
            for (uint32_t s = 0; s < nSplits; ++s) {
                uint32_t lo[2], hi[2];
                if (!commonSpace(b, splits[s], lo, hi)) continue;
                c += ((hi[0] - 1) / 4 - lo[0] / 4 + 1) * ((hi[1] - 1) / 4 - lo[1] / 4 + 1);
            }
        }
        counts[t] = c;
    }
}

// One thread per (triangle, subspace, 4x4 tile) candidate.  The candidate is
// a member of the tile's work list iff one voxel centre of the tile inside
// the triangle's clipped bounding box passes the inclusive edge test with
// tN-oriented normals (traverseTilesForOverlaps, src/voxelizer.cu:980-1033).
// A member then runs generateVoxelization's per-centre work
// (src/voxelizer.cu:1344-1462) on all 16 centres of the tile inside the
// subspace and toggles bit voxelX of the centre's row.
__global__ void solidToggleKernel(const float* __restrict__ V, const uint32_t* __restrict__ I, uint32_t nT,
                                  PassGeom g, const SplitYZ* __restrict__ splits, uint32_t nSplits,
                                  const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ totalPtr,
                                  uint32_t* __restrict__ toggles) {
    const uint32_t total = *totalPtr;
    const double d = g.d;
    for (uint32_t item = blockIdx.x * blockDim.x + threadIdx.x; item < total; item += gridDim.x * blockDim.x) {
        const uint32_t t = findOwner(offsets, nT, item);
        uint32_t local = item - __ldg(offsets + t);
        BinTri b;
        binSetup(V, I, t, g, b);
        uint32_t lo[2] = {0, 0}, hi[2] = {0, 0};
        SplitYZ sp = splits[0];
        for (uint32_t s = 0; s < nSplits; ++s) {
            if (!commonSpace(b, splits[s], lo, hi)) continue;
            uint32_t nty = (hi[0] - 1) / 4 - lo[0] / 4 + 1, ntz = (hi[1] - 1) / 4 - lo[1] / 4 + 1;
            if (local < nty * ntz) { sp = splits[s]; break; }
            local -= nty * ntz;
        }
        const uint32_t nty = (hi[0] - 1) / 4 - lo[0] / 4 + 1;
        const uint32_t tileY = lo[0] / 4 + local % nty, tileZ = lo[1] / 4 + local / nty;
        const D3* v = b.v;
        // Binning edge functions (orientation by the sign of tN).
        double bnx[3], bny[3], bd[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const D3& p = v[i];
            const D3& q = v[(i + 1) % 3];
            if (b.tN > 0.0) { bnx[i] = __dsub_rn(p.z, q.z); bny[i] = __dsub_rn(q.y, p.y); }
            else { bnx[i] = __dsub_rn(q.z, p.z); bny[i] = __dsub_rn(p.y, q.y); }
            bd[i] = -sum2<site::D_BIN>(bnx[i], p.y, bny[i], p.z);
        }
        bool member = false;
        for (uint32_t iy = tileY * 4; iy < tileY * 4 + 4 && iy < hi[0] && !member; ++iy) {
            if (iy < lo[0]) continue;
            const double py = lin<site::P_BIN>((double)iy, d, g.mn[1]);
            for (uint32_t iz = tileZ * 4; iz < tileZ * 4 + 4 && iz < hi[1]; ++iz) {
                if (iz < lo[1]) continue;
                const double pz = lin<site::P_BIN>((double)iz, d, g.mn[2]);
                bool ok = true;
#pragma unroll
                for (int k = 0; k < 3; ++k) ok &= sum2p1<site::E_BIN>(bnx[k], py, bny[k], pz, bd[k]) >= 0.0;
                if (ok) { member = true; break; }
            }
        }
        if (!member) continue;
        // Generation: normal cross(v0 - v2, v1 - v0), edges oriented by n.x.
        const D3 U{__dsub_rn(v[0].x, v[2].x), __dsub_rn(v[0].y, v[2].y), __dsub_rn(v[0].z, v[2].z)};
        const D3 W{__dsub_rn(v[1].x, v[0].x), __dsub_rn(v[1].y, v[0].y), __dsub_rn(v[1].z, v[0].z)};
        const D3 n{diff2<site::CR_GEN>(U.y, W.z, U.z, W.y), diff2<site::CR_GEN>(U.z, W.x, U.x, W.z),
                   diff2<site::CR_GEN>(U.x, W.y, U.y, W.x)};
        double ex[3], ey[3], ed[3];
        bool tl[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const D3& p = v[i];
            const D3& q = v[(i + 1) % 3];
            if (n.x > 0.0) { ex[i] = __dsub_rn(p.z, q.z); ey[i] = __dsub_rn(q.y, p.y); }
            else { ex[i] = __dsub_rn(q.z, p.z); ey[i] = __dsub_rn(p.y, q.y); }
            ed[i] = -sum2<site::D_GEN>(ex[i], p.y, ey[i], p.z);
            tl[i] = ex[i] > 0.0 || (ex[i] == 0.0 && ey[i] < 0.0);
        }
        for (uint32_t c = 0; c < 16; ++c) {
            const uint32_t vz = tileZ * 4 + c / 4, vy = tileY * 4 + c % 4;
            if (vy < sp.y0 || vy >= sp.y1 || vz < sp.z0 || vz >= sp.z1) continue;
            const double py = lin<site::P_GEN>((double)vy, d, g.mn[1]);
            const double pz = lin<site::P_GEN>((double)vz, d, g.mn[2]);
            int pass = 0;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                double r = sum2p1<site::E_GEN>(ex[i], py, ey[i], pz, ed[i]);
                if (tl[i]) r = __dadd_rn(r, kDblMin);
                pass += r > 0.0;
            }
            if (pass != 3) continue;
            const double ax = __dsub_rn(v[0].x, g.mn[0]), ay = __dsub_rn(v[0].y, py), az = __dsub_rn(v[0].z, pz);
            const double B = sum3<site::B_GEN>(ax, n.x, ay, n.y, az, n.z);
            double px = __ddiv_rn(B, n.x);
            px = px < 0.0 ? 0.0 : px;
            const uint32_t vx = __double2uint_rz(ceil(__ddiv_rn(px, d))) + 1u;
            if (vx >= g.X) continue;
            const uint32_t row = (vz + 1) * g.AY + (vy + 1);
            atomicXor(toggles + (size_t)row * g.ipx + (vx >> 5), 0x80000000u >> (vx & 31u));
        }
    }
}

// Toggle bits -> solid runs, one warp per row: bit x = XOR of toggles <= x.
__global__ void rowFillKernel(uint32_t* __restrict__ words, uint32_t rows, uint32_t ipx) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warpsPerBlock = blockDim.x >> 5;
    for (uint32_t row = blockIdx.x * warpsPerBlock + (threadIdx.x >> 5); row < rows;
         row += gridDim.x * warpsPerBlock) {
        uint32_t* r = words + (size_t)row * ipx;
        uint32_t carry = 0;
        for (uint32_t base = 0; base < ipx; base += 32) {
            const uint32_t k = base + lane;
            const uint32_t w = k < ipx ? r[k] : 0u;
            uint32_t p = w;
            p ^= p >> 1; p ^= p >> 2; p ^= p >> 4; p ^= p >> 8; p ^= p >> 16;
            const uint32_t bal = __ballot_sync(0xffffffffu, __popc(w) & 1u);
            const uint32_t before = (__popc(bal & laneMaskLt()) & 1u) ^ carry;
            if (k < ipx) r[k] = before ? ~p : p;
            carry ^= __popc(bal) & 1u;
        }
    }
}

// ---------------------------------------------------------------------------
// Surface voxelization (FP32): classifyTriangles / analyzeBoundingBox /
// encodeTriangleType (src/voxelizer.cu:3040-3221) and the 1D / 2D / 3D
// processing kernels (3306-3955).

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

// Work items of one (triangle, material subspace): voxels along the axis for
// 1D boxes, columns of the projection plane otherwise.
__device__ __forceinline__ uint32_t surfItems(const IBox& b, uint32_t code) {
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
                c += surfItems(b, code);
            }
        }
        counts[t] = c;
    }
}

struct Overlap { float nx[3], ny[3], de[3]; };

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
        const float s = sum2f<DE>(o.nx[i], pa, o.ny[i], pb);
        o.de[i] = __fadd_rn(__fadd_rn(-s, fmaxf(0.0f, __fmul_rn(d, o.nx[i]))), fmaxf(0.0f, __fmul_rn(d, o.ny[i])));
    }
    return o;
}

template <int OT> __device__ __forceinline__ bool overlapTest(const Overlap& o, float a, float b) {
    bool r = true;
#pragma unroll
    for (int i = 0; i < 3; ++i) r &= sum2p1f<OT>(o.nx[i], a, o.ny[i], b, o.de[i]) >= 0.0f;
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

// Records one processVoxel (src/voxelizer.cu:2946-2989) of the surface pass.
template <int K> struct SurfaceSink {
    uint32_t* bits;
    typename NodeT<K>::slot_t* slots;
    typename NodeT<K>::slot_t key;
    PassGeom g;
    int gridType;
    int mode;
    __device__ __forceinline__ void operator()(int x, int y, int z) const {
        const uint32_t X = g.X, AY = g.AY;
        size_t node;
        if (NodeT<K>::fcc) {
            const size_t l = 2 * (size_t)X, a = l * AY;
            const size_t zz = 2 * (size_t)(uint32_t)z + (gridType >= 3 ? 1 : 0);
            node = a * zz + l * (uint32_t)y + 2 * (size_t)(uint32_t)x + ((gridType & 1) == 0 ? 1 : 0);
        } else {
            node = ((size_t)(uint32_t)z * AY + (uint32_t)y) * X + (uint32_t)x;
        }
        if (mode == 0) {
            const size_t w = ((size_t)(uint32_t)z * AY + (uint32_t)y) * g.ipx + ((uint32_t)x >> 5);
            const uint32_t bit = 0x80000000u >> ((uint32_t)x & 31u);
            const uint32_t old = atomicOr(bits + w, bit);
            if (!(old & bit)) slots[node] = key;
        } else {
            slotMax(slots + node, key);
        }
    }
};

template <int K>
__global__ void surfaceWorkKernel(int mode, const float* __restrict__ V, const uint32_t* __restrict__ I,
                                  const uint8_t* __restrict__ M, uint32_t nT, PassGeom g, int gridType,
                                  const Split3* __restrict__ splits, uint32_t nSplits,
                                  const uint32_t* __restrict__ codes, const uint32_t* __restrict__ offsets,
                                  const uint32_t* __restrict__ totalPtr, uint32_t* __restrict__ bits, void* nodes) {
    const uint32_t total = *totalPtr;
    const float d = g.df;
    for (uint32_t item = blockIdx.x * blockDim.x + threadIdx.x; item < total; item += gridDim.x * blockDim.x) {
        const uint32_t t = findOwner(offsets, nT, item);
        uint32_t local = item - __ldg(offsets + t);
        const uint32_t code = __ldg(codes + t);
        F3 v[3];
        loadTriF(V, I, t, v);
        const IBox full = voxBoundsHalf(v, g);
        IBox b = full;
        for (uint32_t s = 0; s < nSplits; ++s) {
            b = full;
            if (!clampBox(b, splits[s])) continue;
            const uint32_t n = surfItems(b, code);
            if (local < n) break;
            local -= n;
        }
        const uint32_t bb = code >> 30, axis = (code >> 28) & 3u;
        SurfaceSink<K> sink;
        sink.bits = bits;
        sink.slots = reinterpret_cast<typename NodeT<K>::slot_t*>(nodes);
        sink.key = NodeT<K>::key(bb, __ldg(M + t), t);
        sink.g = g;
        sink.gridType = gridType;
        sink.mode = mode;
        const uint32_t ex = (uint32_t)(b.hi[0] - b.lo[0] + 1), ey = (uint32_t)(b.hi[1] - b.lo[1] + 1);
        if (bb == 1) {
            // process1DTriangles (3306-3411): every voxel of the line, no test.
            if (axis == 0) sink(b.lo[0] + (int)local + 1, b.lo[1] + 1, b.lo[2] + 1);
            else if (axis == 1) sink(b.lo[0] + 1, b.lo[1] + (int)local + 1, b.lo[2] + 1);
            else sink(b.lo[0] + 1, b.lo[1] + 1, b.lo[2] + (int)local + 1);
            continue;
        }
        if (bb == 2) {
            // process2DTriangles (3418-3596): the dominant projection only.
            const F3 n = crossF<site::CRF_2D>(subF(v[0], v[2]), subF(v[1], v[0]));
            if (axis == 0) {
                const int j = b.lo[1] + (int)(local % ey), k = b.lo[2] + (int)(local / ey);
                const Overlap o = setupOverlap<0, site::DE_2D_YZ>(v, n, d);
                if (overlapTest<site::OT_2D_YZ>(o, vbComp<site::PC_2D>(j, g.mnf[1], d), vbComp<site::PC_2D>(k, g.mnf[2], d)))
                    sink(b.lo[0] + 1, j + 1, k + 1);
            } else if (axis == 1) {
                const int i = b.lo[0] + (int)(local % ex), k = b.lo[2] + (int)(local / ex);
                const Overlap o = setupOverlap<1, site::DE_2D_ZX>(v, n, d);
                if (overlapTest<site::OT_2D_ZX>(o, vbComp<site::PC_2D>(k, g.mnf[2], d), vbComp<site::PC_2D>(i, g.mnf[0], d)))
                    sink(i + 1, b.lo[1] + 1, k + 1);
            } else {
                const int i = b.lo[0] + (int)(local % ex), j = b.lo[1] + (int)(local / ex);
                const Overlap o = setupOverlap<2, site::DE_2D_XY>(v, n, d);
                if (overlapTest<site::OT_2D_XY>(o, vbComp<site::PC_2D>(i, g.mnf[0], d), vbComp<site::PC_2D>(j, g.mnf[1], d)))
                    sink(i + 1, j + 1, b.lo[2] + 1);
            }
            continue;
        }
        // process3DTriangles (3603-3955): dominant projection, depth range
        // from the plane, then the other two projections per voxel unless the
        // range is a single voxel.
        const F3 n = crossF<site::CRF_3D>(subF(v[0], v[2]), subF(v[1], v[0]));
        const Overlap o0 = setupOverlap<0, site::DE_3D_YZ>(v, n, d);
        const Overlap o1 = setupOverlap<1, site::DE_3D_ZX>(v, n, d);
        const Overlap o2 = setupOverlap<2, site::DE_3D_XY>(v, n, d);
        if (axis == 0) {
            const int j = b.lo[1] + (int)(local % ey), k = b.lo[2] + (int)(local / ey);
            F3 p{0.0f, vbComp<site::PC_3D>(j, g.mnf[1], d), vbComp<site::PC_3D>(k, g.mnf[2], d)};
            if (!overlapTest<site::OT_3D_YZ>(o0, p.y, p.z)) continue;
            int r0, r1;
            depthRange<0, site::DT_3DX>(v, p, n, g, r0, r1);
            if (r0 > b.hi[0] || r1 < b.lo[0]) continue;
            r0 = r0 < b.lo[0] ? b.lo[0] : r0;
            r1 = r1 > b.hi[0] ? b.hi[0] : r1;
            if (r0 == r1) { sink(r0 + 1, j + 1, k + 1); continue; }
            for (int i = r0; i <= r1; ++i) {
                p.x = vbComp<site::PC_3DL>(i, g.mnf[0], d);
                if (overlapTest<site::OT_3DX_ZX>(o1, p.z, p.x) && overlapTest<site::OT_3DX_XY>(o2, p.x, p.y))
                    sink(i + 1, j + 1, k + 1);
            }
        } else if (axis == 1) {
            const int i = b.lo[0] + (int)(local % ex), k = b.lo[2] + (int)(local / ex);
            F3 p{vbComp<site::PC_3D>(i, g.mnf[0], d), 0.0f, vbComp<site::PC_3D>(k, g.mnf[2], d)};
            if (!overlapTest<site::OT_3D_ZX>(o1, p.z, p.x)) continue;
            int r0, r1;
            depthRange<1, site::DT_3DY>(v, p, n, g, r0, r1);
            if (r0 > b.hi[1] || r1 < b.lo[1]) continue;
            r0 = r0 < b.lo[1] ? b.lo[1] : r0;
            r1 = r1 > b.hi[1] ? b.hi[1] : r1;
            if (r0 == r1) { sink(i + 1, r0 + 1, k + 1); continue; }
            for (int j = r0; j <= r1; ++j) {
                p.y = vbComp<site::PC_3DL>(j, g.mnf[1], d);
                if (overlapTest<site::OT_3DY_XY>(o2, p.x, p.y) && overlapTest<site::OT_3DY_YZ>(o0, p.y, p.z))
                    sink(i + 1, j + 1, k + 1);
            }
        } else {
            const int i = b.lo[0] + (int)(local % ex), j = b.lo[1] + (int)(local / ex);
            F3 p{vbComp<site::PC_3D>(i, g.mnf[0], d), vbComp<site::PC_3D>(j, g.mnf[1], d), 0.0f};
            if (!overlapTest<site::OT_3D_XY>(o2, p.x, p.y)) continue;
            int r0, r1;
            depthRange<2, site::DT_3DZ>(v, p, n, g, r0, r1);
            if (r0 > b.hi[2] || r1 < b.lo[2]) continue;
            r0 = r0 < b.lo[2] ? b.lo[2] : r0;
            r1 = r1 > b.hi[2] ? b.hi[2] : r1;
            if (r0 == r1) { sink(i + 1, j + 1, r0 + 1); continue; }
            for (int k = r0; k <= r1; ++k) {
                p.z = vbComp<site::PC_3DL>(k, g.mnf[2], d);
                if (overlapTest<site::OT_3DZ_YZ>(o0, p.y, p.z) && overlapTest<site::OT_3DZ_ZX>(o1, p.z, p.x))
                    sink(i + 1, j + 1, k + 1);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Node classification on packed bits.

__global__ void combineKernel(const uint4* __restrict__ a, const uint4* __restrict__ b, uint4* __restrict__ out,
                              uint64_t n4) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += (uint64_t)gridDim.x * blockDim.x) {
        uint4 x = a[i], y = b[i];
        out[i] = make_uint4(x.x | y.x, x.y | y.y, x.z | y.z, x.w | y.w);
    }
}

// One pruning pass over one yz subspace (fillNodeList2 and the host loop,
// src/voxelizer.cu:1790-1913, src/host_side.cpp:1183-1206): a solid node
// stays solid iff each axis has a solid neighbour.  Words are updated in
// place; the host repeats passes until none changes, which reaches the same
// greatest fixed point as the reference's in-place node passes.
__global__ void pruneKernel(uint32_t* solid, PassGeom g, SplitYZ sp, uint32_t* changed) {
    const uint32_t ny = sp.y1 - sp.y0;
    const uint64_t nWords = (uint64_t)ny * (sp.z1 - sp.z0) * g.ipx;
    const size_t plane = (size_t)g.ipx * g.AY;
    bool any = false;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nWords; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = (uint32_t)(i % g.ipx);
        const uint64_t r = i / g.ipx;
        const uint32_t y = sp.y0 + (uint32_t)(r % ny), z = sp.z0 + (uint32_t)(r / ny);
        const size_t idx = ((size_t)z * g.AY + y) * g.ipx + k;
        const uint32_t w = solid[idx];
        if (w == 0) continue;
        const uint32_t prev = k > 0 ? solid[idx - 1] : 0u;
        const uint32_t next = k + 1 < g.ipx ? solid[idx + 1] : 0u;
        const uint32_t L = (w >> 1) | (prev << 31), R = (w << 1) | (next >> 31);
        const uint32_t In = y > 0 ? solid[idx - g.ipx] : 0u, Out = y + 1 < g.AY ? solid[idx + g.ipx] : 0u;
        const uint32_t Dn = z > 0 ? solid[idx - plane] : 0u, Up = z + 1 < g.AZ ? solid[idx + plane] : 0u;
        const uint32_t nw = w & (L | R) & (In | Out) & (Dn | Up);
        if (nw != w) {
            solid[idx] = nw;
            any = true;
        }
    }
    if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(changed, 1u);
}

// Node emission, Cartesian lattices.  One thread writes 16 bytes of nodes
// (G nodes of one row, all inside one 32-bit word of the bit grids).
// Boundary ids follow fillNodeList2 in split order: a neighbour in a later
// yz subspace is read from the unpruned grid (its subspace was still
// unpruned when this one converged), every other neighbour from the final
// grid.
template <int K>
__global__ void emitCartesianKernel(const uint32_t* __restrict__ fin, const uint32_t* __restrict__ fill,
                                    const uint32_t* __restrict__ surf, PassGeom g,
                                    const uint8_t* __restrict__ yLater, const uint8_t* __restrict__ zLater,
                                    void* __restrict__ nodes, int materials) {
    typedef NodeT<K> NT;
    constexpr int G = 16 / NT::bytes;
    __shared__ uint8_t lut[64];
    if (threadIdx.x < 64) lut[threadIdx.x] = kOrientTable[threadIdx.x];
    __syncthreads();
    const uint32_t groupsPerRow = g.X / G;
    const uint64_t nGroups = (uint64_t)groupsPerRow * g.AY * g.AZ;
    const size_t plane = (size_t)g.ipx * g.AY;
    for (uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gi < nGroups;
         gi += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t row = gi / groupsPerRow;
        const uint32_t x0 = (uint32_t)(gi % groupsPerRow) * G;
        const uint32_t y = (uint32_t)(row % g.AY), z = (uint32_t)(row / g.AY);
        const uint32_t k = x0 >> 5;
        const size_t idx = (size_t)row * g.ipx + k;
        const uint32_t c = __ldg(fin + idx);
        const uint32_t s0 = materials ? __ldg(surf + idx) : 0u;
        uint4 outv = make_uint4(0, 0, 0, 0);
        uint64_t* out64 = reinterpret_cast<uint64_t*>(&outv);
        const uint32_t sh = x0 & 31u;
        const uint32_t gmask = (G == 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << (32 - G - sh)));
        if ((c | s0) & gmask) {
            const uint32_t prev = k > 0 ? __ldg(fin + idx - 1) : 0u;
            const uint32_t next = k + 1 < g.ipx ? __ldg(fin + idx + 1) : 0u;
            const uint32_t L = (c >> 1) | (prev << 31), R = (c << 1) | (next >> 31);
            const uint32_t In = y > 0 ? __ldg(fin + idx - g.ipx) : 0u;
            uint32_t Out = 0u, Up = 0u;
            if (y + 1 < g.AY) {
                Out = __ldg(fin + idx + g.ipx);
                if (yLater[y]) Out = __ldg(fill + idx + g.ipx) | (materials ? __ldg(surf + idx + g.ipx) : 0u);
            }
            const uint32_t Dn = z > 0 ? __ldg(fin + idx - plane) : 0u;
            if (z + 1 < g.AZ) {
                Up = __ldg(fin + idx + plane);
                if (zLater[z]) Up = __ldg(fill + idx + plane) | (materials ? __ldg(surf + idx + plane) : 0u);
            }
            const uint32_t f0 = NT::bytes == 8 ? __ldg(fill + idx) : 0u;
            uint4 keys = make_uint4(0, 0, 0, 0);
            const size_t nodeBase = (size_t)row * g.X + x0;
            if (s0 & gmask) keys = *reinterpret_cast<const uint4*>(reinterpret_cast<const uint8_t*>(nodes) + nodeBase * NT::bytes);
            const typename NT::slot_t* ks = reinterpret_cast<const typename NT::slot_t*>(&keys);
#pragma unroll
            for (int n = 0; n < G; ++n) {
                const uint32_t q = 31u - (sh + n);
                uint32_t bid = 0;
                if ((c >> q) & 1u) {
                    const uint32_t perm = ((L >> q) & 1u) | (((R >> q) & 1u) << 1) | (((In >> q) & 1u) << 2) |
                                          (((Out >> q) & 1u) << 3) | (((Dn >> q) & 1u) << 4) | (((Up >> q) & 1u) << 5);
                    bid = lut[perm];
                }
                const bool isSurf = (s0 >> q) & 1u;
                const uint32_t mat = isSurf ? NT::keyMat((uint64_t)ks[n]) : 0u;
                float r = 0.0f;
                if (NT::bytes == 8) r = ((f0 >> q) & 1u) ? 1.0f : 0.0f;
                const uint64_t val = NT::pack(bid, mat, r);
                if (NT::bytes == 1) reinterpret_cast<uint8_t*>(&outv)[n] = (uint8_t)val;
                else if (NT::bytes == 2) reinterpret_cast<uint16_t*>(&outv)[n] = (uint16_t)val;
                else if (NT::bytes == 4) reinterpret_cast<uint32_t*>(&outv)[n] = (uint32_t)val;
                else out64[n] = val;
            }
        }
        reinterpret_cast<uint4*>(nodes)[(size_t)gi] = outv;
    }
}

struct FccGrids {
    const uint32_t* fill[4];
    const uint32_t* surf[4];
};

// Node emission, FCC lattices (convertToFCCGrid + calculateFCCBoundaries,
// src/voxelizer.cu:1710-1776, 1929-2048).  FCC node (X, y, Z) belongs to
// sub-lattice 1 + (X & 1) + 2 * (Z & 1) at voxel (X / 2, y, Z / 2); its id is
// the 12-bit mask of solid FCC neighbours.  The neighbour relation is
// symmetric, so the reference's in-place pass equals this snapshot
// evaluation.
__device__ __forceinline__ uint32_t fccSolid(const FccGrids& G, const PassGeom& g, uint32_t X2, uint32_t y, uint32_t Z2,
                                             int materials) {
    const int gt = (int)(X2 & 1u) + 2 * (int)(Z2 & 1u);
    const uint32_t x = X2 >> 1, z = Z2 >> 1;
    const size_t w = ((size_t)z * g.AY + y) * g.ipx + (x >> 5);
    uint32_t word = __ldg(G.fill[gt] + w);
    if (materials) word |= __ldg(G.surf[gt] + w);
    return (word >> (31u - (x & 31u))) & 1u;
}

template <int K>
__global__ void emitFccKernel(FccGrids G, PassGeom g, void* __restrict__ nodes, int materials) {
    typedef NodeT<K> NT;
    constexpr int GN = 16 / NT::bytes;
    const uint32_t NX = 2 * g.X, NY = g.AY, NZ = 2 * g.AZ;
    const uint32_t groupsPerRow = NX / GN;
    const uint64_t nGroups = (uint64_t)groupsPerRow * NY * NZ;
    const size_t npx = NX;
    for (uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gi < nGroups;
         gi += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t row = gi / groupsPerRow;
        const uint32_t X0 = (uint32_t)(gi % groupsPerRow) * GN;
        const uint32_t y = (uint32_t)(row % NY), Z2 = (uint32_t)(row / NY);
        uint4 outv = make_uint4(0, 0, 0, 0);
        uint4 keys = make_uint4(0, 0, 0, 0);
        bool keysLoaded = false;
#pragma unroll
        for (int n = 0; n < GN; ++n) {
            const uint32_t X2 = X0 + n;
            const int gt = (int)(X2 & 1u) + 2 * (int)(Z2 & 1u);
            const uint32_t x = X2 >> 1, z = Z2 >> 1;
            const size_t w = ((size_t)z * g.AY + y) * g.ipx + (x >> 5);
            const uint32_t q = 31u - (x & 31u);
            const uint32_t fb = (__ldg(G.fill[gt] + w) >> q) & 1u;
            const uint32_t sb = materials ? (__ldg(G.surf[gt] + w) >> q) & 1u : 0u;
            uint32_t bid = 0;
            if (fb | sb) {
                const bool left = X2 > 0, right = X2 < NX - 1, in = y > 0, out = y < NY - 1;
                const bool down = Z2 > 0, up = Z2 < NZ - 1, xe = ((X2 + Z2) & 1u) == 0;
                const uint32_t ym = xe ? y - 1 : y;   // y - xEven
                const uint32_t yp = xe ? y : y + 1;   // y + !xEven
                const bool cIn = (xe && in) || !xe, cOut = (!xe && out) || xe;
                if (down && cIn && fccSolid(G, g, X2, ym, Z2 - 1, materials)) bid |= 1u;
                if (down && left && fccSolid(G, g, X2 - 1, y, Z2 - 1, materials)) bid |= 2u;
                if (down && right && fccSolid(G, g, X2 + 1, y, Z2 - 1, materials)) bid |= 4u;
                if (down && cOut && fccSolid(G, g, X2, yp, Z2 - 1, materials)) bid |= 8u;
                if (left && cIn && fccSolid(G, g, X2 - 1, ym, Z2, materials)) bid |= 16u;
                if (right && cIn && fccSolid(G, g, X2 + 1, ym, Z2, materials)) bid |= 32u;
                if (left && cOut && fccSolid(G, g, X2 - 1, yp, Z2, materials)) bid |= 64u;
                if (right && cOut && fccSolid(G, g, X2 + 1, yp, Z2, materials)) bid |= 128u;
                if (up && cIn && fccSolid(G, g, X2, ym, Z2 + 1, materials)) bid |= 256u;
                if (up && left && fccSolid(G, g, X2 - 1, y, Z2 + 1, materials)) bid |= 512u;
                if (up && right && fccSolid(G, g, X2 + 1, y, Z2 + 1, materials)) bid |= 1024u;
                if (up && cOut && fccSolid(G, g, X2, yp, Z2 + 1, materials)) bid |= 2048u;
            }
            uint32_t mat = 0;
            if (sb) {
                if (!keysLoaded) {
                    keys = *reinterpret_cast<const uint4*>(reinterpret_cast<const uint8_t*>(nodes) +
                                                           ((size_t)row * npx + X0) * NT::bytes);
                    keysLoaded = true;
                }
                mat = NT::keyMat((uint64_t)reinterpret_cast<const typename NT::slot_t*>(&keys)[n]);
            }
            const uint64_t val = NT::pack(bid, mat, 0.0f);
            if (NT::bytes == 2) reinterpret_cast<uint16_t*>(&outv)[n] = (uint16_t)val;
            else reinterpret_cast<uint32_t*>(&outv)[n] = (uint32_t)val;
        }
        reinterpret_cast<uint4*>(nodes)[(size_t)gi] = outv;
    }
}

inline uint32_t gridFor(uint64_t work, uint32_t threads, uint32_t cap = 148u * 32u) {
    uint64_t b = (work + threads - 1) / threads;
    if (b == 0) b = 1;
    return (uint32_t)(b < cap ? b : cap);
}

}  // namespace

// ---------------------------------------------------------------------------
// Launch wrappers.

void launch_scan(const uint32_t* in, uint32_t* offsets, uint32_t n, uint32_t* blockSums, uint32_t* total,
                 uint32_t* overflow, cudaStream_t s, uint32_t* launches) {
    const uint32_t tiles = n == 0 ? 1 : (n + kScanTile - 1) / kScanTile;
    scanTileKernel<<<tiles, kScanThreads, 0, s>>>(in, offsets, n, blockSums);
    scanSumsKernel<<<1, kScanThreads, 0, s>>>(blockSums, tiles, total, overflow);
    scanAddKernel<<<(n + 1 + 255) / 256, 256, 0, s>>>(offsets, n, blockSums, total);
    *launches += 3;
}

void launch_solid_count(const float* V, const uint32_t* I, uint32_t nT, PassGeom g, const SplitYZ* splits,
                        uint32_t nSplits, uint32_t* counts, cudaStream_t s, uint32_t* launches) {
    solidCountKernel<<<gridFor(nT, 256), 256, 0, s>>>(V, I, nT, g, splits, nSplits, counts);
    *launches += 1;
}

void launch_solid_toggle(const float* V, const uint32_t* I, uint32_t nT, PassGeom g, const SplitYZ* splits,
                         uint32_t nSplits, const uint32_t* offsets, const uint32_t* total, uint32_t* toggles,
                         cudaStream_t s, uint32_t* launches) {
    solidToggleKernel<<<148 * 8, 256, 0, s>>>(V, I, nT, g, splits, nSplits, offsets, total, toggles);
    *launches += 1;
}

void launch_row_fill(uint32_t* words, uint32_t rows, uint32_t ipx, cudaStream_t s, uint32_t* launches) {
    rowFillKernel<<<gridFor((uint64_t)rows * 32, 256), 256, 0, s>>>(words, rows, ipx);
    *launches += 1;
}

void launch_surface_count(const float* V, const uint32_t* I, uint32_t nT, PassGeom g, const Split3* splits,
                          uint32_t nSplits, uint32_t* codes, uint32_t* counts, cudaStream_t s, uint32_t* launches) {
    surfaceCountKernel<<<gridFor(nT, 256), 256, 0, s>>>(V, I, nT, g, splits, nSplits, codes, counts);
    *launches += 1;
}

void launch_surface_work(int nodeKind, int mode, const float* V, const uint32_t* I, const uint8_t* M, uint32_t nT,
                         PassGeom g, int gridType, const Split3* splits, uint32_t nSplits, const uint32_t* codes,
                         const uint32_t* offsets, const uint32_t* total, uint32_t* surfBits, void* nodes,
                         cudaStream_t s, uint32_t* launches) {
    const dim3 grid(148 * 8), block(256);
    switch (nodeKind) {
    case kShort: surfaceWorkKernel<kShort><<<grid, block, 0, s>>>(mode, V, I, M, nT, g, gridType, splits, nSplits, codes, offsets, total, surfBits, nodes); break;
    case kLong: surfaceWorkKernel<kLong><<<grid, block, 0, s>>>(mode, V, I, M, nT, g, gridType, splits, nSplits, codes, offsets, total, surfBits, nodes); break;
    case kPartial: surfaceWorkKernel<kPartial><<<grid, block, 0, s>>>(mode, V, I, M, nT, g, gridType, splits, nSplits, codes, offsets, total, surfBits, nodes); break;
    case kShortFcc: surfaceWorkKernel<kShortFcc><<<grid, block, 0, s>>>(mode, V, I, M, nT, g, gridType, splits, nSplits, codes, offsets, total, surfBits, nodes); break;
    default: surfaceWorkKernel<kLongFcc><<<grid, block, 0, s>>>(mode, V, I, M, nT, g, gridType, splits, nSplits, codes, offsets, total, surfBits, nodes); break;
    }
    *launches += 1;
}

void launch_combine(const uint32_t* a, const uint32_t* b, uint32_t* out, uint64_t n, cudaStream_t s,
                    uint32_t* launches) {
    const uint64_t n4 = n / 4;
    combineKernel<<<gridFor(n4, 256), 256, 0, s>>>(reinterpret_cast<const uint4*>(a), reinterpret_cast<const uint4*>(b),
                                                    reinterpret_cast<uint4*>(out), n4);
    *launches += 1;
}

void launch_prune(uint32_t* solid, PassGeom g, SplitYZ split, uint32_t* changed, cudaStream_t s, uint32_t* launches) {
    const uint64_t n = (uint64_t)(split.y1 - split.y0) * (split.z1 - split.z0) * g.ipx;
    pruneKernel<<<gridFor(n, 256), 256, 0, s>>>(solid, g, split, changed);
    *launches += 1;
}

void launch_emit_cartesian(int nodeKind, const uint32_t* finalSolid, const uint32_t* fill, const uint32_t* surf,
                           PassGeom g, const uint8_t* yLater, const uint8_t* zLater, void* nodes, int materials,
                           cudaStream_t s, uint32_t* launches) {
    const int bytes = nodeKind == kShort ? 1 : nodeKind == kLong ? 2 : 8;
    const uint64_t groups = (uint64_t)g.X * g.AY * g.AZ * bytes / 16;
    const uint32_t grid = gridFor(groups, 256, 148u * 64u);
    switch (nodeKind) {
    case kShort: emitCartesianKernel<kShort><<<grid, 256, 0, s>>>(finalSolid, fill, surf, g, yLater, zLater, nodes, materials); break;
    case kLong: emitCartesianKernel<kLong><<<grid, 256, 0, s>>>(finalSolid, fill, surf, g, yLater, zLater, nodes, materials); break;
    default: emitCartesianKernel<kPartial><<<grid, 256, 0, s>>>(finalSolid, fill, surf, g, yLater, zLater, nodes, materials); break;
    }
    *launches += 1;
}

void launch_emit_fcc(int nodeKind, const uint32_t* const* fill, const uint32_t* const* surf, PassGeom g, void* nodes,
                     int materials, cudaStream_t s, uint32_t* launches) {
    FccGrids G;
    for (int i = 0; i < 4; ++i) { G.fill[i] = fill[i]; G.surf[i] = surf[i]; }
    const int bytes = nodeKind == kShortFcc ? 2 : 4;
    const uint64_t groups = (uint64_t)(2 * g.X) * g.AY * (2 * g.AZ) * bytes / 16;
    const uint32_t grid = gridFor(groups, 256, 148u * 64u);
    if (nodeKind == kShortFcc) emitFccKernel<kShortFcc><<<grid, 256, 0, s>>>(G, g, nodes, materials);
    else emitFccKernel<kLongFcc><<<grid, 256, 0, s>>>(G, g, nodes, materials);
    *launches += 1;
}

}  // namespace vxb
