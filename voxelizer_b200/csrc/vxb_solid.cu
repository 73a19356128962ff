// Solid (parity) voxelization kernels: calculateTileOverlap /
// constructWorkQueue / generateVoxelization (src/voxelizer.cu:840-1617),
// FP64 as in the reference.
//
// The reference sorts (tile, triangle) pairs and voxelizes one tile per
// block.  Here the work list is the flat set of (work triangle, yz subspace,
// 4x4 tile) candidates of every unit of the batch over an exclusive scan of
// per-triangle candidate counts;
// a candidate is a member of the tile's list iff one voxel centre of the
// tile inside the triangle's clipped bounding box passes the binning test,
// and a member toggles, for each centre of the tile inside the subspace that
// passes the strict generation test, the bit of its x-intercept voxel in the
// centre's row.  Toggles commute (XOR), so no sort is needed; a row prefix
// XOR then turns toggles into solid runs.  A block stages its candidates'
// triangles (vertices, tN, voxel box, both edge-function sets, the normal)
// in shared memory once.

#include "vxb_common.cuh"
#include "vxb_device.cuh"
#include "vxb_kernels.cuh"

namespace vxb {

using namespace detail;

namespace {

constexpr double kDblMin = 2.2250738585072014e-308;  // DBL_MIN, src/voxelizer.cu:1443
constexpr int kBlock = 256;
constexpr uint32_t kSlots = 160;   // 160 staged triangles: 44 KB of static shared memory

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

// The unit and mesh triangle of work triangle wt.
__device__ __forceinline__ uint32_t workUnit(const Batch& b, uint32_t wt, uint32_t* t) {
    const uint32_t u = unitOf(b.workBase, b.nUnits, wt);
    *t = wt - __ldg(b.workBase + u);
    return u;
}

__global__ void solidCountKernel(Batch b, uint32_t nWork, uint32_t* __restrict__ counts) {
    for (uint32_t wt = blockIdx.x * blockDim.x + threadIdx.x; wt < nWork; wt += gridDim.x * blockDim.x) {
        uint32_t t;
        const Unit& U = b.units[workUnit(b, wt, &t)];
        const PassGeom g = U.g;
        BinTri bt;
        binSetup(U.V, U.I, t, g, bt);
        uint32_t c = 0;
        if (!binRejected(bt)) {
            const SplitYZ* splits = b.splits + U.splitBase;
            for (uint32_t s = 0; s < U.nSplits; ++s) {
                uint32_t lo[2], hi[2];
                if (!commonSpace(bt, splits[s], lo, hi)) continue;
                c += ((hi[0] - 1) / 4 - lo[0] / 4 + 1) * ((hi[1] - 1) / 4 - lo[1] / 4 + 1);
            }
        }
        counts[wt] = c;
    }
}

// Staged triangle: binning data plus the generation edge functions.
struct SolidStage {
    BinTri b;
    double bnx[3], bny[3], bd[3];   // binning edges (oriented by tN)
    D3 n;                           // cross(v0 - v2, v1 - v0)
    double ex[3], ey[3], ed[3];     // generation edges (oriented by n.x)
    uint32_t tl;                    // top-left flags of the generation edges
    uint32_t unit;
};

__device__ __forceinline__ void stageSolid(SolidStage& st, const Batch& b, uint32_t wt) {
    uint32_t t;
    st.unit = workUnit(b, wt, &t);
    const Unit& unit = b.units[st.unit];
    binSetup(unit.V, unit.I, t, unit.g, st.b);
    const D3* v = st.b.v;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const D3& p = v[i];
        const D3& q = v[(i + 1) % 3];
        if (st.b.tN > 0.0) { st.bnx[i] = __dsub_rn(p.z, q.z); st.bny[i] = __dsub_rn(q.y, p.y); }
        else { st.bnx[i] = __dsub_rn(q.z, p.z); st.bny[i] = __dsub_rn(p.y, q.y); }
        st.bd[i] = -sum2<site::D_BIN>(st.bnx[i], p.y, st.bny[i], p.z);
    }
    const D3 U{__dsub_rn(v[0].x, v[2].x), __dsub_rn(v[0].y, v[2].y), __dsub_rn(v[0].z, v[2].z)};
    const D3 W{__dsub_rn(v[1].x, v[0].x), __dsub_rn(v[1].y, v[0].y), __dsub_rn(v[1].z, v[0].z)};
    st.n = D3{diff2<site::CR_GEN>(U.y, W.z, U.z, W.y), diff2<site::CR_GEN>(U.z, W.x, U.x, W.z),
              diff2<site::CR_GEN>(U.x, W.y, U.y, W.x)};
    st.tl = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const D3& p = v[i];
        const D3& q = v[(i + 1) % 3];
        if (st.n.x > 0.0) { st.ex[i] = __dsub_rn(p.z, q.z); st.ey[i] = __dsub_rn(q.y, p.y); }
        else { st.ex[i] = __dsub_rn(q.z, p.z); st.ey[i] = __dsub_rn(p.y, q.y); }
        st.ed[i] = -sum2<site::D_GEN>(st.ex[i], p.y, st.ey[i], p.z);
        if (st.ex[i] > 0.0 || (st.ex[i] == 0.0 && st.ey[i] < 0.0)) st.tl |= 1u << i;
    }
}

// One (triangle, subspace, tile) candidate: binning membership
// (traverseTilesForOverlaps, src/voxelizer.cu:980-1033), then
// generateVoxelization's per-centre work (1344-1462) for the tile's centres
// inside the subspace.
__device__ __forceinline__ void solidCandidate(const SolidStage& st, const Batch& b, uint32_t local,
                                               uint32_t* __restrict__ fill) {
    const Unit& U = b.units[st.unit];
    const PassGeom& g = U.g;
    const SplitYZ* __restrict__ splits = b.splits + U.splitBase;
    const uint32_t nSplits = U.nSplits;
    uint32_t* __restrict__ toggles = fill + U.wordBase;
    const double d = g.d;
    uint32_t lo[2] = {0, 0}, hi[2] = {0, 0};
    SplitYZ sp = splits[0];
    for (uint32_t s = 0; s < nSplits; ++s) {
        if (!commonSpace(st.b, splits[s], lo, hi)) continue;
        const uint32_t nty = (hi[0] - 1) / 4 - lo[0] / 4 + 1, ntz = (hi[1] - 1) / 4 - lo[1] / 4 + 1;
        if (local < nty * ntz) { sp = splits[s]; break; }
        local -= nty * ntz;
    }
    const uint32_t nty = (hi[0] - 1) / 4 - lo[0] / 4 + 1;
    const uint32_t tileY = lo[0] / 4 + local % nty, tileZ = lo[1] / 4 + local / nty;
    // Unfused edge functions (the pinned forms of E_BIN and E_GEN) keep the
    // product of the row's coordinate across the row: the same operations
    // in the same order as evaluating each centre from scratch.
    static_assert(site::E_BIN == 0 && site::E_GEN == 0, "row products assume the unfused edge forms");
    static_assert(site::P_BIN == 0, "corner test assumes the unfused centre form");
    // Every operation of an unfused binning edge function is monotone in the
    // centre's row and column (d > 0), so its largest value over the tile's
    // centres is at the corner its normal points to: a tile where one edge
    // is negative even there has no member centre.
    {
        const uint32_t y0 = max(tileY * 4, lo[0]), y1 = min(tileY * 4 + 4, hi[0]);
        const uint32_t z0 = max(tileZ * 4, lo[1]), z1 = min(tileZ * 4 + 4, hi[1]);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double py = lin<site::P_BIN>((double)(st.bnx[k] > 0.0 ? y1 - 1 : y0), d, g.mn[1]);
            const double pz = lin<site::P_BIN>((double)(st.bny[k] > 0.0 ? z1 - 1 : z0), d, g.mn[2]);
            if (__dadd_rn(__dadd_rn(__dmul_rn(st.bnx[k], py), __dmul_rn(st.bny[k], pz)), st.bd[k]) < 0.0) return;
        }
    }
    bool member = false;
    for (uint32_t iy = tileY * 4; iy < tileY * 4 + 4 && iy < hi[0] && !member; ++iy) {
        if (iy < lo[0]) continue;
        const double py = lin<site::P_BIN>((double)iy, d, g.mn[1]);
        double ry[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) ry[k] = __dmul_rn(st.bnx[k], py);
        for (uint32_t iz = tileZ * 4; iz < tileZ * 4 + 4 && iz < hi[1]; ++iz) {
            if (iz < lo[1]) continue;
            const double pz = lin<site::P_BIN>((double)iz, d, g.mn[2]);
            bool ok = true;
#pragma unroll
            for (int k = 0; k < 3; ++k) ok &= __dadd_rn(__dadd_rn(ry[k], __dmul_rn(st.bny[k], pz)), st.bd[k]) >= 0.0;
            if (ok) { member = true; break; }
        }
    }
    if (!member) return;
    const D3* v = st.b.v;
    for (uint32_t cz = 0; cz < 4; ++cz) {
        const uint32_t vz = tileZ * 4 + cz;
        if (vz < sp.z0 || vz >= sp.z1) continue;
        const double pz = lin<site::P_GEN>((double)vz, d, g.mn[2]);
        double rz[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) rz[i] = __dmul_rn(st.ey[i], pz);
        for (uint32_t cy = 0; cy < 4; ++cy) {
            const uint32_t vy = tileY * 4 + cy;
            if (vy < sp.y0 || vy >= sp.y1) continue;
            const double py = lin<site::P_GEN>((double)vy, d, g.mn[1]);
            int pass = 0;
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                double r = __dadd_rn(__dadd_rn(__dmul_rn(st.ex[i], py), rz[i]), st.ed[i]);
                if ((st.tl >> i) & 1u) r = __dadd_rn(r, kDblMin);
                pass += r > 0.0;
            }
            if (pass != 3) continue;
            const double ax = __dsub_rn(v[0].x, g.mn[0]), ay = __dsub_rn(v[0].y, py), az = __dsub_rn(v[0].z, pz);
            const double B = sum3<site::B_GEN>(ax, st.n.x, ay, st.n.y, az, st.n.z);
            double px = __ddiv_rn(B, st.n.x);
            px = px < 0.0 ? 0.0 : px;
            const uint32_t vx = __double2uint_rz(ceil(__ddiv_rn(px, d))) + 1u;
            if (vx >= g.X) continue;
            const uint32_t row = (vz + g.padZ) * g.AY + (vy + g.padY);
            atomicXor(toggles + (size_t)row * g.ipx + (vx >> 5), 0x80000000u >> (vx & 31u));
        }
    }
}

__global__ void __launch_bounds__(kBlock, 3) solidToggleKernel(Batch b, uint32_t nWork,
                                                               const uint32_t* __restrict__ offsets,
                                                               const uint32_t* __restrict__ totalPtr,
                                                               uint32_t* __restrict__ fill, uint32_t* queue) {
    __shared__ SolidStage stage[kSlots];
    __shared__ uint32_t stOff[kSlots + 1];
    __shared__ uint32_t tFirst, tLast, nextBase;
    const uint32_t total = *totalPtr;
    // Batches of kBlock candidates in a fixed grid-stride order, or
    // (queue != NULL) taken from a device work queue, one atomic per batch.
    uint32_t base = blockIdx.x * kBlock;
    if (queue) {
        if (threadIdx.x == 0) nextBase = atomicAdd(queue, kBlock);
        __syncthreads();
        base = nextBase;
    }
    while (base < total) {
        const uint32_t last = min(base + kBlock, total) - 1;
        // Owners of the batch's first and last items, one warp each.
        if (threadIdx.x < 64) {
            const uint32_t t = warpFindOwner(offsets, nWork, threadIdx.x < 32 ? base : last, threadIdx.x & 31u);
            if (threadIdx.x == 0) tFirst = t;
            if (threadIdx.x == 32) tLast = t;
        }
        __syncthreads();
        const uint32_t t0 = tFirst, t1 = tLast, ns = min(t1 - t0 + 1, kSlots);
        // Triangles without candidates between them are never selected
        // (their offset equals the next one) and are not staged.
        if (threadIdx.x < ns) {
            const uint32_t o = __ldg(offsets + t0 + threadIdx.x);
            stOff[threadIdx.x] = o;
            if (__ldg(offsets + t0 + threadIdx.x + 1) > o) stageSolid(stage[threadIdx.x], b, t0 + threadIdx.x);
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
                solidCandidate(stage[lo], b, item - stOff[lo], fill);
            } else {
                // The owner lies past the staged triangles and at most at
                // the batch's last owner: offsets[t0 + ns] <= item <
                // offsets[t1 + 1].
                uint32_t lo = t0 + ns, hi = t1 + 1;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (__ldg(offsets + mid) <= item) lo = mid;
                    else hi = mid;
                }
                const uint32_t wt = lo;
                SolidStage st;
                stageSolid(st, b, wt);
                solidCandidate(st, b, item - __ldg(offsets + wt), fill);
            }
        }
        if (queue && threadIdx.x == 0) nextBase = atomicAdd(queue, kBlock);
        __syncthreads();
        base = queue ? nextBase : base + gridDim.x * kBlock;
    }
}

// Toggle bits -> solid runs: bit x of a row = XOR of the row's toggles at or
// before x.  A warp takes kFillRows whole rows (consecutive words) and walks
// them as 32-word chunks, one word per lane, so loads and stores are
// coalesced: a lane turns its word into the prefix XOR of its bits and
// inverts it when the words before it in its row hold an odd number of
// toggles.  That parity is a segmented XOR scan over the lanes (a ballot of
// word parities, cut at the lanes that start a row) plus the parity carried
// from the previous chunk for the row that continues into this one.
constexpr uint32_t kFillRows = 16;

__global__ void rowFillKernel(Batch b, uint64_t nRows, uint32_t* __restrict__ fill) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nWarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g * kFillRows < nRows; g += nWarps) {
        uint64_t row = g * kFillRows;
        const uint64_t rowEnd = min(row + kFillRows, nRows);
        while (row < rowEnd) {
            // The rows of [row, rowEnd) in one unit.
            const uint32_t u = b.nUnits > 1 ? unitOf(b.rowBase, b.nUnits, row) : 0u;
            const uint64_t uRow0 = __ldg(b.rowBase + u), uRow1 = __ldg(b.rowBase + u + 1);
            const uint64_t r1 = min(rowEnd, uRow1);
            const Unit& U = b.units[u];
            const uint32_t ipx = U.g.ipx;
            uint32_t* words = fill + U.wordBase;
            const uint32_t w0 = (uint32_t)(row - uRow0) * ipx, w1 = (uint32_t)(r1 - uRow0) * ipx;
            uint32_t carry = 0u;
            for (uint32_t cb = w0; cb < w1; cb += 32u) {
                const uint32_t w = cb + lane;
                const bool valid = w < w1;
                const uint32_t x = valid ? words[w] : 0u;
                const uint32_t starts = __ballot_sync(0xffffffffu, valid && (w - w0) % ipx == 0u);
                const uint32_t odd = __ballot_sync(0xffffffffu, __popc(x) & 1u);
                const uint32_t upTo = starts & ((2u << lane) - 1u);   // row starts at lanes <= lane
                uint32_t below = (1u << lane) - 1u;                  // lanes < lane
                uint32_t pre;
                if (upTo) {
                    below &= ~((1u << (31u - __clz(upTo))) - 1u);
                    pre = __popc(odd & below) & 1u;
                } else {
                    pre = (__popc(odd & below) & 1u) ^ carry;
                }
                uint32_t p = x;
                p ^= p >> 1; p ^= p >> 2; p ^= p >> 4; p ^= p >> 8; p ^= p >> 16;
                if (pre) p = ~p;
                if (valid && p != x) words[w] = p;
                carry = __shfl_sync(0xffffffffu, pre ^ (__popc(x) & 1u), 31);
            }
            row = r1;
        }
    }
}

}  // namespace

void launch_solid_count(const Batch& b, uint32_t nWork, uint32_t* counts, cudaStream_t s, uint32_t* launches) {
    solidCountKernel<<<gridFor(nWork, 256), 256, 0, s>>>(b, nWork, counts);
    *launches += 1;
}

void launch_solid_toggle(const Batch& b, uint32_t nWork, const uint32_t* offsets, const uint32_t* total,
                         uint32_t* fill, uint32_t blocksPerSm, uint32_t* queue, cudaStream_t s, uint32_t* launches) {
    if (queue) cudaMemsetAsync(queue, 0, sizeof(uint32_t), s);
    solidToggleKernel<<<148u * blocksPerSm, kBlock, 0, s>>>(b, nWork, offsets, total, fill, queue);
    *launches += 1;
}

void launch_row_fill(const Batch& b, uint64_t nRows, uint32_t* fill, cudaStream_t s, uint32_t* launches) {
    rowFillKernel<<<gridFor((nRows + kFillRows - 1) / kFillRows * 32u, 256), 256, 0, s>>>(b, nRows, fill);
    *launches += 1;
}

}  // namespace vxb
