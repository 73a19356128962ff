// Solid (parity) voxelization kernels.
#include "vxb_common.cuh"
#include "vxb_device.cuh"
#include "vxb_kernels.cuh"

#include <cfloat>

namespace vxb {

using namespace detail;

namespace {

constexpr double kDblMin = 2.2250738585072014e-308;  // DBL_MIN, src/voxelizer.cu:1443

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
}  // namespace

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
}  // namespace vxb
