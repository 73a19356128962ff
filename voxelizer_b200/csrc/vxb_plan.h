// Host-side sizing: bounding box, voxel length, grid dimensions and the
// internal split sequence, restating src/host_side.cpp of the reference
// (calculateBoundingBox 2462-2488, determineDimensions 2497-2609,
// adjustResolution 2620-2634, splitResolutionByMaxDim / ByNrOfParts
// 2942-3239, allocResolution padding 953-957).  The split sequence is part of
// the output contract: pruning runs per yz subspace in this order and the
// x padding depends on the number of x passes.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

#ifdef __CUDACC__
#define VXB_HD __host__ __device__
#else
#define VXB_HD
#endif

namespace vxb {

struct Range { uint32_t lo, hi; };

struct Plan {
    double mn[3], mx[3];   // bounding box (float vertices widened to double); mn: the voxelized box's corner
    double mnHost[3];      // the mesh's minimum corner (getMinVertex)
    double d;              // voxel length
    uint32_t res[3];       // resolution.max: x padded (+2) and rounded to 32 * xSplits
    uint32_t xSplits, xRes;
    uint32_t alloc[3];     // res + (0, 2, 2)
    std::vector<Range> ySplitsExt, zSplitsExt;        // voxSplitRes over [0, res)
    std::vector<Range> ySplitsAlloc, zSplitsAlloc;    // voxSplitRes over [0, alloc)
    std::vector<Range> xMat, yMat, zMat;              // matSplitRes over [0, res)
    // Device space (src/host_side.cpp:782-1011): a yz partition of the full
    // grid whose voxelized box is extended by one voxel towards each
    // neighbouring partition.  Row `padY` of the allocation holds local
    // voxel row 0 (1 without a neighbour below in y, the zero padding row;
    // 0 with one, the overlap row), likewise `padZ`; `border` zeroes the
    // allocation's faces after the boundary ids (zeroPadding).  A full grid
    // is the device space without neighbours.
    uint32_t padY = 1, padZ = 1;
    bool border = false;
    uint32_t part[4] = {0, 0, 0, 0};   // partition y0, y1, z0, z1 (voxels of the full grid)
};

// Reference conversion semantics for uint(ceil(...)): NaN and negatives to 0.
inline uint32_t toUint(double v) {
    if (!(v > 0.0)) return 0u;
    if (v >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

// splitResolutionByNrOfParts: floor division, the remainder goes to the
// first part (src/host_side.cpp:3025-3105).  Writes the parts of [0, len)
// into out (room for ceil(len / maxPart) ranges) and returns their number.
inline uint32_t splitInto(uint32_t len, uint32_t maxPart, Range* out) {
    const uint32_t n = (len + maxPart - 1) / maxPart;
    uint32_t prev = len;
    for (uint32_t i = n; i > 0; --i) {
        out[i - 1].hi = prev;
        out[i - 1].lo = prev - prev / i;
        prev = out[i - 1].lo;
    }
    return n;
}

// Part i alone of the same split (for device code that has no room for the
// whole list).
VXB_HD inline Range splitPart(uint32_t len, uint32_t maxPart, uint32_t i) {
    const uint32_t n = (len + maxPart - 1) / maxPart;
    uint32_t prev = len;
    for (uint32_t k = n; k > i + 1; --k) prev -= prev / k;
    Range r;
    r.hi = prev;
    r.lo = prev - prev / (i + 1);
    return r;
}

inline std::vector<Range> splitLength(uint32_t len, uint32_t maxPart) {
    std::vector<Range> out((len + maxPart - 1) / maxPart);
    splitInto(len, maxPart, out.data());
    return out;
}

inline void boundingBox(const float* v, uint32_t nV, double* mn, double* mx) {
    for (int a = 0; a < 3; ++a) mn[a] = mx[a] = v[a];
    for (uint32_t i = 1; i < nV; ++i)
        for (int a = 0; a < 3; ++a) {
            if (v[3 * i + a] > mx[a]) mx[a] = v[3 * i + a];
            if (v[3 * i + a] < mn[a]) mn[a] = v[3 * i + a];
        }
}

// The grid of determineDimensions and adjustResolution without the split
// lists.
struct GridSize {
    double d;              // voxel length
    uint32_t res[3];       // resolution.max: x padded (+2) and rounded to 32 * xSplits
    uint32_t xSplits, xRes;
    uint32_t alloc[3];     // res + (0, 2, 2)
};

// uint(ceil(extent / d)) + 1 of determineDimensions; false where the count
// leaves no room for the padding rows in 32 bits (the reference would wrap
// to an empty grid there).
inline bool axisRes(double extent, double d, uint32_t& r) {
    const double c = std::ceil(extent / d);
    if (c >= 4294967290.0) return false;
    r = toUint(c) + 1;
    return true;
}

// Returns 0, or -1 for arguments the path cannot honour.
inline int sizeGrid(const double* mn, const double* mx, int byCube, uint32_t maxDim, double cube,
                    const uint32_t* voxSplit, GridSize& g) {
    const double dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    uint32_t r[3];
    double d;
    bool ok = true;
    if (byCube) {
        if (!(cube > 0.0)) return -1;
        d = cube;
        ok = axisRes(dx, d, r[0]) && axisRes(dy, d, r[1]) && axisRes(dz, d, r[2]);
    } else {
        if (maxDim < 2) return -1;
        const uint32_t m = maxDim;
        if (dx > dy && dx > dz) {
            d = dx / double(m - 1);
            r[0] = m; ok = axisRes(dy, d, r[1]) && axisRes(dz, d, r[2]);
        } else if (dx > dy) {
            d = dz / double(m - 1);
            r[2] = m; ok = axisRes(dx, d, r[0]) && axisRes(dy, d, r[1]);
        } else if (dy > dz) {
            d = dy / double(m - 1);
            r[1] = m; ok = axisRes(dx, d, r[0]) && axisRes(dz, d, r[2]);
        } else {
            d = dz / double(m - 1);
            r[2] = m; ok = axisRes(dx, d, r[0]) && axisRes(dy, d, r[1]);
        }
        if (!(d > 0.0)) return -1;
    }
    if (!ok || r[0] > 0xFFFFFFFFu - 2u || r[1] > 0xFFFFFFFFu - 2u || r[2] > 0xFFFFFFFFu - 2u) return -1;
    r[0] += 2;
    for (int a = 0; a < 3; ++a)
        if (voxSplit[a] == 0) return -1;
    g.d = d;
    g.xSplits = (r[0] + voxSplit[0] - 1) / voxSplit[0];
    const uint32_t xMod = 32u * g.xSplits;
    if (r[0] % xMod != 0) r[0] += xMod - r[0] % xMod;
    g.xRes = r[0] / g.xSplits;
    // The reference's per-split word mask (src/voxelizer.cu:1579-1616) holds
    // 32 words, so an x pass longer than 1024 voxels is undefined there.
    if (g.xRes > 1024) return -1;
    for (int a = 0; a < 3; ++a) g.res[a] = r[a];
    g.alloc[0] = r[0];
    g.alloc[1] = r[1] + 2;
    g.alloc[2] = r[2] + 2;
    return 0;
}

// Returns 0, or a negative vxb status for arguments the path cannot honour.
inline int makePlan(const double* mn, const double* mx, int byCube, uint32_t maxDim, double cube,
                    const uint32_t* voxSplit, const uint32_t* matSplit, Plan& p) {
    for (int a = 0; a < 3; ++a) { p.mn[a] = mn[a]; p.mx[a] = mx[a]; p.mnHost[a] = mn[a]; }
    GridSize g;
    if (sizeGrid(mn, mx, byCube, maxDim, cube, voxSplit, g)) return -1;
    const uint32_t* r = g.res;
    p.d = g.d;
    p.xSplits = g.xSplits;
    p.xRes = g.xRes;
    for (int a = 0; a < 3; ++a) {
        p.res[a] = g.res[a];
        p.alloc[a] = g.alloc[a];
    }
    p.ySplitsExt = splitLength(r[1], voxSplit[1]);
    p.zSplitsExt = splitLength(r[2], voxSplit[2]);
    p.ySplitsAlloc = splitLength(p.alloc[1], voxSplit[1]);
    p.zSplitsAlloc = splitLength(p.alloc[2], voxSplit[2]);
    // A zero material split size (the reference passes 0 where no surface
    // pass runs, src/host_side.cpp:2301) means one pass over the extent.
    p.xMat = splitLength(r[0], matSplit[0] ? matSplit[0] : r[0]);
    p.yMat = splitLength(r[1], matSplit[1] ? matSplit[1] : r[1]);
    p.zMat = splitLength(r[2], matSplit[2] ? matSplit[2] : r[2]);
    p.padY = p.padZ = 1;
    p.border = false;
    p.part[0] = 0;
    p.part[1] = r[1];
    p.part[2] = 0;
    p.part[3] = r[2];
    return 0;
}

// The device space of partition [y0, y1) x [z0, z1) of the full plan `p`
// (voxelizeWorker, src/host_side.cpp:911-1011): neighbour flags from the
// partition's position, the extended box, its minimum corner in double
// (hostMin + extMin * d), the allocation (partition + 2 rows each way) and
// the split lists over the extended box and the allocation.
inline int devicePlan(const Plan& p, uint32_t y0, uint32_t y1, uint32_t z0, uint32_t z1, const uint32_t* voxSplit,
                      const uint32_t* matSplit, Plan& q) {
    if (!(y0 < y1 && y1 <= p.res[1] && z0 < z1 && z1 <= p.res[2])) return -1;
    bool left = false, right = false, down = false, up = false;
    if (y0 == 0 && y1 != p.res[1]) right = true;
    else if (y1 == p.res[1] && y0 != 0) left = true;
    else if (y0 != 0 && y1 != p.res[1]) left = right = true;
    if (z0 == 0 && z1 != p.res[2]) up = true;
    else if (z1 == p.res[2] && z0 != 0) down = true;
    else if (z0 != 0 && z1 != p.res[2]) down = up = true;
    const uint32_t ey0 = y0 - (left ? 1u : 0u), ey1 = y1 + (right ? 1u : 0u);
    const uint32_t ez0 = z0 - (down ? 1u : 0u), ez1 = z1 + (up ? 1u : 0u);
    q = p;
    q.mn[0] = p.mn[0] + double(0u) * p.d;
    q.mn[1] = p.mn[1] + double(ey0) * p.d;
    q.mn[2] = p.mn[2] + double(ez0) * p.d;
    q.res[1] = ey1 - ey0;
    q.res[2] = ez1 - ez0;
    q.alloc[1] = (y1 - y0) + 2;
    q.alloc[2] = (z1 - z0) + 2;
    q.ySplitsExt = splitLength(q.res[1], voxSplit[1]);
    q.zSplitsExt = splitLength(q.res[2], voxSplit[2]);
    q.ySplitsAlloc = splitLength(q.alloc[1], voxSplit[1]);
    q.zSplitsAlloc = splitLength(q.alloc[2], voxSplit[2]);
    q.yMat = splitLength(q.res[1], matSplit[1] ? matSplit[1] : q.res[1]);
    q.zMat = splitLength(q.res[2], matSplit[2] ? matSplit[2] : q.res[2]);
    q.padY = left ? 0u : 1u;
    q.padZ = down ? 0u : 1u;
    q.border = left || right || down || up;
    q.part[0] = y0;
    q.part[1] = y1;
    q.part[2] = z0;
    q.part[3] = z1;
    return 0;
}

// splitResolutionByNrOfParts over one axis (src/host_side.cpp:3025-3105):
// `parts` pieces of [0, len), floor division, the remainder to the first.
inline std::vector<Range> splitParts(uint32_t len, uint32_t parts) {
    std::vector<Range> out(parts);
    uint32_t prev = len;
    for (uint32_t i = parts; i > 0; --i) {
        Range r;
        r.hi = prev;
        r.lo = r.hi - r.hi / i;
        prev = r.lo;
        out[i - 1] = r;
    }
    return out;
}

}  // namespace vxb
