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

namespace vxb {

struct Range { uint32_t lo, hi; };

struct Plan {
    double mn[3], mx[3];   // bounding box (float vertices widened to double)
    double d;              // voxel length
    uint32_t res[3];       // resolution.max: x padded (+2) and rounded to 32 * xSplits
    uint32_t xSplits, xRes;
    uint32_t alloc[3];     // res + (0, 2, 2)
    std::vector<Range> ySplitsExt, zSplitsExt;        // voxSplitRes over [0, res)
    std::vector<Range> ySplitsAlloc, zSplitsAlloc;    // voxSplitRes over [0, alloc)
    std::vector<Range> xMat, yMat, zMat;              // matSplitRes over [0, res)
};

// Reference conversion semantics for uint(ceil(...)): NaN and negatives to 0.
inline uint32_t toUint(double v) {
    if (!(v > 0.0)) return 0u;
    if (v >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

// splitResolutionByNrOfParts: floor division, the remainder goes to the
// first part (src/host_side.cpp:3025-3105).
inline std::vector<Range> splitLength(uint32_t len, uint32_t maxPart) {
    const uint32_t n = (len + maxPart - 1) / maxPart;
    std::vector<Range> out(n);
    uint32_t prev = len;
    for (uint32_t i = n; i > 0; --i) {
        Range r;
        r.hi = prev;
        r.lo = r.hi - r.hi / i;
        prev = r.lo;
        out[i - 1] = r;
    }
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

// Returns 0, or a negative vxb status for arguments the path cannot honour.
inline int makePlan(const double* mn, const double* mx, int byCube, uint32_t maxDim, double cube,
                    const uint32_t* voxSplit, const uint32_t* matSplit, Plan& p) {
    for (int a = 0; a < 3; ++a) { p.mn[a] = mn[a]; p.mx[a] = mx[a]; }
    const double dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    uint32_t r[3];
    double d;
    if (byCube) {
        if (!(cube > 0.0)) return -1;
        d = cube;
        r[0] = toUint(std::ceil(dx / d)) + 1;
        r[1] = toUint(std::ceil(dy / d)) + 1;
        r[2] = toUint(std::ceil(dz / d)) + 1;
    } else {
        if (maxDim < 2) return -1;
        const uint32_t m = maxDim;
        if (dx > dy && dx > dz) {
            d = dx / double(m - 1);
            r[0] = m; r[1] = toUint(std::ceil(dy / d)) + 1; r[2] = toUint(std::ceil(dz / d)) + 1;
        } else if (dx > dy) {
            d = dz / double(m - 1);
            r[2] = m; r[0] = toUint(std::ceil(dx / d)) + 1; r[1] = toUint(std::ceil(dy / d)) + 1;
        } else if (dy > dz) {
            d = dy / double(m - 1);
            r[1] = m; r[0] = toUint(std::ceil(dx / d)) + 1; r[2] = toUint(std::ceil(dz / d)) + 1;
        } else {
            d = dz / double(m - 1);
            r[2] = m; r[0] = toUint(std::ceil(dx / d)) + 1; r[1] = toUint(std::ceil(dy / d)) + 1;
        }
        if (!(d > 0.0)) return -1;
    }
    r[0] += 2;
    for (int a = 0; a < 3; ++a)
        if (voxSplit[a] == 0) return -1;
    p.d = d;
    p.xSplits = (r[0] + voxSplit[0] - 1) / voxSplit[0];
    const uint32_t xMod = 32u * p.xSplits;
    if (r[0] % xMod != 0) r[0] += xMod - r[0] % xMod;
    p.xRes = r[0] / p.xSplits;
    // The reference's per-split word mask (src/voxelizer.cu:1579-1616) holds
    // 32 words, so an x pass longer than 1024 voxels is undefined there.
    if (p.xRes > 1024) return -1;
    for (int a = 0; a < 3; ++a) p.res[a] = r[a];
    p.alloc[0] = r[0];
    p.alloc[1] = r[1] + 2;
    p.alloc[2] = r[2] + 2;
    p.ySplitsExt = splitLength(r[1], voxSplit[1]);
    p.zSplitsExt = splitLength(r[2], voxSplit[2]);
    p.ySplitsAlloc = splitLength(p.alloc[1], voxSplit[1]);
    p.zSplitsAlloc = splitLength(p.alloc[2], voxSplit[2]);
    // A zero material split size (the reference passes 0 where no surface
    // pass runs, src/host_side.cpp:2301) means one pass over the extent.
    p.xMat = splitLength(r[0], matSplit[0] ? matSplit[0] : r[0]);
    p.yMat = splitLength(r[1], matSplit[1] ? matSplit[1] : r[1]);
    p.zMat = splitLength(r[2], matSplit[2] ? matSplit[2] : r[2]);
    return 0;
}

}  // namespace vxb
