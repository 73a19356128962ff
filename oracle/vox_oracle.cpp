// CPU restatement of hakarlss/Voxelizer's mesh -> node-grid path.
//
// TEST INFRASTRUCTURE ONLY (see vox_oracle.h).  Follows the reference step by
// step; each function cites the reference lines it restates.  Integer and
// index arithmetic keeps the reference's 32-bit unsigned wrap-around.
// Floating-point expressions are written with explicit std::fma according to
// the contraction model in orc_params::fma_model; this file is compiled with
// -ffp-contract=off so the compiler adds no contraction of its own.

#include "vox_oracle.h"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <limits>
#include <cstring>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef uint32_t uint;
typedef uint8_t uchar;

struct d2 { double x, y; };
struct d3 { double x, y, z; };
struct f2 { float x, y; };
struct f3 { float x, y, z; };
struct i2 { int x, y; };
struct i3 { int x, y, z; };
struct u2 { uint x, y; };
struct u3 { uint x, y, z; };
template <class T> struct Bounds { T min, max; };

// ---------------------------------------------------------------------------
// CUDA conversion semantics (PTX cvt.rzi with the default clamping):
// NaN -> 0, values beyond the destination range clamp to it.
static inline uint cvt_d2u(double v) {
    if (std::isnan(v)) return 0u;
    if (v <= 0.0) return 0u;
    if (v >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint)v;
}
static inline int cvt_d2i(double v) {
    if (std::isnan(v)) return 0;
    if (v <= -2147483648.0) return INT_MIN;
    if (v >= 2147483647.0) return INT_MAX;
    return (int)v;
}
static inline int cvt_f2i(float v) { return cvt_d2i((double)v); }

// ---------------------------------------------------------------------------
// Contraction model (see vox_oracle.h).
struct Fma {
    uint8_t s[ORC_NSITES];
    explicit Fma(const uint8_t* sites) { memcpy(s, sites, sizeof(s)); }
    int operator[](int i) const { return s[i]; }
};

template <class T> static inline T fmaT(T a, T b, T c) { return std::fma(a, b, c); }

// a*b + c*d + e
template <class T> static inline T sum2p1(T a, T b, T c, T d, T e, int mode) {
    switch (mode) {
    case 0: return (a * b + c * d) + e;
    case 1: return fmaT(a, b, c * d) + e;
    case 2: return fmaT(c, d, a * b) + e;
    default: return fmaT(a, b, fmaT(c, d, e));
    }
}
// a*b + c*d
template <class T> static inline T sum2(T a, T b, T c, T d, int mode) {
    switch (mode) {
    case 0: return a * b + c * d;
    case 1: return fmaT(a, b, c * d);
    default: return fmaT(c, d, a * b);
    }
}
// a*b - c*d
template <class T> static inline T diff2(T a, T b, T c, T d, int mode) {
    switch (mode) {
    case 0: return a * b - c * d;
    case 1: return fmaT(a, b, -(c * d));
    default: return fmaT(-c, d, a * b);
    }
}
// a*b + c*d + e*f
template <class T> static inline T sum3(T a, T b, T c, T d, T e, T f, int mode) {
    switch (mode) {
    case 0: return (a * b + c * d) + e * f;
    case 1: return fmaT(e, f, fmaT(a, b, c * d));
    case 2: return fmaT(e, f, fmaT(c, d, a * b));
    case 3: return fmaT(a, b, c * d) + e * f;
    case 4: return fmaT(e, f, a * b + c * d);
    default: return fmaT(c, d, a * b) + e * f;
    }
}

// ---------------------------------------------------------------------------
// Node layouts, include/node_types.h:19-706 (same byte layout, own code).
struct ShortN { uchar bim; };
struct LongN { uchar bid, mat; };
struct PartialN { uchar bid, mat, pad0, pad1; float r; };
struct SFccN { uint16_t bim; };
struct LFccN { uint16_t bid; uchar mat, pad; };

template <class N> struct Tr;
template <> struct Tr<ShortN> {
    static const bool fcc = false, ratio = false;
    static uint bid(const ShortN& n) { return n.bim & 31u; }
    static uint mat(const ShortN& n) { return n.bim >> 5; }
    static void setBid(ShortN& n, uint b) { n.bim = (uchar)((b & 31u) | (n.bim & 224u)); }
    static ShortN make(uint b, uint m) { ShortN n; n.bim = (uchar)((m << 5) | (b & 31u)); return n; }
    static void setR(ShortN&, float) {}
};
template <> struct Tr<LongN> {
    static const bool fcc = false, ratio = false;
    static uint bid(const LongN& n) { return n.bid; }
    static uint mat(const LongN& n) { return n.mat; }
    static void setBid(LongN& n, uint b) { n.bid = (uchar)b; }
    static LongN make(uint b, uint m) { LongN n; n.bid = (uchar)b; n.mat = (uchar)m; return n; }
    static void setR(LongN&, float) {}
};
template <> struct Tr<PartialN> {
    static const bool fcc = false, ratio = true;
    static uint bid(const PartialN& n) { return n.bid; }
    static uint mat(const PartialN& n) { return n.mat; }
    static void setBid(PartialN& n, uint b) { n.bid = (uchar)b; }
    static PartialN make(uint b, uint m) { PartialN n; n.bid = (uchar)b; n.mat = (uchar)m; n.pad0 = n.pad1 = 0; n.r = 0.f; return n; }
    static void setR(PartialN& n, float r) { n.r = r; }
};
template <> struct Tr<SFccN> {
    static const bool fcc = true, ratio = false;
    static uint bid(const SFccN& n) { return n.bim & 4095u; }
    static uint mat(const SFccN& n) { return n.bim >> 12; }
    static void setBid(SFccN& n, uint b) { n.bim = (uint16_t)((b & 4095u) | (n.bim & 61440u)); }
    static SFccN make(uint b, uint m) { SFccN n; n.bim = (uint16_t)((m << 12) | (b & 4095u)); return n; }
    static void setR(SFccN&, float) {}
};
template <> struct Tr<LFccN> {
    static const bool fcc = true, ratio = false;
    static uint bid(const LFccN& n) { return n.bid; }
    static uint mat(const LFccN& n) { return n.mat; }
    static void setBid(LFccN& n, uint b) { n.bid = (uint16_t)b; }
    static LFccN make(uint b, uint m) { LFccN n; n.bid = (uint16_t)b; n.mat = (uchar)m; n.pad = 0; return n; }
    static void setR(LFccN&, float) {}
};

// ---------------------------------------------------------------------------
// Boundary-id lookup, src/voxelizer.cu:2142-2236.  Bits of the 6-neighbour
// permutation: -x 1, +x 2, -y 4, +y 8, -z 16, +z 32.  A node keeps a
// non-zero id iff each axis has at least one solid neighbour; ids follow the
// reference's numbering (include/voxelizer.h:47-83).
static const uchar kOrient[64] = {
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
    0, 0, 0, 0, 0, 1, 2, 9, 0, 3, 4, 10, 0, 11, 12, 21,
    0, 0, 0, 0, 0, 5, 6, 13, 0, 7, 8, 14, 0, 15, 16, 26,
    0, 0, 0, 0, 0, 17, 18, 23, 0, 19, 20, 22, 0, 25, 24, 27,
};

// ---------------------------------------------------------------------------
// Splits, src/host_side.cpp:2942-3239.
static void splitLen(uint len, uint n, std::vector<Bounds<uint> >& out) {
    out.assign(n, Bounds<uint>());
    uint prev = len;
    for (uint i = n; i > 0; --i) {
        Bounds<uint> b; b.max = prev; b.min = b.max - (b.max / i); prev = b.min;
        out[i - 1] = b;
    }
}
static std::vector<Bounds<u2> > splitYZ(u2 maxDim, Bounds<u3> r) {
    uint ry = r.max.y - r.min.y, rz = r.max.z - r.min.z;
    uint ny = (ry + maxDim.x - 1) / maxDim.x, nz = (rz + maxDim.y - 1) / maxDim.y;
    std::vector<Bounds<uint> > yb, zb;
    splitLen(ry, ny, yb);
    splitLen(rz, nz, zb);
    std::vector<Bounds<u2> > s;
    for (uint z = 0; z < nz; ++z)
        for (uint y = 0; y < ny; ++y) {
            Bounds<u2> b;
            b.min = u2{r.min.y + yb[y].min, r.min.z + zb[z].min};
            b.max = u2{r.min.y + yb[y].max, r.min.z + zb[z].max};
            s.push_back(b);
        }
    return s;
}
static std::vector<Bounds<u3> > split3(u3 maxDim, Bounds<u3> r) {
    u3 res{r.max.x - r.min.x, r.max.y - r.min.y, r.max.z - r.min.z};
    uint nx = (res.x + maxDim.x - 1) / maxDim.x, ny = (res.y + maxDim.y - 1) / maxDim.y,
         nz = (res.z + maxDim.z - 1) / maxDim.z;
    std::vector<Bounds<uint> > xb, yb, zb;
    splitLen(res.x, nx, xb);
    splitLen(res.y, ny, yb);
    splitLen(res.z, nz, zb);
    std::vector<Bounds<u3> > s;
    for (uint z = 0; z < nz; ++z)
        for (uint y = 0; y < ny; ++y)
            for (uint x = 0; x < nx; ++x) {
                Bounds<u3> b;
                b.min = u3{r.min.x + xb[x].min, r.min.y + yb[y].min, r.min.z + zb[z].min};
                b.max = u3{r.min.x + xb[x].max, r.min.y + yb[y].max, r.min.z + zb[z].max};
                s.push_back(b);
            }
    return s;
}

// ---------------------------------------------------------------------------
// Bounding box and dimensions: src/host_side.cpp:2462-2488, 2497-2609,
// 2620-2634, 730-738.
struct Plan {
    d3 mn, mx;
    double d;
    u3 res;       // resolution.max (x includes padding and rounding)
    uint xSplits, xRes;
    u3 alloc;     // res + (0,2,2); a device space: partition + (0,2,2)
    int err;
    // Device space, voxelizeWorker (src/host_side.cpp:911-1011): the
    // voxelized (extended) box `ext` (local extents), its minimum corner
    // (extMinVertex), the allocation row of local row 0 (padding: 1, overlap
    // with a neighbour: 0) and whether zeroPadding clears the faces.
    d3 mnExt;
    u3 ext;
    uint padY, padZ;
    bool border;
};

static Plan makePlan(const orc_params* p, const float* v, uint nV) {
    Plan pl;
    memset(&pl, 0, sizeof(pl));
    if (nV == 0) { pl.err = -10; return pl; }
    pl.mn = d3{v[0], v[1], v[2]};
    pl.mx = pl.mn;
    for (uint i = 1; i < nV; i++) {
        if (v[3*i] > pl.mx.x) pl.mx.x = v[3*i];
        if (v[3*i+1] > pl.mx.y) pl.mx.y = v[3*i+1];
        if (v[3*i+2] > pl.mx.z) pl.mx.z = v[3*i+2];
        if (v[3*i] < pl.mn.x) pl.mn.x = v[3*i];
        if (v[3*i+1] < pl.mn.y) pl.mn.y = v[3*i+1];
        if (v[3*i+2] < pl.mn.z) pl.mn.z = v[3*i+2];
    }
    d3 diff{pl.mx.x - pl.mn.x, pl.mx.y - pl.mn.y, pl.mx.z - pl.mn.z};
    u3 res{0, 0, 0};
    double d;
    if (p->by_cube_length) {
        d = p->cube_length;
        res.x = cvt_d2u(std::ceil(diff.x / d)) + 1;
        res.y = cvt_d2u(std::ceil(diff.y / d)) + 1;
        res.z = cvt_d2u(std::ceil(diff.z / d)) + 1;
    } else {
        uint m = p->max_dim;
        if (diff.x > diff.y && diff.x > diff.z) {
            d = diff.x / double(m - 1);
            res.x = m;
            res.y = cvt_d2u(std::ceil(diff.y / d)) + 1;
            res.z = cvt_d2u(std::ceil(diff.z / d)) + 1;
        } else if (diff.x > diff.y) {
            d = diff.z / double(m - 1);
            res.z = m;
            res.x = cvt_d2u(std::ceil(diff.x / d)) + 1;
            res.y = cvt_d2u(std::ceil(diff.y / d)) + 1;
        } else if (diff.y > diff.z) {
            d = diff.y / double(m - 1);
            res.y = m;
            res.x = cvt_d2u(std::ceil(diff.x / d)) + 1;
            res.z = cvt_d2u(std::ceil(diff.z / d)) + 1;
        } else {
            d = diff.z / double(m - 1);
            res.z = m;
            res.x = cvt_d2u(std::ceil(diff.x / d)) + 1;
            res.y = cvt_d2u(std::ceil(diff.y / d)) + 1;
        }
    }
    res.x += 2;
    pl.d = d;
    if (p->vox_split[0] == 0 || p->vox_split[1] == 0 || p->vox_split[2] == 0) { pl.err = -11; return pl; }
    pl.xSplits = (res.x + p->vox_split[0] - 1) / p->vox_split[0];
    uint xMod = 32u * pl.xSplits;
    if (res.x % xMod != 0) res.x += xMod - (res.x % xMod);
    pl.res = res;
    pl.xRes = res.x / pl.xSplits;
    pl.alloc = u3{res.x, res.y + 2, res.z + 2};
    pl.mnExt = pl.mn;
    pl.ext = res;
    pl.padY = pl.padZ = 1;
    pl.border = false;
    // The solid voxelizer's per-split word mask holds at most 32 words
    // (src/voxelizer.cu:1579-1616): larger x passes are undefined there.
    if (pl.xRes > 1024) pl.err = -12;
    return pl;
}

// rotateVertices (src/host_side.cpp:3261-3280): the mesh turned about z by
// x' = a - y, y' = b + x with a = cy + cx, b = cy - cx from the half extents
// of its bounding box (in double), rounded to float.
static std::vector<float> turnedVertices(const float* v, uint nV) {
    std::vector<float> r(v, v + 3 * (size_t)nV);
    if (nV == 0) return r;
    double mn[2] = {v[0], v[1]}, mx[2] = {v[0], v[1]};
    for (uint i = 1; i < nV; ++i)
        for (int a = 0; a < 2; ++a) {
            mn[a] = std::min(mn[a], (double)v[3 * i + a]);
            mx[a] = std::max(mx[a], (double)v[3 * i + a]);
        }
    const double cx = (mx[0] - mn[0]) / 2.0, cy = (mx[1] - mn[1]) / 2.0;
    const double a = cy + cx, b = cy - cx;
    for (uint i = 0; i < nV; ++i) {
        const double x = v[3 * i];
        r[3 * i] = float(a - double(v[3 * i + 1]));
        r[3 * i + 1] = float(b + x);
    }
    return r;
}

// The device space of partition p->part (voxelizeWorker,
// src/host_side.cpp:911-1011): neighbour flags from the partition's
// position, the box extended by one voxel towards each neighbour, its
// minimum corner hostMin + extMin * d, the allocation partition + 2.
static void applySpace(const orc_params* p, Plan& pl) {
    if (!p->space || pl.err) return;
    const uint y0 = p->part[0], y1 = p->part[1], z0 = p->part[2], z1 = p->part[3];
    if (!(y0 < y1 && y1 <= pl.res.y && z0 < z1 && z1 <= pl.res.z)) { pl.err = -15; return; }
    bool left = false, right = false, down = false, up = false;
    if (y0 == 0 && y1 != pl.res.y) right = true;
    else if (y1 == pl.res.y && y0 != 0) left = true;
    else if (y0 != 0 && y1 != pl.res.y) left = right = true;
    if (z0 == 0 && z1 != pl.res.z) up = true;
    else if (z1 == pl.res.z && z0 != 0) down = true;
    else if (z0 != 0 && z1 != pl.res.z) down = up = true;
    const uint ey0 = y0 - (left ? 1 : 0), ey1 = y1 + (right ? 1 : 0);
    const uint ez0 = z0 - (down ? 1 : 0), ez1 = z1 + (up ? 1 : 0);
    pl.mnExt = d3{pl.mn.x + double(0u) * pl.d, pl.mn.y + double(ey0) * pl.d, pl.mn.z + double(ez0) * pl.d};
    pl.ext = u3{pl.res.x, ey1 - ey0, ez1 - ez0};
    pl.alloc = u3{pl.res.x, (y1 - y0) + 2, (z1 - z0) + 2};
    pl.padY = left ? 0 : 1;
    pl.padZ = down ? 0 : 1;
    pl.border = left || right || down || up;
}

// ---------------------------------------------------------------------------
// Tile binning, src/voxelizer.cu:840-1232 (restated for the CPU).
struct TriSetupD {
    d3 v[3];
    bool valid;      // passed the tN / bounding-box / subspace rejections
    Bounds<u2> cs;   // commonSpace
    d2 n[3];
    double dist[3];
};

static inline void fetchD(const float* V, const uint* I, uint t, d3* v) {
    for (int k = 0; k < 3; ++k) {
        uint a = I[3*t + k];
        v[k] = d3{V[3*a], V[3*a+1], V[3*a+2]};
    }
}

// calculateTileOverlap / constructWorkQueue setup, src/voxelizer.cu:861-945 and 1086-1144.
static TriSetupD binSetup(const float* V, const uint* I, uint t, d3 mn, double d, Bounds<u2> space,
                          const Fma& F, bool checkReject) {
    TriSetupD s;
    fetchD(V, I, t, s.v);
    const d3* v = s.v;
    // getTriangleBounds (double2 y/z), src/voxelizer.cu:2397-2418
    d2 bmin{v[0].y, v[0].z}, bmax = bmin;
    for (int i = 1; i < 3; i++) {
        bmin.x = v[i].y < bmin.x ? v[i].y : bmin.x;
        bmin.y = v[i].z < bmin.y ? v[i].z : bmin.y;
        bmax.x = v[i].y > bmax.x ? v[i].y : bmax.x;
        bmax.y = v[i].z > bmax.y ? v[i].z : bmax.y;
    }
    // getVoxelBoundsDouble, src/voxelizer.cu:2446-2458
    d2 vmin{(bmin.x - mn.y) / d, (bmin.y - mn.z) / d};
    d2 vmax{(bmax.x - mn.y) / d, (bmax.y - mn.z) / d};
    i2 vlo{cvt_d2i(std::ceil(vmin.x)), cvt_d2i(std::ceil(vmin.y))};
    i2 vhi{cvt_d2i(std::floor(vmax.x) + 1.0), cvt_d2i(std::floor(vmax.y) + 1.0)};
    // tN, src/voxelizer.cu:882-884 (two 3-product sums, then a difference)
    double tN = sum3(v[0].y, v[1].z, v[2].y, v[0].z, v[2].z, v[1].y, F[ORC_S_TN]) -
                sum3(v[2].y, v[1].z, v[0].z, v[1].y, v[2].z, v[0].y, F[ORC_S_TN]);
    s.valid = true;
    if (checkReject) {
        if (tN == 0.0) { s.valid = false; return s; }
        if (vlo.x >= vhi.x || vlo.y >= vhi.y) { s.valid = false; return s; }
        if (vhi.x <= (int)space.min.x || vhi.y <= (int)space.min.y) { s.valid = false; return s; }
        if (vlo.x >= (int)space.max.x || vlo.y >= (int)space.max.y) { s.valid = false; return s; }
    }
    i2 smin{(int)space.min.x, (int)space.min.y};
    s.cs.min = u2{(uint)std::max(smin.x, vlo.x), (uint)std::max(smin.y, vlo.y)};
    s.cs.max = u2{std::min(space.max.x, (uint)vhi.x), std::min(space.max.y, (uint)vhi.y)};
    for (int i = 0; i < 3; i++) {
        const d3& a = v[i];
        const d3& b = v[(i + 1) % 3];
        if (tN > 0.0) s.n[i] = d2{a.z - b.z, b.y - a.y};
        else s.n[i] = d2{b.z - a.z, a.y - b.y};
    }
    for (int i = 0; i < 3; i++)
        s.dist[i] = -sum2(s.n[i].x, v[i].y, s.n[i].y, v[i].z, F[ORC_S_D_BIN]);
    return s;
}

static inline double pcoord(uint i, double d, double m, int mode) {
    return mode ? std::fma(double(i), d, m) : double(i) * d + m;
}

// traverseTilesForOverlaps / traverseTilesForWorkQueue, src/voxelizer.cu:980-1033, 1168-1232.
template <class Emit>
static void traverseTiles(const TriSetupD& s, d3 mn, double d, const Fma& F, Emit emit) {
    Bounds<u2> tiles{u2{s.cs.min.x / 4, s.cs.min.y / 4}, u2{(s.cs.max.x - 1) / 4, (s.cs.max.y - 1) / 4}};
    for (uint t = tiles.min.x; t <= tiles.max.x; t++) {
        for (uint u = tiles.min.y; u <= tiles.max.y; u++) {
            bool skip = false;
            for (uint i = t * 4; i < t * 4 + 4 && i < s.cs.max.x && !skip; i++) {
                for (uint j = u * 4; j < u * 4 + 4 && j < s.cs.max.y && !skip; j++) {
                    if (i >= s.cs.min.x && j >= s.cs.min.y) {
                        double px = pcoord(i, d, mn.y, F[ORC_S_P_BIN]), py = pcoord(j, d, mn.z, F[ORC_S_P_BIN]);
                        bool ok = true;
                        for (int k = 0; k < 3; k++)
                            ok &= sum2p1(s.n[k].x, px, s.n[k].y, py, s.dist[k], F[ORC_S_E_BIN]) >= 0.0;
                        if (ok) { emit(t, u); skip = true; }
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Solid voxelization of one yz subspace, src/host_side.cpp:274-397 with the
// kernels src/voxelizer.cu:840-1617.
static void performVoxelization(const float* V, const uint* I, uint nT, d3 mn, double d, Bounds<u3> extRes,
                                Bounds<u2> yz, uint xRes, uint nX, uint32_t* voxels, u3 alloc, const Fma& F,
                                uint padY, uint padZ) {
    Bounds<u2> space{u2{yz.min.x - extRes.min.y, yz.min.y - extRes.min.z},
                     u2{yz.max.x - extRes.min.y, yz.max.y - extRes.min.z}};
    u3 resExt{extRes.max.x - extRes.min.x, extRes.max.y - extRes.min.y, extRes.max.z - extRes.min.z};
    const uint tilesY = (resExt.y + 3) / 4;
    // calculateTileOverlap
    std::vector<uint> counts(nT, 0);
#pragma omp parallel for schedule(dynamic, 256)
    for (long long tt = 0; tt < (long long)nT; ++tt) {
        uint t = (uint)tt;
        TriSetupD s = binSetup(V, I, t, mn, d, space, F, true);
        if (!s.valid) continue;
        uint c = 0;
        traverseTiles(s, mn, d, F, [&](uint, uint) { c++; });
        counts[t] = c;
    }
    // prepareForConstructWorkQueue, src/host_side.cpp:2645-2668
    std::vector<uint> offs(nT, 0);
    uint W = 0;
    int first = -1;
    for (uint i = 0; i < nT; i++) {
        if (counts[i] == 0) offs[i] = 0;
        else {
            if (first < 0) first = (int)i;
            offs[i] = W;
            W += counts[i];
        }
    }
    if (W == 0) return;
    // constructWorkQueue
    std::vector<uint> wqTri(W), wqTile(W);
#pragma omp parallel for schedule(dynamic, 256)
    for (long long tt = 0; tt < (long long)nT; ++tt) {
        uint t = (uint)tt;
        if (t < (uint)first) continue;
        uint off = offs[t];
        if (t != (uint)first && off == 0) continue;
        TriSetupD s = binSetup(V, I, t, mn, d, space, F, false);
        uint cur = 0;
        traverseTiles(s, mn, d, F, [&](uint tcol, uint urow) {
            wqTri[off + cur] = t;
            wqTile[off + cur] = urow * tilesY + tcol;
            cur++;
        });
    }
    // sortWorkQueue + compactWorkQueue (src/voxelizer.cu:39-111): stable sort
    // by tile id, then the first position of every distinct tile.
    std::vector<uint> order(W);
    for (uint i = 0; i < W; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint a, uint b) { return wqTile[a] < wqTile[b]; });
    std::vector<uint> tileList, tileStart;
    for (uint i = 0; i < W; i++) {
        if (i == 0 || wqTile[order[i]] != wqTile[order[i - 1]]) {
            tileList.push_back(wqTile[order[i]]);
            tileStart.push_back(i);
        }
    }
    tileStart.push_back(W);
    const uint ipx = alloc.x >> 5;
    // Row stride: the allocation (src/voxelizer.cu:1486-1501 grows the
    // extended box by the padding rows that no neighbour overlaps).
    const uint resY2 = alloc.y;
    // generateVoxelization, src/voxelizer.cu:1273-1617, once per x subspace.
    for (uint xs = 0; xs < nX; ++xs) {
        Bounds<u3> sub{u3{xs * xRes, yz.min.x, yz.min.y}, u3{(xs + 1) * xRes, yz.max.x, yz.max.y}};
        Bounds<u2> sp{u2{sub.min.y - extRes.min.y, sub.min.z - extRes.min.z},
                      u2{sub.max.y - extRes.min.y, sub.max.z - extRes.min.z}};
        const uint intsPerDim = (sub.max.x - sub.min.x) >> 5;
        const uint minIx = (sub.min.x + 2) >> 5;
        const uint endIx = (sub.max.x + 2) >> 5;
        const uint lastIX = (sub.max.x + 1) >> 5;
#pragma omp parallel for schedule(dynamic, 16)
        for (long long tl = 0; tl < (long long)tileList.size(); ++tl) {
            uint tileNr = tileList[tl];
            uint tileZ = tileNr / tilesY, tileY = tileNr % tilesY;
            // Per voxel centre: XOR accumulation of "active segment" words and
            // the per-split word mask (activeSegments / bitmasks in the kernel).
            for (uint k = 0; k < 16; ++k) {
                uint voxelZ = (k / 4) + tileZ * 4;
                uint voxelY = (k % 4) + tileY * 4;
                if (!(voxelY >= sp.min.x && voxelY < sp.max.x && voxelZ >= sp.min.y && voxelZ < sp.max.y)) continue;
                uint32_t bitmask = 0;
                bool any = false;
                uint rowBase = resY2 * ipx * (voxelZ + padZ) + ipx * (voxelY + padY);
                double px = pcoord(voxelY, d, mn.y, F[ORC_S_P_GEN]), py = pcoord(voxelZ, d, mn.z, F[ORC_S_P_GEN]);
                for (uint w = tileStart[tl]; w < tileStart[tl + 1]; ++w) {
                    uint tri = wqTri[order[w]];
                    d3 v[3];
                    fetchD(V, I, tri, v);
                    d3 U{v[0].x - v[2].x, v[0].y - v[2].y, v[0].z - v[2].z};
                    d3 W2{v[1].x - v[0].x, v[1].y - v[0].y, v[1].z - v[0].z};
                    // cross(U, V), include/helper_math.h:1998-2004
                    d3 n{diff2(U.y, W2.z, U.z, W2.y, F[ORC_S_CR_GEN]), diff2(U.z, W2.x, U.x, W2.z, F[ORC_S_CR_GEN]),
                         diff2(U.x, W2.y, U.y, W2.x, F[ORC_S_CR_GEN])};
                    d2 en[3];
                    double dist[3];
                    for (int i = 0; i < 3; i++) {
                        const d3& a = v[i];
                        const d3& b = v[(i + 1) % 3];
                        if (n.x > 0.0) en[i] = d2{a.z - b.z, b.y - a.y};
                        else en[i] = d2{b.z - a.z, a.y - b.y};
                        dist[i] = -sum2(en[i].x, a.y, en[i].y, a.z, F[ORC_S_D_GEN]);
                    }
                    uint pass = 0;
                    for (int i = 0; i < 3; i++) {
                        double r = sum2p1(en[i].x, px, en[i].y, py, dist[i], (F[ORC_S_E_GEN] >> (2 * i)) & 3);
                        if (en[i].x > 0.0 || (en[i].x == 0.0 && en[i].y < 0.0)) r += DBL_MIN;
                        if (r > 0.0) pass++;
                    }
                    if (pass != 3) continue;
                    d3 A{v[0].x - mn.x, v[0].y - px, v[0].z - py};
                    double B = sum3(A.x, n.x, A.y, n.y, A.z, n.z, F[ORC_S_B_GEN]);
                    double pxx = B / n.x;
                    pxx = pxx < 0.0 ? 0.0 : pxx;
                    uint voxelX = cvt_d2u(std::ceil(pxx / d)) + 1u;
                    uint ix = voxelX >> 5;
                    if (ix >= endIx) {
                        // beyond this x subspace: ignored
                    } else if (ix < minIx) {
                        bitmask ^= 0xFFFFFFFFu;
                        any = true;
                    } else {
                        voxels[rowBase + ix] ^= (0xFFFFFFFFu >> (voxelX % 32u));
                        uint sh = ix % intsPerDim + 1;
                        uint32_t bm = ix < lastIX ? (sh >= 32 ? 0u : (0xFFFFFFFFu >> sh)) : 0u;
                        bitmask ^= bm;
                        any = true;
                    }
                }
                if (!any) continue;
                uint start = rowBase + minIx;  // == currentSegment - currentSegment % intsPerDim
                for (uint i = 0; i < intsPerDim; i++)
                    if (bitmask & (1u << (31 - i))) voxels[start + i] ^= 0xFFFFFFFFu;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Surface voxelization, src/voxelizer.cu:2358-2989, 3040-4201.
struct SurfHit { uint idx; uint key; uint tri; };

struct TriClass { uint code; };

static inline f3 sub3(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }

static inline f3 crossF(f3 a, f3 b, int mode) {
    return f3{diff2(a.y, b.z, a.z, b.y, mode), diff2(a.z, b.x, a.x, b.z, mode), diff2(a.x, b.y, a.y, b.x, mode)};
}
static inline float dot3F(f3 a, f3 b, int mode) { return sum3(a.x, b.x, a.y, b.y, a.z, b.z, mode); }

static inline void fetchF(const float* V, const uint* I, uint t, f3* v) {
    for (int k = 0; k < 3; ++k) {
        uint a = I[3*t + k];
        v[k] = f3{V[3*a], V[3*a+1], V[3*a+2]};
    }
}

// getTriangleBounds (float3), src/voxelizer.cu:2366-2390
static inline void triBoundsF(const f3* v, f3& mn, f3& mx) {
    mn = v[0]; mx = v[0];
    for (int i = 1; i < 3; i++) {
        if (v[i].x < mn.x) mn.x = v[i].x;
        if (v[i].y < mn.y) mn.y = v[i].y;
        if (v[i].z < mn.z) mn.z = v[i].z;
        if (v[i].x > mx.x) mx.x = v[i].x;
        if (v[i].y > mx.y) mx.y = v[i].y;
        if (v[i].z > mx.z) mx.z = v[i].z;
    }
}
// getVoxelBoundsHalf, src/voxelizer.cu:2471-2492
static inline Bounds<i3> voxBoundsHalf(f3 bmin, f3 bmax, f3 m, float d) {
    Bounds<i3> b;
    b.min = i3{cvt_f2i(std::ceil((bmin.x - m.x) / d - 0.5f)), cvt_f2i(std::ceil((bmin.y - m.y) / d - 0.5f)),
               cvt_f2i(std::ceil((bmin.z - m.z) / d - 0.5f))};
    b.max = i3{cvt_f2i(std::floor((bmax.x - m.x) / d + 0.5f)), cvt_f2i(std::floor((bmax.y - m.y) / d + 0.5f)),
               cvt_f2i(std::floor((bmax.z - m.z) / d + 0.5f))};
    return b;
}
static inline int vcMin(float v, float m, float d) { return cvt_f2i(std::ceil((v - m) / d - 0.5f)); }
static inline int vcMax(float v, float m, float d) { return cvt_f2i(std::floor((v - m) / d + 0.5f)); }

// classifyTriangles / analyzeBoundingBox / encodeTriangleType, src/voxelizer.cu:3040-3221
static uint classify(const f3* v, f3 m, float d, const Fma& F) {
    f3 n = crossF(sub3(v[0], v[2]), sub3(v[1], v[0]), F[ORC_S_CRF_CLS]);
    if (!(n.x != 0.0f || n.y != 0.0f || n.z != 0.0f)) return 0u;
    f3 bmin, bmax;
    triBoundsF(v, bmin, bmax);
    Bounds<i3> vb = voxBoundsHalf(bmin, bmax, m, d);
    i3 df{vb.max.x - vb.min.x, vb.max.y - vb.min.y, vb.max.z - vb.min.z};
    uint bb, axis, cols;
    if (df.x == 0) {
        if (df.y == 0) {
            if (df.z == 0) { bb = 1; axis = 0; cols = 1; }
            else { bb = 1; axis = 2; cols = (uint)df.z; }
        } else if (df.z == 0) { bb = 1; axis = 1; cols = (uint)df.y; }
        else { bb = 2; axis = 0; cols = (uint)(df.y * df.z); }
    } else if (df.y == 0) {
        if (df.z == 0) { bb = 1; axis = 0; cols = (uint)df.x; }
        else { bb = 2; axis = 1; cols = (uint)(df.x * df.z); }
    } else if (df.z == 0) { bb = 2; axis = 2; cols = (uint)(df.x * df.y); }
    else {
        bb = 3;
        // determineDominantAxis, src/voxelizer.cu:2526-2546
        float ax = std::fabs(n.x), ay = std::fabs(n.y), az = std::fabs(n.z);
        if (ax > ay && ax > az) axis = 0;
        else if (ay > ax && ay > az) axis = 1;
        else axis = 2;
        cols = axis == 0 ? (uint)(df.y * df.z) : axis == 1 ? (uint)(df.x * df.z) : (uint)(df.x * df.y);
    }
    return cols | (axis << 28) | (bb << 30);
}

struct Overlap { f2 ne[3]; float de[3]; };

// setupYZ/ZX/XYOverlapTest, src/voxelizer.cu:2675-2757.  `axis` selects
// which pair of coordinates (a, b) the edge functions live in:
// 0: (y, z) oriented by n.x; 1: (z, x) by n.y; 2: (x, y) by n.z.
static inline Overlap setupOverlap(const f3* t, f3 n, float d, int axis, int deMode) {
    Overlap o;
    for (int i = 0; i < 3; i++) {
        const f3& p = t[i];
        const f3& q = t[(i + 1) % 3];
        float pa, pb, qa, qb, nn;
        if (axis == 0) { pa = p.y; pb = p.z; qa = q.y; qb = q.z; nn = n.x; }
        else if (axis == 1) { pa = p.z; pb = p.x; qa = q.z; qb = q.x; nn = n.y; }
        else { pa = p.x; pb = p.y; qa = q.x; qb = q.y; nn = n.z; }
        if (nn >= 0.0f) o.ne[i] = f2{pb - qb, qa - pa};
        else o.ne[i] = f2{qb - pb, pa - qa};
        float s = sum2(o.ne[i].x, pa, o.ne[i].y, pb, (deMode >> (2 * i)) & 3);
        o.de[i] = (-s + std::fmax(0.0f, d * o.ne[i].x)) + std::fmax(0.0f, d * o.ne[i].y);
    }
    return o;
}
// overlapTestYZ/ZX/XY, src/voxelizer.cu:2890-2942
static inline bool overlapTest(const Overlap& o, float a, float b, int mode) {
    bool r = true;
    for (int i = 0; i < 3; i++) r &= sum2p1(o.ne[i].x, a, o.ne[i].y, b, o.de[i], (mode >> (2 * i)) & 3) >= 0.0f;
    return r;
}
// getSingleVoxelBoundsComponent, src/voxelizer.cu:2575-2586
static inline float vbComp(int c, float m, float d, int mode) {
    float a = float(c) - 0.5f;
    return mode ? std::fma(a, d, m) : m + a * d;
}

struct SurfaceCtx {
    const float* V; const uint* I; const uchar* M;
    f3 m; float d;
    u3 res;          // the allocation: extResolution plus the padding rows
    bool fcc; int gridType;
    const Fma* F;
    int padY, padZ;  // adjustment (1, left ? 0 : 1, down ? 0 : 1), src/voxelizer.cu:3362-3368
};

static inline uint nodeIndex(const SurfaceCtx& c, int x, int y, int z) {
    if (c.fcc) {
        uint l = 2 * c.res.x, a = l * c.res.y;
        if (c.gridType == 1) return a * 2 * uint(z) + l * uint(y) + 2 * uint(x);
        if (c.gridType == 2) return a * 2 * uint(z) + l * uint(y) + 2 * uint(x) + 1;
        if (c.gridType == 3) return a * (2 * uint(z) + 1) + l * uint(y) + 2 * uint(x);
        return a * (2 * uint(z) + 1) + l * uint(y) + 2 * uint(x) + 1;
    }
    return c.res.x * c.res.y * uint(z) + c.res.x * uint(y) + uint(x);
}

// adjustVoxelRange, src/voxelizer.cu:3963-3993
static inline bool adjustRange(Bounds<i3>& b, Bounds<u3> sub) {
    i3 smin{(int)sub.min.x, (int)sub.min.y, (int)sub.min.z};
    i3 smax{(int)sub.max.x - 1, (int)sub.max.y - 1, (int)sub.max.z - 1};
    if (smin.x > b.max.x || smin.y > b.max.y || smin.z > b.max.z) return false;
    if (b.min.x > smax.x || b.min.y > smax.y || b.min.z > smax.z) return false;
    b.min = i3{std::max(b.min.x, smin.x), std::max(b.min.y, smin.y), std::max(b.min.z, smin.z)};
    b.max = i3{std::min(b.max.x, smax.x), std::min(b.max.y, smax.y), std::min(b.max.z, smax.z)};
    return true;
}

// determineDepthRangeX/Y/Z, src/voxelizer.cu:3994-4119 with intersectWithPlane*.
static inline i2 depthRange(const f3* t, f3 p, f3 n, f3 m, float d, int axis, int dt) {
    f3 pmin, pmax;
    float a, b;
    if (axis == 0) {
        bool ny = n.y > 0.0f, nz = n.z > 0.0f;
        pmin = f3{0.0f, p.y + float(ny) * d, p.z + float(nz) * d};
        pmax = f3{0.0f, p.y + float(!ny) * d, p.z + float(!nz) * d};
        a = dot3F(sub3(t[0], pmin), n, dt) / n.x;
        b = dot3F(sub3(t[0], pmax), n, dt) / n.x;
    } else if (axis == 1) {
        bool nx = n.x > 0.0f, nz = n.z > 0.0f;
        pmin = f3{p.x + float(nx) * d, 0.0f, p.z + float(nz) * d};
        pmax = f3{p.x + float(!nx) * d, 0.0f, p.z + float(!nz) * d};
        a = dot3F(sub3(t[0], pmin), n, dt) / n.y;
        b = dot3F(sub3(t[0], pmax), n, dt) / n.y;
    } else {
        bool nx = n.x > 0.0f, ny = n.y > 0.0f;
        pmin = f3{p.x + float(nx) * d, p.y + float(ny) * d, 0.0f};
        pmax = f3{p.x + float(!nx) * d, p.y + float(!ny) * d, 0.0f};
        a = dot3F(sub3(t[0], pmin), n, dt) / n.z;
        b = dot3F(sub3(t[0], pmax), n, dt) / n.z;
    }
    if (a > b) std::swap(a, b);  // boundsCheck, src/voxelizer.cu:4165-4177
    float mm = axis == 0 ? m.x : axis == 1 ? m.y : m.z;
    return i2{vcMin(a, mm, d), vcMax(b, mm, d)};
}

// Form of the edge functions at iteration `pos` of a loop of `n` iterations
// that the reference build unrolled `unr` times with a prolog: the prolog
// runs the first n mod unr iterations.
static inline int loopForm(int pos, int n, int unr, int mainMode, int proMode) {
    if (unr <= 1) return mainMode;
    return pos < n % unr ? proMode : mainMode;
}

// process1D/2D/3DTriangles for one triangle inside one material subspace,
// src/voxelizer.cu:3306-3955.  Calls hit(nodeIndex) for every processVoxel.
template <class Hit>
static void surfaceTriangle(const SurfaceCtx& c, uint tri, uint code, Bounds<u3> sub, Hit hit) {
    const Fma& F = *c.F;
    uint bb = code >> 30;
    if (bb == 0) return;
    f3 t[3];
    fetchF(c.V, c.I, tri, t);
    f3 bmin, bmax;
    triBoundsF(t, bmin, bmax);
    Bounds<i3> vb = voxBoundsHalf(bmin, bmax, c.m, c.d);
    if (!adjustRange(vb, sub)) return;
    uint axis = (code >> 28) & 3u;
    const int ax = 1, ay = c.padY, az = c.padZ;  // padding adjustment
    if (bb == 1) {
        vb.min = i3{vb.min.x + ax, vb.min.y + ay, vb.min.z + az};
        vb.max = i3{vb.max.x + ax, vb.max.y + ay, vb.max.z + az};
        if (axis == 0) for (int i = vb.min.x; i <= vb.max.x; i++) hit(nodeIndex(c, i, vb.min.y, vb.min.z));
        else if (axis == 1) for (int j = vb.min.y; j <= vb.max.y; j++) hit(nodeIndex(c, vb.min.x, j, vb.min.z));
        else for (int k = vb.min.z; k <= vb.max.z; k++) hit(nodeIndex(c, vb.min.x, vb.min.y, k));
        return;
    }
    if (bb == 2) {
        f3 n = crossF(sub3(t[0], t[2]), sub3(t[1], t[0]), F[ORC_S_CRF_2D]);
        const int pc = F[ORC_S_PC_2D];
        // The inner loop (z for the x and y axes, y for the z axis) runs its
        // first (trip count mod UNR_2D) iterations in the prolog forms.
        const int unr = F[ORC_S_UNR_2D];
        auto form = [&](int inner, int lo, int hi, int mainMode, int proMode) {
            return loopForm(inner - lo, hi - lo + 1, unr, mainMode, proMode);
        };
        if (axis == 0) {
            Overlap o = setupOverlap(t, n, c.d, 0, F[ORC_S_DE_2D_YZ]);
            for (int j = vb.min.y; j <= vb.max.y; j++)
                for (int k = vb.min.z; k <= vb.max.z; k++)
                    if (overlapTest(o, vbComp(j, c.m.y, c.d, pc), vbComp(k, c.m.z, c.d, pc),
                                    form(k, vb.min.z, vb.max.z, F[ORC_S_OT_2D_YZ], F[ORC_S_OT_2DP_YZ])))
                        hit(nodeIndex(c, vb.min.x + ax, j + ay, k + az));
        } else if (axis == 1) {
            Overlap o = setupOverlap(t, n, c.d, 1, F[ORC_S_DE_2D_ZX]);
            for (int i = vb.min.x; i <= vb.max.x; i++)
                for (int k = vb.min.z; k <= vb.max.z; k++)
                    if (overlapTest(o, vbComp(k, c.m.z, c.d, pc), vbComp(i, c.m.x, c.d, pc),
                                    form(k, vb.min.z, vb.max.z, F[ORC_S_OT_2D_ZX], F[ORC_S_OT_2DP_ZX])))
                        hit(nodeIndex(c, i + ax, vb.min.y + ay, k + az));
        } else {
            Overlap o = setupOverlap(t, n, c.d, 2, F[ORC_S_DE_2D_XY]);
            for (int i = vb.min.x; i <= vb.max.x; i++)
                for (int j = vb.min.y; j <= vb.max.y; j++)
                    if (overlapTest(o, vbComp(i, c.m.x, c.d, pc), vbComp(j, c.m.y, c.d, pc),
                                    form(j, vb.min.y, vb.max.y, F[ORC_S_OT_2D_XY], F[ORC_S_OT_2DP_XY])))
                        hit(nodeIndex(c, i + ax, j + ay, vb.min.z + az));
        }
        return;
    }
    f3 n = crossF(sub3(t[0], t[2]), sub3(t[1], t[0]), F[ORC_S_CRF_3D]);
    Overlap o0 = setupOverlap(t, n, c.d, 0, F[ORC_S_DE_3D_YZ]);
    Overlap o1 = setupOverlap(t, n, c.d, 1, F[ORC_S_DE_3D_ZX]);
    Overlap o2 = setupOverlap(t, n, c.d, 2, F[ORC_S_DE_3D_XY]);
    const int pc = F[ORC_S_PC_3D], pl = F[ORC_S_PC_3DL];
    const int ul = F[ORC_S_UNR_3DL];
    if (axis == 0) {
        for (int j = vb.min.y; j <= vb.max.y; j++)
            for (int k = vb.min.z; k <= vb.max.z; k++) {
                f3 p{0.0f, vbComp(j, c.m.y, c.d, pc), vbComp(k, c.m.z, c.d, pc)};
                if (!overlapTest(o0, p.y, p.z, F[ORC_S_OT_3D_YZ])) continue;
                i2 r = depthRange(t, p, n, c.m, c.d, 0, F[ORC_S_DT_3DX]);
                if (r.x > vb.max.x || r.y < vb.min.x) continue;
                r.x = r.x < vb.min.x ? vb.min.x : r.x;
                r.y = r.y > vb.max.x ? vb.max.x : r.y;
                if (r.x == r.y) { hit(nodeIndex(c, r.x + ax, j + ay, k + az)); continue; }
                for (int i = r.x; i <= r.y; i++) {
                    p.x = vbComp(i, c.m.x, c.d, pl);
                    const int q = i - r.x, nl = r.y - r.x + 1;
                    if (overlapTest(o1, p.z, p.x, loopForm(q, nl, ul, F[ORC_S_OT_3DX_ZX], F[ORC_S_OT_3DXP_ZX])) &&
                        overlapTest(o2, p.x, p.y, loopForm(q, nl, ul, F[ORC_S_OT_3DX_XY], F[ORC_S_OT_3DXP_XY])))
                        hit(nodeIndex(c, i + ax, j + ay, k + az));
                }
            }
    } else if (axis == 1) {
        for (int k = vb.min.z; k <= vb.max.z; k++)
            for (int i = vb.min.x; i <= vb.max.x; i++) {
                f3 p{vbComp(i, c.m.x, c.d, pc), 0.0f, vbComp(k, c.m.z, c.d, pc)};
                if (!overlapTest(o1, p.z, p.x, F[ORC_S_OT_3D_ZX])) continue;
                i2 r = depthRange(t, p, n, c.m, c.d, 1, F[ORC_S_DT_3DY]);
                if (r.x > vb.max.y || r.y < vb.min.y) continue;
                r.x = r.x < vb.min.y ? vb.min.y : r.x;
                r.y = r.y > vb.max.y ? vb.max.y : r.y;
                if (r.x == r.y) { hit(nodeIndex(c, i + ax, r.x + ay, k + az)); continue; }
                for (int j = r.x; j <= r.y; j++) {
                    p.y = vbComp(j, c.m.y, c.d, pl);
                    const int q = j - r.x, nl = r.y - r.x + 1;
                    if (overlapTest(o2, p.x, p.y, loopForm(q, nl, ul, F[ORC_S_OT_3DY_XY], F[ORC_S_OT_3DYP_XY])) &&
                        overlapTest(o0, p.y, p.z, loopForm(q, nl, ul, F[ORC_S_OT_3DY_YZ], F[ORC_S_OT_3DYP_YZ])))
                        hit(nodeIndex(c, i + ax, j + ay, k + az));
                }
            }
    } else {
        for (int i = vb.min.x; i <= vb.max.x; i++)
            for (int j = vb.min.y; j <= vb.max.y; j++) {
                f3 p{vbComp(i, c.m.x, c.d, pc), vbComp(j, c.m.y, c.d, pc), 0.0f};
                if (!overlapTest(o2, p.x, p.y, F[ORC_S_OT_3D_XY])) continue;
                i2 r = depthRange(t, p, n, c.m, c.d, 2, F[ORC_S_DT_3DZ]);
                if (r.x > vb.max.z || r.y < vb.min.z) continue;
                r.x = r.x < vb.min.z ? vb.min.z : r.x;
                r.y = r.y > vb.max.z ? vb.max.z : r.y;
                if (r.x == r.y) { hit(nodeIndex(c, i + ax, j + ay, r.x + az)); continue; }
                for (int k = r.x; k <= r.y; k++) {
                    p.z = vbComp(k, c.m.z, c.d, pl);
                    const int q = k - r.x, nl = r.y - r.x + 1;
                    if (overlapTest(o0, p.y, p.z, loopForm(q, nl, ul, F[ORC_S_OT_3DZ_YZ], F[ORC_S_OT_3DZP_YZ])) &&
                        overlapTest(o1, p.z, p.x, loopForm(q, nl, ul, F[ORC_S_OT_3DZ_ZX], F[ORC_S_OT_3DZP_ZX])))
                        hit(nodeIndex(c, i + ax, j + ay, k + az));
                }
            }
    }
}

// ---------------------------------------------------------------------------
// PartialNode volume ratio: processVoxel<PartialNode> and
// calculateVoxelPlaneIntersectionVolume with its helpers,
// src/voxelizer.cu:2996-3033, 4220-4807 (a Salama-Kolb style plane-box cut).
// The reference computes, in FP32, the volume of the part of a voxel behind
// the triangle's plane and stores |1 - volume / d^3|.  Facts of the
// reference that the result depends on, restated here:
//  * the voxel is the one centred at minCorner + d * (node coordinates), the
//    node coordinates including the one-voxel padding, i.e. one voxel further
//    along x, y and z than the voxel that passed the overlap test;
//  * the plane normal is the class kernel's unnormalised cross product
//    (zero for 1D-class triangles, which makes the ratio NaN);
//  * |n.x|, |n.y| or |n.z| exactly 1 takes the axis-parallel shortcut;
//  * when the plane misses the voxel the reference reads an unset array
//    element for the cut polygon's pyramid; that pyramid counts as empty.
// Operation order follows the reference; the reference build contracts some
// multiply-adds and its normalize() uses rsqrtf, so this restatement (plain
// IEEE operations, 1 / sqrtf) agrees with it to a tolerance, not bit for bit.
namespace ratio {

static inline f3 add(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline f3 mul(float s, f3 a) { return f3{s * a.x, s * a.y, s * a.z}; }
static inline float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline f3 rotX(f3 v, float s, float c) { return f3{v.x, v.y * c - v.z * s, v.y * s + v.z * c}; }
static inline f3 rotY(f3 v, float s, float c) { return f3{v.x * c + v.z * s, v.y, v.z * c - v.x * s}; }

struct Poly { f3 p[6]; int n = 0; void push(f3 v) { if (n < 6) p[n++] = v; } };

// Pyramid over `base` (rotated into a plane z = const) with apex `top`:
// surveyor's formula for the base area.
static float pyramid(const Poly& b, f3 top) {
    float area = 0.0f;
    for (int i = 0; i < b.n; i++) {
        f3 u = b.p[i], w = b.p[(i + 1) % b.n];
        area += 0.5f * (u.x * w.y - w.x * u.y);
    }
    float base0z = b.n ? b.p[0].z : 0.0f;
    return std::fabs((1.0f / 3.0f) * area * (top.z - base0z));
}

// Rotates `poly` (and the apex) so that `rn` becomes the z axis: about x
// when rn.y != 0, then about y when the (rotated) rn.x != 0.
static float rotatedPyramid(Poly poly, f3 rn, f3 apex) {
    f3 top = apex;
    if (rn.y != 0.0f) {
        float pl = std::sqrt(rn.y * rn.y + rn.z * rn.z);
        float sn = rn.y / pl, cs = rn.z / pl;
        top = rotX(top, sn, cs);
        for (int i = 0; i < poly.n; i++) poly.p[i] = rotX(poly.p[i], sn, cs);
        rn = rotX(rn, sn, cs);
    }
    if (rn.x != 0.0f) {
        float pl = std::sqrt(rn.z * rn.z + rn.x * rn.x);
        float sn = -rn.x / pl, cs = rn.z / pl;
        top = rotY(top, sn, cs);
        for (int i = 0; i < poly.n; i++) poly.p[i] = rotY(poly.p[i], sn, cs);
    }
    return pyramid(poly, top);
}

// `unstable` is set when an edge is (nearly) parallel to the plane (its
// parameter is then 0 / 0, an infinity or a huge quotient) or when the plane
// passes (nearly) through a voxel corner (a parameter near 0 or 1): which
// side of [0, 1] the parameter falls on then depends on the last bits of the
// products, so arithmetic with and without multiply-add contraction can take
// different branches.
static float cutVolume(const f3* t, f3 n, int x, int y, int z, f3 m, float d, bool& unstable) {
    f3 vc = add(m, mul(d, f3{float(x), float(y), float(z)}));
    if (std::fabs(n.x) == 1.0f) return (d * d) * ((d / 2.0f) + t[0].x - vc.x);
    if (std::fabs(n.y) == 1.0f) return (d * d) * ((d / 2.0f) + t[0].y - vc.y);
    if (std::fabs(n.z) == 1.0f) return (d * d) * ((d / 2.0f) + t[0].z - vc.z);
    const bool sx = n.x > 0.0f, sy = n.y > 0.0f, sz = n.z > 0.0f;
    // Steps along x, y, z away from the corner nearest the plane (the corner
    // on the normal's side); the y and z steps trade places when an odd
    // number of normal components are positive, keeping the frame
    // right-handed.
    const float ex = sx ? -d : d, ey = sy ? -d : d, ez = sz ? -d : d;
    const bool even = ((int)sx + (int)sy + (int)sz) % 2 == 0;
    const f3 dx{ex, 0.0f, 0.0f};
    const f3 dy = even ? f3{0.0f, ey, 0.0f} : f3{0.0f, 0.0f, ez};
    const f3 dz = even ? f3{0.0f, 0.0f, ez} : f3{0.0f, ey, 0.0f};
    const float h = d / 2.0f;
    f3 c[8];
    c[0] = add(vc, f3{sx ? h : -h, sy ? h : -h, sz ? h : -h});
    c[1] = add(c[0], dx);
    c[2] = add(c[0], dy);
    c[3] = add(c[0], dz);
    c[4] = add(c[1], dz);
    c[5] = add(c[2], dx);
    c[6] = add(c[3], dy);
    c[7] = add(c[4], dy);
    // Walk three corner paths 0 -> A -> B -> 7 with a side edge A -> S; path
    // k builds face k and closes the previous face where it turns at B.
    static const int A[3] = {1, 2, 3}, B[3] = {4, 5, 6}, S[3] = {5, 6, 4};
    const float nscale = (std::fabs(n.x) + std::fabs(n.y) + std::fabs(n.z)) * d;
    auto along = [&](f3 p, f3 q) {
        const float den = dot(n, f3{q.x - p.x, q.y - p.y, q.z - p.z});
        if (!(std::fabs(den) > 1e-5f * nscale)) unstable = true;
        const float tt = dot(n, f3{t[0].x - p.x, t[0].y - p.y, t[0].z - p.z}) / den;
        if (std::fabs(tt) < 1e-4f || std::fabs(tt - 1.0f) < 1e-4f) unstable = true;
        return tt;
    };
    auto point = [&](f3 p, f3 q, float tt) { return add(p, mul(tt, f3{q.x - p.x, q.y - p.y, q.z - p.z})); };
    // A NaN tt (edge in the plane) is neither: the first two edges of a path
    // are tested for "outside", the others for "inside", as in the reference.
    auto inside = [](float tt) { return tt >= 0.0f && tt <= 1.0f; };
    auto outside = [](float tt) { return tt < 0.0f || tt > 1.0f; };
    Poly cut, face[3];
    for (int k = 0; k < 3; k++) {
        Poly& own = face[k];
        Poly& prev = face[(k + 2) % 3];
        const f3 a = c[A[k]], b = c[B[k]];
        float tt = along(c[0], a);
        if (outside(tt)) {
            own.push(a);
            tt = along(a, b);
            if (outside(tt)) {
                tt = along(b, c[7]);
                if (inside(tt)) {
                    f3 ip = point(b, c[7], tt);
                    own.push(b); own.push(ip);
                    prev.push(ip); prev.push(b);
                    cut.push(ip);
                } else {
                    own.push(b);
                    prev.push(b);
                }
            } else {
                f3 ip = point(a, b, tt);
                own.push(ip);
                cut.push(ip);
            }
        } else {
            cut.push(point(c[0], a, tt));
        }
        tt = along(a, c[S[k]]);
        if (inside(tt)) {
            f3 ip = point(a, c[S[k]], tt);
            own.push(ip);
            cut.push(ip);
        }
    }
    float vol = rotatedPyramid(cut, n, c[0]);
    for (int k = 0; k < 3; k++) {
        const Poly& f = face[k];
        if (f.n <= 2) continue;
        f3 e0{f.p[0].x - f.p[2].x, f.p[0].y - f.p[2].y, f.p[0].z - f.p[2].z};
        f3 e1{f.p[1].x - f.p[0].x, f.p[1].y - f.p[0].y, f.p[1].z - f.p[0].z};
        f3 fn{e0.y * e1.z - e0.z * e1.y, e0.z * e1.x - e0.x * e1.z, e0.x * e1.y - e0.y * e1.x};
        fn = mul(1.0f / std::sqrt(dot(fn, fn)), fn);
        vol += rotatedPyramid(f, fn, c[0]);
    }
    return vol;
}

// The stored ratio for surface node (x, y, z) written by triangle `tri` of
// class `cls` (1, 2, 3).
static float nodeRatio(const SurfaceCtx& cx, uint tri, uint cls, int x, int y, int z, bool& unstable) {
    f3 t[3];
    fetchF(cx.V, cx.I, tri, t);
    f3 n{0.0f, 0.0f, 0.0f};
    if (cls >= 2)
        n = crossF(sub3(t[0], t[2]), sub3(t[1], t[0]), (*cx.F)[cls == 2 ? ORC_S_CRF_2D : ORC_S_CRF_3D]);
    else
        return std::numeric_limits<float>::quiet_NaN();   // zero normal: every edge parameter is 0 / 0
    float vol = cutVolume(t, n, x, y, z, cx.m, cx.d, unstable);
    return std::fabs(1.0f - vol / (cx.d * cx.d * cx.d));
}

}  // namespace ratio

// Deterministic material resolution.  The reference stores Node(1, mat)
// with plain racing stores (src/voxelizer.cu:2988) from the 1D, 2D and 3D
// kernels in that order, so a node ends with the material of *some*
// triangle of the highest class that touched it.  This restatement (and the
// CUDA path) picks the largest (class, material) key among those triangles.
// For PartialNode the stored ratio comes from one racing triangle as well;
// here it is the largest (class, material, triangle index), and `topHits`
// counts the triangles of the winning class (more than one: the reference's
// ratio is not determined).
struct SurfaceRec { uint key; uint minMatTop; uint tri; uint topHits; };

static void surfacePass(const SurfaceCtx& c, uint nT, const std::vector<Bounds<u3> >& splits,
                        std::unordered_map<uint, SurfaceRec>& rec) {
    const Fma& F = *c.F;
    std::vector<uint> codes(nT);
#pragma omp parallel for schedule(static)
    for (long long tt = 0; tt < (long long)nT; ++tt) {
        f3 t[3];
        fetchF(c.V, c.I, (uint)tt, t);
        codes[tt] = classify(t, c.m, c.d, F);
    }
    // thrust::sort_by_key(triTypes, tris) (src/voxelizer.cu:553-586): the
    // processing order; results do not depend on it under the max rule.
    std::vector<uint> order(nT);
    for (uint i = 0; i < nT; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint a, uint b) { return codes[a] < codes[b]; });
#ifdef _OPENMP
    int nth = omp_get_max_threads();
#else
    int nth = 1;
#endif
    for (const Bounds<u3>& sub : splits) {
        std::vector<std::vector<SurfHit> > local(nth);
#pragma omp parallel
        {
#ifdef _OPENMP
            int tid = omp_get_thread_num();
#else
            int tid = 0;
#endif
#pragma omp for schedule(dynamic, 64)
            for (long long k = 0; k < (long long)nT; ++k) {
                uint tri = order[k];
                uint code = codes[tri];
                uint cls = code >> 30;
                uint key = (cls << 8) | c.M[tri];
                surfaceTriangle(c, tri, code, sub, [&](uint idx) { local[tid].push_back(SurfHit{idx, key, tri}); });
            }
        }
        for (auto& l : local)
            for (auto& h : l) {
                auto it = rec.find(h.idx);
                if (it == rec.end()) rec[h.idx] = SurfaceRec{h.key, h.key & 255u, h.tri, 1u};
                else {
                    SurfaceRec& r = it->second;
                    uint cls = h.key >> 8, rc = r.key >> 8;
                    if (cls > rc) r = SurfaceRec{h.key, h.key & 255u, h.tri, 1u};
                    else if (cls == rc) {
                        if (h.key > r.key || (h.key == r.key && h.tri > r.tri)) { r.key = h.key; r.tri = h.tri; }
                        r.minMatTop = std::min(r.minMatTop, h.key & 255u);
                        r.topHits++;
                    }
                }
            }
    }
}

// ---------------------------------------------------------------------------
template <class N>
static int run(const orc_params* p, const Plan& pl, const float* V, uint nV, const uint* I, uint nT,
               const uchar* M, void* out, uint8_t* conflict, orc_info* info, uint32_t* winTri = nullptr,
               uint8_t* winCls = nullptr) {
    typedef Tr<N> T;
    const Fma F(p->fma_sites);
    const bool fcc = T::fcc;
    u3 alloc = pl.alloc;
    const uint nInts = (alloc.x * alloc.y * alloc.z) >> 5;
    std::vector<uint32_t> voxels(nInts, 0u);
    Bounds<u3> ext{u3{0, 0, 0}, pl.ext};
    Bounds<u3> allocPart{u3{0, 0, 0}, alloc};
    const u2 vs{p->vox_split[1], p->vox_split[2]};
    std::vector<Bounds<u2> > extYz = splitYZ(vs, ext);
    std::vector<Bounds<u2> > allocYz = splitYZ(vs, allocPart);
    // Slices along x: nodes are built on the turned grid and turned back
    // before the boundary ids (src/host_side.cpp:1144-1206).
    const bool turn = p->rotate_x && p->node_output;
    const bool mats = p->materials && p->node_output;
    if (!p->node_output) {
        for (auto& s : extYz)
            performVoxelization(V, I, nT, pl.mnExt, pl.d, ext, s, pl.xRes, pl.xSplits, voxels.data(), alloc, F, pl.padY,
                                pl.padZ);
        memcpy(out, voxels.data(), sizeof(uint32_t) * (size_t)nInts);
        return 0;
    }
    const size_t nNodes = fcc ? (size_t)(2 * alloc.x) * alloc.y * (2 * alloc.z) : (size_t)alloc.x * alloc.y * alloc.z;
    if (conflict) memset(conflict, 0, nNodes);
    std::vector<N> turned(turn ? nNodes : 0);
    std::vector<uint8_t> turnedConf(turn && conflict ? nNodes : 0);
    uint8_t* const outConflict = conflict;
    if (turn && conflict) conflict = turnedConf.data();
    N* nodes = turn ? turned.data() : (N*)out;
    N zero = T::make(0, 0);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)nNodes; ++i) nodes[i] = zero;
    std::vector<Bounds<u3> > matSplits = split3(u3{p->mat_split[0], p->mat_split[1], p->mat_split[2]}, ext);
    std::unordered_map<uint, SurfaceRec> rec;
    if (!fcc) {
        for (auto& s : extYz)
            performVoxelization(V, I, nT, pl.mnExt, pl.d, ext, s, pl.xRes, pl.xSplits, voxels.data(), alloc, F, pl.padY,
                                pl.padZ);
        // constructNodeList2, src/voxelizer.cu:1626-1681 (all alloc splits together)
#pragma omp parallel for schedule(static)
        for (long long w = 0; w < (long long)nInts; ++w) {
            uint32_t word = voxels[w];
            for (uint b = 0; b < 32; ++b) {
                uint bit = (word >> (31 - b)) & 1u;
                N nd = T::make(bit, 0);
                T::setR(nd, float(bit > 0));
                nodes[(size_t)w * 32 + b] = nd;
            }
        }
        if (mats) {
            SurfaceCtx c{V, I, M, f3{float(pl.mnExt.x), float(pl.mnExt.y), float(pl.mnExt.z)}, float(pl.d), alloc,
                         false, 1, &F, (int)pl.padY, (int)pl.padZ};
            surfacePass(c, nT, matSplits, rec);
        }
    } else {
        // Sub-lattice g goes to FCC slot g (1 + (x & 1) + 2 (z & 1)).  For a
        // turned mesh the reference shifts grid g by the z-swapped pattern and
        // writes it to slot (g + 1) % 4 + 1 (src/host_side.cpp:1438-1476),
        // i.e. slot g gets its usual shift with the y part toggled.
        const double h = pl.d / 2.0;
        auto shift = [&](int g) {
            d3 sh = g == 1 ? d3{0, 0, 0} : g == 2 ? d3{h, h, 0} : g == 3 ? d3{0, h, h} : d3{h, 0, h};
            if (turn) sh.y = sh.y == 0.0 ? h : 0.0;
            return sh;
        };
        for (int g = 1; g <= 4; ++g) {
            d3 sh = shift(g);
            d3 m{pl.mnExt.x + sh.x, pl.mnExt.y + sh.y, pl.mnExt.z + sh.z};
            std::fill(voxels.begin(), voxels.end(), 0u);
            for (auto& s : extYz)
                performVoxelization(V, I, nT, m, pl.d, ext, s, pl.xRes, pl.xSplits, voxels.data(), alloc, F, pl.padY,
                                    pl.padZ);
            // convertToFCCGrid, src/voxelizer.cu:1710-1776
            const uint rx = alloc.x, ry = alloc.y;
#pragma omp parallel for schedule(static)
            for (long long w = 0; w < (long long)nInts; ++w) {
                uint ipx = rx >> 5, ipy = ry * ipx;
                uint y = (uint)(w % ipy) / ipx, z = (uint)(w / ipy);
                uint32_t word = voxels[w];
                for (uint b = 0; b < 32; ++b) {
                    uint x = (uint)(w % ipx) * 32 + b;
                    size_t idx;
                    size_t L = 2 * (size_t)rx, A = L * ry;
                    if (g == 1) idx = A * 2 * z + L * y + 2 * x;
                    else if (g == 2) idx = A * 2 * z + L * y + 2 * x + 1;
                    else if (g == 3) idx = A * (2 * z + 1) + L * y + 2 * x;
                    else idx = A * (2 * z + 1) + L * y + 2 * x + 1;
                    nodes[idx] = T::make((word >> (31 - b)) & 1u, 0);
                }
            }
        }
        if (mats) {
            for (int g = 1; g <= 4; ++g) {
                d3 sh = shift(g);
                f3 m{float(pl.mnExt.x + sh.x), float(pl.mnExt.y + sh.y), float(pl.mnExt.z + sh.z)};
                SurfaceCtx c{V, I, M, m, float(pl.d), alloc, true, g, &F, (int)pl.padY, (int)pl.padZ};
                surfacePass(c, nT, matSplits, rec);
            }
        }
    }
    // processVoxel's Node(1, mat) for every surface node (max rule); the
    // PartialNode ratio of the winning triangle.  Conflict bits: 1 = the
    // winning class saw more than one material, 2 = more than one triangle.
    uint64_t nConf = 0;
    const SurfaceCtx rc{V, I, M, f3{float(pl.mnExt.x), float(pl.mnExt.y), float(pl.mnExt.z)}, float(pl.d), alloc,
                        false, 1, &F, (int)pl.padY, (int)pl.padZ};
    std::vector<std::pair<uint, SurfaceRec> > recs(rec.begin(), rec.end());
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : nConf)
    for (long long i = 0; i < (long long)recs.size(); ++i) {
        const uint idx = recs[i].first;
        const SurfaceRec& r = recs[i].second;
        uint matv = r.key & 255u;
        N nd = T::make(1, matv);
        if (T::ratio) {
            const int x = (int)(idx % alloc.x), y = (int)(idx / alloc.x % alloc.y), z = (int)(idx / alloc.x / alloc.y);
            bool unstable = false;
            T::setR(nd, ratio::nodeRatio(rc, r.tri, r.key >> 8, x, y, z, unstable));
            if (unstable && conflict) conflict[idx] |= 4;
        }
        nodes[idx] = nd;
        if (winTri) winTri[idx] = r.tri;
        if (winCls) winCls[idx] = (uint8_t)(r.key >> 8);
        uint8_t cf = (r.minMatTop != matv ? 1u : 0u) | (r.topHits > 1 ? 2u : 0u);
        if (r.minMatTop != matv) nConf++;
        if (conflict && cf) conflict[idx] |= cf;
    }
    info->n_conflicts = nConf;
    info->n_surface = rec.size();
    if (turn) {
        // unRotateNodes (src/voxelizer.cu:2061-2124): (x, y, z) of the X x Y
        // x Z array goes to (y, X - 1 - x, z) of the Y x X x Z array; an FCC
        // node (x, y, z) of the 2X x Y x 2Z array goes to (2y + (x + z + 1) %
        // 2, X - 1 - x / 2, z) of the 2Y x X x 2Z array.  The allocation and
        // its yz subspaces become the turned-back ones.
        N* dst = (N*)out;
        const size_t X = fcc ? 2 * (size_t)alloc.x : alloc.x, Y = alloc.y, Zn = fcc ? 2 * (size_t)alloc.z : alloc.z;
#pragma omp parallel for schedule(static)
        for (long long z = 0; z < (long long)Zn; ++z)
            for (size_t y = 0; y < Y; ++y)
                for (size_t x = 0; x < X; ++x) {
                    const size_t i = (size_t)z * X * Y + y * X + x;
                    const size_t j = fcc ? (size_t)z * X * Y + (X / 2 - 1 - x / 2) * (2 * Y) + 2 * y + (x + z + 1) % 2
                                         : (size_t)z * X * Y + (X - 1 - x) * Y + y;
                    dst[j] = nodes[i];
                    if (outConflict) outConflict[j] = conflict[i];
                }
        nodes = dst;
        conflict = outConflict;
        alloc = u3{alloc.y, alloc.x, alloc.z};
        allocPart = Bounds<u3>{u3{0, 0, 0}, alloc};
        allocYz = splitYZ(vs, allocPart);
    }
    if (!fcc) {
        // fillNodeList2 + the host loop, src/voxelizer.cu:1790-1913 and
        // src/host_side.cpp:1183-1206: per alloc yz split, in order, prune
        // until no node loses its id.  The in-place kernel converges to the
        // greatest set in which every node has a solid neighbour on each axis
        // (ids are monotone in the neighbour set), so Jacobi passes give the
        // same result.
        const uint npx = alloc.x, npy = npx * alloc.y;
        std::vector<uchar> solid(nNodes);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)nNodes; ++i) solid[i] = T::bid(nodes[i]) > 0;
        uint passes = 0;
        auto perm = [&](size_t n, uint x, uint y, uint z) {
            uint pm = 0;
            if (x > 0 && solid[n - 1]) pm += 1;
            if (x < alloc.x - 1 && solid[n + 1]) pm += 2;
            if (y > 0 && solid[n - npx]) pm += 4;
            if (y < alloc.y - 1 && solid[n + npx]) pm += 8;
            if (z > 0 && solid[n - npy]) pm += 16;
            if (z < alloc.z - 1 && solid[n + npy]) pm += 32;
            return pm;
        };
        for (auto& s : allocYz) {
            for (;;) {
                passes++;
                std::vector<size_t> drop;
#pragma omp parallel
                {
                    std::vector<size_t> mine;
#pragma omp for schedule(static)
                    for (long long z = s.min.y; z < (long long)s.max.y; ++z)
                        for (uint y = s.min.x; y < s.max.x; ++y)
                            for (uint x = 0; x < alloc.x; ++x) {
                                size_t n = (size_t)z * npy + (size_t)y * npx + x;
                                if (!solid[n]) continue;
                                if (kOrient[perm(n, x, y, (uint)z)] == 0) mine.push_back(n);
                            }
#pragma omp critical
                    drop.insert(drop.end(), mine.begin(), mine.end());
                }
                for (size_t n : drop) solid[n] = 0;
                if (drop.empty()) break;
            }
#pragma omp parallel for schedule(static)
            for (long long z = s.min.y; z < (long long)s.max.y; ++z)
                for (uint y = s.min.x; y < s.max.x; ++y)
                    for (uint x = 0; x < alloc.x; ++x) {
                        size_t n = (size_t)z * npy + (size_t)y * npx + x;
                        if (T::bid(nodes[n]) == 0) continue;
                        T::setBid(nodes[n], solid[n] ? kOrient[perm(n, x, y, (uint)z)] : 0u);
                    }
        }
        info->prune_passes = passes;
        // zeroPadding (src/voxelizer.cu:4811-4844) in a device space with
        // neighbours: every node on a face of the allocation.
        if (pl.border) {
#pragma omp parallel for schedule(static)
            for (long long z = 0; z < (long long)alloc.z; ++z)
                for (uint y = 0; y < alloc.y; ++y)
                    for (uint x = 0; x < alloc.x; ++x)
                        if (x == 0 || x + 1 == alloc.x || y == 0 || y + 1 == alloc.y || z == 0 || z + 1 == alloc.z)
                            nodes[(size_t)z * npy + (size_t)y * npx + x] = zero;
        }
    } else {
        // calculateFCCBoundaries, src/voxelizer.cu:1929-2048.  The 12
        // neighbour offsets are symmetric, so the in-place kernel equals a
        // snapshot evaluation; splits (z doubled) therefore need no ordering.
        const uint NX = 2 * alloc.x, NY = alloc.y, NZ = 2 * alloc.z;
        const size_t npx = NX, npy = (size_t)NX * NY;
        std::vector<uchar> solid(nNodes);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)nNodes; ++i) solid[i] = T::bid(nodes[i]) > 0;
#pragma omp parallel for schedule(static)
        for (long long z = 0; z < (long long)NZ; ++z)
            for (uint y = 0; y < NY; ++y)
                for (uint x = 0; x < NX; ++x) {
                    size_t n = (size_t)z * npy + (size_t)y * npx + x;
                    if (!solid[n]) continue;
                    bool left = x > 0, right = x < NX - 1, in = y > 0, outy = y < NY - 1;
                    bool down = z > 0, up = z < NZ - 1, xe = ((x + (uint)z) % 2) == 0;
                    uint b = 0;
                    size_t ye = xe ? npx : 0, yo = xe ? 0 : npx;
                    if (down && ((xe && in) || !xe) && solid[n - npy - ye]) b += 1;
                    if (down && left && solid[n - npy - 1]) b += 2;
                    if (down && right && solid[n - npy + 1]) b += 4;
                    if (down && ((!xe && outy) || xe) && solid[n - npy + yo]) b += 8;
                    if (left && ((xe && in) || !xe) && solid[n - 1 - ye]) b += 16;
                    if (right && ((xe && in) || !xe) && solid[n + 1 - ye]) b += 32;
                    if (left && ((!xe && outy) || xe) && solid[n - 1 + yo]) b += 64;
                    if (right && ((!xe && outy) || xe) && solid[n + 1 + yo]) b += 128;
                    if (up && ((xe && in) || !xe) && solid[n + npy - ye]) b += 256;
                    if (up && left && solid[n + npy - 1]) b += 512;
                    if (up && right && solid[n + npy + 1]) b += 1024;
                    if (up && ((!xe && outy) || xe) && solid[n + npy + yo]) b += 2048;
                    T::setBid(nodes[n], b);
                }
        // zeroPadding (src/voxelizer.cu:4827-4834) of an FCC device space with
        // neighbours: two node layers at the x and z faces, one at the y faces.
        if (pl.border) {
#pragma omp parallel for schedule(static)
            for (long long z = 0; z < (long long)NZ; ++z)
                for (uint y = 0; y < NY; ++y)
                    for (uint x = 0; x < NX; ++x)
                        if (x < 2 || x + 2 >= NX || y == 0 || y + 1 == NY || z < 2 || z + 2 >= (long long)NZ)
                            nodes[(size_t)z * npy + (size_t)y * npx + x] = zero;
        }
    }
    return 0;
}

}  // namespace

extern "C" int orc_plan(const orc_params* p, const float* verts, uint32_t nV, orc_info* info) {
    std::vector<float> tv;
    if (p->rotate_x) {
        tv = turnedVertices(verts, nV);
        verts = tv.data();
    }
    Plan pl = makePlan(p, verts, nV);
    applySpace(p, pl);
    memset(info, 0, sizeof(*info));
    if (pl.err) return pl.err;
    bool fcc = p->node_type == ORC_SHORT_FCC || p->node_type == ORC_LONG_FCC;
    static const uint nb[5] = {1, 2, 8, 2, 4};
    if (p->node_type < 0 || p->node_type > 4) return -13;
    if (p->node_output) {
        const bool back = p->rotate_x && p->space;   // turned back: x and y trade places
        const uint ax = back ? pl.alloc.y : pl.alloc.x, ay = back ? pl.alloc.x : pl.alloc.y;
        info->dims[0] = fcc ? 2 * ax : ax;
        info->dims[1] = ay;
        info->dims[2] = fcc ? 2 * pl.alloc.z : pl.alloc.z;
        info->out_bytes = (uint64_t)info->dims[0] * info->dims[1] * info->dims[2] * nb[p->node_type];
    } else {
        info->dims[0] = pl.alloc.x; info->dims[1] = pl.alloc.y; info->dims[2] = pl.alloc.z;
        info->out_bytes = (uint64_t)pl.alloc.x * pl.alloc.y * pl.alloc.z / 8;
    }
    info->voxel_length = pl.d;
    info->min_vertex[0] = pl.mn.x; info->min_vertex[1] = pl.mn.y; info->min_vertex[2] = pl.mn.z;
    info->resolution[0] = pl.res.x; info->resolution[1] = pl.res.y; info->resolution[2] = pl.res.z;
    info->x_splits = pl.xSplits;
    return 0;
}

extern "C" int orc_voxelize(const orc_params* p, const float* verts, uint32_t nV, const uint32_t* idx,
                            uint32_t nT, const uint8_t* mats, uint32_t nMat, void* out, uint64_t out_bytes,
                            uint8_t* conflict, orc_info* info) {
    (void)nMat;
    int rc = orc_plan(p, verts, nV, info);
    if (rc) return rc;
    if (out_bytes < info->out_bytes) return -14;
    std::vector<float> tv;
    if (p->rotate_x) {
        tv = turnedVertices(verts, nV);
        verts = tv.data();
    }
    Plan pl = makePlan(p, verts, nV);
    applySpace(p, pl);
#ifdef _OPENMP
    if (p->threads > 0) omp_set_num_threads(p->threads);
#endif
    if (!p->node_output) return run<ShortN>(p, pl, verts, nV, idx, nT, mats, out, conflict, info);
    switch (p->node_type) {
    case ORC_SHORT: return run<ShortN>(p, pl, verts, nV, idx, nT, mats, out, conflict, info);
    case ORC_LONG: return run<LongN>(p, pl, verts, nV, idx, nT, mats, out, conflict, info);
    case ORC_PARTIAL: return run<PartialN>(p, pl, verts, nV, idx, nT, mats, out, conflict, info);
    case ORC_SHORT_FCC: return run<SFccN>(p, pl, verts, nV, idx, nT, mats, out, conflict, info);
    case ORC_LONG_FCC: return run<LFccN>(p, pl, verts, nV, idx, nT, mats, out, conflict, info);
    }
    return -13;
}

// Cartesian node outputs with, per node, the triangle and class that won its
// surface record (0xFFFFFFFF / 0 where the node is not a surface node): the
// inputs of the PartialNode ratio, for tests that evaluate it separately.
extern "C" int orc_voxelize_winners(const orc_params* p, const float* verts, uint32_t nV, const uint32_t* idx,
                                    uint32_t nT, const uint8_t* mats, uint32_t nMat, void* out, uint64_t out_bytes,
                                    uint8_t* conflict, orc_info* info, uint32_t* win_tri, uint8_t* win_cls) {
    if (!p->node_output || p->node_type != ORC_PARTIAL || !p->materials) return -13;
    int rc = orc_plan(p, verts, nV, info);
    if (rc) return rc;
    if (out_bytes < info->out_bytes) return -14;
    Plan pl = makePlan(p, verts, nV);
    applySpace(p, pl);
    return run<PartialN>(p, pl, verts, nV, idx, nT, mats, out, conflict, info, win_tri, win_cls);
}

// The PartialNode ratio one triangle would give one node (the restatement
// above), for tests that attribute a ratio to its triangle.
extern "C" float orc_node_ratio(const orc_params* p, const float* verts, const uint32_t* idx, uint32_t tri,
                                uint32_t cls, int x, int y, int z, const float* min_corner, float d) {
    const Fma F(p->fma_sites);
    const SurfaceCtx c{verts, idx, nullptr, f3{min_corner[0], min_corner[1], min_corner[2]}, d, u3{0, 0, 0},
                       false, 1, &F, 1, 1};
    bool unstable = false;
    return ratio::nodeRatio(c, tri, cls, x, y, z, unstable);
}

// Every surface hit (triangle << 32 | node index) of one lattice of the
// planned grid (grid 0: Cartesian; 1-4: FCC sub-lattice g), evaluated with
// the site modes in p->fma_sites, in triangle order within each material
// subspace.  Returns the number of hits (pairs beyond `cap` are counted, not
// stored).  Used to fit and check the contraction model one triangle at a
// time against the reference's output.
extern "C" long long orc_surface_hits(const orc_params* p, const float* verts, uint32_t nV, const uint32_t* idx,
                                      uint32_t nT, int grid, uint64_t* pairs, uint64_t cap) {
    Plan pl = makePlan(p, verts, nV);
    applySpace(p, pl);
    if (pl.err) return pl.err;
    if (grid < 0 || grid > 4) return -13;
    const Fma F(p->fma_sites);
    Bounds<u3> ext{u3{0, 0, 0}, pl.ext};
    std::vector<Bounds<u3> > matSplits = split3(u3{p->mat_split[0], p->mat_split[1], p->mat_split[2]}, ext);
    const double h = pl.d / 2.0;
    d3 sh = grid <= 1 ? d3{0, 0, 0} : grid == 2 ? d3{h, h, 0} : grid == 3 ? d3{0, h, h} : d3{h, 0, h};
    d3 m{pl.mnExt.x + sh.x, pl.mnExt.y + sh.y, pl.mnExt.z + sh.z};
    const SurfaceCtx c{verts, idx, nullptr, f3{float(m.x), float(m.y), float(m.z)}, float(pl.d), pl.alloc,
                       grid > 0, grid > 0 ? grid : 1, &F, (int)pl.padY, (int)pl.padZ};
    std::vector<uint> codes(nT);
    for (uint t = 0; t < nT; ++t) {
        f3 v[3];
        fetchF(verts, idx, t, v);
        codes[t] = classify(v, c.m, c.d, F);
    }
    unsigned long long n = 0;
    for (const Bounds<u3>& sub : matSplits)
        for (uint t = 0; t < nT; ++t)
            surfaceTriangle(c, t, codes[t], sub, [&](uint i) {
                if (n < cap) pairs[n] = ((uint64_t)t << 32) | i;
                ++n;
            });
    return (long long)n;
}
