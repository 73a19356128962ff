// Node classification kernels: packed-bit pruning and node emission.
//
// Emission reads three bit grids (final solid, unpruned fill, surface) and
// writes the node grid once.  One thread owns one 32-bit word (32 nodes of a
// row): it forms the six neighbour masks of its word with shifts of the word
// and of the words around it, so a whole word of boundary ids costs a few
// bitwise operations when the word is uniform (all empty, or all solid with
// all six neighbours solid: id 27).  For 1- and 2-byte nodes the ids of a
// mixed word are computed bit-sliced (five planes, one per id bit) and
// transposed to bytes; PartialNodes and FCC nodes take a per-node table
// lookup where solid meets empty.  A warp's 32 words are staged in shared
// memory and stored as contiguous 512-byte rows with 16-byte vector stores.
//
// Grids of one unit hold fewer than 2^32 voxels, so word indices inside a
// unit fit 32 bits; arena offsets (unit word bases) are 64-bit.

#include "vxb_common.cuh"
#include "vxb_device.cuh"
#include "vxb_kernels.cuh"
#include "vxb_ratio.cuh"

namespace vxb {

using namespace detail;

namespace {

__global__ void combineKernel(const uint4* __restrict__ a, const uint4* __restrict__ b, uint4* __restrict__ out,
                              uint64_t n4) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += (uint64_t)gridDim.x * blockDim.x) {
        uint4 x = a[i], y = b[i];
        out[i] = make_uint4(x.x | y.x, x.y | y.y, x.z | y.z, x.w | y.w);
    }
}

// Pruning (fillNodeList2 and the host loop, src/voxelizer.cu:1790-1913,
// src/host_side.cpp:1183-1206): a solid node stays solid iff each axis has a
// solid neighbour.  Passes repeat until nothing changes, which reaches the
// same greatest fixed point as the reference's in-place node passes.
// Neighbours in a later subspace are read from the unpruned grid (fill |
// surf): the reference prunes subspaces in order, so they are still unpruned
// when this one converges.  Reading them explicitly makes a subspace's
// result independent of how far later subspaces have been pruned, which lets
// the host queue passes for all subspaces before checking convergence.
//
// The first pass visits every word of the subspace index's regions and lists
// the words it changed; each later pass revisits only the words next to the
// previous pass's changes (a word can only change when a neighbour did).
// Later passes may visit a word from several threads, so they clear bits with
// atomicAnd: the solid set only shrinks, and every change schedules its
// neighbours, so the passes converge to the same fixed point.

// The data of one pruning region.
struct PruneView {
    uint32_t* S;
    const uint32_t* F;
    const uint32_t* Sf;        // NULL without materials
    const uint8_t* yLater;
    uint32_t ipx, AY, AZ, y0, y1, z0, z1;
};

__device__ __forceinline__ PruneView pruneView(const Batch& b, const PruneRegion& R, uint32_t* solid,
                                               const uint32_t* fill, const uint32_t* surf) {
    const Unit& U = b.units[R.unit];
    PruneView v;
    v.S = solid + U.wordBase;
    v.F = fill + U.wordBase;
    v.Sf = (surf && U.materials) ? surf + U.wordBase : nullptr;
    v.yLater = b.later + U.laterBase;
    v.ipx = U.g.ipx;
    v.AY = U.g.AY;
    v.AZ = U.g.AZ;
    v.y0 = R.split.y0;
    v.y1 = R.split.y1;
    v.z0 = R.split.z0;
    v.z1 = R.split.z1;
    return v;
}

// The pruned value of word (k, y, z) given its current neighbourhood.
// kFresh reads the solid words past L1.
template <bool kFresh = false>
__device__ __forceinline__ uint32_t prunedWord(const PruneView& v, uint32_t w, uint32_t idx, uint32_t k, uint32_t y,
                                               uint32_t z) {
    uint32_t* S = v.S;
    auto ld = [&](uint32_t i) { return kFresh ? __ldcg(S + i) : S[i]; };
    const uint32_t plane = v.ipx * v.AY;
    const uint32_t prev = k > 0 ? ld(idx - 1) : 0u;
    const uint32_t next = k + 1 < v.ipx ? ld(idx + 1) : 0u;
    const uint32_t L = (w >> 1) | (prev << 31), Rt = (w << 1) | (next >> 31);
    const uint32_t In = y > 0 ? ld(idx - v.ipx) : 0u;
    uint32_t Out = 0u, Up = 0u;
    if (y + 1 < v.AY) {
        if (v.yLater[y]) Out = __ldg(v.F + idx + v.ipx) | (v.Sf ? __ldg(v.Sf + idx + v.ipx) : 0u);
        else Out = ld(idx + v.ipx);
    }
    const uint32_t Dn = z > 0 ? ld(idx - plane) : 0u;
    if (z + 1 < v.AZ) {
        const uint8_t* zLater = v.yLater + v.AY;
        if (zLater[z]) Up = __ldg(v.F + idx + plane) | (v.Sf ? __ldg(v.Sf + idx + plane) : 0u);
        else Up = ld(idx + plane);
    }
    return w & (L | Rt) & (In | Out) & (Dn | Up);
}

// Appends (region, word) to a change list; past `cap` it sets *overflow.
__device__ __forceinline__ void listAppend(unsigned long long* list, uint32_t* count, uint32_t cap,
                                           uint32_t* overflow, uint32_t rg, uint32_t idx) {
    const uint32_t at = atomicAdd(count, 1u);
    if (at < cap) list[at] = ((unsigned long long)rg << 32) | idx;
    else *overflow = 1u;
}

// Pass 0: every word of the regions of one subspace index.  Warps walk 32
// consecutive words; the region of a warp's first word is one search, the
// others step forward from it.
__global__ void pruneKernel(Batch b, const PruneRegion* __restrict__ regions, uint32_t n, uint32_t total,
                            uint32_t* solid, const uint32_t* __restrict__ fill, const uint32_t* __restrict__ surf,
                            uint32_t* flags, uint32_t flagBase, uint32_t passes, unsigned long long* list,
                            uint32_t* count, uint32_t cap, uint32_t* overflow) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nWarps = (gridDim.x * blockDim.x) >> 5;
    uint32_t dirty = 0xFFFFFFFFu;   // region this thread changed last (flag not yet set)
    uint32_t cur = 0xFFFFFFFFu, wordStart = 0, ny = 0;
    PruneView v{};
    for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u; base < total; base += nWarps * 32u) {
        uint32_t r0 = 0;
        if (lane == 0 && n > 1) {
            uint32_t lo = 0, hi = n;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (__ldg(&regions[mid].wordStart) <= base) lo = mid;
                else hi = mid;
            }
            r0 = lo;
        }
        r0 = __shfl_sync(0xffffffffu, r0, 0);
        const uint32_t i = base + lane;
        if (i >= total) continue;
        uint32_t r = r0;
        while (r + 1 < n && __ldg(&regions[r + 1].wordStart) <= i) ++r;
        if (r != cur) {
            cur = r;
            const PruneRegion R = regions[r];
            v = pruneView(b, R, solid, fill, surf);
            wordStart = R.wordStart;
            ny = v.y1 - v.y0;
        }
        const uint32_t li = i - wordStart;
        const uint32_t row = li / v.ipx;
        const uint32_t k = li - row * v.ipx;
        const uint32_t zz = row / ny;
        const uint32_t y = v.y0 + (row - zz * ny), z = v.z0 + zz;
        const uint32_t idx = (z * v.AY + y) * v.ipx + k;
        const uint32_t w = v.S[idx];
        if (w == 0) continue;
        const uint32_t nw = prunedWord(v, w, idx, k, y, z);
        if (nw != w) {
            v.S[idx] = nw;
            listAppend(list, count, cap, overflow, r, idx);
            if (dirty != r) {
                if (dirty != 0xFFFFFFFFu) atomicOr(flags + (flagBase + dirty) * passes, 1u);
                dirty = r;
            }
        }
    }
    const uint32_t peers = __match_any_sync(0xffffffffu, dirty);
    if (dirty != 0xFFFFFFFFu && lane == (uint32_t)(__ffs(peers) - 1)) atomicOr(flags + (flagBase + dirty) * passes, 1u);
}

// One entry of a list pass (pass >= 1): the listed word and its six
// neighbours inside the region's subspace.  kFresh reads the solid words
// past L1 (passes of one launch see the previous pass's atomics).
template <bool kFresh>
__device__ __forceinline__ void pruneListEntry(const Batch& b, const PruneRegion* __restrict__ regions,
                                               uint32_t* solid, const uint32_t* __restrict__ fill,
                                               const uint32_t* __restrict__ surf, uint32_t* flags, uint32_t flagBase,
                                               uint32_t passes, uint32_t pass, unsigned long long ent,
                                               unsigned long long* out, uint32_t* outCount, uint32_t cap,
                                               uint32_t* overflow) {
    const uint32_t rg = (uint32_t)(ent >> 32), c = (uint32_t)ent;
    const PruneView v = pruneView(b, regions[rg], solid, fill, surf);
    const uint32_t plane = v.ipx * v.AY;
    const uint32_t cz = c / plane, rem = c - cz * plane, cy = rem / v.ipx, ck = rem - cy * v.ipx;
    bool changed = false;
#pragma unroll 1
    for (int q = 0; q < 7; ++q) {
        uint32_t k = ck, y = cy, z = cz;
        if (q == 1) { if (k == 0) continue; --k; }
        else if (q == 2) { if (k + 1 >= v.ipx) continue; ++k; }
        else if (q == 3) { if (y == v.y0) continue; --y; }
        else if (q == 4) { if (y + 1 >= v.y1) continue; ++y; }
        else if (q == 5) { if (z == v.z0) continue; --z; }
        else if (q == 6) { if (z + 1 >= v.z1) continue; ++z; }
        const uint32_t idx = (z * v.AY + y) * v.ipx + k;
        const uint32_t w = kFresh ? __ldcg(v.S + idx) : v.S[idx];
        if (w == 0) continue;
        const uint32_t nw = prunedWord<kFresh>(v, w, idx, k, y, z);
        if (nw != w) {
            const uint32_t old = atomicAnd(v.S + idx, nw);
            if (old & ~nw) {
                listAppend(out, outCount, cap, overflow, rg, idx);
                changed = true;
            }
        }
    }
    if (changed) atomicOr(flags + (flagBase + rg) * passes + pass, 1u);
}

// Pass `pass` >= 1: the words next to the previous pass's changes (and the
// changed words themselves), inside their region's subspace.
__global__ void pruneListKernel(Batch b, const PruneRegion* __restrict__ regions, uint32_t* solid,
                                const uint32_t* __restrict__ fill, const uint32_t* __restrict__ surf, uint32_t* flags,
                                uint32_t flagBase, uint32_t passes, uint32_t pass,
                                const unsigned long long* __restrict__ in, const uint32_t* __restrict__ inCount,
                                unsigned long long* out, uint32_t* outCount, uint32_t cap, uint32_t* overflow) {
    const uint32_t nIn = min(*inCount, cap);
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < nIn; e += gridDim.x * blockDim.x)
        pruneListEntry<false>(b, regions, solid, fill, surf, flags, flagBase, passes, pass, in[e], out, outCount, cap,
                              overflow);
}

// Passes firstPass .. passes - 1 in one block with a block barrier between
// passes (the lists alternate as they do between single-pass launches).  It
// stops once a list is empty.  A list longer than `escapeAt` is left to the
// host: every region of the subspace index is marked as changed in the last
// pass, so the host runs full passes until the index is stable.
__global__ void __launch_bounds__(1024) pruneListLoopKernel(Batch b, const PruneRegion* __restrict__ regions,
                                                            uint32_t nRegions, uint32_t* solid,
                                                            const uint32_t* __restrict__ fill,
                                                            const uint32_t* __restrict__ surf, uint32_t* flags,
                                                            uint32_t flagBase, uint32_t passes, uint32_t firstPass,
                                                            unsigned long long* list0, unsigned long long* list1,
                                                            uint32_t* counts, uint32_t cap, uint32_t escapeAt,
                                                            uint32_t* overflow) {
    for (uint32_t pass = firstPass; pass < passes; ++pass) {
        __syncthreads();
        const uint32_t nIn = min(*reinterpret_cast<volatile uint32_t*>(counts + pass - 1), cap);
        if (nIn == 0) return;
        if (nIn > escapeAt) {
            for (uint32_t r = threadIdx.x; r < nRegions; r += blockDim.x)
                atomicOr(flags + (flagBase + r) * passes + passes - 1, 1u);
            return;
        }
        const unsigned long long* in = (pass - 1) & 1u ? list1 : list0;
        unsigned long long* out = pass & 1u ? list1 : list0;
        for (uint32_t e = threadIdx.x; e < nIn; e += blockDim.x)
            pruneListEntry<true>(b, regions, solid, fill, surf, flags, flagBase, passes, pass, __ldcg(in + e), out,
                                 counts + pass, cap, overflow);
    }
}

// The words of one unit a kernel reads.
struct UnitWords {
    const uint32_t* fin;
    const uint32_t* fill;
    const uint32_t* surf;     // NULL without materials
    const uint8_t* yLater;
    const uint8_t* zLater;
    uint32_t ipx, AY, AZ, border;
};

// Nodes of word w that zeroPadding (src/voxelizer.cu:4811-4844) clears in a
// device space with neighbours: every node on a face of the allocation.
__device__ __forceinline__ uint32_t borderMask(const UnitWords& u, uint32_t w) {
    if (!u.border) return 0u;
    const uint32_t row = w / u.ipx, k = w - row * u.ipx;
    const uint32_t z = row / u.AY, y = row - z * u.AY;
    if (y == 0 || y + 1 == u.AY || z == 0 || z + 1 == u.AZ) return 0xFFFFFFFFu;
    return (k == 0 ? 0x80000000u : 0u) | (k + 1 == u.ipx ? 1u : 0u);
}

struct EmitArgs {
    Batch b;
    const uint32_t* fin;     // pruned solid arena
    const uint32_t* fill;    // parity fill arena (unpruned)
    const uint32_t* surf;    // surface arena
    const WordRank* ranks;   // surface words with their ranks (arena-wide)
    const void* keys;        // merged material keys by rank
    uint32_t keysCap;        // keys past it read as 0
};

__device__ __forceinline__ UnitWords unitWords(const EmitArgs& a, const Unit& U) {
    UnitWords uw;
    uw.fin = a.fin + U.wordBase;
    uw.fill = a.fill + U.wordBase;
    uw.surf = U.materials ? a.surf + U.wordBase : nullptr;
    uw.yLater = a.b.later + U.laterBase;
    uw.zLater = uw.yLater + U.g.AY;
    uw.ipx = U.g.ipx;
    uw.AY = U.g.AY;
    uw.AZ = U.g.AZ;
    uw.border = U.g.border;
    return uw;
}

// Node emission, Cartesian lattices.  Boundary ids follow fillNodeList2 in
// split order: a neighbour in a later yz subspace is read from the unpruned
// grid (its subspace was still unpruned when this one converged), every
// other neighbour from the final grid.  Pruned surface nodes keep their
// material (node.bid(0) keeps mat, include/node_types.h).
struct WordNbrs {
    uint32_t c, s0, f0, L, R, In, Out, Dn, Up;
};

template <int K>
__device__ __forceinline__ WordNbrs loadNbrs(const UnitWords& u, uint32_t w) {
    typedef NodeT<K> NT;
    WordNbrs n;
    n.c = __ldg(u.fin + w);
    n.s0 = u.surf ? __ldg(u.surf + w) : 0u;
    n.f0 = NT::bytes == 8 ? __ldg(u.fill + w) : 0u;
    n.L = n.R = n.In = n.Out = n.Dn = n.Up = 0u;
    if (n.c | n.s0 | n.f0) {
        const uint32_t row = w / u.ipx;
        const uint32_t k = w - row * u.ipx;
        const uint32_t z = row / u.AY, y = row - z * u.AY;
        const uint32_t plane = u.ipx * u.AY;
        const uint32_t prev = k > 0 ? __ldg(u.fin + w - 1) : 0u;
        const uint32_t next = k + 1 < u.ipx ? __ldg(u.fin + w + 1) : 0u;
        n.L = (n.c >> 1) | (prev << 31);
        n.R = (n.c << 1) | (next >> 31);
        n.In = y > 0 ? __ldg(u.fin + w - u.ipx) : 0u;
        if (y + 1 < u.AY)
            n.Out = u.yLater[y] ? (__ldg(u.fill + w + u.ipx) | (u.surf ? __ldg(u.surf + w + u.ipx) : 0u))
                                : __ldg(u.fin + w + u.ipx);
        n.Dn = z > 0 ? __ldg(u.fin + w - plane) : 0u;
        if (z + 1 < u.AZ)
            n.Up = u.zLater[z] ? (__ldg(u.fill + w + plane) | (u.surf ? __ldg(u.surf + w + plane) : 0u))
                               : __ldg(u.fin + w + plane);
    }
    return n;
}

// Boundary ids of the nodes `cm` of a word as five bit planes: plane k holds
// bit k of every node's id.  Along each axis a node has a solid neighbour
// below only (1), above only (2) or on both sides (3); the id is
// kOrientTable[x | y << 2 | z << 4] for those three codes (0 when an axis has
// none), and each plane is the union of the code combinations whose id has
// that bit set, evaluated on whole words at once.
__device__ __forceinline__ void idPlanes(const WordNbrs& n, uint32_t cm, uint32_t P[5]) {
    const uint32_t L = n.L, R = n.R;
    const uint32_t X1 = L & ~R, X3 = L & R, Xo = L ^ R, Xa = L | R, X2 = R & ~L;
    const uint32_t Y1 = n.In & ~n.Out, Y2 = n.Out & ~n.In, Y3 = n.In & n.Out, Ya = n.In | n.Out;
    const uint32_t Z1 = n.Dn & ~n.Up, Z2 = n.Up & ~n.Dn, Z3 = n.Dn & n.Up, Za = n.Dn | n.Up, Zo = n.Dn ^ n.Up;
    P[0] = ((Za & ((Y1 & L) | (Y2 & X1))) | (Y3 & ((n.Dn & L) | (Z2 & X1)))) & cm;
    P[1] = ((Y1 & ((Zo & X2) | (Z3 & R))) | (Za & Y2 & L) | (Y3 & ((Z1 & X1) | (Z2 & L) | (Z3 & X3)))) & cm;
    P[2] = ((Z1 & ((Y2 & X2) | (Y3 & R))) | (Z2 & ((Y1 & Xa) | (Y2 & L) | (Y3 & X1))) | (Z3 & ((Y1 & X3) | (Y2 & R)))) &
           cm;
    P[3] = ((Z1 & (((Y1 | Y2) & X3) | (Y3 & Xo))) | (Z2 & ((Y1 & X3) | (Y2 & R) | (Y3 & L))) | (Z3 & Y3 & Xa)) & cm;
    P[4] = ((Y3 & ((Z1 & X3) | (Z2 & R))) | (Z3 & Ya & Xa)) & cm;
}

// The planes as bytes in node order: N[m] holds the ids of nodes 4m .. 4m+3
// (node t of a word is bit 31 - t), one per byte.  An 8x8 bit transpose in
// each byte lane of the bit-reversed planes leaves the id of node 8b + i in
// byte b of row i; 4x4 byte transposes put the nodes in order.
__device__ __forceinline__ void idBytes(const uint32_t P[5], uint32_t N[8]) {
    uint32_t r[8];
#pragma unroll
    for (int k = 0; k < 5; ++k) r[k] = __brev(P[k]);
    r[5] = r[6] = r[7] = 0u;
#pragma unroll
    for (int s = 4; s >= 1; s >>= 1) {
        const uint32_t m = s == 4 ? 0x0F0F0F0Fu : s == 2 ? 0x33333333u : 0x55555555u;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if ((k / s) % 2 == 0) {
                const uint32_t t = ((r[k] >> s) ^ r[k + s]) & m;
                r[k + s] ^= t;
                r[k] ^= t << s;
            }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint32_t t0 = __byte_perm(r[4 * h], r[4 * h + 1], 0x5140), t1 = __byte_perm(r[4 * h], r[4 * h + 1], 0x7362);
        const uint32_t t2 = __byte_perm(r[4 * h + 2], r[4 * h + 3], 0x5140),
                       t3 = __byte_perm(r[4 * h + 2], r[4 * h + 3], 0x7362);
        N[h] = __byte_perm(t0, t2, 0x5410);
        N[2 + h] = __byte_perm(t0, t2, 0x7632);
        N[4 + h] = __byte_perm(t1, t3, 0x5410);
        N[6 + h] = __byte_perm(t1, t3, 0x7632);
    }
}

__device__ __forceinline__ uint32_t permOf(const WordNbrs& n, uint32_t q) {
    return ((n.L >> q) & 1u) | (((n.R >> q) & 1u) << 1) | (((n.In >> q) & 1u) << 2) | (((n.Out >> q) & 1u) << 3) |
           (((n.Dn >> q) & 1u) << 4) | (((n.Up >> q) & 1u) << 5);
}

// 1- and 2-byte nodes.  Each lane owns one word and builds its 32 nodes in
// its own shared-memory row: the ids of all 32 come from the bit planes of
// idPlanes (or a constant for empty and all-interior words), the materials
// of surface nodes from the merged keys, which are consecutive by rank (a
// word whose 32 nodes are all surface nodes loads its 32 keys without a
// per-node loop).  The warp's 32 rows are then stored as one contiguous
// span.  Unit word bases are multiples of 32, so a warp's words belong to
// one unit.
template <int K>
__global__ void __launch_bounds__(256, 6) emitNarrowKernel(EmitArgs a, uint64_t wordBegin, uint64_t totalWords) {
    typedef NodeT<K> NT;
    static_assert(NT::bytes <= 2, "narrow nodes only");
    constexpr int NB = NT::bytes;
    constexpr int WB = 32 * NB;                  // bytes of one word's nodes
    constexpr int CH = WB / 16;                  // 16-byte chunks per word
    constexpr int PITCH = (CH + 1) * 16;         // padded smem row (conflict-free)
    __shared__ __align__(16) uint8_t stage[8][32 * PITCH];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint8_t* my = stage[warp] + lane * PITCH;
    const uint32_t v27 = (uint32_t)NT::pack(27u, 0u, 0.0f);
    // Data of the unit last visited (a warp's words belong to one unit).
    uint32_t cur = 0xFFFFFFFFu, nWords = 0;
    uint64_t uBase = 0;
    uint8_t* uOut = nullptr;
    UnitWords uw{};
    for (uint64_t gbase = wordBegin + ((uint64_t)blockIdx.x * 8u + warp) * 32u; gbase < totalWords;
         gbase += (uint64_t)gridDim.x * 8u * 32u) {
        const uint32_t u = a.b.nUnits > 1 ? unitOf(a.b.wordBase, a.b.nUnits, gbase) : 0u;
        if (u != cur) {
            cur = u;
            const Unit& U = a.b.units[u];
            nWords = U.g.ipx * U.g.AY * U.g.AZ;
            uBase = U.wordBase;
            uOut = static_cast<uint8_t*>(U.out);
            uw = unitWords(a, U);
        }
        const uint32_t wbase = (uint32_t)(gbase - uBase);
        if (wbase >= nWords) continue;            // padding after the unit's grid (whole warp)
        const uint32_t w = wbase + lane;
        WordNbrs n{};
        uint32_t zero = 0u;
        if (w < nWords) {
            n = loadNbrs<K>(uw, w);
            zero = borderMask(uw, w);
        }
        // Ids: none, all 27 (every node solid with six solid neighbours), or
        // the bit-sliced planes.  Materials of surface nodes follow by rank
        // (the rank is loaded first, so that its latency overlaps the ids).
        const uint32_t cm = n.c & ~zero, sm = n.s0 & ~zero;
        const uint32_t rank0 = sm ? a.ranks[uBase + w].rank : 0u;
        if (cm == 0u || (cm & n.L & n.R & n.In & n.Out & n.Dn & n.Up) == 0xFFFFFFFFu) {
            const uint32_t rep = cm == 0u ? 0u : NB == 1 ? v27 * 0x01010101u : v27 * 0x00010001u;
#pragma unroll
            for (int i = 0; i < CH; ++i) *reinterpret_cast<uint4*>(my + 16 * i) = make_uint4(rep, rep, rep, rep);
        } else {
            uint32_t N[8];
            {
                uint32_t P[5];
                idPlanes(n, cm, P);
                idBytes(P, N);
            }
#pragma unroll
            for (int i = 0; i < CH; ++i) {
                uint4 q;
                if (NB == 1) {
                    q = make_uint4(N[4 * i], N[4 * i + 1], N[4 * i + 2], N[4 * i + 3]);
                } else {
                    q = make_uint4(__byte_perm(N[2 * i], 0u, 0x4140), __byte_perm(N[2 * i], 0u, 0x4342),
                                   __byte_perm(N[2 * i + 1], 0u, 0x4140), __byte_perm(N[2 * i + 1], 0u, 0x4342));
                }
                *reinterpret_cast<uint4*>(my + 16 * i) = q;
            }
        }
        if (sm) {
            const uint32_t* keys = reinterpret_cast<const uint32_t*>(a.keys);
            if (sm == 0xFFFFFFFFu && (uint64_t)rank0 + 32u <= a.keysCap) {
                // 32 surface nodes: their keys are the 32 from rank0 on.
#pragma unroll 8
                for (uint32_t j = 0; j < 32u; ++j) {
                    const uint32_t mat = NT::keyMat(__ldg(keys + rank0 + j));
                    if (NB == 1) my[j] |= (uint8_t)(mat << 5);
                    else my[2 * j + 1] = (uint8_t)mat;
                }
            } else {
                // Four surface nodes per step, so that their key loads are
                // in flight together.
                constexpr int kKeys = 4;
                uint32_t rest = sm;
                do {
                    uint32_t bt[kKeys], mat[kKeys];
#pragma unroll
                    for (int q = 0; q < kKeys; ++q) {
                        bt[q] = 32u;
                        if (rest) {
                            bt[q] = __clz(rest);       // node index in the word
                            rest &= ~(0x80000000u >> bt[q]);
                        }
                    }
#pragma unroll
                    for (int q = 0; q < kKeys; ++q) {
                        const uint32_t r = rank0 + (bt[q] ? __popc(n.s0 >> (32u - bt[q])) : 0u);
                        mat[q] = bt[q] < 32u && r < a.keysCap ? NT::keyMat(__ldg(keys + r)) : 0u;
                    }
#pragma unroll
                    for (int q = 0; q < kKeys; ++q) {
                        if (bt[q] == 32u) break;
                        if (NB == 1) my[bt[q]] |= (uint8_t)(mat[q] << 5);
                        else my[2 * bt[q] + 1] = (uint8_t)mat[q];
                    }
                } while (rest);
            }
        }
        __syncwarp();
        const uint32_t wend = wbase + 32u <= nWords ? 32u : nWords - wbase;
        uint4* out = reinterpret_cast<uint4*>(uOut + (size_t)wbase * WB);
#pragma unroll
        for (int i = 0; i < CH; ++i) {
            const uint32_t chunk = i * 32 + lane;       // 16-byte chunk of the warp's span
            const uint32_t wi = chunk / CH, ci = chunk % CH;
            if (wi < wend) out[chunk] = *reinterpret_cast<const uint4*>(stage[warp] + wi * PITCH + 16 * ci);
        }
        __syncwarp();
    }
}

// 8-byte PartialNodes: one lane per word, nodes stored from registers.  The
// ratio of a node is 1 where the parity fill is set and the node is not a
// surface node.
__global__ void __launch_bounds__(256) emitPartialKernel(EmitArgs a, uint64_t wordBegin, uint64_t totalWords) {
    typedef NodeT<kPartial> NT;
    __shared__ uint8_t lut[64];
    if (threadIdx.x < 64) lut[threadIdx.x] = kOrientTable[threadIdx.x];
    __syncthreads();
    for (uint64_t gw = wordBegin + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gw < totalWords;
         gw += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t u = unitOf(a.b.wordBase, a.b.nUnits, gw);
        const Unit& U = a.b.units[u];
        const uint32_t w = (uint32_t)(gw - U.wordBase);
        if (w >= U.g.ipx * U.g.AY * U.g.AZ) continue;
        const UnitWords uw = unitWords(a, U);
        const WordNbrs n = loadNbrs<kPartial>(uw, w);
        const uint32_t zero = borderMask(uw, w);
        uint4* out = reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(U.out) + (size_t)w * 32 * 8);
        if (((n.c | n.s0 | n.f0) & ~zero) == 0u) {
#pragma unroll
            for (int i = 0; i < 16; ++i) out[i] = make_uint4(0, 0, 0, 0);
            continue;
        }
        uint32_t matRank = n.s0 ? a.ranks[U.wordBase + w].rank : 0u;
        // Node coordinates of the word's first node (ratio of surface nodes).
        const int x0 = (int)(w % U.g.ipx) * 32, y0 = (int)(w / U.g.ipx % U.g.AY), z0 = (int)(w / U.g.ipx / U.g.AY);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            uint32_t v32[4];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const uint32_t bt = 2 * i + j, q = 31u - bt;
                uint32_t bid = 0, mat = 0;
                if ((n.c >> q) & 1u) bid = lut[permOf(n, q)];
                // constructNodeList2 writes float(solid); processVoxel<PartialNode>
                // overwrites surface nodes with the winning triangle's ratio.
                float r = ((n.f0 >> q) & 1u) ? 1.0f : 0.0f;
                if ((n.s0 >> q) & 1u) {
                    if (matRank < a.keysCap && !((zero >> q) & 1u)) {
                        const uint64_t key = reinterpret_cast<const unsigned long long*>(a.keys)[matRank];
                        mat = NT::keyMat(key);
                        r = ratio::nodeRatio(U.V, U.I, (uint32_t)key, (uint32_t)(key >> 40), x0 + (int)bt, y0, z0,
                                             detail::F3{U.g.mnf[0], U.g.mnf[1], U.g.mnf[2]}, U.g.df);
                    }
                    ++matRank;
                }
                const uint64_t nv = (zero >> q) & 1u ? 0ull : NT::pack(bid, mat, r);
                v32[2 * j] = (uint32_t)nv;
                v32[2 * j + 1] = (uint32_t)(nv >> 32);
            }
            out[i] = make_uint4(v32[0], v32[1], v32[2], v32[3]);
        }
    }
}

struct FccArgs {
    Batch b;
    const FccMesh* meshes;
    const uint64_t* groupBase;
    uint32_t nMeshes;
    const uint32_t* fill;
    const uint32_t* surf;
    const WordRank* ranks;
    const void* keys;
    uint32_t keysCap;
    uint32_t raw;   // nodes before the boundaries: id = solid bit, no face clearing
};

// The four sub-lattice grids of one FCC mesh.
struct FccGrids {
    const uint32_t* fill[4];
    const uint32_t* surf[4];   // NULL without materials
    uint64_t wordBase[4];      // arena word of each sub-lattice (rank space)
    uint32_t ipx, AY;
};

// Node emission, FCC lattices (convertToFCCGrid + calculateFCCBoundaries,
// src/voxelizer.cu:1710-1776, 1929-2048).  FCC node (X, y, Z) belongs to
// sub-lattice 1 + (X & 1) + 2 * (Z & 1) at voxel (X / 2, y, Z / 2); its id is
// the 12-bit mask of solid FCC neighbours.  The neighbour relation is
// symmetric, so the reference's in-place pass equals this snapshot
// evaluation.
__device__ __forceinline__ uint32_t fccSolid(const FccGrids& G, uint32_t X2, uint32_t y, uint32_t Z2) {
    const int gt = (int)(X2 & 1u) + 2 * (int)(Z2 & 1u);
    const uint32_t x = X2 >> 1, z = Z2 >> 1;
    const uint32_t w = (z * G.AY + y) * G.ipx + (x >> 5);
    uint32_t word = __ldg(G.fill[gt] + w);
    if (G.surf[gt]) word |= __ldg(G.surf[gt] + w);
    return (word >> (31u - (x & 31u))) & 1u;
}

template <int K>
__global__ void emitFccKernel(FccArgs A, uint64_t totalGroups) {
    typedef NodeT<K> NT;
    constexpr int GN = 16 / NT::bytes;
    for (uint64_t gg = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gg < totalGroups;
         gg += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t m = unitOf(A.groupBase, A.nMeshes, gg);
        const FccMesh M = A.meshes[m];
        FccGrids G;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const Unit& U = A.b.units[M.unit0 + l];
            G.fill[l] = A.fill + U.wordBase;
            G.surf[l] = U.materials ? A.surf + U.wordBase : nullptr;
            G.wordBase[l] = U.wordBase;
        }
        const PassGeom& g = A.b.units[M.unit0].g;
        G.ipx = g.ipx;
        G.AY = g.AY;
        const uint32_t NX = 2 * g.X, NY = g.AY, NZ = 2 * g.AZ;
        const uint32_t groupsPerRow = NX / GN;
        const uint32_t gi = (uint32_t)(gg - __ldg(A.groupBase + m));
        const uint32_t row = gi / groupsPerRow;
        const uint32_t X0 = (gi - row * groupsPerRow) * GN;
        const uint32_t Z2 = row / NY, y = row - Z2 * NY;
        uint4 outv = make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int n = 0; n < GN; ++n) {
            const uint32_t X2 = X0 + n;
            const int gt = (int)(X2 & 1u) + 2 * (int)(Z2 & 1u);
            const uint32_t x = X2 >> 1, z = Z2 >> 1;
            const uint32_t w = (z * G.AY + y) * G.ipx + (x >> 5);
            const uint32_t q = 31u - (x & 31u);
            const uint32_t fb = (__ldg(G.fill[gt] + w) >> q) & 1u;
            const uint32_t sw = G.surf[gt] ? __ldg(G.surf[gt] + w) : 0u;
            const uint32_t sb = (sw >> q) & 1u;
            uint32_t bid = 0;
            if ((fb | sb) && A.raw) {
                bid = 1;
            } else if (fb | sb) {
                const bool left = X2 > 0, right = X2 < NX - 1, in = y > 0, out = y < NY - 1;
                const bool down = Z2 > 0, up = Z2 < NZ - 1, xe = ((X2 + Z2) & 1u) == 0;
                const uint32_t ym = xe ? y - 1 : y;   // y - xEven
                const uint32_t yp = xe ? y : y + 1;   // y + !xEven
                const bool cIn = (xe && in) || !xe, cOut = (!xe && out) || xe;
                if (down && cIn && fccSolid(G, X2, ym, Z2 - 1)) bid |= 1u;
                if (down && left && fccSolid(G, X2 - 1, y, Z2 - 1)) bid |= 2u;
                if (down && right && fccSolid(G, X2 + 1, y, Z2 - 1)) bid |= 4u;
                if (down && cOut && fccSolid(G, X2, yp, Z2 - 1)) bid |= 8u;
                if (left && cIn && fccSolid(G, X2 - 1, ym, Z2)) bid |= 16u;
                if (right && cIn && fccSolid(G, X2 + 1, ym, Z2)) bid |= 32u;
                if (left && cOut && fccSolid(G, X2 - 1, yp, Z2)) bid |= 64u;
                if (right && cOut && fccSolid(G, X2 + 1, yp, Z2)) bid |= 128u;
                if (up && cIn && fccSolid(G, X2, ym, Z2 + 1)) bid |= 256u;
                if (up && left && fccSolid(G, X2 - 1, y, Z2 + 1)) bid |= 512u;
                if (up && right && fccSolid(G, X2 + 1, y, Z2 + 1)) bid |= 1024u;
                if (up && cOut && fccSolid(G, X2, yp, Z2 + 1)) bid |= 2048u;
            }
            uint32_t mat = 0;
            if (sb) {
                const uint32_t bt = x & 31u;
                const uint32_t r = A.ranks[G.wordBase[gt] + w].rank + (bt ? __popc(sw >> (32 - bt)) : 0u);
                mat = r < A.keysCap ? NT::keyMat(reinterpret_cast<const uint32_t*>(A.keys)[r]) : 0u;
            }
            // zeroPadding of an FCC device space with neighbours
            // (src/voxelizer.cu:4827-4834): two node layers at the x and z
            // faces, one at the y faces.
            const bool face = g.border && !A.raw && (X2 < 2 || X2 + 2 >= NX || y == 0 || y + 1 == NY || Z2 < 2 || Z2 + 2 >= NZ);
            const uint64_t val = face ? 0ull : NT::pack(bid, mat, 0.0f);
            if (NT::bytes == 2) reinterpret_cast<uint16_t*>(&outv)[n] = (uint16_t)val;
            else reinterpret_cast<uint32_t*>(&outv)[n] = (uint32_t)val;
        }
        reinterpret_cast<uint4*>(M.out)[gi] = outv;
    }
}

}  // namespace

void launch_combine(const uint32_t* a, const uint32_t* b, uint32_t* out, uint64_t n, cudaStream_t s,
                    uint32_t* launches) {
    const uint64_t n4 = n / 4;
    combineKernel<<<gridFor(n4, 256), 256, 0, s>>>(reinterpret_cast<const uint4*>(a), reinterpret_cast<const uint4*>(b),
                                                    reinterpret_cast<uint4*>(out), n4);
    *launches += 1;
}

void launch_prune(const Batch& b, const PruneRegion* regions, uint32_t n, uint32_t groupWords, uint32_t* solid,
                  const uint32_t* fill, const uint32_t* surf, uint32_t* flags, uint32_t flagBase, uint32_t passes,
                  unsigned long long* list, uint32_t* count, uint32_t cap, uint32_t* overflow, cudaStream_t s,
                  uint32_t* launches) {
    pruneKernel<<<gridFor(groupWords, 256, 148u * 8u), 256, 0, s>>>(b, regions, n, groupWords, solid, fill, surf,
                                                                    flags, flagBase, passes, list, count, cap,
                                                                    overflow);
    *launches += 1;
}

void launch_prune_list_loop(const Batch& b, const PruneRegion* regions, uint32_t nRegions, uint32_t* solid,
                            const uint32_t* fill, const uint32_t* surf, uint32_t* flags, uint32_t flagBase,
                            uint32_t passes, uint32_t firstPass, unsigned long long* list0, unsigned long long* list1,
                            uint32_t* counts, uint32_t cap, uint32_t escapeAt, uint32_t* overflow, cudaStream_t s,
                            uint32_t* launches) {
    pruneListLoopKernel<<<1, 1024, 0, s>>>(b, regions, nRegions, solid, fill, surf, flags, flagBase, passes, firstPass,
                                           list0, list1, counts, cap, escapeAt, overflow);
    *launches += 1;
}

void launch_prune_list(const Batch& b, const PruneRegion* regions, uint32_t* solid, const uint32_t* fill,
                       const uint32_t* surf, uint32_t* flags, uint32_t flagBase, uint32_t passes, uint32_t pass,
                       const unsigned long long* in, const uint32_t* inCount, unsigned long long* out,
                       uint32_t* outCount, uint32_t cap, uint32_t* overflow, cudaStream_t s, uint32_t* launches) {
    pruneListKernel<<<148 * 8, 256, 0, s>>>(b, regions, solid, fill, surf, flags, flagBase, passes, pass, in, inCount,
                                            out, outCount, cap, overflow);
    *launches += 1;
}

void launch_emit_cartesian(int nodeKind, const Batch& b, uint64_t wordBegin, uint64_t totalWords,
                           const uint32_t* finalSolid,
                           const uint32_t* fill, const uint32_t* surf, const WordRank* ranks, const void* keys,
                           uint32_t keysCap, uint32_t blocksPerSm, cudaStream_t s, uint32_t* launches) {
    EmitArgs a;
    a.keysCap = keysCap;
    a.b = b;
    a.fin = finalSolid;
    a.fill = fill;
    a.surf = surf;
    a.ranks = ranks;
    a.keys = keys;
    const uint64_t words = totalWords - wordBegin;
    const uint32_t grid = gridFor(words, 256, 148u * blocksPerSm);
    switch (nodeKind) {
    case kShort: emitNarrowKernel<kShort><<<grid, 256, 0, s>>>(a, wordBegin, totalWords); break;
    case kLong: emitNarrowKernel<kLong><<<grid, 256, 0, s>>>(a, wordBegin, totalWords); break;
    default: emitPartialKernel<<<gridFor(words, 256, 148u * 8u), 256, 0, s>>>(a, wordBegin, totalWords); break;
    }
    *launches += 1;
}

void launch_emit_fcc(int nodeKind, const Batch& b, const FccMesh* meshes, const uint64_t* groupBase,
                     uint32_t nMeshes, uint64_t totalGroups, const uint32_t* fill, const uint32_t* surf,
                     const WordRank* ranks, const void* keys, uint32_t keysCap, bool raw, cudaStream_t s,
                     uint32_t* launches) {
    FccArgs A;
    A.keysCap = keysCap;
    A.raw = raw ? 1u : 0u;
    A.b = b;
    A.meshes = meshes;
    A.groupBase = groupBase;
    A.nMeshes = nMeshes;
    A.fill = fill;
    A.surf = surf;
    A.ranks = ranks;
    A.keys = keys;
    const uint32_t grid = gridFor(totalGroups, 256, 148u * 64u);
    if (nodeKind == kShortFcc) emitFccKernel<kShortFcc><<<grid, 256, 0, s>>>(A, totalGroups);
    else emitFccKernel<kLongFcc><<<grid, 256, 0, s>>>(A, totalGroups);
    *launches += 1;
}

}  // namespace vxb
