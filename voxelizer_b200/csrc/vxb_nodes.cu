// Node classification kernels: packed-bit pruning and node emission.
//
// Emission reads three bit grids (final solid, unpruned fill, surface) and
// writes the node grid once.  One thread owns one 32-bit word (32 nodes of a
// row): it forms the six neighbour masks of its word with shifts of the word
// and of the words around it, so a whole word of boundary ids costs a few
// bitwise operations when the word is uniform (all empty, or all solid with
// all six neighbours solid: id 27) and a per-node table lookup only where
// solid meets empty.  A warp's 32 words are staged in shared memory and
// stored as contiguous 512-byte rows with 16-byte vector stores.

#include "vxb_common.cuh"
#include "vxb_device.cuh"
#include "vxb_kernels.cuh"

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

// One pruning pass over one yz subspace (fillNodeList2 and the host loop,
// src/voxelizer.cu:1790-1913, src/host_side.cpp:1183-1206): a solid node
// stays solid iff each axis has a solid neighbour.  Words are updated in
// place; passes repeat until none changes, which reaches the same greatest
// fixed point as the reference's in-place node passes.  Neighbours in a
// later subspace are read from the unpruned grid (fill | surf): the
// reference prunes subspaces in order, so they are still unpruned when this
// one converges.  Reading them explicitly makes a subspace's result
// independent of how far later subspaces have been pruned, which lets the
// host queue passes for all subspaces before checking convergence.
__global__ void pruneKernel(uint32_t* solid, const uint32_t* __restrict__ fill, const uint32_t* __restrict__ surf,
                            const uint8_t* __restrict__ yLater, const uint8_t* __restrict__ zLater, PassGeom g,
                            SplitYZ sp, uint32_t* changed) {
    // Grids hold fewer than 2^32 voxels, so word indices fit 32 bits.
    const uint32_t ny = sp.y1 - sp.y0;
    const uint32_t nWords = ny * (sp.z1 - sp.z0) * g.ipx;
    const uint32_t plane = g.ipx * g.AY;
    bool any = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nWords; i += gridDim.x * blockDim.x) {
        const uint32_t r = i / g.ipx;
        const uint32_t k = i - r * g.ipx;
        const uint32_t zz = r / ny;
        const uint32_t y = sp.y0 + (r - zz * ny), z = sp.z0 + zz;
        const uint32_t idx = (z * g.AY + y) * g.ipx + k;
        const uint32_t w = solid[idx];
        if (w == 0) continue;
        const uint32_t prev = k > 0 ? solid[idx - 1] : 0u;
        const uint32_t next = k + 1 < g.ipx ? solid[idx + 1] : 0u;
        const uint32_t L = (w >> 1) | (prev << 31), R = (w << 1) | (next >> 31);
        const uint32_t In = y > 0 ? solid[idx - g.ipx] : 0u;
        uint32_t Out = 0u, Up = 0u;
        if (y + 1 < g.AY) {
            if (yLater[y]) Out = __ldg(fill + idx + g.ipx) | (surf ? __ldg(surf + idx + g.ipx) : 0u);
            else Out = solid[idx + g.ipx];
        }
        const uint32_t Dn = z > 0 ? solid[idx - plane] : 0u;
        if (z + 1 < g.AZ) {
            if (zLater[z]) Up = __ldg(fill + idx + plane) | (surf ? __ldg(surf + idx + plane) : 0u);
            else Up = solid[idx + plane];
        }
        const uint32_t nw = w & (L | R) & (In | Out) & (Dn | Up);
        if (nw != w) {
            solid[idx] = nw;
            any = true;
        }
    }
    if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(changed, 1u);
}

struct EmitArgs {
    const uint32_t* fin;     // pruned solid
    const uint32_t* fill;    // parity fill (unpruned)
    const uint32_t* surf;    // surface voxels (nullptr without materials)
    const uint32_t* ranks;   // exclusive popcount prefix of surf words
    const void* keys;        // merged material keys by rank
    const uint8_t* yLater;
    const uint8_t* zLater;
    void* nodes;
    PassGeom g;
    int materials;
};

// Node emission, Cartesian lattices.  Boundary ids follow fillNodeList2 in
// split order: a neighbour in a later yz subspace is read from the unpruned
// grid (its subspace was still unpruned when this one converged), every
// other neighbour from the final grid.  Pruned surface nodes keep their
// material (node.bid(0) keeps mat, include/node_types.h).

// The seven words around word w and its coordinates.  Grids hold fewer than
// 2^32 voxels, so word indices fit 32 bits.
struct WordNbrs {
    uint32_t c, s0, f0, L, R, In, Out, Dn, Up;
};

template <int K>
__device__ __forceinline__ WordNbrs loadNbrs(const EmitArgs& a, uint32_t w) {
    typedef NodeT<K> NT;
    const PassGeom& g = a.g;
    WordNbrs n;
    n.c = __ldg(a.fin + w);
    n.s0 = a.materials ? __ldg(a.surf + w) : 0u;
    n.f0 = NT::bytes == 8 ? __ldg(a.fill + w) : 0u;
    n.L = n.R = n.In = n.Out = n.Dn = n.Up = 0u;
    if (n.c | n.s0 | n.f0) {
        const uint32_t row = w / g.ipx;
        const uint32_t k = w - row * g.ipx;
        const uint32_t z = row / g.AY, y = row - z * g.AY;
        const uint32_t plane = g.ipx * g.AY;
        const uint32_t prev = k > 0 ? __ldg(a.fin + w - 1) : 0u;
        const uint32_t next = k + 1 < g.ipx ? __ldg(a.fin + w + 1) : 0u;
        n.L = (n.c >> 1) | (prev << 31);
        n.R = (n.c << 1) | (next >> 31);
        n.In = y > 0 ? __ldg(a.fin + w - g.ipx) : 0u;
        if (y + 1 < g.AY)
            n.Out = a.yLater[y] ? (__ldg(a.fill + w + g.ipx) | (a.materials ? __ldg(a.surf + w + g.ipx) : 0u))
                                : __ldg(a.fin + w + g.ipx);
        n.Dn = z > 0 ? __ldg(a.fin + w - plane) : 0u;
        if (z + 1 < g.AZ)
            n.Up = a.zLater[z] ? (__ldg(a.fill + w + plane) | (a.materials ? __ldg(a.surf + w + plane) : 0u))
                               : __ldg(a.fin + w + plane);
    }
    return n;
}

__device__ __forceinline__ uint32_t permOf(const WordNbrs& n, uint32_t q) {
    return ((n.L >> q) & 1u) | (((n.R >> q) & 1u) << 1) | (((n.In >> q) & 1u) << 2) | (((n.Out >> q) & 1u) << 3) |
           (((n.Dn >> q) & 1u) << 4) | (((n.Up >> q) & 1u) << 5);
}

// 1- and 2-byte nodes.  Each lane owns one word and builds its 32 nodes in
// its own shared-memory row: nodes whose six neighbours are all solid and
// that carry no material (id 27) come from a bit expansion, and only the
// remaining set bits (solid next to empty, surface nodes) are visited one by
// one.  The warp's 32 rows are then stored as one contiguous span.
template <int K>
__global__ void __launch_bounds__(256) emitNarrowKernel(EmitArgs a) {
    typedef NodeT<K> NT;
    static_assert(NT::bytes <= 2, "narrow nodes only");
    constexpr int NB = NT::bytes;
    constexpr int WB = 32 * NB;                  // bytes of one word's nodes
    constexpr int CH = WB / 16;                  // 16-byte chunks per word
    constexpr int PITCH = (CH + 1) * 16;         // padded smem row (conflict-free)
    __shared__ __align__(16) uint8_t stage[8][32 * PITCH];
    __shared__ uint8_t lut[64];
    if (threadIdx.x < 64) lut[threadIdx.x] = kOrientTable[threadIdx.x];
    __syncthreads();
    const PassGeom& g = a.g;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nWords = g.ipx * g.AY * g.AZ;
    uint8_t* my = stage[warp] + lane * PITCH;
    const uint32_t v27 = (uint32_t)NT::pack(27u, 0u, 0.0f);
    for (uint32_t wbase = (blockIdx.x * 8u + warp) * 32u; wbase < nWords; wbase += gridDim.x * 8u * 32u) {
        const uint32_t w = wbase + lane;
        WordNbrs n{};
        if (w < nWords) n = loadNbrs<K>(a, w);
        const uint32_t interior = n.c & n.L & n.R & n.In & n.Out & n.Dn & n.Up & ~n.s0;
        uint32_t rest = (n.c & ~interior) | n.s0;
        uint32_t v[CH * 4];
        if (interior == 0u) {
#pragma unroll
            for (int i = 0; i < CH * 4; ++i) v[i] = 0u;
        } else if (interior == 0xFFFFFFFFu) {
            const uint32_t rep = NB == 1 ? v27 * 0x01010101u : v27 * 0x00010001u;
#pragma unroll
            for (int i = 0; i < CH * 4; ++i) v[i] = rep;
        } else {
#pragma unroll
            for (int i = 0; i < CH * 4; ++i) {
                uint32_t x = 0u;
#pragma unroll
                for (int j = 0; j < 4 / NB; ++j) {
                    const uint32_t b = (uint32_t)(i * (4 / NB) + j);
                    x |= ((interior >> (31u - b)) & 1u) * (v27 << (8 * NB * j));
                }
                v[i] = x;
            }
        }
#pragma unroll
        for (int i = 0; i < CH; ++i)
            *reinterpret_cast<uint4*>(my + 16 * i) = make_uint4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
        if (rest) {
            const uint32_t rank0 = n.s0 ? __ldg(a.ranks + w) : 0u;
            do {
                const uint32_t b = __clz(rest);        // node index in the word
                const uint32_t q = 31u - b;           // its bit
                uint32_t bid = 0u, mat = 0u;
                if ((n.c >> q) & 1u) bid = lut[permOf(n, q)];
                if ((n.s0 >> q) & 1u) {
                    const uint32_t r = rank0 + (b ? __popc(n.s0 >> (32u - b)) : 0u);
                    mat = NT::keyMat(reinterpret_cast<const uint32_t*>(a.keys)[r]);
                }
                const uint32_t nv = (uint32_t)NT::pack(bid, mat, 0.0f);
                if (NB == 1) my[b] = (uint8_t)nv;
                else reinterpret_cast<uint16_t*>(my)[b] = (uint16_t)nv;
                rest &= ~(0x80000000u >> b);
            } while (rest);
        }
        __syncwarp();
        const uint32_t wend = wbase + 32u <= nWords ? 32u : nWords - wbase;
        uint4* out = reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(a.nodes) + (size_t)wbase * WB);
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
__global__ void __launch_bounds__(256) emitPartialKernel(EmitArgs a) {
    typedef NodeT<kPartial> NT;
    __shared__ uint8_t lut[64];
    if (threadIdx.x < 64) lut[threadIdx.x] = kOrientTable[threadIdx.x];
    __syncthreads();
    const PassGeom& g = a.g;
    const uint32_t nWords = g.ipx * g.AY * g.AZ;
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < nWords; w += gridDim.x * blockDim.x) {
        const WordNbrs n = loadNbrs<kPartial>(a, w);
        uint4* out = reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(a.nodes) + (size_t)w * 32 * 8);
        if ((n.c | n.s0 | n.f0) == 0u) {
#pragma unroll
            for (int i = 0; i < 16; ++i) out[i] = make_uint4(0, 0, 0, 0);
            continue;
        }
        const uint32_t rank0 = n.s0 ? __ldg(a.ranks + w) : 0u;
        uint32_t matRank = rank0;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            uint32_t v32[4];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const uint32_t b = 2 * i + j, q = 31u - b;
                uint32_t bid = 0, mat = 0;
                if ((n.c >> q) & 1u) bid = lut[permOf(n, q)];
                if ((n.s0 >> q) & 1u) {
                    mat = NT::keyMat(reinterpret_cast<const unsigned long long*>(a.keys)[matRank]);
                    ++matRank;
                }
                const float r = ((n.f0 >> q) & 1u) && !((n.s0 >> q) & 1u) ? 1.0f : 0.0f;
                const uint64_t nv = NT::pack(bid, mat, r);
                v32[2 * j] = (uint32_t)nv;
                v32[2 * j + 1] = (uint32_t)(nv >> 32);
            }
            out[i] = make_uint4(v32[0], v32[1], v32[2], v32[3]);
        }
    }
}

struct FccArgs {
    const uint32_t* fill[4];
    const uint32_t* surf[4];
    uint64_t surfWordBase[4];   // word offset of surf[g] in the rank space
    const uint32_t* ranks;
    const void* keys;
    void* nodes;
    PassGeom g;
    int materials;
};

// Node emission, FCC lattices (convertToFCCGrid + calculateFCCBoundaries,
// src/voxelizer.cu:1710-1776, 1929-2048).  FCC node (X, y, Z) belongs to
// sub-lattice 1 + (X & 1) + 2 * (Z & 1) at voxel (X / 2, y, Z / 2); its id is
// the 12-bit mask of solid FCC neighbours.  The neighbour relation is
// symmetric, so the reference's in-place pass equals this snapshot
// evaluation.
__device__ __forceinline__ uint32_t fccSolid(const FccArgs& A, uint32_t X2, uint32_t y, uint32_t Z2) {
    const PassGeom& g = A.g;
    const int gt = (int)(X2 & 1u) + 2 * (int)(Z2 & 1u);
    const uint32_t x = X2 >> 1, z = Z2 >> 1;
    const size_t w = ((size_t)z * g.AY + y) * g.ipx + (x >> 5);
    uint32_t word = __ldg(A.fill[gt] + w);
    if (A.materials) word |= __ldg(A.surf[gt] + w);
    return (word >> (31u - (x & 31u))) & 1u;
}

template <int K>
__global__ void emitFccKernel(FccArgs A) {
    typedef NodeT<K> NT;
    constexpr int GN = 16 / NT::bytes;
    const PassGeom& g = A.g;
    const uint32_t NX = 2 * g.X, NY = g.AY, NZ = 2 * g.AZ;
    const uint32_t groupsPerRow = NX / GN;
    const uint64_t nGroups = (uint64_t)groupsPerRow * NY * NZ;
    for (uint64_t gi = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gi < nGroups;
         gi += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t row = gi / groupsPerRow;
        const uint32_t X0 = (uint32_t)(gi % groupsPerRow) * GN;
        const uint32_t y = (uint32_t)(row % NY), Z2 = (uint32_t)(row / NY);
        uint4 outv = make_uint4(0, 0, 0, 0);
#pragma unroll
        for (int n = 0; n < GN; ++n) {
            const uint32_t X2 = X0 + n;
            const int gt = (int)(X2 & 1u) + 2 * (int)(Z2 & 1u);
            const uint32_t x = X2 >> 1, z = Z2 >> 1;
            const size_t w = ((size_t)z * g.AY + y) * g.ipx + (x >> 5);
            const uint32_t q = 31u - (x & 31u);
            const uint32_t fb = (__ldg(A.fill[gt] + w) >> q) & 1u;
            const uint32_t sw = A.materials ? __ldg(A.surf[gt] + w) : 0u;
            const uint32_t sb = (sw >> q) & 1u;
            uint32_t bid = 0;
            if (fb | sb) {
                const bool left = X2 > 0, right = X2 < NX - 1, in = y > 0, out = y < NY - 1;
                const bool down = Z2 > 0, up = Z2 < NZ - 1, xe = ((X2 + Z2) & 1u) == 0;
                const uint32_t ym = xe ? y - 1 : y;   // y - xEven
                const uint32_t yp = xe ? y : y + 1;   // y + !xEven
                const bool cIn = (xe && in) || !xe, cOut = (!xe && out) || xe;
                if (down && cIn && fccSolid(A, X2, ym, Z2 - 1)) bid |= 1u;
                if (down && left && fccSolid(A, X2 - 1, y, Z2 - 1)) bid |= 2u;
                if (down && right && fccSolid(A, X2 + 1, y, Z2 - 1)) bid |= 4u;
                if (down && cOut && fccSolid(A, X2, yp, Z2 - 1)) bid |= 8u;
                if (left && cIn && fccSolid(A, X2 - 1, ym, Z2)) bid |= 16u;
                if (right && cIn && fccSolid(A, X2 + 1, ym, Z2)) bid |= 32u;
                if (left && cOut && fccSolid(A, X2 - 1, yp, Z2)) bid |= 64u;
                if (right && cOut && fccSolid(A, X2 + 1, yp, Z2)) bid |= 128u;
                if (up && cIn && fccSolid(A, X2, ym, Z2 + 1)) bid |= 256u;
                if (up && left && fccSolid(A, X2 - 1, y, Z2 + 1)) bid |= 512u;
                if (up && right && fccSolid(A, X2 + 1, y, Z2 + 1)) bid |= 1024u;
                if (up && cOut && fccSolid(A, X2, yp, Z2 + 1)) bid |= 2048u;
            }
            uint32_t mat = 0;
            if (sb) {
                const uint32_t b = x & 31u;
                const uint32_t r = __ldg(A.ranks + A.surfWordBase[gt] + w) + (b ? __popc(sw >> (32 - b)) : 0u);
                mat = NT::keyMat(reinterpret_cast<const uint32_t*>(A.keys)[r]);
            }
            const uint64_t val = NT::pack(bid, mat, 0.0f);
            if (NT::bytes == 2) reinterpret_cast<uint16_t*>(&outv)[n] = (uint16_t)val;
            else reinterpret_cast<uint32_t*>(&outv)[n] = (uint32_t)val;
        }
        reinterpret_cast<uint4*>(A.nodes)[(size_t)gi] = outv;
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

void launch_prune(uint32_t* solid, const uint32_t* fill, const uint32_t* surf, const uint8_t* yLater,
                  const uint8_t* zLater, PassGeom g, SplitYZ split, uint32_t* changed, cudaStream_t s,
                  uint32_t* launches) {
    const uint64_t n = (uint64_t)(split.y1 - split.y0) * (split.z1 - split.z0) * g.ipx;
    pruneKernel<<<gridFor(n, 256), 256, 0, s>>>(solid, fill, surf, yLater, zLater, g, split, changed);
    *launches += 1;
}

void launch_emit_cartesian(int nodeKind, const uint32_t* finalSolid, const uint32_t* fill, const uint32_t* surf,
                           const uint32_t* ranks, const void* keys, PassGeom g, const uint8_t* yLater,
                           const uint8_t* zLater, void* nodes, int materials, cudaStream_t s, uint32_t* launches) {
    EmitArgs a;
    a.fin = finalSolid;
    a.fill = fill;
    a.surf = surf;
    a.ranks = ranks;
    a.keys = keys;
    a.yLater = yLater;
    a.zLater = zLater;
    a.nodes = nodes;
    a.g = g;
    a.materials = materials;
    const uint64_t words = (uint64_t)g.ipx * g.AY * g.AZ;
    const uint32_t grid = gridFor(words, 256, 148u * 16u);
    switch (nodeKind) {
    case kShort: emitNarrowKernel<kShort><<<grid, 256, 0, s>>>(a); break;
    case kLong: emitNarrowKernel<kLong><<<grid, 256, 0, s>>>(a); break;
    default: emitPartialKernel<<<gridFor(words, 256, 148u * 8u), 256, 0, s>>>(a); break;
    }
    *launches += 1;
}

void launch_emit_fcc(int nodeKind, const uint32_t* const* fill, const uint32_t* const* surf,
                     const uint64_t* surfWordBase, const uint32_t* ranks, const void* keys, PassGeom g, void* nodes,
                     int materials, cudaStream_t s, uint32_t* launches) {
    FccArgs A;
    for (int i = 0; i < 4; ++i) {
        A.fill[i] = fill[i];
        A.surf[i] = surf[i];
        A.surfWordBase[i] = surfWordBase[i];
    }
    A.ranks = ranks;
    A.keys = keys;
    A.nodes = nodes;
    A.g = g;
    A.materials = materials;
    const int bytes = nodeKind == kShortFcc ? 2 : 4;
    const uint64_t groups = (uint64_t)(2 * g.X) * g.AY * (2 * g.AZ) * bytes / 16;
    const uint32_t grid = gridFor(groups, 256, 148u * 64u);
    if (nodeKind == kShortFcc) emitFccKernel<kShortFcc><<<grid, 256, 0, s>>>(A);
    else emitFccKernel<kLongFcc><<<grid, 256, 0, s>>>(A);
    *launches += 1;
}

}  // namespace vxb
