// Slices along x (voxelizeSlice with direction 0, hakarlss/Voxelizer
// src/host_side.cpp:704-718, 1144-1236, 3261-3309): the reference rotates the
// mesh 90 degrees about z, slices the rotated grid along y, and un-rotates
// the node array before it computes the boundary ids.  Kernels here:
//  * the vertex rotation (rotateVertices, in double, rounded to float);
//  * the node array as it stands before fillNodeList2 (constructNodeList2
//    plus the surface pass: bid = solid bit, material and ratio of the
//    surface winner) for the rotated slice;
//  * unRotateNodes (src/voxelizer.cu:2061-2124), the boundary-id passes of
//    fillNodeList2 (1790-1913) over the un-rotated array, in place, one yz
//    subspace at a time until no node loses its id, and zeroPadding
//    (4811-4844);
//  * for FCC lattices, unRotateNodes' FCC branch, calculateFCCBoundaries
//    (1929-2048) on the un-rotated array and zeroPadding's FCC branch.
// Slices are small (three node layers), so these are plain node-per-thread
// kernels.

#include "vxb_common.cuh"
#include "vxb_device.cuh"
#include "vxb_kernels.cuh"
#include "vxb_ratio.cuh"

#include <type_traits>

namespace vxb {

using namespace detail;

namespace {

__global__ void rotateKernel(const float* __restrict__ V, float* __restrict__ R, uint32_t n, double a, double b) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x = (double)V[3 * (size_t)i], y = (double)V[3 * (size_t)i + 1];
        R[3 * (size_t)i] = __double2float_rn(__dsub_rn(a, y));
        R[3 * (size_t)i + 1] = __double2float_rn(__dadd_rn(b, x));
        R[3 * (size_t)i + 2] = V[3 * (size_t)i + 2];
    }
}

// Nodes before the boundary ids, one thread per 32-node word of the unit.
template <int K>
__global__ void emitRawKernel(Batch b, uint64_t totalWords, const uint32_t* __restrict__ fill,
                              const uint32_t* __restrict__ surf, const WordRank* __restrict__ ranks, const void* keys,
                              uint32_t keysCap) {
    typedef NodeT<K> NT;
    for (uint64_t gw = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gw < totalWords;
         gw += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t u = unitOf(b.wordBase, b.nUnits, gw);
        const Unit& U = b.units[u];
        const uint32_t w = (uint32_t)(gw - U.wordBase);
        if (w >= U.g.ipx * U.g.AY * U.g.AZ) continue;
        const uint32_t f = __ldg(fill + U.wordBase + w);
        const uint32_t s = U.materials ? __ldg(surf + U.wordBase + w) : 0u;
        uint32_t rank = s ? ranks[U.wordBase + w].rank : 0u;
        const int x0 = (int)(w % U.g.ipx) * 32, y0 = (int)(w / U.g.ipx % U.g.AY), z0 = (int)(w / U.g.ipx / U.g.AY);
        uint8_t* out = static_cast<uint8_t*>(U.out) + (size_t)w * 32 * NT::bytes;
        for (uint32_t bt = 0; bt < 32; ++bt) {
            const uint32_t q = 31u - bt;
            const uint32_t fb = (f >> q) & 1u, sb = (s >> q) & 1u;
            uint32_t mat = 0;
            float r = fb ? 1.0f : 0.0f;
            if (sb) {
                if (rank < keysCap) {
                    if (NT::bytes == 8) {
                        const uint64_t key = reinterpret_cast<const unsigned long long*>(keys)[rank];
                        mat = NT::keyMat(key);
                        r = ratio::nodeRatio(U.V, U.I, (uint32_t)key, (uint32_t)(key >> 40), x0 + (int)bt, y0, z0,
                                             detail::F3{U.g.mnf[0], U.g.mnf[1], U.g.mnf[2]}, U.g.df);
                    } else {
                        mat = NT::keyMat(reinterpret_cast<const uint32_t*>(keys)[rank]);
                    }
                }
                ++rank;
            }
            const uint64_t nv = NT::pack((fb | sb) ? 1u : 0u, mat, r);
            for (int k = 0; k < NT::bytes; ++k) out[bt * NT::bytes + k] = (uint8_t)(nv >> (8 * k));
        }
    }
}

// unRotateNodes: node (x, y, z) of the rotated X x Y x Z array goes to
// (y, X - 1 - x, z) of the Y x X x Z array.
__global__ void unrotateKernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, uint32_t X, uint32_t Y,
                               uint32_t Z, uint32_t nb) {
    const uint64_t n = (uint64_t)X * Y * Z;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)(i % X), y = (uint32_t)(i / X % Y), z = (uint32_t)(i / X / Y);
        const uint64_t j = (uint64_t)X * Y * z + (uint64_t)Y * (X - 1 - x) + y;
        for (uint32_t k = 0; k < nb; ++k) out[j * nb + k] = in[i * nb + k];
    }
}

// One fillNodeList2 pass over subspace [y0, y1) x [z0, z1) of an X x Y x Z
// array, in place: solid nodes get the id of their neighbour pattern; a node
// whose pattern has no id loses its solidity and sets *changed.  The id is
// byte 0 of every node layout (the low 5 bits of a ShortNode).
__global__ void idPassKernel(uint8_t* nodes, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nb, uint32_t idMask,
                             uint32_t y0, uint32_t y1, uint32_t z0, uint32_t z1, uint32_t* changed) {
    __shared__ uint8_t lut[64];
    if (threadIdx.x < 64) lut[threadIdx.x] = kOrientTable[threadIdx.x];
    __syncthreads();
    const uint64_t n = (uint64_t)X * (y1 - y0) * (z1 - z0);
    const uint64_t px = nb, py = (uint64_t)X * nb, pz = (uint64_t)X * Y * nb;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)(i % X);
        const uint32_t y = y0 + (uint32_t)(i / X % (y1 - y0)), z = z0 + (uint32_t)(i / X / (y1 - y0));
        uint8_t* p = nodes + ((uint64_t)z * Y * X + (uint64_t)y * X + x) * nb;
        const uint32_t b0 = p[0];
        if ((b0 & idMask) == 0) continue;
        uint32_t perm = 0;
        if (x > 0 && (p[-(int64_t)px] & idMask)) perm += 1;
        if (x + 1 < X && (p[px] & idMask)) perm += 2;
        if (y > 0 && (*(p - py) & idMask)) perm += 4;
        if (y + 1 < Y && (p[py] & idMask)) perm += 8;
        if (z > 0 && (*(p - pz) & idMask)) perm += 16;
        if (z + 1 < Z && (p[pz] & idMask)) perm += 32;
        const uint32_t id = lut[perm];
        p[0] = (uint8_t)((b0 & ~idMask) | id);
        if (id == 0) atomicOr(changed, 1u);
    }
}

// zeroPadding: every node on a face of the array becomes zero; FCC arrays
// lose two node layers at the x and z faces (src/voxelizer.cu:4811-4844).
__global__ void zeroFacesKernel(uint8_t* nodes, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nb, uint32_t fcc) {
    const uint64_t n = (uint64_t)X * Y * Z;
    const uint32_t w = fcc ? 2u : 1u;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)(i % X), y = (uint32_t)(i / X % Y), z = (uint32_t)(i / X / Y);
        if (x < w || x + w >= X || y == 0 || y + 1 == Y || z < w || z + w >= Z)
            for (uint32_t k = 0; k < nb; ++k) nodes[i * nb + k] = 0;
    }
}

// unRotateNodes, FCC branch (src/voxelizer.cu:2104-2110): node (x, y, z) of
// the turned X x Y x Z FCC array goes to (2y + (x + z + 1) % 2, X / 2 - 1 -
// x / 2, z) of the 2Y x X/2 x Z array.
__global__ void unrotateFccKernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, uint32_t X, uint32_t Y,
                                  uint32_t Z, uint32_t nb) {
    const uint64_t n = (uint64_t)X * Y * Z;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)(i % X), y = (uint32_t)(i / X % Y), z = (uint32_t)(i / X / Y);
        const uint32_t nx = 2 * y + (x + z + 1) % 2, ny = X / 2 - 1 - x / 2;
        const uint64_t j = (uint64_t)X * Y * z + (uint64_t)(2 * Y) * ny + nx;
        for (uint32_t k = 0; k < nb; ++k) out[j * nb + k] = in[i * nb + k];
    }
}

// calculateFCCBoundaries (src/voxelizer.cu:1929-2048) in place over an X x Y
// x Z FCC node array of 2-byte (12-bit id) or 4-byte (16-bit id) nodes: a
// solid node's id becomes the mask of its solid FCC neighbours.  A node
// whose mask is zero has no solid neighbour, so no other node reads it; the
// in-place pass equals a snapshot evaluation.
template <int NB>
__global__ void fccBoundaryKernel(uint8_t* nodes, uint32_t X, uint32_t Y, uint32_t Z) {
    typedef typename std::conditional<NB == 2, uint16_t, uint32_t>::type T;
    constexpr uint32_t kId = NB == 2 ? 0x0FFFu : 0xFFFFu;
    T* v = reinterpret_cast<T*>(nodes);
    const uint64_t n = (uint64_t)X * Y * Z;
    const uint64_t px = 1, py = X, pz = (uint64_t)X * Y;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const T cur = v[i];
        if ((cur & kId) == 0) continue;
        const uint32_t x = (uint32_t)(i % X), y = (uint32_t)(i / X % Y), z = (uint32_t)(i / X / Y);
        const bool left = x > 0, right = x + 1 < X, in = y > 0, out = y + 1 < Y, down = z > 0, up = z + 1 < Z;
        const bool xe = ((x + z) & 1u) == 0;
        const bool cIn = (xe && in) || !xe, cOut = (!xe && out) || xe;
        const uint64_t ye = xe ? py : 0, yo = xe ? 0 : py;
        auto on = [&](uint64_t j) { return (v[j] & kId) != 0; };
        uint32_t b = 0;
        if (down && cIn && on(i - pz - ye)) b |= 1u;
        if (down && left && on(i - pz - px)) b |= 2u;
        if (down && right && on(i - pz + px)) b |= 4u;
        if (down && cOut && on(i - pz + yo)) b |= 8u;
        if (left && cIn && on(i - px - ye)) b |= 16u;
        if (right && cIn && on(i + px - ye)) b |= 32u;
        if (left && cOut && on(i - px + yo)) b |= 64u;
        if (right && cOut && on(i + px + yo)) b |= 128u;
        if (up && cIn && on(i + pz - ye)) b |= 256u;
        if (up && left && on(i + pz - px)) b |= 512u;
        if (up && right && on(i + pz + px)) b |= 1024u;
        if (up && cOut && on(i + pz + yo)) b |= 2048u;
        v[i] = (T)((cur & ~(T)kId) | (T)b);
    }
}

}  // namespace

void launch_rotate_vertices(const float* V, float* R, uint32_t n, double a, double b, cudaStream_t s,
                            uint32_t* launches) {
    rotateKernel<<<gridFor(n, 256, 148u * 8u), 256, 0, s>>>(V, R, n, a, b);
    *launches += 1;
}

void launch_emit_raw(int nodeKind, const Batch& b, uint64_t totalWords, const uint32_t* fill, const uint32_t* surf,
                     const WordRank* ranks, const void* keys, uint32_t keysCap, cudaStream_t s, uint32_t* launches) {
    const uint32_t grid = gridFor(totalWords, 128, 148u * 8u);
    switch (nodeKind) {
    case kShort: emitRawKernel<kShort><<<grid, 128, 0, s>>>(b, totalWords, fill, surf, ranks, keys, keysCap); break;
    case kLong: emitRawKernel<kLong><<<grid, 128, 0, s>>>(b, totalWords, fill, surf, ranks, keys, keysCap); break;
    default: emitRawKernel<kPartial><<<grid, 128, 0, s>>>(b, totalWords, fill, surf, ranks, keys, keysCap); break;
    }
    *launches += 1;
}

void launch_unrotate(const void* in, void* out, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nodeBytes,
                     cudaStream_t s, uint32_t* launches) {
    unrotateKernel<<<gridFor((uint64_t)X * Y * Z, 256, 148u * 8u), 256, 0, s>>>(
        static_cast<const uint8_t*>(in), static_cast<uint8_t*>(out), X, Y, Z, nodeBytes);
    *launches += 1;
}

void launch_id_pass(void* nodes, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nodeBytes, uint32_t idMask,
                    uint32_t y0, uint32_t y1, uint32_t z0, uint32_t z1, uint32_t* changed, cudaStream_t s,
                    uint32_t* launches) {
    idPassKernel<<<gridFor((uint64_t)X * (y1 - y0) * (z1 - z0), 256, 148u * 8u), 256, 0, s>>>(
        static_cast<uint8_t*>(nodes), X, Y, Z, nodeBytes, idMask, y0, y1, z0, z1, changed);
    *launches += 1;
}

void launch_zero_faces(void* nodes, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nodeBytes, bool fcc, cudaStream_t s,
                       uint32_t* launches) {
    zeroFacesKernel<<<gridFor((uint64_t)X * Y * Z, 256, 148u * 8u), 256, 0, s>>>(static_cast<uint8_t*>(nodes), X, Y,
                                                                                  Z, nodeBytes, fcc ? 1u : 0u);
    *launches += 1;
}

void launch_unrotate_fcc(const void* in, void* out, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nodeBytes,
                         cudaStream_t s, uint32_t* launches) {
    unrotateFccKernel<<<gridFor((uint64_t)X * Y * Z, 256, 148u * 8u), 256, 0, s>>>(
        static_cast<const uint8_t*>(in), static_cast<uint8_t*>(out), X, Y, Z, nodeBytes);
    *launches += 1;
}

void launch_fcc_boundaries(void* nodes, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nodeBytes, cudaStream_t s,
                           uint32_t* launches) {
    const uint32_t grid = gridFor((uint64_t)X * Y * Z, 256, 148u * 8u);
    if (nodeBytes == 2) fccBoundaryKernel<2><<<grid, 256, 0, s>>>(static_cast<uint8_t*>(nodes), X, Y, Z);
    else fccBoundaryKernel<4><<<grid, 256, 0, s>>>(static_cast<uint8_t*>(nodes), X, Y, Z);
    *launches += 1;
}

}  // namespace vxb
