// vox::Voxelizer<Node>: source-compatible C++ front end of the B200
// voxelizer, for code written against hakarlss/Voxelizer's public API
// (include/voxelizer.h and include/node_types.h of the reference).  Class,
// member and node names, argument order, defaults, node byte layouts and
// ownership rules are the reference's; the work runs through the C ABI in
// vxb.h (libvxb.so).
//
// Ownership (as in the reference, src/host_side.cpp:3561-3625):
//  * *ToRAM calls return host arrays allocated with new[]; the caller
//    delete[]s them (NodePointer::ptr or ::vptr).
//  * voxelize / voxelizeToNodes return device pointers allocated with
//    cudaMalloc on device 0; the caller cudaFree()s them.
// One GPU: devConfig (dy, dz) partitions the grid as the reference's
// devices do (each partition voxelized with its overlap rows, faces zeroed in
// node output) but runs every partition on this voxelizer's device; the
// NodePointers carry each partition's dim and loc.  Inside
// simulateMultidevice the results are host arrays (new[]), as the
// reference's collectData uploads them.  Slices are provided along x, y and
// z (devConfig 1); slices along x turn the mesh as the reference does, but
// leave the voxelizer's stored mesh as it is.
#ifndef VOX_VOXELIZER_B200_H
#define VOX_VOXELIZER_B200_H

#include <cuda_runtime.h>
#include <vector_functions.h>
#include <vector_types.h>

#include <climits>
#include <cstdint>
#include <exception>
#include <functional>
#include <string>
#include <vector>

#include "../vxb.h"

namespace vox {

typedef unsigned int uint;
typedef uint16_t ushort;
typedef uint8_t uchar;
typedef uint32_t VoxInt;

// Error type thrown by every member below (what() carries the message).
class Exception : public std::exception {
public:
    explicit Exception(std::string message) throw() : msg(message) {}
    explicit Exception(char const* message) throw() : msg(message) {}
    ~Exception() throw() {}
    const char* what() const throw() { return msg.c_str(); }
private:
    const std::string msg;
};

// ---------------------------------------------------------------------------
// Node layouts.  Byte layout and accessors match include/node_types.h of the
// reference so that node arrays can be exchanged with code built against it.

// 1 byte: boundary id in bits 0-4, material in bits 5-7.
class ShortNode {
public:
    __host__ __device__ ShortNode() : bim(0) {}
    __host__ __device__ ShortNode(uchar b) : bim(b) {}
    __host__ __device__ ShortNode(uchar b, uchar m) { set(m, b); }
    __host__ __device__ uchar mat() const { return bim >> 5; }
    __host__ __device__ uchar bid() const { return bim & 31; }
    __host__ __device__ float r() const { return 0.0f; }
    __host__ __device__ void mat(uchar m) { bim = (uchar)((m << 5) | (bim & 31)); }
    __host__ __device__ void bid(uchar b) { bim = (uchar)((b & 31) | (bim & 224)); }
    __host__ __device__ void r(float) {}
    __host__ __device__ void set(uchar m, uchar b) { bim = (uchar)((m << 5) | (b & 31)); }
    static __host__ __device__ uchar maxMat() { return 7; }
    static __host__ __device__ uchar maxBid() { return 31; }
    static __host__ __device__ bool hasRatio() { return false; }
    static __host__ __device__ bool isFCCNode() { return false; }
    static const int kind = VXB_SHORT_NODE;
private:
    uchar bim;
};

// 2 bytes: boundary id, material.
class LongNode {
public:
    __host__ __device__ LongNode() : _bid(0), _mat(0) {}
    __host__ __device__ LongNode(uchar b) : _bid(b), _mat(0) {}
    __host__ __device__ LongNode(uchar b, uchar m) : _bid(b), _mat(m) {}
    __host__ __device__ uchar mat() const { return _mat; }
    __host__ __device__ uchar bid() const { return _bid; }
    __host__ __device__ float r() const { return 0.0f; }
    __host__ __device__ void mat(uchar m) { _mat = m; }
    __host__ __device__ void bid(uchar b) { _bid = b; }
    __host__ __device__ void r(float) {}
    __host__ __device__ void set(uchar m, uchar b) { _mat = m; _bid = b; }
    static __host__ __device__ uchar maxMat() { return UCHAR_MAX; }
    static __host__ __device__ uchar maxBid() { return UCHAR_MAX; }
    static __host__ __device__ bool hasRatio() { return false; }
    static __host__ __device__ bool isFCCNode() { return false; }
    static const int kind = VXB_LONG_NODE;
private:
    uchar _bid;
    uchar _mat;
};

// 8 bytes: boundary id, material, 2 padding bytes, solid volume ratio.
class PartialNode {
public:
    __host__ __device__ PartialNode() : _bid(0), _mat(0), _r(0.0f) {}
    __host__ __device__ PartialNode(uchar b) : _bid(b), _mat(0), _r(0.0f) {}
    __host__ __device__ PartialNode(uchar b, uchar m) : _bid(b), _mat(m), _r(0.0f) {}
    __host__ __device__ PartialNode(uchar b, uchar m, float ratio) : _bid(b), _mat(m), _r(ratio) {}
    __host__ __device__ uchar mat() const { return _mat; }
    __host__ __device__ uchar bid() const { return _bid; }
    __host__ __device__ float r() const { return _r; }
    __host__ __device__ void mat(uchar m) { _mat = m; }
    __host__ __device__ void bid(uchar b) { _bid = b; }
    __host__ __device__ void r(float ratio) { _r = ratio; }
    __host__ __device__ void set(uchar m, uchar b) { _mat = m; _bid = b; }
    __host__ __device__ void set(uchar m, uchar b, float ratio) { _mat = m; _bid = b; _r = ratio; }
    static __host__ __device__ uchar maxMat() { return UCHAR_MAX; }
    static __host__ __device__ uchar maxBid() { return UCHAR_MAX; }
    static __host__ __device__ bool hasRatio() { return true; }
    static __host__ __device__ bool isFCCNode() { return false; }
    static const int kind = VXB_PARTIAL_NODE;
private:
    uchar _bid;
    uchar _mat;
    float _r;
};

// 2 bytes: 12-bit FCC neighbour mask, 4-bit material.
class ShortFCCNode {
public:
    __host__ __device__ ShortFCCNode() : bim(0) {}
    __host__ __device__ ShortFCCNode(ushort b) : bim(b) {}
    __host__ __device__ ShortFCCNode(ushort b, ushort m) { set(m, b); }
    __host__ __device__ ushort mat() const { return bim >> 12; }
    __host__ __device__ ushort bid() const { return bim & 4095; }
    __host__ __device__ float r() const { return 0.0f; }
    __host__ __device__ void mat(ushort m) { bim = (ushort)((m << 12) | (bim & 4095)); }
    __host__ __device__ void bid(ushort b) { bim = (ushort)((b & 4095) | (bim & 61440)); }
    __host__ __device__ void r(float) {}
    __host__ __device__ void set(ushort m, ushort b) { bim = (ushort)((m << 12) | (b & 4095)); }
    static __host__ __device__ ushort maxMat() { return 15; }
    static __host__ __device__ bool hasRatio() { return false; }
    static __host__ __device__ bool isFCCNode() { return true; }
    static const int kind = VXB_SHORT_FCC_NODE;
private:
    ushort bim;
};

// 4 bytes: uint16 FCC neighbour mask, material, 1 padding byte.
class LongFCCNode {
public:
    __host__ __device__ LongFCCNode() : _bid(0), _mat(0) {}
    __host__ __device__ LongFCCNode(ushort b) : _bid(b), _mat(0) {}
    __host__ __device__ LongFCCNode(ushort b, uchar m) : _bid(b), _mat(m) {}
    __host__ __device__ uchar mat() const { return _mat; }
    __host__ __device__ ushort bid() const { return _bid; }
    __host__ __device__ float r() const { return 0.0f; }
    __host__ __device__ void mat(uchar m) { _mat = m; }
    __host__ __device__ void bid(ushort b) { _bid = b; }
    __host__ __device__ void r(float) {}
    __host__ __device__ void set(uchar m, ushort b) { _bid = b; _mat = m; }
    static __host__ __device__ ushort maxMat() { return UCHAR_MAX; }
    static __host__ __device__ bool hasRatio() { return false; }
    static __host__ __device__ bool isFCCNode() { return true; }
    static const int kind = VXB_LONG_FCC_NODE;
private:
    ushort _bid;
    uchar _mat;
};

// Result of a voxelization (include/voxelizer.h:674-684 of the reference).
template <class Node>
struct NodePointer {
    union {
        Node* ptr;     // node grid
        VoxInt* vptr;  // plain bit array
    };
    int dev;
    uint3 dim;
    uint3 loc;
};

template <class Node = ShortNode>
class Voxelizer {
public:
    Voxelizer(float const* _vertices, uint const* _indices, uint _nrOfVertices, uint _nrOfTriangles);
    Voxelizer(float const* _vertices, uint const* _indices, uchar const* _materials, uint _nrOfVertices,
              uint _nrOfTriangles, uint _nrOfUniqueMaterials);
    ~Voxelizer();

    std::vector<NodePointer<Node> > voxelize(uint maxDimension = 256, uint2 devConfig = make_uint2(1, 1),
                                             uint3 voxSplitRes = make_uint3(1024, 512, 512));
    std::vector<NodePointer<Node> > voxelize(double cubeLength, uint2 devConfig = make_uint2(1, 1),
                                             uint3 voxSplitRes = make_uint3(1024, 512, 512));
    NodePointer<Node> voxelizeToRAM(uint maxDimension = 256, uint3 voxSplitRes = make_uint3(1024, 512, 512));
    NodePointer<Node> voxelizeToRAM(double cubeLength, uint3 voxSplitRes = make_uint3(1024, 512, 512));
    std::vector<NodePointer<Node> > voxelizeToNodes(uint maxDimension = 256, uint2 devConfig = make_uint2(1, 1),
                                                    uint3 voxSplitRes = make_uint3(1024, 512, 512),
                                                    uint3 matSplitRes = make_uint3(512, 512, 512));
    std::vector<NodePointer<Node> > voxelizeToNodes(double cubeLength, uint2 devConfig = make_uint2(1, 1),
                                                    uint3 voxSplitRes = make_uint3(1024, 512, 512),
                                                    uint3 matSplitRes = make_uint3(512, 512, 512));
    NodePointer<Node> voxelizeToNodesToRAM(uint maxDimension = 256, uint3 voxSplitRes = make_uint3(1024, 512, 512),
                                           uint3 matSplitRes = make_uint3(512, 512, 512));
    NodePointer<Node> voxelizeToNodesToRAM(double cubeLength, uint3 voxSplitRes = make_uint3(1024, 512, 512),
                                           uint3 matSplitRes = make_uint3(512, 512, 512));

    // Slices (src/host_side.cpp:1927-2262): direction 0 (x), 1 (y) or 2
    // (z); a three-layer node array whose middle layer is slice `slice`.
    std::vector<NodePointer<Node> > voxelizeSlice(uint maxDimension, int direction, uint slice, uint devConfig = 1,
                                                  uint2 voxSplitRes = make_uint2(1024, 512),
                                                  uint2 matSplitRes = make_uint2(512, 512));
    std::vector<NodePointer<Node> > voxelizeSlice(double cubeLength, int direction, uint slice, uint devConfig = 1,
                                                  uint2 voxSplitRes = make_uint2(1024, 512),
                                                  uint2 matSplitRes = make_uint2(512, 512));
    NodePointer<Node> voxelizeSliceToRAM(uint maxDimension, int direction, uint slice,
                                         uint2 voxSplitRes = make_uint2(1024, 512),
                                         uint2 matSplitRes = make_uint2(512, 512));
    NodePointer<Node> voxelizeSliceToRAM(double cubeLength, int direction, uint slice,
                                         uint2 voxSplitRes = make_uint2(1024, 512),
                                         uint2 matSplitRes = make_uint2(512, 512));

    double getVoxelLength() const throw() { return voxelLength; }
    double3 getMinVertex() const throw() { return minVertex; }
    double3 getMaxVertex() const throw() { return maxVertex; }
    uint3 getResolution() const throw() { return resolution; }
    std::vector<float> getVertices() const throw() { return vertices; }
    std::vector<uint> getIndices() const throw() { return indices; }
    uint getNrOfTriangles() const throw() { return nrOfTriangles; }

    void setMaterials(uchar const* _materials, uint _nrOfUniqueMaterials);
    void setMaterialOutput(bool _materials) throw();
    void verboseOutput(bool verbose) throw();
    uint3 getArrayDimensions(uint longestSizeInVoxels, uint maxInternalXSize, bool sliceAlongX);
    uint3 getArrayDimensions(double cubeLength, uint maxInternalXSize, bool sliceAlongX);
    std::vector<NodePointer<Node> > simulateMultidevice(std::function<std::vector<NodePointer<Node> >()> func);

private:
    Voxelizer(const Voxelizer&);
    Voxelizer& operator=(const Voxelizer&);

    NodePointer<Node> run(bool toHost, uint3 voxSplitRes, uint3 matSplitRes);
    std::vector<NodePointer<Node> > runParts(uint2 devConfig, uint3 voxSplitRes, uint3 matSplitRes);
    NodePointer<Node> runSlice(bool toHost, int direction, uint slice, uint2 voxSplitRes, uint2 matSplitRes);
    vxb_request request(uint3 voxSplitRes, uint3 matSplitRes) const;

    vxb_voxelizer* handle;
    std::vector<float> vertices;
    std::vector<uint> indices;
    uint nrOfTriangles;
    // Option state that persists between calls, as in the reference's
    // Options struct (include/host_support.h:39-56).
    bool nodeOutput;
    bool voxelDistanceGiven;
    bool simulate = false;   // inside simulateMultidevice
    uint maxDimensionSetting;
    double voxelLength;
    double3 minVertex, maxVertex;
    uint3 resolution;
};

}  // namespace vox

#endif
