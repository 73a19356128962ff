// Implementation of vox::Voxelizer<Node> (include/vox/voxelizer.h) on top
// of the C ABI.  Control flow per call follows the reference's public
// members in src/host_side.cpp (constructors 29-99, setMaterials 218-243,
// voxelize 562-650, voxelizeToNodes 1734-1814, voxelizeToNodesToRAM
// 1829-1886, voxelizeToRAM 2275-2337, getArrayDimensions 3329-3475,
// collectData 3561-3625), including its option state that persists between
// calls.

#include "vox/voxelizer.h"

#include <cuda_runtime.h>

#include <iostream>
#include <string>

namespace vox {

namespace {

void check(vxb_status rc) {
    if (rc != VXB_OK) throw Exception(std::string(vxb_last_error()));
}

vxb_uint3 u3(uint3 v) { vxb_uint3 r; r.x = v.x; r.y = v.y; r.z = v.z; return r; }

}  // namespace

template <class Node>
Voxelizer<Node>::Voxelizer(float const* _vertices, uint const* _indices, uint _nrOfVertices, uint _nrOfTriangles)
    : handle(nullptr), nrOfTriangles(_nrOfTriangles), nodeOutput(false), voxelDistanceGiven(false),
      maxDimensionSetting(256), voxelLength(0.0) {
    check(vxb_create(&handle, Node::kind, _vertices, _indices, _nrOfVertices, _nrOfTriangles, 0));
    vertices.assign(_vertices, _vertices + 3 * (size_t)_nrOfVertices);
    indices.assign(_indices, _indices + 3 * (size_t)_nrOfTriangles);
    // calculateBoundingBox, src/host_side.cpp:2462-2488
    minVertex = make_double3(0, 0, 0);
    maxVertex = make_double3(0, 0, 0);
    if (_nrOfVertices > 0) {
        double mn[3] = {_vertices[0], _vertices[1], _vertices[2]}, mx[3] = {mn[0], mn[1], mn[2]};
        for (uint i = 1; i < _nrOfVertices; ++i)
            for (int a = 0; a < 3; ++a) {
                if (_vertices[3 * i + a] > mx[a]) mx[a] = _vertices[3 * i + a];
                if (_vertices[3 * i + a] < mn[a]) mn[a] = _vertices[3 * i + a];
            }
        minVertex = make_double3(mn[0], mn[1], mn[2]);
        maxVertex = make_double3(mx[0], mx[1], mx[2]);
    }
    resolution = make_uint3(256, 0, 0);
}

template <class Node>
Voxelizer<Node>::Voxelizer(float const* _vertices, uint const* _indices, uchar const* _materials, uint _nrOfVertices,
                           uint _nrOfTriangles, uint _nrOfUniqueMaterials)
    : Voxelizer(_vertices, _indices, _nrOfVertices, _nrOfTriangles) {
    setMaterials(_materials, _nrOfUniqueMaterials);
}

template <class Node>
Voxelizer<Node>::~Voxelizer() {
    if (handle) vxb_destroy(handle);
}

template <class Node>
void Voxelizer<Node>::setMaterials(uchar const* _materials, uint _nrOfUniqueMaterials) {
    check(vxb_set_materials(handle, _materials, _nrOfUniqueMaterials));
}

template <class Node>
void Voxelizer<Node>::setMaterialOutput(bool _materials) throw() {
    vxb_set_material_output(handle, _materials ? 1 : 0);
}

template <class Node>
void Voxelizer<Node>::verboseOutput(bool verbose) throw() {
    vxb_verbose_output(handle, verbose ? 1 : 0);
}

// One voxelization with the current option state.  As in the reference,
// a cube length given by an earlier call stays in effect
// (voxelDistanceGiven is never cleared, src/host_side.cpp:704-720).
template <class Node>
NodePointer<Node> Voxelizer<Node>::run(bool toHost, uint3 voxSplitRes, uint3 matSplitRes) {
    vxb_request r;
    r.by_cube_length = voxelDistanceGiven ? 1 : 0;
    r.max_dimension = maxDimensionSetting;
    r.cube_length = voxelLength;
    r.vox_split_res = u3(voxSplitRes);
    r.mat_split_res = u3(matSplitRes);
    const int nodes = nodeOutput ? 1 : 0;
    vxb_grid_info gi;
    check(vxb_plan(handle, nodes, &r, &gi));
    NodePointer<Node> res = NodePointer<Node>();
    res.dev = 0;
    res.loc = make_uint3(0, 0, 0);
    res.dim = make_uint3(gi.dim.x, gi.dim.y, gi.dim.z);
    if (toHost) {
        void* host = nodes ? static_cast<void*>(new Node[gi.count]) : static_cast<void*>(new VoxInt[gi.count]);
        vxb_status rc = vxb_voxelize_to_host(handle, nodes, &r, host, gi.bytes, &gi);
        if (rc != VXB_OK) {
            if (nodes) delete[] static_cast<Node*>(host);
            else delete[] static_cast<VoxInt*>(host);
            check(rc);
        }
        if (nodes) res.ptr = static_cast<Node*>(host);
        else res.vptr = static_cast<VoxInt*>(host);
    } else {
        void* dev = nullptr;
        if (cudaMalloc(&dev, gi.bytes) != cudaSuccess) {
            cudaGetLastError();
            throw Exception("cudaMalloc of the result failed");
        }
        vxb_status rc = vxb_voxelize_to_device(handle, nodes, &r, dev, gi.bytes, nullptr, &gi);
        if (rc == VXB_OK && cudaDeviceSynchronize() != cudaSuccess) rc = VXB_ECUDA;
        if (rc != VXB_OK) {
            cudaFree(dev);
            check(rc);
        }
        if (nodes) res.ptr = static_cast<Node*>(dev);
        else res.vptr = static_cast<VoxInt*>(dev);
    }
    voxelLength = gi.voxel_length;
    resolution = make_uint3(gi.resolution.x, gi.resolution.y, gi.resolution.z);
    return res;
}

template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::voxelize(uint maxDimension, uint2 devConfig, uint3 voxSplitRes) {
    std::vector<NodePointer<Node> > result;
    if (Node::isFCCNode()) {
        std::cout << "Please use a standard Node-type when producing a plain voxelization.\n";
        return result;
    }
    if (devConfig.x * devConfig.y != 1) throw Exception("Only one device is supported (devConfig must be (1, 1)).");
    nodeOutput = false;
    maxDimensionSetting = maxDimension;
    result.push_back(run(false, voxSplitRes, make_uint3(512, 512, 512)));
    return result;
}

template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::voxelize(double cubeLength, uint2 devConfig, uint3 voxSplitRes) {
    std::vector<NodePointer<Node> > result;
    if (Node::isFCCNode()) {
        std::cout << "Please use a standard Node-type when producing a plain voxelization.\n";
        return result;
    }
    if (devConfig.x * devConfig.y != 1) throw Exception("Only one device is supported (devConfig must be (1, 1)).");
    nodeOutput = false;
    voxelDistanceGiven = true;
    voxelLength = cubeLength;
    result.push_back(run(false, voxSplitRes, make_uint3(512, 512, 512)));
    return result;
}

template <class Node>
NodePointer<Node> Voxelizer<Node>::voxelizeToRAM(uint maxDimension, uint3 voxSplitRes) {
    if (Node::isFCCNode()) {
        std::cout << "Please use a standard Node-type when producing a plain voxelization" << std::endl;
        return NodePointer<Node>();
    }
    maxDimensionSetting = maxDimension;
    return run(true, voxSplitRes, make_uint3(512, 512, 512));
}

template <class Node>
NodePointer<Node> Voxelizer<Node>::voxelizeToRAM(double cubeLength, uint3 voxSplitRes) {
    if (Node::isFCCNode()) {
        std::cout << "Please use a standard Node-type when producing a plain voxelization" << std::endl;
        return NodePointer<Node>();
    }
    voxelDistanceGiven = true;
    voxelLength = cubeLength;
    return run(true, voxSplitRes, make_uint3(512, 512, 512));
}

template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::voxelizeToNodes(uint maxDimension, uint2 devConfig, uint3 voxSplitRes,
                                                                 uint3 matSplitRes) {
    std::vector<NodePointer<Node> > result;
    nodeOutput = true;
    if (Node::isFCCNode()) {
        std::cout << "FCC Nodes can currently only be defined through the side length of their cubic cells";
        return result;
    }
    if (devConfig.x * devConfig.y != 1) throw Exception("Only one device is supported (devConfig must be (1, 1)).");
    maxDimensionSetting = maxDimension;
    result.push_back(run(false, voxSplitRes, matSplitRes));
    return result;
}

template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::voxelizeToNodes(double cubeLength, uint2 devConfig,
                                                                 uint3 voxSplitRes, uint3 matSplitRes) {
    std::vector<NodePointer<Node> > result;
    if (devConfig.x * devConfig.y != 1) throw Exception("Only one device is supported (devConfig must be (1, 1)).");
    nodeOutput = true;
    voxelDistanceGiven = true;
    voxelLength = cubeLength;
    result.push_back(run(false, voxSplitRes, matSplitRes));
    return result;
}

template <class Node>
NodePointer<Node> Voxelizer<Node>::voxelizeToNodesToRAM(uint maxDimension, uint3 voxSplitRes, uint3 matSplitRes) {
    if (Node::isFCCNode()) {
        std::cout << "FCC Nodes can currently only be defined through the length of their cubic cells";
        return NodePointer<Node>();
    }
    nodeOutput = true;
    maxDimensionSetting = maxDimension;
    return run(true, voxSplitRes, matSplitRes);
}

template <class Node>
NodePointer<Node> Voxelizer<Node>::voxelizeToNodesToRAM(double cubeLength, uint3 voxSplitRes, uint3 matSplitRes) {
    nodeOutput = true;
    voxelDistanceGiven = true;
    voxelLength = cubeLength;
    return run(true, voxSplitRes, matSplitRes);
}

template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::voxelizeSlice(uint, int, uint, uint, uint2, uint2) {
    throw Exception("voxelizeSlice is not provided by this library");
}
template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::voxelizeSlice(double, int, uint, uint, uint2, uint2) {
    throw Exception("voxelizeSlice is not provided by this library");
}
template <class Node>
NodePointer<Node> Voxelizer<Node>::voxelizeSliceToRAM(uint, int, uint, uint2, uint2) {
    throw Exception("voxelizeSliceToRAM is not provided by this library");
}
template <class Node>
NodePointer<Node> Voxelizer<Node>::voxelizeSliceToRAM(double, int, uint, uint2, uint2) {
    throw Exception("voxelizeSliceToRAM is not provided by this library");
}

template <class Node>
uint3 Voxelizer<Node>::getArrayDimensions(uint longestSizeInVoxels, uint maxInternalXSize, bool sliceAlongX) {
    vxb_uint3 d;
    check(vxb_get_array_dimensions(handle, 0, longestSizeInVoxels, 0.0, maxInternalXSize, sliceAlongX ? 1 : 0, &d));
    maxDimensionSetting = longestSizeInVoxels;  // setResolution(), src/host_side.cpp:3375
    return make_uint3(d.x, d.y, d.z);
}

template <class Node>
uint3 Voxelizer<Node>::getArrayDimensions(double cubeLength, uint maxInternalXSize, bool sliceAlongX) {
    vxb_uint3 d;
    check(vxb_get_array_dimensions(handle, 1, 0, cubeLength, maxInternalXSize, sliceAlongX ? 1 : 0, &d));
    return make_uint3(d.x, d.y, d.z);
}

template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::simulateMultidevice(
    std::function<std::vector<NodePointer<Node> >()>) {
    throw Exception("simulateMultidevice is not provided by this library (single device only)");
}

template class Voxelizer<ShortNode>;
template class Voxelizer<LongNode>;
template class Voxelizer<PartialNode>;
template class Voxelizer<ShortFCCNode>;
template class Voxelizer<LongFCCNode>;

}  // namespace vox
