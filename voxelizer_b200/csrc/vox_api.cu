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
    // calculateBoundingBox (src/host_side.cpp:2462-2488) ran in vxb_create,
    // on the device when there is one.
    double mn[3], mx[3];
    check(vxb_bounding_box(handle, mn, mx));
    minVertex = make_double3(mn[0], mn[1], mn[2]);
    maxVertex = make_double3(mx[0], mx[1], mx[2]);
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
    nodeOutput = false;
    maxDimensionSetting = maxDimension;
    if (devConfig.x * devConfig.y != 1 || simulate) return runParts(devConfig, voxSplitRes, make_uint3(512, 512, 512));
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
    nodeOutput = false;
    voxelDistanceGiven = true;
    voxelLength = cubeLength;
    if (devConfig.x * devConfig.y != 1 || simulate) return runParts(devConfig, voxSplitRes, make_uint3(512, 512, 512));
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
    maxDimensionSetting = maxDimension;
    if (devConfig.x * devConfig.y != 1 || simulate) return runParts(devConfig, voxSplitRes, matSplitRes);
    result.push_back(run(false, voxSplitRes, matSplitRes));
    return result;
}

template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::voxelizeToNodes(double cubeLength, uint2 devConfig,
                                                                 uint3 voxSplitRes, uint3 matSplitRes) {
    std::vector<NodePointer<Node> > result;
    nodeOutput = true;
    voxelDistanceGiven = true;
    voxelLength = cubeLength;
    if (devConfig.x * devConfig.y != 1 || simulate) return runParts(devConfig, voxSplitRes, matSplitRes);
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

// The reference's slice members take uint2 split sizes (a, b) and use
// (a, b, b) (src/host_side.cpp:1966-1972).
template <class Node>
vxb_request Voxelizer<Node>::request(uint3 voxSplitRes, uint3 matSplitRes) const {
    vxb_request r;
    r.by_cube_length = voxelDistanceGiven ? 1 : 0;
    r.max_dimension = maxDimensionSetting;
    r.cube_length = voxelLength;
    r.vox_split_res = u3(voxSplitRes);
    r.mat_split_res = u3(matSplitRes);
    return r;
}

// Partitions of devConfig, each voxelized as the reference voxelizes it on
// its own device (vxb_voxelize_parts_*).  All run on this voxelizer's GPU;
// the results are device pointers there, or host arrays (new[]) inside
// simulateMultidevice, whose collectData uploads to the host
// (src/host_side.cpp:3535-3543).
template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::runParts(uint2 devConfig, uint3 voxSplitRes, uint3 matSplitRes) {
    const vxb_request r = request(voxSplitRes, matSplitRes);
    const int nodes = nodeOutput ? 1 : 0;
    const uint n = devConfig.x * devConfig.y;
    if (n == 0) throw Exception("devConfig needs at least one device along each axis");
    std::vector<vxb_grid_info> gi(n);
    check(vxb_plan_parts(handle, nodes, &r, devConfig.x, devConfig.y, gi.data()));
    std::vector<void*> bufs(n, nullptr);
    std::vector<uint64_t> bytes(n);
    const bool host = simulate;
    int device = 0;
    cudaGetDevice(&device);
    auto release = [&]() {
        for (uint i = 0; i < n; ++i) {
            if (!bufs[i]) continue;
            if (!host) cudaFree(bufs[i]);
            else if (nodes) delete[] static_cast<Node*>(bufs[i]);
            else delete[] static_cast<VoxInt*>(bufs[i]);
        }
    };
    for (uint i = 0; i < n; ++i) {
        bytes[i] = gi[i].bytes;
        if (host) {
            bufs[i] = nodes ? static_cast<void*>(new Node[gi[i].count]) : static_cast<void*>(new VoxInt[gi[i].count]);
        } else if (cudaMalloc(&bufs[i], gi[i].bytes) != cudaSuccess) {
            cudaGetLastError();
            bufs[i] = nullptr;
            release();
            throw Exception("cudaMalloc of a partition result failed");
        }
    }
    vxb_status rc = host ? vxb_voxelize_parts_to_host(handle, nodes, &r, devConfig.x, devConfig.y, bufs.data(),
                                                      bytes.data(), gi.data())
                         : vxb_voxelize_parts_to_device(handle, nodes, &r, devConfig.x, devConfig.y, bufs.data(),
                                                        bytes.data(), nullptr, gi.data());
    if (rc != VXB_OK) {
        release();
        check(rc);
    }
    std::vector<NodePointer<Node> > result(n);
    for (uint i = 0; i < n; ++i) {
        NodePointer<Node>& np = result[i];
        if (nodes) np.ptr = static_cast<Node*>(bufs[i]);
        else np.vptr = static_cast<VoxInt*>(bufs[i]);
        np.dev = device;
        np.dim = make_uint3(gi[i].dim.x, gi[i].dim.y, gi[i].dim.z);
        np.loc = make_uint3(gi[i].location.x, gi[i].location.y, gi[i].location.z);
    }
    voxelLength = gi[0].voxel_length;
    resolution = make_uint3(gi[0].resolution.x, gi[0].resolution.y, gi[0].resolution.z);
    return result;
}

// One slice (vxb_voxelize_slice_*): node output, a device pointer or, with
// toHost (or inside simulateMultidevice), a host array.
template <class Node>
NodePointer<Node> Voxelizer<Node>::runSlice(bool toHost, int direction, uint slice, uint2 voxSplitRes,
                                            uint2 matSplitRes) {
    nodeOutput = true;   // the slice members set nodeOutput (src/host_side.cpp:1946)
    const vxb_request r = request(make_uint3(voxSplitRes.x, voxSplitRes.y, voxSplitRes.y),
                                  make_uint3(matSplitRes.x, matSplitRes.y, matSplitRes.y));
    vxb_grid_info gi;
    check(vxb_plan_slice(handle, &r, direction, slice, &gi));
    NodePointer<Node> res = NodePointer<Node>();
    int device = 0;
    cudaGetDevice(&device);
    res.dev = device;
    res.loc = make_uint3(0, 0, 0);
    res.dim = make_uint3(gi.dim.x, gi.dim.y, gi.dim.z);
    if (toHost || simulate) {
        Node* host = new Node[gi.count];
        vxb_status rc = vxb_voxelize_slice_to_host(handle, &r, direction, slice, host, gi.bytes, &gi);
        if (rc != VXB_OK) {
            delete[] host;
            check(rc);
        }
        res.ptr = host;
    } else {
        void* dev = nullptr;
        if (cudaMalloc(&dev, gi.bytes) != cudaSuccess) {
            cudaGetLastError();
            throw Exception("cudaMalloc of the result failed");
        }
        vxb_status rc = vxb_voxelize_slice_to_device(handle, &r, direction, slice, dev, gi.bytes, nullptr, &gi);
        if (rc != VXB_OK) {
            cudaFree(dev);
            check(rc);
        }
        res.ptr = static_cast<Node*>(dev);
    }
    voxelLength = gi.voxel_length;
    resolution = make_uint3(gi.resolution.x, gi.resolution.y, gi.resolution.z);
    return res;
}

template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::voxelizeSlice(uint maxDimension, int direction, uint slice,
                                                               uint devConfig, uint2 voxSplitRes,
                                                               uint2 matSplitRes) {
    std::vector<NodePointer<Node> > result;
    if (Node::isFCCNode()) {
        std::cout << "FCC Nodes can currently only be defined through the length of their cubic cells";
        return result;
    }
    if (devConfig != 1) throw Exception("slices are voxelized on one device (devConfig 1)");
    maxDimensionSetting = maxDimension;
    result.push_back(runSlice(false, direction, slice, voxSplitRes, matSplitRes));
    return result;
}

template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::voxelizeSlice(double cubeLength, int direction, uint slice,
                                                               uint devConfig, uint2 voxSplitRes,
                                                               uint2 matSplitRes) {
    std::vector<NodePointer<Node> > result;
    if (devConfig != 1) throw Exception("slices are voxelized on one device (devConfig 1)");
    voxelDistanceGiven = true;
    voxelLength = cubeLength;
    result.push_back(runSlice(false, direction, slice, voxSplitRes, matSplitRes));
    return result;
}

template <class Node>
NodePointer<Node> Voxelizer<Node>::voxelizeSliceToRAM(uint maxDimension, int direction, uint slice, uint2 voxSplitRes,
                                                      uint2 matSplitRes) {
    if (Node::isFCCNode()) {
        std::cout << "FCC Nodes can currently only be defined through the length of their cubic cells";
        return NodePointer<Node>();
    }
    maxDimensionSetting = maxDimension;
    return runSlice(true, direction, slice, voxSplitRes, matSplitRes);
}

template <class Node>
NodePointer<Node> Voxelizer<Node>::voxelizeSliceToRAM(double cubeLength, int direction, uint slice,
                                                      uint2 voxSplitRes, uint2 matSplitRes) {
    voxelDistanceGiven = true;
    voxelLength = cubeLength;
    return runSlice(true, direction, slice, voxSplitRes, matSplitRes);
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

// simulateMultidevice (src/host_side.cpp): runs `func` with every partition
// on one device and host results.
template <class Node>
std::vector<NodePointer<Node> > Voxelizer<Node>::simulateMultidevice(
    std::function<std::vector<NodePointer<Node> >()> func) {
    simulate = true;
    try {
        std::vector<NodePointer<Node> > result = func();
        simulate = false;
        return result;
    } catch (...) {
        simulate = false;
        throw;
    }
}

template class Voxelizer<ShortNode>;
template class Voxelizer<LongNode>;
template class Voxelizer<PartialNode>;
template class Voxelizer<ShortFCCNode>;
template class Voxelizer<LongFCCNode>;

}  // namespace vox
