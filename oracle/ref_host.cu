// TEST INFRASTRUCTURE ONLY.  A C ABI over the reference's own public API:
// vox::Voxelizer<Node> (include/voxelizer.h:704-1000) as src/host_side.cpp
// implements it, compiled unmodified from the reference's sources together
// with src/voxelizer.cu (oracle/Makefile, target refhost; Boost replaced by
// the std-based shims in oracle/boost_shim).  Only tests/ and bench.py's
// reference arm load the resulting oracle/_ref/libvoxhost.so; the product
// library never does.
//
//   refh_dims:      Voxelizer<Node>::getArrayDimensions (host_side.cpp:3329-3475),
//                   host code only, so it runs without a GPU.
//   refh_voxelize:  voxelizeToNodesToRAM (host_side.cpp:1829-1886) or
//                   voxelizeToRAM (2275-2337): the reference's whole single-
//                   device flow, host arrays in, host array out.

#include "voxelizer.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>

using namespace vox;

namespace {

char g_error[1024] = "";

int fail(int code, const char* msg) {
    snprintf(g_error, sizeof(g_error), "%s", msg);
    return code;
}

template <class Node>
Voxelizer<Node>* make(const float* v, uint32_t nV, const uint32_t* idx, uint32_t nT, const uint8_t* mats,
                      uint32_t nMat) {
    if (mats) return new Voxelizer<Node>(v, idx, mats, nV, nT, nMat);
    return new Voxelizer<Node>(v, idx, nV, nT);
}

template <class Node>
int dims(const float* v, uint32_t nV, const uint32_t* idx, uint32_t nT, int byCube, uint32_t maxDim, double cube,
         uint32_t maxX, int sliceX, uint32_t* out) {
    Voxelizer<Node>* vx = make<Node>(v, nV, idx, nT, nullptr, 0);
    const uint3 d = byCube ? vx->getArrayDimensions(cube, maxX, sliceX != 0)
                           : vx->getArrayDimensions(maxDim, maxX, sliceX != 0);
    delete vx;
    out[0] = d.x;
    out[1] = d.y;
    out[2] = d.z;
    return 0;
}

template <class Node>
int voxelize(int nodes, int byCube, uint32_t maxDim, double cube, const uint32_t* vs, const uint32_t* ms,
             const float* v, uint32_t nV, const uint32_t* idx, uint32_t nT, const uint8_t* mats, uint32_t nMat,
             void* out, uint64_t outBytes, uint32_t* dimsOut, double* msOut) {
    const auto t0 = std::chrono::steady_clock::now();
    Voxelizer<Node>* vx = make<Node>(v, nV, idx, nT, mats, nMat);
    const uint3 vox = make_uint3(vs[0], vs[1], vs[2]), mat = make_uint3(ms[0], ms[1], ms[2]);
    NodePointer<Node> np;
    memset(&np, 0, sizeof(np));
    if (nodes)
        np = byCube ? vx->voxelizeToNodesToRAM(cube, vox, mat) : vx->voxelizeToNodesToRAM(maxDim, vox, mat);
    else
        np = byCube ? vx->voxelizeToRAM(cube, vox) : vx->voxelizeToRAM(maxDim, vox);
    const auto t1 = std::chrono::steady_clock::now();
    delete vx;
    if (!np.ptr) return fail(-2, "the reference returned no array (unsupported combination)");
    const uint64_t count = (uint64_t)np.dim.x * np.dim.y * np.dim.z;
    const uint64_t bytes = nodes ? count * sizeof(Node) : count / 8;
    dimsOut[0] = np.dim.x;
    dimsOut[1] = np.dim.y;
    dimsOut[2] = np.dim.z;
    if (msOut) *msOut = std::chrono::duration<double, std::milli>(t1 - t0).count();
    int rc = 0;
    if (out) {
        if (outBytes < bytes) rc = fail(-3, "output buffer too small");
        else memcpy(out, nodes ? (const void*)np.ptr : (const void*)np.vptr, bytes);
    }
    if (nodes) delete[] np.ptr;
    else delete[] np.vptr;
    return rc;
}

}  // namespace

extern "C" const char* refh_last_error() { return g_error; }

extern "C" int refh_dims(int node_type, const float* v, uint32_t nV, const uint32_t* idx, uint32_t nT, int by_cube,
                         uint32_t max_dim, double cube, uint32_t max_x, int slice_x, uint32_t* out) {
    try {
        switch (node_type) {
        case 0: return dims<ShortNode>(v, nV, idx, nT, by_cube, max_dim, cube, max_x, slice_x, out);
        case 1: return dims<LongNode>(v, nV, idx, nT, by_cube, max_dim, cube, max_x, slice_x, out);
        case 2: return dims<PartialNode>(v, nV, idx, nT, by_cube, max_dim, cube, max_x, slice_x, out);
        case 3: return dims<ShortFCCNode>(v, nV, idx, nT, by_cube, max_dim, cube, max_x, slice_x, out);
        case 4: return dims<LongFCCNode>(v, nV, idx, nT, by_cube, max_dim, cube, max_x, slice_x, out);
        }
        return fail(-4, "unknown node type");
    } catch (const std::exception& e) {
        return fail(-1, e.what());
    }
}

extern "C" int refh_voxelize(int node_type, int nodes, int by_cube, uint32_t max_dim, double cube,
                             const uint32_t* vox_split, const uint32_t* mat_split, const float* v, uint32_t nV,
                             const uint32_t* idx, uint32_t nT, const uint8_t* mats, uint32_t nMat, void* out,
                             uint64_t out_bytes, uint32_t* dims_out, double* ms) {
    try {
        switch (node_type) {
        case 0: return voxelize<ShortNode>(nodes, by_cube, max_dim, cube, vox_split, mat_split, v, nV, idx, nT,
                                           mats, nMat, out, out_bytes, dims_out, ms);
        case 1: return voxelize<LongNode>(nodes, by_cube, max_dim, cube, vox_split, mat_split, v, nV, idx, nT,
                                          mats, nMat, out, out_bytes, dims_out, ms);
        case 2: return voxelize<PartialNode>(nodes, by_cube, max_dim, cube, vox_split, mat_split, v, nV, idx, nT,
                                             mats, nMat, out, out_bytes, dims_out, ms);
        case 3: return voxelize<ShortFCCNode>(nodes, by_cube, max_dim, cube, vox_split, mat_split, v, nV, idx, nT,
                                              mats, nMat, out, out_bytes, dims_out, ms);
        case 4: return voxelize<LongFCCNode>(nodes, by_cube, max_dim, cube, vox_split, mat_split, v, nV, idx, nT,
                                             mats, nMat, out, out_bytes, dims_out, ms);
        }
        return fail(-4, "unknown node type");
    } catch (const std::exception& e) {
        return fail(-1, e.what());
    }
}
