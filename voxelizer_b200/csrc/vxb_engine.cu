// The C ABI (include/vxb.h): single voxelizers and batches.
//
// One vxb_voxelizer holds a copy of the mesh (as the reference's constructor
// does, src/host_side.cpp:72-99), its device copy, and the buffers of its
// pipeline, which grow on demand and are reused across calls.  A
// voxelization is one stream-ordered sequence of launches followed by one
// host check (vxb_pipeline.cu).  A vxb_batch runs many voxelizers' meshes
// through the same sequence at once, optionally replayed from a CUDA graph.

#include "vxb.h"
#include "vxb_host.h"
#include "vxb_kernels.cuh"
#include "vxb_pipeline.h"
#include "vxb_plan.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

using vxb::failf;

namespace {

const uint32_t kMaxMat[5] = {7, 255, 255, 15, 255};

bool isFcc(int t) { return t == VXB_SHORT_FCC_NODE || t == VXB_LONG_FCC_NODE; }

}  // namespace

struct vxb_voxelizer {
    int nodeType = 0;
    int device = 0;
    bool materialsOn = false;
    bool verbose = false;
    uint32_t nUniqueMaterials = 0;
    uint32_t nV = 0, nT = 0;
    std::vector<float> vertices;
    std::vector<uint32_t> indices;
    std::vector<uint8_t> materials;
    double mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
    bool meshOnDevice = false, matsOnDevice = false;
    bool hasMaterials = false;   // setMaterials was called (materials live on the host or the device)
    vxb::DevBuf dV, dI, dM, outStage, dCheck;
    cudaStream_t copyStream = nullptr;   // device-to-host copies of streamed output
    ~vxb_voxelizer() {
        if (copyStream) cudaStreamDestroy(copyStream);
    }
    // Slices along x: the rotated mesh (made on the first such call) and the
    // rotated slice's node array before the boundary ids.
    vxb::DevBuf dVrot, xStage, xFlag;
    bool rotOnDevice = false;
    vxb::Pipeline pipe;
    vxb::StageTimer timer;
    uint32_t launches = 0;
    // Set while work of a call may still be queued on the device (a call
    // that failed half-way); vxb_destroy then waits for the device before
    // its buffers return to the block cache.  Calls that succeed end with
    // their work complete.
    bool busy = false;

    int plan(int nodes, const vxb_request* r, vxb::Plan& p, vxb_grid_info* info) const;
    // The request's plan of the whole grid, without the output size checks
    // (of the mesh's bounding box, or of bmn / bmx).
    int fullPlan(const vxb_request* r, vxb::Plan& p, const double* bmn = nullptr, const double* bmx = nullptr) const;
    // Combinations the reference refuses (src/host_side.cpp:568-573,
    // 1744-1749, 1836-1841, 2280-2285) and missing materials.
    int validate(int nodes, const vxb_request* r) const {
        if (!nodes && isFcc(nodeType))
            return failf(VXB_EUNSUPPORTED, "Please use a standard Node-type when producing a plain voxelization.");
        if (nodes && isFcc(nodeType) && !r->by_cube_length)
            return failf(VXB_EUNSUPPORTED,
                         "FCC Nodes can currently only be defined through the side length of their cubic cells");
        if (nodes && materialsOn && !hasMaterials)
            return failf(VXB_ENOMATERIALS, "material output requested but no materials were set");
        return 0;
    }
    int upload(cudaStream_t s);
    // Copies caller arrays to the device; false (nothing kept) when there is
    // no usable device.
    bool uploadFrom(const float* vertices, const uint32_t* indices);
    bool uploadMaterials(const uint8_t* mats);
    void job(int nodes, const vxb_request* r, void* dout, uint64_t bytes, vxb::MeshJob* j) const;
    int run(int nodes, const vxb_request* r, void* dout, uint64_t bytes, cudaStream_t s, vxb_grid_info* info);
    // Device spaces (partitions of the yz voxel range, voxelized as the
    // reference's devices do) of one request: plans and runs them all as one
    // batch.
    struct Space {
        uint32_t part[4];
        vxb_uint3 loc;
    };
    int planSpaces(int nodes, const vxb_request* r, const std::vector<Space>& sp, vxb_grid_info* infos) const;
    int runSpaces(int nodes, const vxb_request* r, const std::vector<Space>& sp, void* const* outs,
                  const uint64_t* bytes, cudaStream_t s, vxb_grid_info* infos);
    // The partitions of devConfig (dev_y, dev_z) (splitResolutionByNrOfParts,
    // src/host_side.cpp:782-813), y fastest.
    int partitions(const vxb_request* r, uint32_t devY, uint32_t devZ, std::vector<Space>* sp) const;
    // The device space of a slice (src/host_side.cpp:748-779): *oob for a
    // slice 0 or past the grid, whose result is all zeros.
    int sliceSpace(const vxb_request* r, int direction, uint32_t slice, Space* sp, bool* oob) const;
    // Slices along x: rotateVertices (src/host_side.cpp:3261-3280) turns the
    // mesh about z (x' = a - y, y' = b + x in double, rounded to float) and
    // the rotated grid is sliced along y.  `rotation` gives a, b and the
    // rotated bounding box (float rounding is monotone, so the box's corners
    // are the rotated corners of the original box); planXSlice the rotated
    // slice's device space and the un-rotated result's shape.
    void rotation(double* a, double* b, double* rmn, double* rmx) const;
    int planXSlice(const vxb_request* r, uint32_t slice, vxb::Plan* q, bool* oob, vxb_grid_info* info) const;
    int runXSlice(const vxb_request* r, uint32_t slice, void* out, uint64_t bytes, cudaStream_t s,
                  vxb_grid_info* info);
};

int vxb_voxelizer::fullPlan(const vxb_request* r, vxb::Plan& p, const double* bmn, const double* bmx) const {
    if (!r) return failf(VXB_EINVAL, "request is NULL");
    if (nV == 0 || nT == 0) return failf(VXB_EINVAL, "empty mesh");
    const uint32_t vs[3] = {r->vox_split_res.x, r->vox_split_res.y, r->vox_split_res.z};
    const uint32_t ms[3] = {r->mat_split_res.x, r->mat_split_res.y, r->mat_split_res.z};
    if (vxb::makePlan(bmn ? bmn : mn, bmx ? bmx : mx, r->by_cube_length, r->max_dimension, r->cube_length, vs, ms, p))
        return failf(VXB_EINVAL, "invalid request (maxDimension >= 2 or cubeLength > 0, split sizes > 0 and an x "
                                 "pass of at most 1024 voxels are required)");
    return 0;
}

int vxb_voxelizer::plan(int nodes, const vxb_request* r, vxb::Plan& p, vxb_grid_info* info) const {
    int rc = fullPlan(r, p);
    if (rc) return rc;
    return vxb::gridInfo(p, nodeType, nodes, info);
}

int vxb_voxelizer::upload(cudaStream_t s) {
    if (!meshOnDevice) {
        int rc;
        if ((rc = dV.ensure(sizeof(float) * 3 * (size_t)nV))) return rc;
        if ((rc = dI.ensure(sizeof(uint32_t) * 3 * (size_t)nT))) return rc;
        VXB_CUDA(cudaMemcpyAsync(dV.p, vertices.data(), sizeof(float) * 3 * (size_t)nV, cudaMemcpyHostToDevice, s));
        VXB_CUDA(cudaMemcpyAsync(dI.p, indices.data(), sizeof(uint32_t) * 3 * (size_t)nT, cudaMemcpyHostToDevice, s));
        meshOnDevice = true;
    }
    if (materialsOn && !matsOnDevice && !materials.empty()) {
        int rc;
        if ((rc = dM.ensure(nT))) return rc;
        VXB_CUDA(cudaMemcpyAsync(dM.p, materials.data(), nT, cudaMemcpyHostToDevice, s));
        matsOnDevice = true;
    }
    return 0;
}

namespace {

// Runs `f` with `device` current, restoring the caller's device; false when
// there is no such device.
template <class F> bool onDevice(int device, F f) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return false;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != device && cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const bool ok = f();
    if (cur != device) cudaSetDevice(cur);
    return ok;
}

}  // namespace

bool vxb_voxelizer::uploadFrom(const float* vertices, const uint32_t* indices) {
    return onDevice(device, [&]() {
        if (dV.ensure(sizeof(float) * 3 * (size_t)nV) || dI.ensure(sizeof(uint32_t) * 3 * (size_t)nT)) return false;
        if (cudaMemcpy(dV.p, vertices, sizeof(float) * 3 * (size_t)nV, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(dI.p, indices, sizeof(uint32_t) * 3 * (size_t)nT, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        meshOnDevice = true;
        return true;
    });
}

bool vxb_voxelizer::uploadMaterials(const uint8_t* mats) {
    if (!meshOnDevice) return false;
    return onDevice(device, [&]() {
        if (dM.ensure(nT)) return false;
        if (cudaMemcpy(dM.p, mats, nT, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        matsOnDevice = true;
        return true;
    });
}

void vxb_voxelizer::job(int nodes, const vxb_request* r, void* dout, uint64_t bytes, vxb::MeshJob* j) const {
    j->V = dV.as<float>();
    j->I = dI.as<uint32_t>();
    j->M = (nodes && materialsOn) ? dM.as<uint8_t>() : nullptr;
    j->nV = nV;
    j->nT = nT;
    for (int a = 0; a < 3; ++a) {
        j->mn[a] = mn[a];
        j->mx[a] = mx[a];
    }
    j->nodeType = nodeType;
    j->nodes = nodes ? 1 : 0;
    j->req = *r;
    j->out = dout;
    j->outBytes = bytes;
}

int vxb_voxelizer::run(int nodes, const vxb_request* r, void* dout, uint64_t bytes, cudaStream_t s,
                       vxb_grid_info* info) {
    vxb::Plan p;
    vxb_grid_info gi;
    int rc = plan(nodes, r, p, &gi);
    if (rc) return rc;
    if (info) *info = gi;
    if (!dout) return failf(VXB_EINVAL, "output buffer is NULL");
    if (bytes < gi.bytes)
        return failf(VXB_EINVAL, "output buffer holds %llu bytes, %llu needed", (unsigned long long)bytes,
                     (unsigned long long)gi.bytes);
    if ((rc = validate(nodes, r))) return rc;
    VXB_CUDA(cudaSetDevice(device));
    launches = 0;
    timer.reset();
    busy = true;
    if ((rc = upload(s))) return rc;
    vxb::MeshJob j;
    job(nodes, r, dout, bytes, &j);
    if ((rc = pipe.prepare(std::vector<vxb::MeshJob>{j}, s))) return rc;
    if ((rc = pipe.enqueue(s, &timer))) return rc;
    rc = pipe.finish(s);
    launches = pipe.launches;
    if (rc == 0) busy = false;
    return rc;
}

int vxb_voxelizer::planSpaces(int nodes, const vxb_request* r, const std::vector<Space>& sp,
                              vxb_grid_info* infos) const {
    vxb::Plan full;
    int rc = fullPlan(r, full);
    if (rc) return rc;
    const uint32_t vs[3] = {r->vox_split_res.x, r->vox_split_res.y, r->vox_split_res.z};
    const uint32_t ms[3] = {r->mat_split_res.x, r->mat_split_res.y, r->mat_split_res.z};
    for (size_t i = 0; i < sp.size(); ++i) {
        vxb::Plan q;
        if (vxb::devicePlan(full, sp[i].part[0], sp[i].part[1], sp[i].part[2], sp[i].part[3], vs, ms, q))
            return failf(VXB_EINVAL, "partition %zu is empty or outside the grid", i);
        if ((rc = vxb::gridInfo(q, nodeType, nodes, infos + i))) return rc;
        infos[i].location = sp[i].loc;
    }
    return 0;
}

int vxb_voxelizer::runSpaces(int nodes, const vxb_request* r, const std::vector<Space>& sp, void* const* outs,
                             const uint64_t* bytes, cudaStream_t s, vxb_grid_info* infos) {
    std::vector<vxb_grid_info> gi(sp.size());
    int rc = planSpaces(nodes, r, sp, gi.data());
    if (rc) return rc;
    for (size_t i = 0; i < sp.size(); ++i) {
        if (infos) infos[i] = gi[i];
        if (!outs || !outs[i]) return failf(VXB_EINVAL, "output buffer %zu is NULL", i);
        if (!bytes || bytes[i] < gi[i].bytes)
            return failf(VXB_EINVAL, "output buffer %zu holds too few bytes (%llu needed)", i,
                         (unsigned long long)gi[i].bytes);
    }
    if ((rc = validate(nodes, r))) return rc;
    VXB_CUDA(cudaSetDevice(device));
    launches = 0;
    timer.reset();
    busy = true;
    if ((rc = upload(s))) return rc;
    std::vector<vxb::MeshJob> jobs(sp.size());
    for (size_t i = 0; i < sp.size(); ++i) {
        job(nodes, r, outs[i], bytes[i], &jobs[i]);
        jobs[i].space = 1;
        for (int k = 0; k < 4; ++k) jobs[i].part[k] = sp[i].part[k];
    }
    if ((rc = pipe.prepare(jobs, s))) return rc;
    if ((rc = pipe.enqueue(s, &timer))) return rc;
    rc = pipe.finish(s);
    launches = pipe.launches;
    if (rc == 0) busy = false;
    return rc;
}

int vxb_voxelizer::partitions(const vxb_request* r, uint32_t devY, uint32_t devZ, std::vector<Space>* sp) const {
    if (devY == 0 || devZ == 0) return failf(VXB_EINVAL, "devConfig needs at least one partition per axis");
    vxb::Plan full;
    int rc = fullPlan(r, full);
    if (rc) return rc;
    const std::vector<vxb::Range> ys = vxb::splitParts(full.res[1], devY), zs = vxb::splitParts(full.res[2], devZ);
    sp->clear();
    for (uint32_t z = 0; z < devZ; ++z)
        for (uint32_t y = 0; y < devY; ++y) {
            Space q;
            q.part[0] = ys[y].lo;
            q.part[1] = ys[y].hi;
            q.part[2] = zs[z].lo;
            q.part[3] = zs[z].hi;
            q.loc = vxb_uint3{0, y, z};
            if (q.part[0] == q.part[1] || q.part[2] == q.part[3])
                return failf(VXB_EINVAL, "devConfig (%u, %u) leaves an empty partition", devY, devZ);
            sp->push_back(q);
        }
    return 0;
}

void vxb_voxelizer::rotation(double* a, double* b, double* rmn, double* rmx) const {
    const double cx = (mx[0] - mn[0]) / 2.0, cy = (mx[1] - mn[1]) / 2.0;
    *a = cy + cx;
    *b = cy - cx;
    rmn[0] = (double)(float)(*a - mx[1]);
    rmx[0] = (double)(float)(*a - mn[1]);
    rmn[1] = (double)(float)(*b + mn[0]);
    rmx[1] = (double)(float)(*b + mx[0]);
    rmn[2] = mn[2];
    rmx[2] = mx[2];
}

int vxb_voxelizer::planXSlice(const vxb_request* r, uint32_t slice, vxb::Plan* q, bool* oob,
                              vxb_grid_info* info) const {
    double a, b, rmn[3], rmx[3];
    rotation(&a, &b, rmn, rmx);
    vxb::Plan full;
    int rc = fullPlan(r, full, rmn, rmx);
    if (rc) return rc;
    *oob = slice == 0 || slice > full.res[1];
    const uint32_t s0 = *oob ? 0u : slice - 1;
    const uint32_t vs[3] = {r->vox_split_res.x, r->vox_split_res.y, r->vox_split_res.z};
    const uint32_t ms[3] = {r->mat_split_res.x, r->mat_split_res.y, r->mat_split_res.z};
    if (vxb::devicePlan(full, s0, s0 + 1, 0, full.res[2], vs, ms, *q))
        return failf(VXB_EINVAL, "slice outside the grid");
    vxb_grid_info gi;
    if ((rc = vxb::gridInfo(*q, nodeType, 1, &gi))) return rc;
    // The un-rotated array: x and y trade places (unRotateCoords,
    // src/host_side.cpp:1160-1175, 1610-1625; an FCC array of 2X x Y x Z
    // nodes becomes 2Y x X x Z).
    const uint32_t t = gi.dim.x;
    gi.dim.x = isFcc(nodeType) ? 2 * gi.dim.y : gi.dim.y;
    gi.dim.y = isFcc(nodeType) ? t / 2 : t;
    gi.location = vxb_uint3{0, 0, 0};
    if (info) *info = gi;
    return 0;
}

int vxb_voxelizer::runXSlice(const vxb_request* r, uint32_t slice, void* out, uint64_t bytes, cudaStream_t s,
                             vxb_grid_info* info) {
    vxb::Plan q;
    bool oob = false;
    vxb_grid_info gi;
    int rc = planXSlice(r, slice, &q, &oob, &gi);
    if (rc) return rc;
    if (info) *info = gi;
    if ((rc = validate(1, r))) return rc;
    if (!out || bytes < gi.bytes) return failf(VXB_EINVAL, "output buffer is NULL or too small");
    VXB_CUDA(cudaSetDevice(device));
    launches = 0;
    timer.reset();
    if (oob) {   // sliceOOB (src/host_side.cpp:1225-1236)
        VXB_CUDA(cudaMemsetAsync(out, 0, gi.bytes, s));
        VXB_CUDA(cudaStreamSynchronize(s));
        return VXB_OK;
    }
    busy = true;
    if ((rc = upload(s))) return rc;
    double a, b, rmn[3], rmx[3];
    rotation(&a, &b, rmn, rmx);
    if (!rotOnDevice) {
        if ((rc = dVrot.ensure(sizeof(float) * 3 * (size_t)nV))) return rc;
        vxb::launch_rotate_vertices(dV.as<float>(), dVrot.as<float>(), nV, a, b, s, &launches);
        VXB_CUDA(cudaGetLastError());
        rotOnDevice = true;
    }
    if ((rc = xStage.ensure(gi.bytes))) return rc;
    if ((rc = xFlag.ensure(4))) return rc;
    vxb::MeshJob j;
    job(1, r, xStage.p, gi.bytes, &j);
    j.V = dVrot.as<float>();
    for (int k = 0; k < 3; ++k) {
        j.mn[k] = rmn[k];
        j.mx[k] = rmx[k];
    }
    j.space = 1;
    for (int k = 0; k < 4; ++k) j.part[k] = q.part[k];
    j.raw = 1;
    j.turned = 1;
    if ((rc = pipe.prepare(std::vector<vxb::MeshJob>{j}, s))) return rc;
    if ((rc = pipe.enqueue(s, &timer))) return rc;
    if ((rc = pipe.finish(s))) return rc;
    launches += pipe.launches;
    const uint32_t nb = (uint32_t)(gi.bytes / gi.count);
    if (isFcc(nodeType)) {
        // fccWorker with xSlicing (src/host_side.cpp:1597-1673):
        // restoreRotatedNodes, calculateFCCBoundaries on the un-rotated
        // array, zeroPadding.
        const uint32_t NX = 2 * q.alloc[0], NY = q.alloc[1], NZ = 2 * q.alloc[2];
        vxb::launch_unrotate_fcc(xStage.p, out, NX, NY, NZ, nb, s, &launches);
        vxb::launch_fcc_boundaries(out, 2 * NY, NX / 2, NZ, nb, s, &launches);
        if (q.border) vxb::launch_zero_faces(out, 2 * NY, NX / 2, NZ, nb, true, s, &launches);
        VXB_CUDA(cudaGetLastError());
        VXB_CUDA(cudaStreamSynchronize(s));
        busy = false;
        return VXB_OK;
    }
    // restoreRotatedNodes, then fillNodeList2 over the un-rotated array one
    // yz subspace at a time until no node loses its id, then zeroPadding
    // (src/host_side.cpp:1144-1223).
    const uint32_t X = q.alloc[0], Y = q.alloc[1], Z = q.alloc[2];
    vxb::launch_unrotate(xStage.p, out, X, Y, Z, nb, s, &launches);
    const uint32_t idMask = nodeType == VXB_SHORT_NODE ? 31u : 255u;
    const std::vector<vxb::Range> ys = vxb::splitLength(X, r->vox_split_res.y);
    const std::vector<vxb::Range> zs = vxb::splitLength(Z, r->vox_split_res.z);
    uint32_t* flag = xFlag.as<uint32_t>();
    for (const vxb::Range& zr : zs)
        for (const vxb::Range& yr : ys)
            for (uint64_t pass = 0;; ++pass) {
                if (pass > (uint64_t)Y * X * Z) return failf(VXB_ETIMEDOUT, "boundary ids did not converge");
                VXB_CUDA(cudaMemsetAsync(flag, 0, 4, s));
                vxb::launch_id_pass(out, Y, X, Z, nb, idMask, yr.lo, yr.hi, zr.lo, zr.hi, flag, s, &launches);
                uint32_t h = 0;
                VXB_CUDA(cudaMemcpyAsync(&h, flag, 4, cudaMemcpyDeviceToHost, s));
                VXB_CUDA(cudaStreamSynchronize(s));
                if (!h) break;
            }
    if (q.border) vxb::launch_zero_faces(out, Y, X, Z, nb, false, s, &launches);
    VXB_CUDA(cudaGetLastError());
    VXB_CUDA(cudaStreamSynchronize(s));
    busy = false;
    return VXB_OK;
}

int vxb_voxelizer::sliceSpace(const vxb_request* r, int direction, uint32_t slice, Space* sp, bool* oob) const {
    if (direction != 1 && direction != 2) return failf(VXB_EINVAL, "slice direction must be 0, 1 or 2");
    vxb::Plan full;
    int rc = fullPlan(r, full);
    if (rc) return rc;
    const uint32_t len = direction == 1 ? full.res[1] : full.res[2];
    *oob = slice == 0 || slice > len;
    const uint32_t s0 = *oob ? 0u : slice - 1;   // slices count the padding row
    sp->loc = vxb_uint3{0, 0, 0};
    if (direction == 1) {
        sp->part[0] = s0; sp->part[1] = s0 + 1; sp->part[2] = 0; sp->part[3] = full.res[2];
    } else {
        sp->part[0] = 0; sp->part[1] = full.res[1]; sp->part[2] = s0; sp->part[3] = s0 + 1;
    }
    return 0;
}

// A batch of voxelizations run together.
struct vxb_batch {
    int device = 0;
    struct Entry {
        vxb_voxelizer* v;
        int nodes;
        vxb_request req;
        void* out;
        uint64_t bytes;
    };
    std::vector<Entry> entries;
    bool prepared = false;       // pipeline tables match `entries`
    vxb::Pipeline pipe;
    cudaStream_t own = nullptr;  // capture stream when the caller passes the legacy default stream
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graphStream = nullptr;
    uint32_t graphKernels = 0;
    uint32_t launches = 0;
    bool busy = false;           // as vxb_voxelizer::busy
    void dropGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        graphKernels = 0;
    }
    ~vxb_batch() {
        dropGraph();
        if (own) cudaStreamDestroy(own);
    }
};

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

const char* vxb_version(void) { return "vxb 0.2 (sm_100a)"; }

vxb_status vxb_create(vxb_voxelizer** out, int node_type, const float* vertices, const uint32_t* indices,
                      uint32_t n_vertices, uint32_t n_triangles, int device) {
    if (!out) return failf(VXB_EINVAL, "out is NULL");
    *out = nullptr;
    if (node_type < 0 || node_type > 4) return failf(VXB_EINVAL, "unknown node type %d", node_type);
    if ((!vertices && n_vertices) || (!indices && n_triangles)) return failf(VXB_EINVAL, "NULL mesh arrays");
    auto badIndex = [&](uint64_t i) {
        return failf(VXB_EINVAL, "index %u of triangle %llu is out of range", indices[i], (unsigned long long)(i / 3));
    };
    vxb_voxelizer* v = new (std::nothrow) vxb_voxelizer();
    if (!v) return failf(VXB_ENOMEM, "out of host memory");
    v->nodeType = node_type;
    v->device = device;
    v->nV = n_vertices;
    v->nT = n_triangles;
    // The copy the reference keeps on the host goes straight to the device
    // when there is one, and the index check and the bounding box run there
    // on that copy; without a device (planning only) the mesh stays on the
    // host until the first voxelization and the checks run here.
    unsigned long long chk[8];
    const bool uploaded = n_vertices && n_triangles && v->uploadFrom(vertices, indices);
    const bool checked = uploaded && onDevice(device, [&]() {
                             return v->dCheck.ensure(sizeof(chk)) == 0 &&
                                    vxb::meshCheck(v->dV.as<float>(), n_vertices, v->dI.as<uint32_t>(),
                                                   3ull * n_triangles, v->dCheck.as<unsigned long long>(), chk,
                                                   0) == 0;
                         });
    if (checked) {
        if (chk[7] != ~0ull) {
            delete v;
            return badIndex(chk[7]);
        }
        for (int a = 0; a < 3; ++a) {
            v->mn[a] = v->mx[a] = vertices[a];
            if (chk[a] != ~0ull) {
                const float f = vertices[3 * (size_t)(uint32_t)chk[a] + a];
                if (f < v->mn[a]) v->mn[a] = f;
            }
            if (chk[3 + a] != ~0ull) {
                const float f = vertices[3 * (size_t)(uint32_t)chk[3 + a] + a];
                if (f > v->mx[a]) v->mx[a] = f;
            }
        }
    } else {
        uint32_t maxIndex = 0;
        for (uint64_t i = 0; i < 3ull * n_triangles; ++i) maxIndex = std::max(maxIndex, indices[i]);
        if (n_triangles && maxIndex >= n_vertices)
            for (uint64_t i = 0; i < 3ull * n_triangles; ++i)
                if (indices[i] >= n_vertices) {
                    delete v;
                    return badIndex(i);
                }
        if (n_vertices) vxb::boundingBox(vertices, n_vertices, v->mn, v->mx);
        if (!uploaded) {
            v->vertices.assign(vertices, vertices + 3 * (size_t)n_vertices);
            v->indices.assign(indices, indices + 3 * (size_t)n_triangles);
        }
    }
    *out = v;
    return VXB_OK;
}

vxb_status vxb_scan_counts(const uint32_t* counts, uint32_t n, uint32_t* offsets, uint32_t* total,
                           uint32_t* overflow, void* stream) {
    if ((!counts && n) || !offsets || !total || !overflow) return failf(VXB_EINVAL, "NULL argument");
    int dev = 0;
    VXB_CUDA(cudaGetDevice(&dev));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    vxb::DevBuf tiles, status;
    tiles.dev = status.dev = dev;
    int rc;
    if ((rc = tiles.ensure(4 * ((size_t)n / 4096 + 2))) || (rc = status.ensure(8))) return rc;
    uint32_t launches = 0;
    vxb::launch_scan(counts, offsets, n, tiles.as<uint32_t>(), status.as<uint32_t>(), status.as<uint32_t>() + 1, s,
                     &launches);
    uint32_t h[2];
    VXB_CUDA(cudaMemcpyAsync(h, status.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    VXB_CUDA(cudaStreamSynchronize(s));
    *total = h[0];
    *overflow = h[1];
    return VXB_OK;
}

vxb_status vxb_bounding_box(const vxb_voxelizer* v, double min_vertex[3], double max_vertex[3]) {
    if (!v || !min_vertex || !max_vertex) return failf(VXB_EINVAL, "NULL argument");
    for (int a = 0; a < 3; ++a) {
        min_vertex[a] = v->mn[a];
        max_vertex[a] = v->mx[a];
    }
    return VXB_OK;
}

vxb_status vxb_destroy(vxb_voxelizer* v) {
    if (!v) return VXB_OK;
    // The instance's buffers go back to the block cache: after a failed
    // call, wait for queued work that may still use them.
    const int dev = v->device;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    if (v->busy) cudaDeviceSynchronize();
    delete v;
    if (cur != dev) cudaSetDevice(cur);
    return VXB_OK;
}

vxb_status vxb_set_materials(vxb_voxelizer* v, const uint8_t* materials, uint32_t n_unique_materials) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    if (!materials) return failf(VXB_EINVAL, "No valid materials provided (Received null pointer) @ setMaterials.");
    if (n_unique_materials > kMaxMat[v->nodeType] + 1)
        return failf(VXB_EINVAL,
                     "The number of unique materials exceeds the capabilities of the node type @ setMaterials.");
    v->nUniqueMaterials = n_unique_materials;
    v->matsOnDevice = false;
    v->materials.clear();
    if (!v->uploadMaterials(materials)) v->materials.assign(materials, materials + v->nT);
    v->hasMaterials = true;
    v->materialsOn = true;
    return VXB_OK;
}

vxb_status vxb_set_material_output(vxb_voxelizer* v, int enable) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    v->materialsOn = enable != 0;
    return VXB_OK;
}

vxb_status vxb_verbose_output(vxb_voxelizer* v, int enable) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    v->verbose = enable != 0;
    return VXB_OK;
}

vxb_status vxb_plan(vxb_voxelizer* v, int nodes, const vxb_request* req, vxb_grid_info* info) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    vxb::Plan p;
    return v->plan(nodes, req, p, info);
}

vxb_status vxb_get_array_dimensions(vxb_voxelizer* v, int by_cube_length, uint32_t max_dimension, double cube_length,
                                    uint32_t max_internal_x, int slice_along_x, vxb_uint3* dims) {
    if (!v || !dims) return failf(VXB_EINVAL, "NULL argument");
    if (slice_along_x) {
        // src/host_side.cpp:3333-3371: the rotated mesh's grid (padding
        // included), its corners un-rotated: x and y trade places; FCC
        // lattices double x and z.
        vxb_request r;
        r.by_cube_length = by_cube_length;
        r.max_dimension = max_dimension;
        r.cube_length = cube_length;
        r.vox_split_res = vxb_uint3{max_internal_x, 512, 512};
        r.mat_split_res = vxb_uint3{512, 512, 512};
        double a, b, rmn[3], rmx[3];
        v->rotation(&a, &b, rmn, rmx);
        vxb::Plan p;
        int rc = v->fullPlan(&r, p, rmn, rmx);
        if (rc) return rc;
        const uint32_t f = isFcc(v->nodeType) ? 2u : 1u;
        dims->x = f * p.alloc[1];
        dims->y = p.alloc[0];
        dims->z = f * p.alloc[2];
        if (f == 2 && !by_cube_length) {
            // The maxDimension overload (src/host_side.cpp:3329-3369) turns
            // the corners of the undoubled grid back with unRotateCoords'
            // FCC branch (3293-3309) and doubles x and z afterwards.
            const uint32_t X = p.alloc[0], Y = p.alloc[1], Z = p.alloc[2];
            auto unrot = [&](uint32_t x, uint32_t y, uint32_t z, uint32_t out[3]) {
                out[0] = 2 * y + (x + z + 1) % 2;
                out[1] = X / 2 - 1 - x / 2;
                out[2] = z;
            };
            uint32_t a[3], b[3];
            unrot(0, 0, 0, a);
            unrot(X - 1, Y - 1, Z - 1, b);
            const uint32_t ext[3] = {std::max(a[0], b[0]) - std::min(a[0], b[0]) + 1,
                                     std::max(a[1], b[1]) - std::min(a[1], b[1]) + 1,
                                     std::max(a[2], b[2]) - std::min(a[2], b[2]) + 1};
            dims->x = 2 * ext[0];
            dims->y = ext[1];
            dims->z = 2 * ext[2];
        }
        return VXB_OK;
    }
    vxb_request r;
    r.by_cube_length = by_cube_length;
    r.max_dimension = max_dimension;
    r.cube_length = cube_length;
    r.vox_split_res = vxb_uint3{max_internal_x, 512, 512};
    r.mat_split_res = vxb_uint3{512, 512, 512};
    vxb_grid_info gi;
    vxb::Plan p;
    int rc = v->plan(1, &r, p, &gi);
    if (rc == VXB_EOVERFLOW) rc = 0;
    if (rc) return rc;
    dims->x = isFcc(v->nodeType) ? 2 * p.alloc[0] : p.alloc[0];
    dims->y = p.alloc[1];
    dims->z = isFcc(v->nodeType) ? 2 * p.alloc[2] : p.alloc[2];
    return VXB_OK;
}

vxb_status vxb_voxelize_to_device(vxb_voxelizer* v, int nodes, const vxb_request* req, void* dev_out,
                                  uint64_t dev_bytes, void* stream, vxb_grid_info* info) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    return v->run(nodes, req, dev_out, dev_bytes, reinterpret_cast<cudaStream_t>(stream), info);
}

vxb_status vxb_plan_parts(vxb_voxelizer* v, int nodes, const vxb_request* req, uint32_t dev_y, uint32_t dev_z,
                          vxb_grid_info* infos) {
    if (!v || !infos) return failf(VXB_EINVAL, "NULL argument");
    std::vector<vxb_voxelizer::Space> sp;
    int rc = v->partitions(req, dev_y, dev_z, &sp);
    if (rc) return rc;
    return v->planSpaces(nodes, req, sp, infos);
}

vxb_status vxb_voxelize_parts_to_device(vxb_voxelizer* v, int nodes, const vxb_request* req, uint32_t dev_y,
                                        uint32_t dev_z, void* const* dev_outs, const uint64_t* dev_bytes,
                                        void* stream, vxb_grid_info* infos) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    std::vector<vxb_voxelizer::Space> sp;
    int rc = v->partitions(req, dev_y, dev_z, &sp);
    if (rc) return rc;
    return v->runSpaces(nodes, req, sp, dev_outs, dev_bytes, reinterpret_cast<cudaStream_t>(stream), infos);
}

vxb_status vxb_voxelize_parts_to_host(vxb_voxelizer* v, int nodes, const vxb_request* req, uint32_t dev_y,
                                      uint32_t dev_z, void* const* host_outs, const uint64_t* host_bytes,
                                      vxb_grid_info* infos) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    std::vector<vxb_voxelizer::Space> sp;
    int rc = v->partitions(req, dev_y, dev_z, &sp);
    if (rc) return rc;
    std::vector<vxb_grid_info> gi(sp.size());
    if ((rc = v->planSpaces(nodes, req, sp, gi.data()))) return rc;
    if (infos)
        for (size_t i = 0; i < sp.size(); ++i) infos[i] = gi[i];
    if (!host_outs || !host_bytes) return failf(VXB_EINVAL, "NULL output arrays");
    uint64_t total = 0;
    std::vector<uint64_t> off(sp.size());
    for (size_t i = 0; i < sp.size(); ++i) {
        if (!host_outs[i] || host_bytes[i] < gi[i].bytes)
            return failf(VXB_EINVAL, "output buffer %zu is NULL or too small", i);
        off[i] = total;
        total += (gi[i].bytes + 255) & ~uint64_t(255);
    }
    VXB_CUDA(cudaSetDevice(v->device));
    if ((rc = v->outStage.ensure(total))) return rc;
    std::vector<void*> outs(sp.size());
    for (size_t i = 0; i < sp.size(); ++i) outs[i] = v->outStage.as<uint8_t>() + off[i];
    std::vector<uint64_t> bytes(sp.size());
    for (size_t i = 0; i < sp.size(); ++i) bytes[i] = gi[i].bytes;
    rc = v->runSpaces(nodes, req, sp, outs.data(), bytes.data(), 0, infos);
    for (size_t i = 0; rc == 0 && i < sp.size(); ++i) {
        cudaError_t e = cudaMemcpy(host_outs[i], outs[i], gi[i].bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = failf(VXB_ECUDA, "%s", cudaGetErrorString(e));
    }
    return rc;
}

vxb_status vxb_plan_slice(vxb_voxelizer* v, const vxb_request* req, int direction, uint32_t slice,
                          vxb_grid_info* info) {
    if (!v || !info) return failf(VXB_EINVAL, "NULL argument");
    if (direction == 0) {
        vxb::Plan q;
        bool oob = false;
        return v->planXSlice(req, slice, &q, &oob, info);
    }
    vxb_voxelizer::Space sp;
    bool oob = false;
    int rc = v->sliceSpace(req, direction, slice, &sp, &oob);
    if (rc) return rc;
    return v->planSpaces(1, req, std::vector<vxb_voxelizer::Space>{sp}, info);
}

vxb_status vxb_voxelize_slice_to_device(vxb_voxelizer* v, const vxb_request* req, int direction, uint32_t slice,
                                        void* dev_out, uint64_t dev_bytes, void* stream, vxb_grid_info* info) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    if (direction == 0)
        return v->runXSlice(req, slice, dev_out, dev_bytes, reinterpret_cast<cudaStream_t>(stream), info);
    vxb_voxelizer::Space sp;
    bool oob = false;
    int rc = v->sliceSpace(req, direction, slice, &sp, &oob);
    if (rc) return rc;
    const std::vector<vxb_voxelizer::Space> one{sp};
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!oob) return v->runSpaces(1, req, one, &dev_out, &dev_bytes, s, info);
    // sliceOOB (src/host_side.cpp:1225-1236): the reference voxelizes slice
    // 0 and then zeroes the array; the result is the zero array.
    vxb_grid_info gi;
    if ((rc = v->planSpaces(1, req, one, &gi))) return rc;
    if (info) *info = gi;
    if ((rc = v->validate(1, req))) return rc;
    if (!dev_out || dev_bytes < gi.bytes) return failf(VXB_EINVAL, "output buffer is NULL or too small");
    VXB_CUDA(cudaSetDevice(v->device));
    VXB_CUDA(cudaMemsetAsync(dev_out, 0, gi.bytes, s));
    VXB_CUDA(cudaStreamSynchronize(s));
    v->launches = 0;
    return VXB_OK;
}

vxb_status vxb_voxelize_slice_to_host(vxb_voxelizer* v, const vxb_request* req, int direction, uint32_t slice,
                                      void* host_out, uint64_t host_bytes, vxb_grid_info* info) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    vxb_grid_info gi;
    int rc = vxb_plan_slice(v, req, direction, slice, &gi);
    if (rc) return rc;
    if (info) *info = gi;
    if (!host_out || host_bytes < gi.bytes) return failf(VXB_EINVAL, "output buffer is NULL or too small");
    VXB_CUDA(cudaSetDevice(v->device));
    if ((rc = v->outStage.ensure(gi.bytes))) return rc;
    rc = vxb_voxelize_slice_to_device(v, req, direction, slice, v->outStage.p, gi.bytes, nullptr, info);
    if (rc == 0) {
        cudaError_t e = cudaMemcpy(host_out, v->outStage.p, gi.bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = failf(VXB_ECUDA, "%s", cudaGetErrorString(e));
    }
    return rc;
}

vxb_status vxb_voxelize_to_host(vxb_voxelizer* v, int nodes, const vxb_request* req, void* host_out,
                                uint64_t host_bytes, vxb_grid_info* info) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    vxb_grid_info gi;
    vxb::Plan p;
    int rc = v->plan(nodes, req, p, &gi);
    if (rc) return rc;
    if (info) *info = gi;
    if ((rc = v->validate(nodes, req))) return rc;
    if (!host_out) return failf(VXB_EINVAL, "output buffer is NULL");
    if (host_bytes < gi.bytes) return failf(VXB_EINVAL, "output buffer too small");
    VXB_CUDA(cudaSetDevice(v->device));
    if ((rc = v->outStage.ensure(gi.bytes))) return rc;
    // A pinned destination takes the node array range by range while it is
    // emitted (the copy overlaps the rest of the emission).
    cudaPointerAttributes pa;
    const bool pinned = cudaPointerGetAttributes(&pa, host_out) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
    if (pinned && !v->copyStream) VXB_CUDA(cudaStreamCreateWithFlags(&v->copyStream, cudaStreamNonBlocking));
    v->pipe.streamOutput(pinned && nodes ? host_out : nullptr, gi.bytes, v->copyStream);
    rc = v->run(nodes, req, v->outStage.p, gi.bytes, 0, info);
    const bool copied = v->pipe.hostCopied();
    v->pipe.streamOutput(nullptr, 0, nullptr);
    if (copied) {
        cudaError_t e = cudaStreamSynchronize(v->copyStream);
        if (rc == 0 && e != cudaSuccess) rc = failf(VXB_ECUDA, "%s", cudaGetErrorString(e));
    } else if (rc == 0) {
        cudaError_t e = cudaMemcpy(host_out, v->outStage.p, gi.bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = failf(VXB_ECUDA, "%s", cudaGetErrorString(e));
    }
    return rc;
}

vxb_status vxb_set_profiling(vxb_voxelizer* v, int enable) {
    if (!v) return failf(VXB_EINVAL, "voxelizer is NULL");
    if (enable < 0 || enable > 2) return failf(VXB_EINVAL, "profiling mode must be 0, 1 or 2");
    v->timer.enabled = enable != 0;
    v->timer.serial = enable == 2;
    return VXB_OK;
}

vxb_status vxb_stage_times(vxb_voxelizer* v, float* ms, uint32_t n) {
    if (!v || !ms) return failf(VXB_EINVAL, "NULL argument");
    for (uint32_t k = 0; k < n && k < (uint32_t)vxb::StageTimer::kStages; ++k) {
        ms[k] = -1.0f;
        if (!v->timer.enabled || !v->timer.used[k]) continue;
        cudaError_t e = cudaEventSynchronize(v->timer.ev[2 * k + 1]);
        if (e != cudaSuccess) return failf(VXB_ECUDA, "%s", cudaGetErrorString(e));
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, v->timer.ev[2 * k], v->timer.ev[2 * k + 1]) == cudaSuccess) ms[k] = t;
    }
    return VXB_OK;
}

vxb_status vxb_stage_timeline(vxb_voxelizer* v, float* start_end, uint32_t n) {
    if (!v || !start_end) return failf(VXB_EINVAL, "NULL argument");
    const vxb::StageTimer& T = v->timer;
    for (uint32_t k = 0; k < 2 * n; ++k) start_end[k] = NAN;
    if (!T.enabled || !T.used[0]) return VXB_OK;
    for (uint32_t k = 0; k < n && k < (uint32_t)vxb::StageTimer::kStages; ++k) {
        if (!T.used[k]) continue;
        cudaError_t e = cudaEventSynchronize(T.ev[2 * k + 1]);
        if (e != cudaSuccess) return failf(VXB_ECUDA, "%s", cudaGetErrorString(e));
        for (int j = 0; j < 2; ++j) {
            float t = 0.0f;
            if (cudaEventElapsedTime(&t, T.ev[0], T.ev[2 * k + j]) == cudaSuccess) start_end[2 * k + j] = t;
        }
    }
    return VXB_OK;
}

vxb_status vxb_last_launch_count(vxb_voxelizer* v, uint32_t* launches) {
    if (!v || !launches) return failf(VXB_EINVAL, "NULL argument");
    *launches = v->launches;
    return VXB_OK;
}

vxb_status vxb_last_stats(vxb_voxelizer* v, vxb_stats* stats) {
    if (!v || !stats) return failf(VXB_EINVAL, "NULL argument");
    *stats = v->pipe.stats;
    return VXB_OK;
}

// ---- batches ----

vxb_status vxb_batch_create(vxb_batch** out, int device) {
    if (!out) return failf(VXB_EINVAL, "out is NULL");
    *out = nullptr;
    vxb_batch* b = new (std::nothrow) vxb_batch();
    if (!b) return failf(VXB_ENOMEM, "out of host memory");
    b->device = device;
    *out = b;
    return VXB_OK;
}

vxb_status vxb_batch_destroy(vxb_batch* b) {
    if (!b) return VXB_OK;
    const int dev = b->device;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    if (b->busy) cudaDeviceSynchronize();
    delete b;
    if (cur != dev) cudaSetDevice(cur);
    return VXB_OK;
}

vxb_status vxb_batch_add(vxb_batch* b, vxb_voxelizer* v, int nodes, const vxb_request* req, void* dev_out,
                         uint64_t dev_bytes, vxb_grid_info* info) {
    if (!b || !v || !req) return failf(VXB_EINVAL, "NULL argument");
    if (v->device != b->device) return failf(VXB_EINVAL, "voxelizer and batch are on different devices");
    vxb::Plan p;
    vxb_grid_info gi;
    int rc = v->plan(nodes, req, p, &gi);
    if (rc) return rc;
    if (info) *info = gi;
    if ((rc = v->validate(nodes, req))) return rc;
    if (!dev_out) return failf(VXB_EINVAL, "output buffer is NULL");
    if (dev_bytes < gi.bytes) return failf(VXB_EINVAL, "output buffer too small");
    if (!b->entries.empty()) {
        const vxb_batch::Entry& e0 = b->entries.front();
        if (e0.v->nodeType != v->nodeType || e0.nodes != (nodes ? 1 : 0))
            return failf(VXB_EINVAL, "all meshes of a batch need the same node type and output kind");
    }
    b->entries.push_back(vxb_batch::Entry{v, nodes ? 1 : 0, *req, dev_out, dev_bytes});
    b->prepared = false;
    b->dropGraph();
    return VXB_OK;
}

vxb_status vxb_batch_clear(vxb_batch* b) {
    if (!b) return failf(VXB_EINVAL, "batch is NULL");
    b->entries.clear();
    b->prepared = false;
    b->dropGraph();
    return VXB_OK;
}

vxb_status vxb_batch_run(vxb_batch* b, void* stream, int flags) {
    if (!b) return failf(VXB_EINVAL, "batch is NULL");
    if (b->entries.empty()) return failf(VXB_EINVAL, "empty batch");
    VXB_CUDA(cudaSetDevice(b->device));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const bool useGraph = (flags & VXB_BATCH_GRAPH) != 0;
    if (useGraph && s == nullptr) {
        // The legacy default stream cannot be captured: run on the batch's
        // own stream, ordered after the caller's default-stream work.
        if (!b->own) VXB_CUDA(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking));
        VXB_CUDA(cudaStreamSynchronize(nullptr));
        s = b->own;
    }
    int rc;
    b->busy = true;
    for (const vxb_batch::Entry& e : b->entries) e.v->busy = true;
    if (!b->prepared) {
        std::vector<vxb::MeshJob> jobs(b->entries.size());
        for (size_t i = 0; i < jobs.size(); ++i) {
            const vxb_batch::Entry& e = b->entries[i];
            if ((rc = e.v->upload(s))) return rc;
            e.v->job(e.nodes, &e.req, e.out, e.bytes, &jobs[i]);
        }
        if ((rc = b->pipe.prepare(jobs, s))) return rc;
        b->prepared = true;
        b->dropGraph();
    }
    if (useGraph) {
        if (!b->exec || b->graphStream != s) {
            b->dropGraph();
            VXB_CUDA(cudaStreamSynchronize(s));
            VXB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            rc = b->pipe.enqueue(s, nullptr);
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(s, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) {
                cudaGetLastError();
                return failf(VXB_ECUDA, "graph capture failed: %s", cudaGetErrorString(e));
            }
            b->graph = g;
            b->graphKernels = b->pipe.launches;
            VXB_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
            b->graphStream = s;
        }
        VXB_CUDA(cudaGraphLaunch(b->exec, s));
        b->pipe.launches = 0;
        rc = b->pipe.finish(s);
        b->launches = b->graphKernels + b->pipe.launches;
    } else {
        if ((rc = b->pipe.enqueue(s, nullptr))) return rc;
        rc = b->pipe.finish(s);
        b->launches = b->pipe.launches;
    }
    if (rc == 0) {
        b->busy = false;
        for (const vxb_batch::Entry& e : b->entries) e.v->busy = false;
    }
    return rc;
}

vxb_status vxb_batch_last_launch_count(vxb_batch* b, uint32_t* launches) {
    if (!b || !launches) return failf(VXB_EINVAL, "NULL argument");
    *launches = b->launches;
    return VXB_OK;
}

}  // extern "C"
