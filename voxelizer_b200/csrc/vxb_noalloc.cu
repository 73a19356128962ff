// vxb_voxelize_bits_noalloc: the plain (solid) voxelization of
// vxb_voxelize_to_device(v, 0, ...) for callers that cannot allocate device
// memory.  Such callers exist because the FDTD codes this library feeds
// often reserve all of a GPU's memory for their field arrays up front and
// hand out slices of that pool themselves, and because cudaFree (and at
// times cudaMalloc) synchronizes the whole device, which a caller that keeps
// several streams busy cannot afford in the middle of a time step.  The
// caller passes the mesh and the output already in device memory; the work
// lists this path needs (a range-checked copy of the indices, per-triangle
// candidate counts, their scan, the yz subspace table and the unit table)
// live in a fixed, statically sized array in device memory instead of
// buffers allocated per call.  The call itself allocates nothing, on the
// device or on the host; its tables are passed to a set-up kernel by value,
// so it copies nothing from host memory either.  The array is placed by the
// CUDA driver when it loads this library's device code.
//
// Limits: at most kMaxTriangles triangles and kMaxSubspaces yz subspaces
// per call, and fewer than 2^32 (triangle, subspace, tile) candidates by the
// bound checked below; larger requests are rejected with VXB_EINVAL.
//
// Errors found on the device (an index >= n_vertices, a candidate count
// that overflows) cannot be returned by the call, which does not wait for
// the GPU; vxb_noalloc_status() reports them for the last call on the
// current device once its stream has finished.
//
// The first call on a device looks up the array's device address (a
// one-time set-up per device, made with that device current); make that
// first call before any stream capture.
//
// The array is shared by every call on a device and keeps the previous
// call's contents; each call clears its status words and overwrites
// everything else it reads before reading it.  Calls whose work overlaps on
// the GPU (two host threads, or two streams without ordering between them)
// race on the array and give undefined results: serialize them.

#include "vxb.h"
#include "vxb_kernels.cuh"
#include "vxb_plan.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

namespace vxb {
int recordError(int code, const char* msg);  // vxb_host.cu
}

namespace {

constexpr uint32_t kMaxTriangles = 1u << 20;  // 1,048,576
constexpr uint32_t kMaxSubspaces = 1024;
constexpr uint32_t kScanTile = 4096;          // items per tile of launch_scan
constexpr int kMaxDevices = 64;

constexpr size_t roundUp(size_t v) { return (v + 255) / 256 * 256; }

// The one-unit batch tables the kernels read.
struct UnitTables {
    vxb::Unit unit;
    uint32_t workBase[2];
    uint32_t pad[2];
    uint64_t rowBase[2];
    uint64_t wordBase[2];
};

// Layout of the scratch array (byte offsets).
constexpr size_t kStatusOff = 0;  // [0] candidate total, [1] overflow flag, [2] index out of range
constexpr size_t kTablesOff = kStatusOff + 256;
constexpr size_t kSubspaceOff = kTablesOff + 768;
static_assert(sizeof(UnitTables) <= 768, "tables region");
constexpr size_t kTileOff = kSubspaceOff + roundUp(kMaxSubspaces * sizeof(vxb::SplitYZ));
constexpr size_t kCountOff = kTileOff + roundUp(4 * (kMaxTriangles / kScanTile + 2));
constexpr size_t kOffsetOff = kCountOff + roundUp(4 * ((size_t)kMaxTriangles + 1));
constexpr size_t kIndexOff = kOffsetOff + roundUp(4 * ((size_t)kMaxTriangles + 2));
constexpr size_t kScratchBytes = kIndexOff + roundUp(12 * (size_t)kMaxTriangles);
static_assert(kScratchBytes == 20990720, "scratch layout changed: update the stated size");

}  // namespace

// 20,990,720 bytes (about 20.0 MiB) of device memory, held by every GPU that
// loads this library until the process exits.
static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

namespace {

void* g_scratchAddress[kMaxDevices] = {};
std::mutex g_setupLock;

int failf(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int failf(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return vxb::recordError(code, buf);
}

// Device address of the scratch array on `device` (the current device).  In
// host code g_noallocScratch names a host-side shadow, not device memory, so
// the address is looked up once per device and cached.
int scratchAddress(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_setupLock);
    if (!g_scratchAddress[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return failf(VXB_ECUDA, "cudaGetSymbolAddress of the scratch array failed on device %d: %s", device,
                         cudaGetErrorString(e));
        }
        g_scratchAddress[device] = p;
    }
    *out = static_cast<unsigned char*>(g_scratchAddress[device]);
    return 0;
}

// Set-up of one call: the unit table (by value), the yz subspaces of the
// solid pass in the reference's order (z outer; splitResolutionByNrOfParts
// per axis) and cleared status words.
__global__ void noallocSetupKernel(UnitTables tab, uint32_t resY, uint32_t resZ, uint32_t splitY, uint32_t splitZ,
                                   UnitTables* dtab, vxb::SplitYZ* dsub, uint32_t* status) {
    if (threadIdx.x == 0) {
        *dtab = tab;
        status[0] = status[1] = status[2] = 0u;
    }
    const uint32_t ny = (resY + splitY - 1) / splitY, nz = (resZ + splitZ - 1) / splitZ;
    for (uint32_t k = threadIdx.x; k < ny * nz; k += blockDim.x) {
        const vxb::Range ry = vxb::splitPart(resY, splitY, k % ny), rz = vxb::splitPart(resZ, splitZ, k / ny);
        dsub[k] = vxb::SplitYZ{ry.lo, ry.hi, rz.lo, rz.hi};
    }
}

// The caller's indices, range-checked: an index >= nV reads vertex 0
// instead and sets status[2], so no kernel reads past the vertex buffer.
__global__ void noallocIndexKernel(const uint32_t* __restrict__ idx, uint32_t n, uint32_t nV, uint32_t* __restrict__ out,
                                   uint32_t* status) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t v = idx[i];
        if (v >= nV) {
            v = 0u;
            status[2] = 1u;
        }
        out[i] = v;
    }
}

}  // namespace

extern "C" vxb_status vxb_voxelize_bits_noalloc(const float* dev_vertices, const uint32_t* dev_indices,
                                                uint32_t n_vertices, uint32_t n_triangles,
                                                const double* min_vertex, const double* max_vertex,
                                                const vxb_request* req, void* dev_out, uint64_t dev_bytes,
                                                void* stream, vxb_grid_info* info) {
    if (!dev_vertices || !dev_indices || !min_vertex || !max_vertex || !req || !dev_out)
        return failf(VXB_EINVAL, "NULL argument");
    if (n_vertices == 0 || n_triangles == 0) return failf(VXB_EINVAL, "empty mesh");
    if (n_triangles > kMaxTriangles)
        return failf(VXB_EINVAL,
                     "%u triangles exceed the %u that the allocation-free path's fixed scratch array holds; "
                     "use vxb_voxelize_to_device",
                     n_triangles, kMaxTriangles);
    vxb::GridSize bg;
    const uint32_t vs[3] = {req->vox_split_res.x, req->vox_split_res.y, req->vox_split_res.z};
    if (vxb::sizeGrid(min_vertex, max_vertex, req->by_cube_length, req->max_dimension, req->cube_length, vs, bg))
        return failf(VXB_EINVAL, "invalid request (maxDimension >= 2 or cubeLength > 0, split sizes > 0 and an x "
                                 "pass of at most 1024 voxels are required)");
    const uint64_t voxels = (uint64_t)bg.alloc[0] * bg.alloc[1] * bg.alloc[2];
    if (voxels > 0xFFFFFFFFull) return failf(VXB_EOVERFLOW, "voxel grid exceeds 32-bit indexing");
    const uint32_t ny = (bg.res[1] + req->vox_split_res.y - 1) / req->vox_split_res.y;
    const uint32_t nz = (bg.res[2] + req->vox_split_res.z - 1) / req->vox_split_res.z;
    if ((uint64_t)ny * nz > kMaxSubspaces)
        return failf(VXB_EINVAL,
                     "%llu yz subspaces exceed the %u that the allocation-free path's fixed scratch array holds; "
                     "use larger split sizes",
                     (unsigned long long)ny * nz, kMaxSubspaces);
    // A triangle is a candidate at most once per (subspace, 4x4 tile) pair
    // it overlaps, and a subspace cut adds at most one partial tile per
    // axis: keep the scan of candidate counts below 2^32.
    const double bound = (double)n_triangles * (double)((bg.res[1] + 3) / 4 + ny) * (double)((bg.res[2] + 3) / 4 + nz);
    if (bound >= 4294967295.0)
        return failf(VXB_EINVAL,
                     "up to %.0f (triangle, tile) candidates: the allocation-free path takes fewer than 2^32; use "
                     "vxb_voxelize_to_device",
                     bound);
    vxb_grid_info gi;
    memset(&gi, 0, sizeof(gi));
    gi.dim.x = bg.alloc[0];
    gi.dim.y = bg.alloc[1];
    gi.dim.z = bg.alloc[2];
    gi.count = voxels / 32;
    gi.bytes = gi.count * 4;
    gi.voxel_length = bg.d;
    for (int a = 0; a < 3; ++a) {
        gi.min_vertex[a] = min_vertex[a];
        gi.max_vertex[a] = max_vertex[a];
    }
    gi.resolution.x = bg.res[0];
    gi.resolution.y = bg.res[1];
    gi.resolution.z = bg.res[2];
    gi.x_splits = bg.xSplits;
    if (info) *info = gi;
    if (dev_bytes < gi.bytes)
        return failf(VXB_EINVAL, "output buffer holds %llu bytes, %llu needed", (unsigned long long)dev_bytes,
                     (unsigned long long)gi.bytes);

    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return failf(VXB_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices) return failf(VXB_EINVAL, "device %d is not supported", device);
    unsigned char* scratch = nullptr;
    if (int rc = scratchAddress(device, &scratch)) return rc;

    const uint32_t nSub = ny * nz;
    UnitTables tab;
    memset(&tab, 0, sizeof(tab));
    vxb::PassGeom& g = tab.unit.g;
    for (int a = 0; a < 3; ++a) {
        g.mn[a] = min_vertex[a];
        g.mnf[a] = (float)min_vertex[a];
    }
    g.d = bg.d;
    g.df = (float)bg.d;
    g.X = bg.res[0];
    g.resY = bg.res[1];
    g.resZ = bg.res[2];
    g.AY = bg.alloc[1];
    g.AZ = bg.alloc[2];
    g.ipx = bg.res[0] / 32;
    g.padY = 1;
    g.padZ = 1;
    g.border = 0;
    uint32_t* checkedIdx = reinterpret_cast<uint32_t*>(scratch + kIndexOff);
    tab.unit.V = dev_vertices;
    tab.unit.I = checkedIdx;
    tab.unit.nT = n_triangles;
    tab.unit.nSplits = nSub;
    tab.unit.out = dev_out;
    tab.workBase[1] = n_triangles;
    tab.rowBase[1] = (uint64_t)g.AY * g.AZ;
    tab.wordBase[1] = (uint64_t)g.ipx * g.AY * g.AZ;

    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t* status = reinterpret_cast<uint32_t*>(scratch + kStatusOff);
    UnitTables* dtab = reinterpret_cast<UnitTables*>(scratch + kTablesOff);
    vxb::SplitYZ* dsub = reinterpret_cast<vxb::SplitYZ*>(scratch + kSubspaceOff);
    uint32_t* tiles = reinterpret_cast<uint32_t*>(scratch + kTileOff);
    uint32_t* counts = reinterpret_cast<uint32_t*>(scratch + kCountOff);
    uint32_t* offsets = reinterpret_cast<uint32_t*>(scratch + kOffsetOff);
    uint32_t* grid = static_cast<uint32_t*>(dev_out);
    vxb::Batch b;
    memset(&b, 0, sizeof(b));
    b.units = &dtab->unit;
    b.nUnits = 1;
    b.workBase = dtab->workBase;
    b.rowBase = dtab->rowBase;
    b.wordBase = dtab->wordBase;
    b.splits = dsub;
    uint32_t launches = 0;
    e = cudaMemsetAsync(grid, 0, gi.bytes, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return failf(VXB_ECUDA, "%s", cudaGetErrorString(e));
    }
    noallocSetupKernel<<<1, 256, 0, s>>>(tab, bg.res[1], bg.res[2], req->vox_split_res.y, req->vox_split_res.z, dtab,
                                         dsub, status);
    const uint32_t nIdx = 3u * n_triangles;
    noallocIndexKernel<<<(nIdx + 255) / 256 < 148u * 8u ? (nIdx + 255) / 256 : 148u * 8u, 256, 0, s>>>(
        dev_indices, nIdx, n_vertices, checkedIdx, status);
    launches += 2;
    vxb::launch_solid_count(b, n_triangles, counts, s, &launches);
    vxb::launch_scan(counts, offsets, n_triangles, tiles, status, status + 1, s, &launches);
    vxb::launch_solid_toggle(b, n_triangles, offsets, status, grid, 3, nullptr, s, &launches);
    vxb::launch_row_fill(b, tab.rowBase[1], grid, s, &launches);
    e = cudaGetLastError();
    if (e != cudaSuccess) return failf(VXB_ECUDA, "%s", cudaGetErrorString(e));
    return VXB_OK;
}

extern "C" vxb_status vxb_noalloc_status(void) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return failf(VXB_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices) return failf(VXB_EINVAL, "device %d is not supported", device);
    unsigned char* scratch = nullptr;
    if (int rc = scratchAddress(device, &scratch)) return rc;
    uint32_t st[3] = {0, 0, 0};
    e = cudaMemcpy(st, scratch + kStatusOff, sizeof(st), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return failf(VXB_ECUDA, "reading the status words: %s", cudaGetErrorString(e));
    }
    if (st[2]) return failf(VXB_EINVAL, "the last call's mesh has an index >= n_vertices; its bit array is undefined");
    if (st[1]) return failf(VXB_EOVERFLOW, "the last call's candidate count overflowed; its bit array is undefined");
    return VXB_OK;
}
