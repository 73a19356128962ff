// Host orchestration and the C ABI (include/vxb.h).
//
// One vxb_voxelizer holds a copy of the mesh (as the reference's constructor
// does, src/host_side.cpp:72-99), its device copy, and scratch buffers that
// grow on demand and are reused across calls.  A voxelization is a fixed
// sequence of stream-ordered launches; the only host round trip is one
// small read after the pruning passes are queued (convergence flags, hit
// list length and surface voxel count), repeated only when a pruning
// subspace needs more passes.

#include "vxb.h"
#include "vxb_kernels.cuh"
#include "vxb_plan.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

namespace {

thread_local std::string g_lastError;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
    return code;
}

#define VXB_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) return fail(VXB_ECUDA, "%s @ %s:%d", cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

const uint32_t kNodeBytes[5] = {1, 2, 8, 2, 4};
const uint32_t kMaxMat[5] = {7, 255, 255, 15, 255};

bool isFcc(int t) { return t == VXB_SHORT_FCC_NODE || t == VXB_LONG_FCC_NODE; }

// Process-wide cache of idle device blocks.  Buffers of destroyed
// voxelizers (and buffers outgrown by a larger request) go here instead of
// cudaFree, and the next allocation of a similar size takes them back, so a
// caller that builds one voxelizer per mesh pays cudaMalloc / cudaFree once.
// Blocks enter the cache only after the device has finished all work, which
// keeps them free of in-flight kernels.  Idle bytes are capped; vxb_trim_cache
// returns them all to the driver.
struct BlockCache {
    std::mutex mu;
    std::multimap<size_t, std::pair<int, void*>> idle;   // bytes -> (device, block)
    size_t idleBytes = 0;
    static constexpr size_t kBudget = 16ull << 30;
};

BlockCache& blockCache() {
    static BlockCache* c = new BlockCache;   // never destroyed: blocks outlive static destructors
    return *c;
}

void* cacheTake(int device, size_t bytes, size_t* got) {
    BlockCache& c = blockCache();
    std::lock_guard<std::mutex> lock(c.mu);
    for (auto it = c.idle.lower_bound(bytes); it != c.idle.end() && it->first <= 2 * bytes + (1u << 20); ++it) {
        if (it->second.first != device) continue;
        void* p = it->second.second;
        *got = it->first;
        c.idleBytes -= it->first;
        c.idle.erase(it);
        return p;
    }
    return nullptr;
}

// `p` must no longer be used by any queued work.
void cacheGive(int device, void* p, size_t bytes) {
    BlockCache& c = blockCache();
    {
        std::lock_guard<std::mutex> lock(c.mu);
        if (c.idleBytes + bytes <= BlockCache::kBudget) {
            c.idle.emplace(bytes, std::make_pair(device, p));
            c.idleBytes += bytes;
            return;
        }
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    cudaFree(p);
    if (cur != device) cudaSetDevice(cur);
}

// A device buffer that only grows, backed by the block cache.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    int dev = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    // Owners call this after the device has drained their work.
    void release() {
        if (p) cacheGive(dev, p, cap);
        p = nullptr;
        cap = 0;
    }
    ~DevBuf() { release(); }
    int ensure(size_t bytes) {
        if (bytes <= cap) return 0;
        if (p) {
            cudaError_t e = cudaDeviceSynchronize();
            if (e != cudaSuccess) return fail(VXB_ECUDA, "%s", cudaGetErrorString(e));
            release();
        }
        cudaGetDevice(&dev);
        size_t got = 0;
        if ((p = cacheTake(dev, bytes, &got))) {
            cap = got;
            return 0;
        }
        size_t want = bytes + bytes / 8 + 256;
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return fail(VXB_ENOMEM, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
        }
        cap = want;
        return 0;
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// Slots of the small device status buffer.
enum : int { kSolidTotal = 0, kSolidOverflow = 1, kSurfTotal = 2, kSurfOverflow = 3, kHitCount = 4,
             kSurfaceVoxels = 5, kFlags = 8 };

}  // namespace

namespace vxb {
// Stores `msg` as the calling thread's vxb_last_error message and returns
// `code`; for entry points defined in other files.
int recordError(int code, const char* msg) { return fail(code, "%s", msg); }
}  // namespace vxb

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
    DevBuf dV, dI, dM;
    // scratch
    DevBuf counts, offsets, tileSums, small, codes, splitsBuf, matSplitsBuf, laterFlags, outStage;
    DevBuf units, perm, buckets, recs, ovl;  // surface pass partition and set-up records
    DevBuf fill[4], surfAll, fin, ranks, rankTiles, hitList, keys;
    uint32_t launches = 0;
    // Optional per-stage CUDA-event timing (vxb_set_profiling): stage k is
    // bracketed by events 2k and 2k+1 on the call's stream.
    static constexpr int kStages = 5;  // 0 solid, 1 surface, 2 prune, 3 emit, 4 material merge
    bool profiling = false;
    cudaEvent_t ev[2 * kStages] = {};
    bool evUsed[kStages] = {};
    void mark(int stage, bool end, cudaStream_t s) {
        if (!profiling) return;
        if (!ev[0])
            for (auto& e : ev) cudaEventCreate(&e);
        cudaEventRecord(ev[2 * stage + (end ? 1 : 0)], s);
        evUsed[stage] = true;
    }
    ~vxb_voxelizer() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }

    int plan(int nodes, const vxb_request* r, vxb::Plan& p, vxb_grid_info* info);
    // Combinations the reference refuses (src/host_side.cpp:568-573,
    // 1744-1749, 1836-1841, 2280-2285) and missing materials.
    int validate(int nodes, const vxb_request* r) const {
        if (!nodes && isFcc(nodeType))
            return fail(VXB_EUNSUPPORTED, "Please use a standard Node-type when producing a plain voxelization.");
        if (nodes && isFcc(nodeType) && !r->by_cube_length)
            return fail(VXB_EUNSUPPORTED,
                        "FCC Nodes can currently only be defined through the side length of their cubic cells");
        if (nodes && materialsOn && materials.empty())
            return fail(VXB_ENOMATERIALS, "material output requested but no materials were set");
        return 0;
    }
    int upload(cudaStream_t s);
    int run(int nodes, const vxb_request* r, void* dout, uint64_t bytes, cudaStream_t s, vxb_grid_info* info);
    int solidPass(const vxb::Plan& p, const vxb::PassGeom& g, uint32_t* grid, cudaStream_t s);
    int surfacePass(const vxb::Plan& p, const vxb::PassGeom& g, int lattice, size_t gridWords, int mode,
                    cudaStream_t s);
    int resolveKeys(const vxb::Plan& p, int lattices, size_t gridWords, uint32_t hitCount, uint32_t surfaceVoxels,
                    cudaStream_t s);
    uint32_t listCap = 0;
};

namespace {

vxb::PassGeom makeGeom(const vxb::Plan& p, double sx, double sy, double sz) {
    vxb::PassGeom g;
    g.mn[0] = p.mn[0] + sx;
    g.mn[1] = p.mn[1] + sy;
    g.mn[2] = p.mn[2] + sz;
    g.d = p.d;
    for (int a = 0; a < 3; ++a) g.mnf[a] = (float)g.mn[a];
    g.df = (float)p.d;
    g.X = p.res[0];
    g.resY = p.res[1];
    g.resZ = p.res[2];
    g.AY = p.alloc[1];
    g.AZ = p.alloc[2];
    g.ipx = p.res[0] / 32;
    return g;
}

// Shifts of the four FCC sub-lattices (src/host_side.cpp:1438-1462).
void latticeShift(const vxb::Plan& p, int lattice, double* sh) {
    const double h = p.d / 2.0;
    const double s[4][3] = {{0.0, 0.0, 0.0}, {h, h, 0.0}, {0.0, h, h}, {h, 0.0, h}};
    for (int a = 0; a < 3; ++a) sh[a] = s[lattice][a];
}

}  // namespace

int vxb_voxelizer::plan(int nodes, const vxb_request* r, vxb::Plan& p, vxb_grid_info* info) {
    if (!r) return fail(VXB_EINVAL, "request is NULL");
    if (nV == 0 || nT == 0) return fail(VXB_EINVAL, "empty mesh");
    const uint32_t vs[3] = {r->vox_split_res.x, r->vox_split_res.y, r->vox_split_res.z};
    const uint32_t ms[3] = {r->mat_split_res.x, r->mat_split_res.y, r->mat_split_res.z};
    int rc = vxb::makePlan(mn, mx, r->by_cube_length, r->max_dimension, r->cube_length, vs, ms, p);
    if (rc) return fail(VXB_EINVAL, "invalid request (maxDimension >= 2 or cubeLength > 0, split sizes > 0 and an x pass of at most 1024 voxels are required)");
    const bool fcc = isFcc(nodeType);
    vxb_grid_info gi;
    memset(&gi, 0, sizeof(gi));
    if (nodes) {
        gi.dim.x = fcc ? 2 * p.alloc[0] : p.alloc[0];
        gi.dim.y = p.alloc[1];
        gi.dim.z = fcc ? 2 * p.alloc[2] : p.alloc[2];
        gi.count = (uint64_t)gi.dim.x * gi.dim.y * gi.dim.z;
        gi.bytes = gi.count * kNodeBytes[nodeType];
        // The reference indexes nodes with 32-bit unsigned integers.
        if (gi.count > 0xFFFFFFFFull) return fail(VXB_EOVERFLOW, "node grid of %llu nodes exceeds 32-bit indexing", (unsigned long long)gi.count);
    } else {
        gi.dim.x = p.alloc[0];
        gi.dim.y = p.alloc[1];
        gi.dim.z = p.alloc[2];
        gi.count = (uint64_t)p.alloc[0] * p.alloc[1] * p.alloc[2] / 32;
        gi.bytes = gi.count * 4;
        if ((uint64_t)p.alloc[0] * p.alloc[1] * p.alloc[2] > 0xFFFFFFFFull)
            return fail(VXB_EOVERFLOW, "voxel grid exceeds 32-bit indexing");
    }
    gi.voxel_length = p.d;
    for (int a = 0; a < 3; ++a) { gi.min_vertex[a] = mn[a]; gi.max_vertex[a] = mx[a]; }
    gi.resolution.x = p.res[0];
    gi.resolution.y = p.res[1];
    gi.resolution.z = p.res[2];
    gi.x_splits = p.xSplits;
    if (info) *info = gi;
    return 0;
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

// Solid voxelization of one (sub-)lattice into `grid` (zeroed here): count
// candidates, scan, toggle, row fill.
int vxb_voxelizer::solidPass(const vxb::Plan& p, const vxb::PassGeom& g, uint32_t* grid, cudaStream_t s) {
    const size_t words = (size_t)g.ipx * g.AY * g.AZ;
    VXB_CUDA(cudaMemsetAsync(grid, 0, words * 4, s));
    std::vector<vxb::SplitYZ> sp;
    for (const auto& z : p.zSplitsExt)
        for (const auto& y : p.ySplitsExt) sp.push_back(vxb::SplitYZ{y.lo, y.hi, z.lo, z.hi});
    int rc;
    if ((rc = splitsBuf.ensure(sp.size() * sizeof(vxb::SplitYZ) + 64))) return rc;
    VXB_CUDA(cudaMemcpyAsync(splitsBuf.p, sp.data(), sp.size() * sizeof(vxb::SplitYZ), cudaMemcpyHostToDevice, s));
    uint32_t* cnt = counts.as<uint32_t>();
    uint32_t* off = offsets.as<uint32_t>();
    uint32_t* sm = small.as<uint32_t>();
    vxb::launch_solid_count(dV.as<float>(), dI.as<uint32_t>(), nT, g, splitsBuf.as<vxb::SplitYZ>(), (uint32_t)sp.size(),
                            cnt, s, &launches);
    vxb::launch_scan(cnt, off, nT, tileSums.as<uint32_t>(), sm + kSolidTotal, sm + kSolidOverflow, s, &launches);
    vxb::launch_solid_toggle(dV.as<float>(), dI.as<uint32_t>(), nT, g, splitsBuf.as<vxb::SplitYZ>(),
                             (uint32_t)sp.size(), off, sm + kSolidTotal, grid, s, &launches);
    vxb::launch_row_fill(grid, g.AY * g.AZ, g.ipx, s, &launches);
    VXB_CUDA(cudaGetLastError());
    return 0;
}

// Surface voxelization of one (sub-)lattice.  mode 0: set its surface bits
// (zeroed here) and append hits to the hit list; mode 1: merge every hit's
// key at its rank (the fallback when the list overflowed, and the path for
// 64-bit PartialNode keys).
int vxb_voxelizer::surfacePass(const vxb::Plan& p, const vxb::PassGeom& g, int lattice, size_t gridWords, int mode,
                               cudaStream_t s) {
    uint32_t* bits = surfAll.as<uint32_t>() + lattice * gridWords;
    if (mode == 0) VXB_CUDA(cudaMemsetAsync(bits, 0, gridWords * 4, s));
    // Material subspace slices per axis (src/host_side.cpp:2301-2337 passes
    // matSplitRes to the surface launches).
    std::vector<uint32_t> sl;
    vxb::SliceTable st;
    const std::vector<vxb::Range>* axes[3] = {&p.xMat, &p.yMat, &p.zMat};
    for (int a = 0; a < 3; ++a) {
        st.off[a] = (uint32_t)(sl.size() / 2);
        st.n[a] = (uint32_t)axes[a]->size();
        for (const auto& r : *axes[a]) { sl.push_back(r.lo); sl.push_back(r.hi); }
    }
    int rc;
    if ((rc = matSplitsBuf.ensure(sl.size() * 4 + 64))) return rc;
    VXB_CUDA(cudaMemcpyAsync(matSplitsBuf.p, sl.data(), sl.size() * 4, cudaMemcpyHostToDevice, s));
    uint32_t* sm = small.as<uint32_t>();
    VXB_CUDA(cudaMemsetAsync(buckets.p, 0, 2 * vxb::kSurfaceBuckets * 4, s));
    VXB_CUDA(cudaMemsetAsync(counts.p, 0, 4 * ((size_t)nT + 1), s));
    vxb::launch_surface_prepare(dV.as<float>(), dI.as<uint32_t>(), dM.as<uint8_t>(), nT, g, codes.as<uint32_t>(),
                                units.as<uint32_t>(), buckets.as<uint32_t>(), perm.as<uint32_t>(), counts.as<uint32_t>(),
                                recs.p, ovl.p, s, &launches);
    vxb::launch_scan(counts.as<uint32_t>(), offsets.as<uint32_t>(), nT, tileSums.as<uint32_t>(), sm + kSurfTotal,
                     sm + kSurfOverflow, s, &launches);
    vxb::launch_surface_work(mode, nodeType == VXB_PARTIAL_NODE ? 1 : 0, recs.p, ovl.p, offsets.as<uint32_t>(), nT,
                             sm + kSurfTotal, buckets.as<uint32_t>(), g, matSplitsBuf.as<uint32_t>(), st, bits,
                             (uint64_t)lattice * gridWords * 32, ranks.as<uint32_t>(), keys.p,
                             hitList.as<unsigned long long>(), sm + kHitCount, listCap, s, &launches);
    VXB_CUDA(cudaGetLastError());
    return 0;
}

// Material keys by surface rank: zero them, then merge the hit list, or
// re-run the surface passes in mode 1 when the list overflowed (or for
// 64-bit keys).  hitCount / surfaceVoxels were read back by the caller.
int vxb_voxelizer::resolveKeys(const vxb::Plan& p, int lattices, size_t gridWords, uint32_t hitCount,
                               uint32_t surfaceVoxels, cudaStream_t s) {
    const bool wide = nodeType == VXB_PARTIAL_NODE;
    int rc;
    if ((rc = keys.ensure((size_t)(surfaceVoxels + 1) * (wide ? 8 : 4)))) return rc;
    uint32_t* sm = small.as<uint32_t>();
    vxb::launch_surface_keys_zero(keys.p, sm + kSurfaceVoxels, wide ? 1 : 0, s, &launches);
    if (!wide && hitCount <= listCap) {
        vxb::launch_surface_merge(hitList.as<unsigned long long>(), sm + kHitCount, listCap, surfAll.as<uint32_t>(),
                                  ranks.as<uint32_t>(), keys.as<uint32_t>(), s, &launches);
        return 0;
    }
    for (int lt = 0; lt < lattices; ++lt) {
        double sh[3];
        latticeShift(p, lt, sh);
        vxb::PassGeom g = makeGeom(p, sh[0], sh[1], sh[2]);
        if ((rc = surfacePass(p, g, lt, gridWords, 1, s))) return rc;
    }
    return 0;
}

int vxb_voxelizer::run(int nodes, const vxb_request* r, void* dout, uint64_t bytes, cudaStream_t s,
                       vxb_grid_info* info) {
    vxb::Plan p;
    vxb_grid_info gi;
    int rc = plan(nodes, r, p, &gi);
    if (rc) return rc;
    if (info) *info = gi;
    if (!dout) return fail(VXB_EINVAL, "output buffer is NULL");
    if (bytes < gi.bytes) return fail(VXB_EINVAL, "output buffer holds %llu bytes, %llu needed",
                                      (unsigned long long)bytes, (unsigned long long)gi.bytes);
    if ((rc = validate(nodes, r))) return rc;
    VXB_CUDA(cudaSetDevice(device));
    launches = 0;
    for (bool& u : evUsed) u = false;
    const bool mats = nodes && materialsOn;
    if ((rc = upload(s))) return rc;
    const size_t words = (size_t)(p.res[0] / 32) * p.alloc[1] * p.alloc[2];
    const size_t gridWords = ((words + 63) / 64) * 64;
    const size_t gridBytes = gridWords * 4;
    if ((rc = counts.ensure(4 * ((size_t)nT + 1)))) return rc;
    if ((rc = offsets.ensure(4 * ((size_t)nT + 2)))) return rc;
    if ((rc = tileSums.ensure(4 * ((size_t)nT / 4096 + 2)))) return rc;
    // Status slots plus three pruning flags per pruning subspace; sized here
    // so that it never moves while kernels of this call use it.
    if ((rc = small.ensure(4 * (kFlags + 3 * p.ySplitsAlloc.size() * p.zSplitsAlloc.size()) + 256))) return rc;
    const int lattices = isFcc(nodeType) ? 4 : 1;
    if (mats) {
        if ((rc = codes.ensure(4 * (size_t)nT))) return rc;
        if ((rc = units.ensure(4 * (size_t)nT))) return rc;
        if ((rc = perm.ensure(4 * (size_t)nT))) return rc;
        if ((rc = buckets.ensure(4 * 2 * vxb::kSurfaceBuckets))) return rc;
        if ((rc = recs.ensure(vxb::kSurfRecBytes * (size_t)nT))) return rc;
        if ((rc = ovl.ensure(vxb::kSurfOvlBytes * (size_t)nT))) return rc;
        if ((rc = surfAll.ensure(gridBytes * lattices))) return rc;
        if ((rc = ranks.ensure(gridBytes * lattices))) return rc;
        if ((rc = rankTiles.ensure(4 * (gridWords * lattices / 2048 + 2)))) return rc;
        // Hit list: 8-byte entries (bit position << 24 | key); PartialNode
        // keys are 64-bit and always take the second traversal.
        const uint64_t want = nodeType == VXB_PARTIAL_NODE
                                  ? 0
                                  : std::min<uint64_t>(96ull << 20, std::max<uint64_t>(8ull << 20, gi.count / 12));
        listCap = (uint32_t)want;
        if (want && (rc = hitList.ensure(want * 8))) return rc;
        VXB_CUDA(cudaMemsetAsync(small.as<uint32_t>() + kHitCount, 0, 4, s));
    }

    if (!nodes) {
        // Plain voxelization: the caller's buffer is the toggle / solid grid.
        vxb::PassGeom g = makeGeom(p, 0.0, 0.0, 0.0);
        if ((rc = solidPass(p, g, reinterpret_cast<uint32_t*>(dout), s))) return rc;
        return 0;
    }
    uint32_t* sm = small.as<uint32_t>();
    if (!isFcc(nodeType)) {
        vxb::PassGeom g = makeGeom(p, 0.0, 0.0, 0.0);
        if ((rc = fill[0].ensure(gridBytes))) return rc;
        if ((rc = fin.ensure(gridBytes))) return rc;
        mark(0, false, s);
        if ((rc = solidPass(p, g, fill[0].as<uint32_t>(), s))) return rc;
        mark(0, true, s);
        const uint32_t* surfp = mats ? surfAll.as<uint32_t>() : nullptr;
        if (mats) {
            mark(1, false, s);
            if ((rc = surfacePass(p, g, 0, gridWords, 0, s))) return rc;
            vxb::launch_surface_rank(surfAll.as<uint32_t>(), gridWords, ranks.as<uint32_t>(), rankTiles.as<uint32_t>(),
                                     sm + kSurfaceVoxels, s, &launches);
            mark(1, true, s);
            mark(2, false, s);
            vxb::launch_combine(fill[0].as<uint32_t>(), surfp, fin.as<uint32_t>(), gridWords, s, &launches);
        } else {
            mark(2, false, s);
            VXB_CUDA(cudaMemcpyAsync(fin.p, fill[0].p, gridBytes, cudaMemcpyDeviceToDevice, s));
        }
        // Split-ordered pruning (src/host_side.cpp:1183-1206).  Passes for
        // every subspace are queued in order with one convergence check at
        // the end: when each subspace's last queued pass changed nothing,
        // every subspace converged before the next one started, exactly as
        // in the reference.  Otherwise the first unconverged subspace gets
        // more passes and every later one is re-run (their state is then a
        // superset of the right answer, from which further passes converge
        // to it).
        std::vector<uint8_t> later(p.alloc[1] + p.alloc[2], 0);
        for (size_t i = 1; i < p.ySplitsAlloc.size(); ++i) later[p.ySplitsAlloc[i].lo - 1] = 1;
        for (size_t i = 1; i < p.zSplitsAlloc.size(); ++i) later[p.alloc[1] + p.zSplitsAlloc[i].lo - 1] = 1;
        if ((rc = laterFlags.ensure(later.size() + 64))) return rc;
        VXB_CUDA(cudaMemcpyAsync(laterFlags.p, later.data(), later.size(), cudaMemcpyHostToDevice, s));
        const uint8_t* yl = laterFlags.as<uint8_t>();
        std::vector<vxb::SplitYZ> psplits;
        for (const auto& z : p.zSplitsAlloc)
            for (const auto& y : p.ySplitsAlloc) psplits.push_back(vxb::SplitYZ{y.lo, y.hi, z.lo, z.hi});
        const size_t nS = psplits.size();
        constexpr int kPasses = 3;
        uint32_t* flags = sm + kFlags;
        std::vector<uint32_t> h(kFlags + nS * kPasses);
        size_t from = 0;
        for (int round = 0;; ++round) {
            VXB_CUDA(cudaMemsetAsync(flags, 0, 4 * nS * kPasses, s));
            for (size_t i = from; i < nS; ++i)
                for (int b = 0; b < kPasses; ++b)
                    vxb::launch_prune(fin.as<uint32_t>(), fill[0].as<uint32_t>(), surfp, yl, yl + p.alloc[1], g,
                                      psplits[i], flags + i * kPasses + b, s, &launches);
            VXB_CUDA(cudaMemcpyAsync(h.data(), sm, 4 * (kFlags + nS * kPasses), cudaMemcpyDeviceToHost, s));
            VXB_CUDA(cudaStreamSynchronize(s));
            size_t bad = nS;
            for (size_t i = from; i < nS; ++i)
                if (h[kFlags + i * kPasses + kPasses - 1]) { bad = i; break; }
            if (bad == nS) break;
            from = bad;
            if (round > 1000000) return fail(VXB_ETIMEDOUT, "pruning did not converge");
        }
        mark(2, true, s);
        if (mats) {
            mark(4, false, s);
            if ((rc = resolveKeys(p, 1, gridWords, h[kHitCount], h[kSurfaceVoxels], s))) return rc;
            mark(4, true, s);
        }
        mark(3, false, s);
        vxb::launch_emit_cartesian(nodeType, fin.as<uint32_t>(), fill[0].as<uint32_t>(), surfp, ranks.as<uint32_t>(),
                                   keys.p, g, yl, yl + p.alloc[1], dout, mats ? 1 : 0, s, &launches);
        mark(3, true, s);
        VXB_CUDA(cudaGetLastError());
        return 0;
    }
    // FCC: four shifted sub-lattices (src/host_side.cpp:1432-1484, 1525-1593).
    const uint32_t* fp[4];
    const uint32_t* sp4[4];
    uint64_t base4[4];
    for (int lt = 0; lt < 4; ++lt)
        if ((rc = fill[lt].ensure(gridBytes))) return rc;
    mark(0, false, s);
    for (int lt = 0; lt < 4; ++lt) {
        double sh[3];
        latticeShift(p, lt, sh);
        vxb::PassGeom g = makeGeom(p, sh[0], sh[1], sh[2]);
        if ((rc = solidPass(p, g, fill[lt].as<uint32_t>(), s))) return rc;
        fp[lt] = fill[lt].as<uint32_t>();
        sp4[lt] = mats ? surfAll.as<uint32_t>() + lt * gridWords : nullptr;
        base4[lt] = lt * gridWords;
        if (mats && (rc = surfacePass(p, g, lt, gridWords, 0, s))) return rc;
    }
    mark(0, true, s);
    if (mats) {
        mark(4, false, s);
        vxb::launch_surface_rank(surfAll.as<uint32_t>(), gridWords * 4, ranks.as<uint32_t>(), rankTiles.as<uint32_t>(),
                                 sm + kSurfaceVoxels, s, &launches);
        uint32_t h[8];
        VXB_CUDA(cudaMemcpyAsync(h, sm, sizeof(h), cudaMemcpyDeviceToHost, s));
        VXB_CUDA(cudaStreamSynchronize(s));
        if ((rc = resolveKeys(p, 4, gridWords, h[kHitCount], h[kSurfaceVoxels], s))) return rc;
        mark(4, true, s);
    }
    vxb::PassGeom g = makeGeom(p, 0.0, 0.0, 0.0);
    mark(3, false, s);
    vxb::launch_emit_fcc(nodeType, fp, sp4, base4, ranks.as<uint32_t>(), keys.p, g, dout, mats ? 1 : 0, s, &launches);
    mark(3, true, s);
    VXB_CUDA(cudaGetLastError());
    return 0;
}

// ---------------------------------------------------------------------------
// C ABI

extern "C" {

const char* vxb_last_error(void) { return g_lastError.c_str(); }
const char* vxb_version(void) { return "vxb 0.1 (sm_100a)"; }

vxb_status vxb_create(vxb_voxelizer** out, int node_type, const float* vertices, const uint32_t* indices,
                      uint32_t n_vertices, uint32_t n_triangles, int device) {
    if (!out) return fail(VXB_EINVAL, "out is NULL");
    *out = nullptr;
    if (node_type < 0 || node_type > 4) return fail(VXB_EINVAL, "unknown node type %d", node_type);
    if ((!vertices && n_vertices) || (!indices && n_triangles)) return fail(VXB_EINVAL, "NULL mesh arrays");
    for (uint64_t i = 0; i < 3ull * n_triangles; ++i)
        if (indices[i] >= n_vertices) return fail(VXB_EINVAL, "index %u of triangle %llu is out of range", indices[i], (unsigned long long)(i / 3));
    vxb_voxelizer* v = new (std::nothrow) vxb_voxelizer();
    if (!v) return fail(VXB_ENOMEM, "out of host memory");
    v->nodeType = node_type;
    v->device = device;
    v->nV = n_vertices;
    v->nT = n_triangles;
    v->vertices.assign(vertices, vertices + 3 * (size_t)n_vertices);
    v->indices.assign(indices, indices + 3 * (size_t)n_triangles);
    if (n_vertices) vxb::boundingBox(vertices, n_vertices, v->mn, v->mx);
    *out = v;
    return VXB_OK;
}

vxb_status vxb_destroy(vxb_voxelizer* v) {
    if (!v) return VXB_OK;
    // The instance's buffers go back to the block cache: wait for queued
    // work that may still use them.
    const int dev = v->device;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    cudaDeviceSynchronize();
    delete v;
    if (cur != dev) cudaSetDevice(cur);
    return VXB_OK;
}

vxb_status vxb_trim_cache(void) {
    BlockCache& c = blockCache();
    std::multimap<size_t, std::pair<int, void*>> idle;
    {
        std::lock_guard<std::mutex> lock(c.mu);
        idle.swap(c.idle);
        c.idleBytes = 0;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto& e : idle) {
        cudaSetDevice(e.second.first);
        cudaFree(e.second.second);
    }
    cudaSetDevice(cur);
    return VXB_OK;
}

vxb_status vxb_set_materials(vxb_voxelizer* v, const uint8_t* materials, uint32_t n_unique_materials) {
    if (!v) return fail(VXB_EINVAL, "voxelizer is NULL");
    if (!materials) return fail(VXB_EINVAL, "No valid materials provided (Received null pointer) @ setMaterials.");
    if (n_unique_materials > kMaxMat[v->nodeType] + 1)
        return fail(VXB_EINVAL, "The number of unique materials exceeds the capabilities of the node type @ setMaterials.");
    v->nUniqueMaterials = n_unique_materials;
    v->materials.assign(materials, materials + v->nT);
    v->matsOnDevice = false;
    v->materialsOn = true;
    return VXB_OK;
}

vxb_status vxb_set_material_output(vxb_voxelizer* v, int enable) {
    if (!v) return fail(VXB_EINVAL, "voxelizer is NULL");
    v->materialsOn = enable != 0;
    return VXB_OK;
}

vxb_status vxb_verbose_output(vxb_voxelizer* v, int enable) {
    if (!v) return fail(VXB_EINVAL, "voxelizer is NULL");
    v->verbose = enable != 0;
    return VXB_OK;
}

vxb_status vxb_plan(vxb_voxelizer* v, int nodes, const vxb_request* req, vxb_grid_info* info) {
    if (!v) return fail(VXB_EINVAL, "voxelizer is NULL");
    vxb::Plan p;
    return v->plan(nodes, req, p, info);
}

vxb_status vxb_get_array_dimensions(vxb_voxelizer* v, int by_cube_length, uint32_t max_dimension, double cube_length,
                                    uint32_t max_internal_x, int slice_along_x, vxb_uint3* dims) {
    if (!v || !dims) return fail(VXB_EINVAL, "NULL argument");
    if (slice_along_x) return fail(VXB_EUNSUPPORTED, "slicing along x is not part of this library");
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
    if (!v) return fail(VXB_EINVAL, "voxelizer is NULL");
    return v->run(nodes, req, dev_out, dev_bytes, reinterpret_cast<cudaStream_t>(stream), info);
}

vxb_status vxb_voxelize_to_host(vxb_voxelizer* v, int nodes, const vxb_request* req, void* host_out,
                                uint64_t host_bytes, vxb_grid_info* info) {
    if (!v) return fail(VXB_EINVAL, "voxelizer is NULL");
    vxb_grid_info gi;
    vxb::Plan p;
    int rc = v->plan(nodes, req, p, &gi);
    if (rc) return rc;
    if (info) *info = gi;
    if ((rc = v->validate(nodes, req))) return rc;
    if (!host_out) return fail(VXB_EINVAL, "output buffer is NULL");
    if (host_bytes < gi.bytes) return fail(VXB_EINVAL, "output buffer too small");
    VXB_CUDA(cudaSetDevice(v->device));
    if ((rc = v->outStage.ensure(gi.bytes))) return rc;
    rc = v->run(nodes, req, v->outStage.p, gi.bytes, 0, info);
    if (rc == 0) {
        cudaError_t e = cudaMemcpy(host_out, v->outStage.p, gi.bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail(VXB_ECUDA, "%s", cudaGetErrorString(e));
    }
    return rc;
}

vxb_status vxb_set_profiling(vxb_voxelizer* v, int enable) {
    if (!v) return fail(VXB_EINVAL, "voxelizer is NULL");
    v->profiling = enable != 0;
    return VXB_OK;
}

vxb_status vxb_stage_times(vxb_voxelizer* v, float* ms, uint32_t n) {
    if (!v || !ms) return fail(VXB_EINVAL, "NULL argument");
    for (uint32_t k = 0; k < n && k < (uint32_t)vxb_voxelizer::kStages; ++k) {
        ms[k] = -1.0f;
        if (!v->profiling || !v->evUsed[k]) continue;
        cudaError_t e = cudaEventSynchronize(v->ev[2 * k + 1]);
        if (e != cudaSuccess) return fail(VXB_ECUDA, "%s", cudaGetErrorString(e));
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, v->ev[2 * k], v->ev[2 * k + 1]) == cudaSuccess) ms[k] = t;
    }
    return VXB_OK;
}

vxb_status vxb_last_launch_count(vxb_voxelizer* v, uint32_t* launches) {
    if (!v || !launches) return fail(VXB_EINVAL, "NULL argument");
    *launches = v->launches;
    return VXB_OK;
}

}  // extern "C"
