// The voxelization pipeline of one batch (vxb_pipeline.h).
//
// All units of a batch go through each stage in one launch: solid
// voxelization, surface voxelization with its hit list and ranks,
// split-ordered pruning, material merge and node emission.  Pruning runs
// kPasses speculative passes per subspace index (for all units at once,
// each region skipping passes once it stops changing); the host checks the
// flags after the batch and adds passes only where a region had not
// converged.

#include "vxb_pipeline.h"

#include <algorithm>
#include <cstring>

namespace vxb {

namespace {

// Slots of the status buffer; pruning flags follow at kFlags.
enum : int { kSolidTotal = 0, kSolidOverflow = 1, kSurfTotal = 2, kSurfOverflow = 3, kHitCount = 4,
             kSurfaceVoxels = 5, kSurfQueue = 6, kToggleQueue = 7, kFlags = 8 };

const uint32_t kNodeBytes[5] = {1, 2, 8, 2, 4};

bool isFccType(int t) { return t == VXB_SHORT_FCC_NODE || t == VXB_LONG_FCC_NODE; }

size_t align16(size_t v) { return (v + 15) & ~size_t(15); }

template <class T> size_t append(std::vector<uint8_t>& blob, const std::vector<T>& v) {
    const size_t off = align16(blob.size());
    blob.resize(off + v.size() * sizeof(T));
    if (!v.empty()) memcpy(blob.data() + off, v.data(), v.size() * sizeof(T));
    return off;
}

}  // namespace

int gridInfo(const Plan& p, int nodeType, int nodes, vxb_grid_info* info) {
    const bool fcc = isFccType(nodeType);
    vxb_grid_info gi;
    memset(&gi, 0, sizeof(gi));
    if (nodes) {
        gi.dim.x = fcc ? 2 * p.alloc[0] : p.alloc[0];
        gi.dim.y = p.alloc[1];
        gi.dim.z = fcc ? 2 * p.alloc[2] : p.alloc[2];
        gi.count = (uint64_t)gi.dim.x * gi.dim.y * gi.dim.z;
        gi.bytes = gi.count * kNodeBytes[nodeType];
        // The reference indexes nodes with 32-bit unsigned integers.
        if (gi.count > 0xFFFFFFFFull)
            return failf(VXB_EOVERFLOW, "node grid of %llu nodes exceeds 32-bit indexing",
                         (unsigned long long)gi.count);
    } else {
        gi.dim.x = p.alloc[0];
        gi.dim.y = p.alloc[1];
        gi.dim.z = p.alloc[2];
        gi.count = (uint64_t)p.alloc[0] * p.alloc[1] * p.alloc[2] / 32;
        gi.bytes = gi.count * 4;
        if ((uint64_t)p.alloc[0] * p.alloc[1] * p.alloc[2] > 0xFFFFFFFFull)
            return failf(VXB_EOVERFLOW, "voxel grid exceeds 32-bit indexing");
    }
    gi.voxel_length = p.d;
    for (int a = 0; a < 3; ++a) {
        gi.min_vertex[a] = p.mnHost[a];
        gi.max_vertex[a] = p.mx[a];
    }
    for (int k = 0; k < 4; ++k) gi.partition[k] = p.part[k];
    gi.resolution.x = p.res[0];
    gi.resolution.y = p.res[1];
    gi.resolution.z = p.res[2];
    gi.x_splits = p.xSplits;
    if (info) *info = gi;
    return 0;
}

// Shifts of the four FCC sub-lattices by their slot in the FCC array (slot
// 1 + (x & 1) + 2 (z & 1), src/host_side.cpp:1438-1462).  For a turned mesh
// (slices along x) the reference shifts grid g by the z-swapped pattern and
// writes it to slot (g + 1) % 4 + 1, which toggles each slot's y shift.
PassGeom makeGeom(const Plan& p, int lattice, bool turned) {
    const double h = p.d / 2.0;
    const double sh[4][3] = {{0.0, 0.0, 0.0}, {h, h, 0.0}, {0.0, h, h}, {h, 0.0, h}};
    const double shTurned[4][3] = {{0.0, h, 0.0}, {h, 0.0, 0.0}, {0.0, 0.0, h}, {h, h, h}};
    PassGeom g;
    for (int a = 0; a < 3; ++a) {
        g.mn[a] = p.mn[a] + (turned ? shTurned : sh)[lattice][a];
        g.mnf[a] = (float)g.mn[a];
    }
    g.d = p.d;
    g.df = (float)p.d;
    g.X = p.res[0];
    g.resY = p.res[1];
    g.resZ = p.res[2];
    g.AY = p.alloc[1];
    g.AZ = p.alloc[2];
    g.ipx = p.res[0] / 32;
    g.padY = p.padY;
    g.padZ = p.padZ;
    g.border = p.border ? 1u : 0u;
    g.pad0 = 0;
    return g;
}

void StageTimer::mark(int stage, bool end, cudaStream_t s) {
    if (!enabled) return;
    if (!ev[0])
        for (auto& e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[2 * stage + (end ? 1 : 0)], s);
    used[stage] = true;
}

StageTimer::~StageTimer() {
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
}

Batch Pipeline::batch() {
    const uint8_t* t = tables.as<uint8_t>();
    Batch b;
    b.units = reinterpret_cast<const Unit*>(t + oUnits_);
    b.nUnits = (uint32_t)units_.size();
    b.workBase = reinterpret_cast<const uint32_t*>(t + oWork_);
    b.rowBase = reinterpret_cast<const uint64_t*>(t + oRow_);
    b.wordBase = reinterpret_cast<const uint64_t*>(t + oWord_);
    b.splits = reinterpret_cast<const SplitYZ*>(t + oSplits_);
    b.slices = reinterpret_cast<const uint32_t*>(t + oSlices_);
    b.later = t + oLater_;
    return b;
}

int Pipeline::prepare(const std::vector<MeshJob>& jobs, cudaStream_t s) {
    if (jobs.empty()) return failf(VXB_EINVAL, "empty batch");
    jobs_ = jobs;
    nodeKind_ = jobs[0].nodeType;
    nodes_ = jobs[0].nodes;
    for (const MeshJob& j : jobs)
        if (j.nodeType != nodeKind_ || j.nodes != nodes_)
            return failf(VXB_EINVAL, "all meshes of a batch need the same node type and output kind");
    const bool fcc = isFccType(nodeKind_);
    wide_ = nodeKind_ == VXB_PARTIAL_NODE;
    raw_ = jobs[0].raw != 0;
    for (const MeshJob& j : jobs)
        if ((j.raw != 0) != raw_ || (raw_ && !j.nodes))
            return failf(VXB_EINVAL, "raw node output is for node grids of a whole batch");
    units_.clear();
    groups_.clear();
    std::vector<uint32_t> workBase{0};
    std::vector<uint64_t> rowBase{0}, wordBase{0};
    std::vector<SplitYZ> splits;
    std::vector<uint32_t> slices;
    std::vector<uint8_t> later;
    std::vector<std::vector<PruneRegion>> regionsBySplit;
    std::vector<FccMesh> fccMeshes;
    std::vector<uint64_t> groupBase{0};
    anyMaterials_ = false;
    anyCartesian_ = false;
    uint64_t nodeCount = 0;
    for (const MeshJob& j : jobs) {
        Plan p;
        const uint32_t vs[3] = {j.req.vox_split_res.x, j.req.vox_split_res.y, j.req.vox_split_res.z};
        const uint32_t ms[3] = {j.req.mat_split_res.x, j.req.mat_split_res.y, j.req.mat_split_res.z};
        if (makePlan(j.mn, j.mx, j.req.by_cube_length, j.req.max_dimension, j.req.cube_length, vs, ms, p))
            return failf(VXB_EINVAL, "invalid request (maxDimension >= 2 or cubeLength > 0, split sizes > 0 and an x "
                                     "pass of at most 1024 voxels are required)");
        if (j.space) {
            Plan full = p;
            if (devicePlan(full, j.part[0], j.part[1], j.part[2], j.part[3], vs, ms, p))
                return failf(VXB_EINVAL, "empty or out-of-range partition");
        }
        vxb_grid_info gi;
        if (int rc = gridInfo(p, j.nodeType, j.nodes, &gi)) return rc;
        if (!j.out) return failf(VXB_EINVAL, "output buffer is NULL");
        if (j.outBytes < gi.bytes)
            return failf(VXB_EINVAL, "output buffer holds %llu bytes, %llu needed", (unsigned long long)j.outBytes,
                         (unsigned long long)gi.bytes);
        nodeCount += gi.count;
        const int lattices = (j.nodes && fcc) ? 4 : 1;
        const uint32_t firstUnit = (uint32_t)units_.size();
        for (int l = 0; l < lattices; ++l) {
            Unit u;
            memset(&u, 0, sizeof(u));
            u.g = makeGeom(p, l, fcc && j.turned);
            u.V = j.V;
            u.I = j.I;
            u.M = j.M;
            u.nT = j.nT;
            u.splitBase = (uint32_t)splits.size();
            for (const auto& z : p.zSplitsExt)
                for (const auto& y : p.ySplitsExt) splits.push_back(SplitYZ{y.lo, y.hi, z.lo, z.hi});
            u.nSplits = (uint32_t)splits.size() - u.splitBase;
            u.sliceBase = (uint32_t)(slices.size() / 2);
            const std::vector<Range>* axes[3] = {&p.xMat, &p.yMat, &p.zMat};
            for (int a = 0; a < 3; ++a) {
                u.sliceN[a] = (uint32_t)axes[a]->size();
                for (const auto& r : *axes[a]) {
                    slices.push_back(r.lo);
                    slices.push_back(r.hi);
                }
            }
            u.laterBase = (uint32_t)later.size();
            later.resize(later.size() + p.alloc[1] + p.alloc[2], 0);
            for (size_t i = 1; i < p.ySplitsAlloc.size(); ++i) later[u.laterBase + p.ySplitsAlloc[i].lo - 1] = 1;
            for (size_t i = 1; i < p.zSplitsAlloc.size(); ++i)
                later[u.laterBase + p.alloc[1] + p.zSplitsAlloc[i].lo - 1] = 1;
            u.materials = (j.nodes && j.M) ? 1u : 0u;
            anyMaterials_ |= u.materials != 0;
            u.wordBase = wordBase.back();
            u.out = l == 0 ? j.out : nullptr;
            const uint64_t nWords = (uint64_t)u.g.ipx * u.g.AY * u.g.AZ;
            wordBase.push_back(u.wordBase + ((nWords + 31) & ~uint64_t(31)));
            rowBase.push_back(rowBase.back() + (uint64_t)u.g.AY * u.g.AZ);
            if ((uint64_t)workBase.back() + j.nT > 0xFFFFFFFFull)
                return failf(VXB_EOVERFLOW, "batch of more than 2^32 work triangles");
            workBase.push_back(workBase.back() + j.nT);
            units_.push_back(u);
            if (j.nodes && !fcc) {
                anyCartesian_ = true;
                size_t k = 0;
                for (const auto& z : p.zSplitsAlloc)
                    for (const auto& y : p.ySplitsAlloc) {
                        if (regionsBySplit.size() <= k) regionsBySplit.resize(k + 1);
                        PruneRegion r;
                        r.unit = firstUnit + (uint32_t)l;
                        r.split = SplitYZ{y.lo, y.hi, z.lo, z.hi};
                        r.wordStart = 0;
                        regionsBySplit[k++].push_back(r);
                    }
            }
        }
        if (j.nodes && fcc) {
            fccMeshes.push_back(FccMesh{firstUnit, j.out});
            groupBase.push_back(groupBase.back() + gi.bytes / 16);
        }
    }
    nWork_ = workBase.back();
    totalWords_ = wordBase.back();
    totalRows_ = rowBase.back();
    nFcc_ = (uint32_t)fccMeshes.size();
    totalGroups_ = groupBase.back();
    // Pruning regions, grouped by subspace index.
    std::vector<PruneRegion> regions;
    for (auto& grp : regionsBySplit) {
        Group gr;
        gr.first = (uint32_t)regions.size();
        gr.count = (uint32_t)grp.size();
        gr.flagBase = gr.first;
        uint64_t words = 0;
        for (PruneRegion& r : grp) {
            r.wordStart = (uint32_t)words;
            const Unit& u = units_[r.unit];
            words += (uint64_t)(r.split.y1 - r.split.y0) * (r.split.z1 - r.split.z0) * u.g.ipx;
            regions.push_back(r);
        }
        if (words > 0xFFFFFFFFull) return failf(VXB_EOVERFLOW, "pruning launch of more than 2^32 words");
        gr.words = (uint32_t)words;
        groups_.push_back(gr);
    }
    nRegions_ = (uint32_t)regions.size();
    // A single plain voxelization writes its solid grid straight into the
    // caller's buffer.
    aliasFill_ = !nodes_ && jobs.size() == 1;
    // Tables.
    blob_.clear();
    oUnits_ = append(blob_, units_);
    oWork_ = append(blob_, workBase);
    oRow_ = append(blob_, rowBase);
    oWord_ = append(blob_, wordBase);
    oSplits_ = append(blob_, splits);
    oSlices_ = append(blob_, slices);
    oLater_ = append(blob_, later);
    oRegions_ = append(blob_, regions);
    oFcc_ = append(blob_, fccMeshes);
    oGroupBase_ = append(blob_, groupBase);
    // Buffers.
    int rc;
    const size_t wordBytes = 4 * (size_t)totalWords_;
    if ((rc = tables.ensure(blob_.size() + 64))) return rc;
    if ((rc = status.ensure(4 * (kFlags + (size_t)nRegions_ * kPasses) + 256))) return rc;
    if ((rc = counts.ensure(4 * ((size_t)nWork_ + 1)))) return rc;
    if ((rc = offsets.ensure(4 * ((size_t)nWork_ + 2)))) return rc;
    if ((rc = tileSums.ensure(4 * ((size_t)nWork_ / 4096 + 2)))) return rc;
    if (!aliasFill_ && (rc = fill.ensure(wordBytes))) return rc;
    if (anyCartesian_ && (rc = fin.ensure(wordBytes))) return rc;
    // Change lists of the pruning passes: the first pass lists every word it
    // changes (a fraction of the boundary words); past the cap the host
    // finishes pruning with full passes.
    uint32_t maxGroupWords = 0;
    for (const Group& gr : groups_) maxGroupWords = std::max(maxGroupWords, gr.words);
    pruneCap_ = std::max<uint32_t>(4u << 20, maxGroupWords / 4);
    if (anyCartesian_ && (rc = pruneScratch.ensure(4 * (groups_.size() * kPasses + 1)))) return rc;
    if (anyCartesian_ && (rc = pruneLists.ensure(2 * 8 * (size_t)pruneCap_))) return rc;
    listCap_ = 0;
    mergeEntries_ = 0;
    keysCap_ = 0;
    if (anyMaterials_) {
        if (!side_) {
            // Pruning and emission (on the way to the result) run on a stream
            // of the greatest priority, so that their blocks are placed
            // before the merge's when both wait for room on the SMs.
            int least = 0, greatest = 0;
            VXB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
            VXB_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
            VXB_CUDA(cudaStreamCreateWithPriority(&hi_, cudaStreamNonBlocking, greatest));
            VXB_CUDA(cudaEventCreateWithFlags(&evFork_, cudaEventDisableTiming));
            VXB_CUDA(cudaEventCreateWithFlags(&evSurfBits_, cudaEventDisableTiming));
            VXB_CUDA(cudaEventCreateWithFlags(&evSurfDone_, cudaEventDisableTiming));
            VXB_CUDA(cudaEventCreateWithFlags(&evSolid_, cudaEventDisableTiming));
            VXB_CUDA(cudaEventCreateWithFlags(&evHiDone_, cudaEventDisableTiming));
        }
        if ((rc = sCounts.ensure(4 * ((size_t)nWork_ + 2)))) return rc;
        if ((rc = sOffsets.ensure(4 * ((size_t)nWork_ + 2)))) return rc;
        if ((rc = sTileSums.ensure(4 * ((size_t)nWork_ / 4096 + 2)))) return rc;
        if ((rc = surf.ensure(wordBytes))) return rc;
        if ((rc = ranks.ensure(2 * wordBytes))) return rc;
        if ((rc = rankTiles.ensure(4 * ((size_t)totalWords_ / 2048 + 2)))) return rc;
        if ((rc = codes.ensure(4 * (size_t)nWork_))) return rc;
        if ((rc = unitCounts.ensure(4 * (size_t)nWork_))) return rc;
        if ((rc = buckets.ensure(4 * 2 * kSurfaceBuckets))) return rc;
        if ((rc = recs.ensure(kSurfRecBytes * (size_t)nWork_))) return rc;
        if ((rc = ovl.ensure(kSurfOvlBytes * (size_t)nWork_))) return rc;
        // Hit list: 8-byte entries (bit position << 24 | key).  PartialNode
        // keys are 64-bit and always take the second traversal.  With the
        // list, the surface voxels are at most its entries.
        if (!wide_) {
            listCap_ = (uint32_t)std::min<uint64_t>(96ull << 20, std::max<uint64_t>(8ull << 20, nodeCount / 12));
            // Entries the merge's non-persistent grid is sized for (more are
            // taken by its blocks' grid-stride loops).
            mergeEntries_ = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(listCap_, nodeCount / 4));
            if ((rc = hitList.ensure((size_t)listCap_ * 8))) return rc;
            keysCap_ = listCap_ + 1;
        } else {
            keysCap_ = (uint32_t)std::min<uint64_t>(totalWords_ * 32 + 1,
                                                     std::max<uint64_t>(1u << 20, totalWords_ * 32 / 16));
        }
        if ((rc = keys.ensure((size_t)keysCap_ * (wide_ ? 8 : 4)))) return rc;
    }
    VXB_CUDA(cudaMemcpyAsync(tables.p, blob_.data(), blob_.size(), cudaMemcpyHostToDevice, s));
    return 0;
}

int Pipeline::enqueue(cudaStream_t s, StageTimer* timer) {
    launches = 0;
    const Batch b = batch();
    uint32_t* st = status.as<uint32_t>();
    uint32_t* fillP = aliasFill_ ? static_cast<uint32_t*>(jobs_[0].out) : fill.as<uint32_t>();
    const size_t wordBytes = aliasFill_ ? (size_t)units_[0].g.ipx * units_[0].g.AY * units_[0].g.AZ * 4
                                        : 4 * (size_t)totalWords_;
    // The stream of the stages on the way to the result: `s`, then (with a
    // surface pass) the high-priority stream from pruning on.
    cudaStream_t ps = s;
    auto mark = [&](int stage, bool end) {
        if (timer) timer->mark(stage, end, ps);
    };
    // Launch shapes of this run; tuning trials are timed per kernel (not
    // while a graph is being captured).
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    VXB_CUDA(cudaStreamIsCapturing(s, &cap));
    bucket_ = tuneBucket(nWork_, totalWords_, nodeKind_, anyMaterials_);
    shape = tunePick(bucket_, &trial_, cap == cudaStreamCaptureStatusNone);
    for (bool& u : tuneUsed_) u = false;
    // Surface voxelization, hit list and surface ranks on the side stream,
    // beside the solid pass (they share no buffer).
    cudaStream_t ss = s;
    const bool serial = timer && timer->enabled && timer->serial;
    if (anyMaterials_) {
        if (!serial) {
            ss = side_;
            VXB_CUDA(cudaEventRecord(evFork_, s));
            VXB_CUDA(cudaStreamWaitEvent(ss, evFork_, 0));
        }
        if (timer) timer->mark(1, false, ss);
        VXB_CUDA(cudaMemsetAsync(surf.p, 0, 4 * (size_t)totalWords_, ss));
        VXB_CUDA(cudaMemsetAsync(buckets.p, 0, 4 * 2 * kSurfaceBuckets, ss));
        VXB_CUDA(cudaMemsetAsync(sCounts.p, 0, 4 * ((size_t)nWork_ + 1), ss));
        VXB_CUDA(cudaMemsetAsync(st + kHitCount, 0, 4, ss));
        launch_surface_prepare(b, nWork_, codes.as<uint32_t>(), unitCounts.as<uint32_t>(), buckets.as<uint32_t>(),
                               sCounts.as<uint32_t>(), recs.p, ovl.p, ss, &launches);
        launch_scan(sCounts.as<uint32_t>(), sOffsets.as<uint32_t>(), nWork_, sTileSums.as<uint32_t>(),
                    st + kSurfTotal, st + kSurfOverflow, ss, &launches);
        // Without a hit list (PartialNode keys, or the tuned strategy) the
        // first traversal sets surface bits only and a second one merges
        // every hit at its rank.
        const bool retraverse = wide_ || shape.surfMerge != 0;
        if (timer) timer->mark(5, false, ss);
        tuneMark(kKnobSurfaceSpan, false, ss);
        tuneMark(kKnobSurface, false, ss);
        launch_surface_work(nodeKind_, retraverse ? 2 : 0, wide_ ? 1 : 0, b, recs.p, ovl.p, sOffsets.as<uint32_t>(), nWork_,
                            st + kSurfTotal, buckets.as<uint32_t>(), surf.as<uint32_t>(), ranks.as<WordRank>(),
                            keys.p, keysCap_, hitList.as<unsigned long long>(), st + kHitCount, listCap_,
                            shape.surfBlocksPerSm, shape.surfBatch, shape.surfQueue ? st + kSurfQueue : nullptr, ss,
                            &launches);
        tuneMark(kKnobSurface, true, ss);
        if (timer) timer->mark(5, true, ss);
        VXB_CUDA(cudaEventRecord(evSurfBits_, ss));
        launch_surface_rank(surf.as<uint32_t>(), totalWords_, ranks.as<WordRank>(), rankTiles.as<uint32_t>(),
                            st + kSurfaceVoxels, ss, &launches);
        if (timer) timer->mark(1, true, ss);
        // Material keys by surface rank (independent of pruning).
        if (timer) timer->mark(4, false, ss);
        launch_surface_keys_zero(keys.p, st + kSurfaceVoxels, keysCap_, wide_ ? 1 : 0, ss, &launches);
        if (!retraverse)
            launch_surface_merge(hitList.as<unsigned long long>(), st + kHitCount, listCap_, ranks.as<WordRank>(),
                                 keys.as<uint32_t>(), keysCap_, shape.mergeBlocksPerSm, mergeEntries_, ss, &launches);
        else
            launch_surface_work(nodeKind_, 1, wide_ ? 1 : 0, b, recs.p, ovl.p, sOffsets.as<uint32_t>(), nWork_,
                                st + kSurfTotal, buckets.as<uint32_t>(), surf.as<uint32_t>(), ranks.as<WordRank>(),
                                keys.p, keysCap_, nullptr, st + kHitCount, 0, shape.surfBlocksPerSm, shape.surfBatch,
                                shape.surfQueue ? st + kSurfQueue : nullptr, ss, &launches);
        tuneMark(kKnobSurfaceSpan, true, ss);
        if (timer) timer->mark(4, true, ss);
        VXB_CUDA(cudaEventRecord(evSurfDone_, ss));
    }
    // Solid voxelization.
    mark(0, false);
    VXB_CUDA(cudaMemsetAsync(fillP, 0, wordBytes, s));
    launch_solid_count(b, nWork_, counts.as<uint32_t>(), s, &launches);
    launch_scan(counts.as<uint32_t>(), offsets.as<uint32_t>(), nWork_, tileSums.as<uint32_t>(), st + kSolidTotal,
                st + kSolidOverflow, s, &launches);
    tuneMark(kKnobToggle, false, s);
    launch_solid_toggle(b, nWork_, offsets.as<uint32_t>(), st + kSolidTotal, fillP, shape.toggleBlocksPerSm,
                        shape.toggleQueue ? st + kToggleQueue : nullptr, s, &launches);
    tuneMark(kKnobToggle, true, s);
    launch_row_fill(b, totalRows_, fillP, s, &launches);
    mark(0, true);
    if (!nodes_) {
        if (!aliasFill_)
            for (const Unit& u : units_)
                VXB_CUDA(cudaMemcpyAsync(u.out, fillP + u.wordBase, (size_t)u.g.ipx * u.g.AY * u.g.AZ * 4,
                                         cudaMemcpyDeviceToDevice, s));
        VXB_CUDA(cudaGetLastError());
        return 0;
    }
    // The merge knob is timed on this stream from the join with the surface
    // bits (pruning runs beside the merge) to the join with the merged keys:
    // the merge's cost on the way to emission, not its own duration.
    bool mergeSpan = false;
    if (anyMaterials_ && !serial) {
        VXB_CUDA(cudaEventRecord(evSolid_, s));
        VXB_CUDA(cudaStreamWaitEvent(hi_, evSolid_, 0));
        ps = hi_;
    }
    // Split-ordered pruning (src/host_side.cpp:1183-1206).
    if (anyCartesian_ && !raw_) {
        if (anyMaterials_) {
            VXB_CUDA(cudaStreamWaitEvent(ps, evSurfBits_, 0));
            tuneMark(kKnobMerge, false, ps);
            mergeSpan = true;
        }
        mark(2, false);
        if (anyMaterials_)
            launch_combine(fillP, surf.as<uint32_t>(), fin.as<uint32_t>(), totalWords_, ps, &launches);
        else
            VXB_CUDA(cudaMemcpyAsync(fin.p, fillP, 4 * (size_t)totalWords_, cudaMemcpyDeviceToDevice, ps));
        VXB_CUDA(cudaMemsetAsync(st + kFlags, 0, 4 * (size_t)nRegions_ * kPasses, ps));
        // Per subspace index and pass: the count of its change list; the
        // last word is the list overflow flag.
        uint32_t* counts = pruneScratch.as<uint32_t>();
        uint32_t* overflow = counts + groups_.size() * kPasses;
        VXB_CUDA(cudaMemsetAsync(counts, 0, 4 * (groups_.size() * kPasses + 1), ps));
        const PruneRegion* regions = reinterpret_cast<const PruneRegion*>(tables.as<uint8_t>() + oRegions_);
        unsigned long long* lists[2] = {pruneLists.as<unsigned long long>(),
                                        pruneLists.as<unsigned long long>() + pruneCap_};
        const uint32_t* surfP = anyMaterials_ ? surf.as<uint32_t>() : nullptr;
        for (size_t gi = 0; gi < groups_.size(); ++gi) {
            const Group& gr = groups_[gi];
            uint32_t* c = counts + gi * kPasses;
            launch_prune(b, regions + gr.first, gr.count, gr.words, fin.as<uint32_t>(), fillP, surfP, st + kFlags,
                         gr.flagBase, kPasses, lists[0], c, pruneCap_, overflow, ps, &launches);
            // Pass 1 over the whole device; later lists are short (usually
            // empty), so passes 2 .. kPasses - 1 run in one block.
            launch_prune_list(b, regions + gr.first, fin.as<uint32_t>(), fillP, surfP, st + kFlags, gr.flagBase,
                              kPasses, 1, lists[0], c, lists[1], c + 1, pruneCap_, overflow, ps, &launches);
            launch_prune_list_loop(b, regions + gr.first, gr.count, fin.as<uint32_t>(), fillP, surfP, st + kFlags,
                                   gr.flagBase, kPasses, 2, lists[0], lists[1], c, pruneCap_, kLoopListMax, overflow, ps,
                                   &launches);
        }
        mark(2, true);
    }
    // Join: emission reads the merged keys.
    if (anyMaterials_) {
        if (!mergeSpan) tuneMark(kKnobMerge, false, ps);
        VXB_CUDA(cudaStreamWaitEvent(ps, evSurfDone_, 0));
        tuneMark(kKnobMerge, true, ps);
    }
    // Node emission.
    mark(3, false);
    if (raw_ && anyCartesian_)
        launch_emit_raw(nodeKind_, b, totalWords_, fillP, surf.as<uint32_t>(), ranks.as<WordRank>(), keys.p, keysCap_,
                        ps, &launches);
    else if (anyCartesian_) {
        tuneMark(kKnobEmit, false, ps);
        if (hostOut_ && units_.size() == 1) {
            // The node array in kOutChunks word ranges, each copied to the
            // caller's pinned host buffer on the copy stream as soon as it
            // is written, so the copy of the first ranges overlaps the rest.
            const Unit& u = units_[0];
            const uint64_t words = (uint64_t)u.g.ipx * u.g.AY * u.g.AZ;
            const uint64_t wordBytes = hostBytes_ / words;
            for (uint32_t k = 0; k < kOutChunks; ++k) {
                const uint64_t w0 = (words * k / kOutChunks) & ~uint64_t(31);
                const uint64_t w1 = k + 1 == kOutChunks ? words : (words * (k + 1) / kOutChunks) & ~uint64_t(31);
                if (w1 <= w0) continue;
                launch_emit_cartesian(nodeKind_, b, w0, w1, fin.as<uint32_t>(), fillP, surf.as<uint32_t>(),
                                      ranks.as<WordRank>(), keys.p, keysCap_, shape.emitBlocksPerSm, ps, &launches);
                if (!outEv_[k]) VXB_CUDA(cudaEventCreateWithFlags(&outEv_[k], cudaEventDisableTiming));
                VXB_CUDA(cudaEventRecord(outEv_[k], ps));
                VXB_CUDA(cudaStreamWaitEvent(copyStream_, outEv_[k], 0));
                VXB_CUDA(cudaMemcpyAsync(static_cast<uint8_t*>(hostOut_) + w0 * wordBytes,
                                         static_cast<const uint8_t*>(u.out) + w0 * wordBytes, (w1 - w0) * wordBytes,
                                         cudaMemcpyDeviceToHost, copyStream_));
            }
            hostCopied_ = true;
        } else {
            launch_emit_cartesian(nodeKind_, b, 0, totalWords_, fin.as<uint32_t>(), fillP, surf.as<uint32_t>(),
                                  ranks.as<WordRank>(), keys.p, keysCap_, shape.emitBlocksPerSm, ps, &launches);
        }
        tuneMark(kKnobEmit, true, ps);
    }
    if (nFcc_)
        launch_emit_fcc(nodeKind_, b, reinterpret_cast<const FccMesh*>(tables.as<uint8_t>() + oFcc_),
                        reinterpret_cast<const uint64_t*>(tables.as<uint8_t>() + oGroupBase_), nFcc_, totalGroups_,
                        fillP, surf.as<uint32_t>(), ranks.as<WordRank>(), keys.p, keysCap_, raw_, ps, &launches);
    mark(3, true);
    if (ps != s) {
        VXB_CUDA(cudaEventRecord(evHiDone_, ps));
        VXB_CUDA(cudaStreamWaitEvent(s, evHiDone_, 0));
    }
    VXB_CUDA(cudaGetLastError());
    return 0;
}

// More passes over one subspace index until no region changes, one full
// pass at a time with a host check in between.
int Pipeline::pruneGroupUntilStable(const Group& gr, cudaStream_t s) {
    const Batch b = batch();
    uint32_t* st = status.as<uint32_t>();
    uint32_t* fillP = aliasFill_ ? static_cast<uint32_t*>(jobs_[0].out) : fill.as<uint32_t>();
    const PruneRegion* regions = reinterpret_cast<const PruneRegion*>(tables.as<uint8_t>() + oRegions_);
    uint32_t* counts = pruneScratch.as<uint32_t>();
    uint32_t* overflow = counts + groups_.size() * kPasses;
    std::vector<uint32_t> h((size_t)gr.count * kPasses);
    for (uint64_t round = 0;; ++round) {
        if (round > (1u << 24)) return failf(VXB_ETIMEDOUT, "pruning did not converge");
        VXB_CUDA(cudaMemsetAsync(st + kFlags + (size_t)gr.flagBase * kPasses, 0, 4 * h.size(), s));
        VXB_CUDA(cudaMemsetAsync(counts, 0, 4, s));
        launch_prune(b, regions + gr.first, gr.count, gr.words, fin.as<uint32_t>(), fillP,
                     anyMaterials_ ? surf.as<uint32_t>() : nullptr, st + kFlags, gr.flagBase, kPasses,
                     pruneLists.as<unsigned long long>(), counts, pruneCap_, overflow, s, &launches);
        VXB_CUDA(cudaMemcpyAsync(h.data(), st + kFlags + (size_t)gr.flagBase * kPasses, 4 * h.size(),
                                 cudaMemcpyDeviceToHost, s));
        VXB_CUDA(cudaStreamSynchronize(s));
        bool changed = false;
        for (uint32_t r = 0; r < gr.count; ++r) changed |= h[(size_t)r * kPasses] != 0;
        if (!changed) return 0;
    }
}

Pipeline::~Pipeline() {
    for (cudaEvent_t e : {evFork_, evSurfBits_, evSurfDone_, evSolid_, evHiDone_})
        if (e) cudaEventDestroy(e);
    if (side_) cudaStreamDestroy(side_);
    if (hi_) cudaStreamDestroy(hi_);
    for (cudaEvent_t& e : tuneEv_)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : outEv_)
        if (e) cudaEventDestroy(e);
}

void Pipeline::tuneMark(int knob, bool end, cudaStream_t s) {
    if (trial_ < 0) return;
    cudaEvent_t& e = tuneEv_[2 * knob + (end ? 1 : 0)];
    if (!e && cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        e = nullptr;
        return;
    }
    cudaEventRecord(e, s);
    if (end) tuneUsed_[knob] = true;
}

// Reports the kernel times of a tuning trial (the stream has drained).
void Pipeline::tuneFinish() {
    if (trial_ < 0) return;
    float ms[kKnobs];
    for (int k = 0; k < kKnobs; ++k) {
        ms[k] = -1.0f;
        if (tuneUsed_[k] && tuneEv_[2 * k] && tuneEv_[2 * k + 1] &&
            cudaEventElapsedTime(&ms[k], tuneEv_[2 * k], tuneEv_[2 * k + 1]) != cudaSuccess) {
            cudaGetLastError();
            ms[k] = -1.0f;
        }
    }
    tuneReport(bucket_, trial_, ms);
    trial_ = -1;
}

int Pipeline::finish(cudaStream_t s) {
    if (!nodes_) {
        VXB_CUDA(cudaStreamSynchronize(s));
        tuneFinish();
        uint32_t h[2];
        VXB_CUDA(cudaMemcpy(h, status.p, sizeof(h), cudaMemcpyDeviceToHost));
        if (h[kSolidOverflow]) return failf(VXB_EOVERFLOW, "solid work list exceeds 2^32 entries");
        return 0;
    }
    std::vector<uint32_t> h(kFlags + (size_t)nRegions_ * kPasses);
    VXB_CUDA(cudaMemcpyAsync(h.data(), status.p, 4 * h.size(), cudaMemcpyDeviceToHost, s));
    uint32_t bk[kSurfaceBuckets] = {0};
    if (anyMaterials_) VXB_CUDA(cudaMemcpyAsync(bk, buckets.p, sizeof(bk), cudaMemcpyDeviceToHost, s));
    VXB_CUDA(cudaStreamSynchronize(s));
    tuneFinish();
    memset(&stats, 0, sizeof(stats));
    stats.units = (uint32_t)units_.size();
    stats.work_triangles = nWork_;
    stats.solid_candidates = h[kSolidTotal];
    stats.surface_columns = anyMaterials_ ? h[kSurfTotal] : 0;
    stats.surface_hits = anyMaterials_ ? h[kHitCount] : 0;
    stats.surface_voxels = anyMaterials_ ? h[kSurfaceVoxels] : 0;
    for (uint32_t k = 0; k < kSurfaceBuckets; ++k) stats.surface_triangles[k / 3] += bk[k];
    stats.grid_words = totalWords_;
    if (h[kSolidOverflow] || (anyMaterials_ && h[kSurfOverflow]))
        return failf(VXB_EOVERFLOW, "work list exceeds 2^32 entries");
    bool reemit = false;
    const Batch b = batch();
    uint32_t* st = status.as<uint32_t>();
    uint32_t* fillP = aliasFill_ ? static_cast<uint32_t*>(jobs_[0].out) : fill.as<uint32_t>();
    if (anyMaterials_) {
        const uint32_t hits = h[kHitCount], surfaceVoxels = h[kSurfaceVoxels];
        const bool listOverflow = !wide_ && hits > listCap_;
        if (listOverflow || (uint64_t)surfaceVoxels + 1 > keysCap_) {
            // Merge every hit straight at its rank (second traversal).
            int rc;
            if ((uint64_t)surfaceVoxels + 1 > keysCap_) {
                if ((rc = keys.ensure(((size_t)surfaceVoxels + 1) * (wide_ ? 8 : 4)))) return rc;
                keysCap_ = surfaceVoxels + 1;
            }
            launch_surface_keys_zero(keys.p, st + kSurfaceVoxels, keysCap_, wide_ ? 1 : 0, s, &launches);
            launch_surface_work(nodeKind_, 1, wide_ ? 1 : 0, b, recs.p, ovl.p, sOffsets.as<uint32_t>(), nWork_,
                                st + kSurfTotal, buckets.as<uint32_t>(), surf.as<uint32_t>(), ranks.as<WordRank>(),
                                keys.p, keysCap_, nullptr, st + kHitCount, 0, shape.surfBlocksPerSm, shape.surfBatch,
                                shape.surfQueue ? st + kSurfQueue : nullptr, s, &launches);
            reemit = true;
        }
    }
    if (anyCartesian_ && !raw_) {
        // The first subspace index with a region that changed in its last
        // queued pass has not converged; it and every later index (pruned
        // against a superset of its final state) get passes until stable.
        uint32_t overflow = 0;
        VXB_CUDA(cudaMemcpy(&overflow, pruneScratch.as<uint32_t>() + groups_.size() * kPasses, 4,
                            cudaMemcpyDeviceToHost));
        size_t first = overflow ? 0 : groups_.size();
        for (size_t gi = 0; gi < groups_.size() && first == groups_.size(); ++gi)
            for (uint32_t r = 0; r < groups_[gi].count; ++r)
                if (h[kFlags + ((size_t)groups_[gi].flagBase + r) * kPasses + kPasses - 1]) {
                    first = gi;
                    break;
                }
        for (size_t gi = first; gi < groups_.size(); ++gi) {
            if (int rc = pruneGroupUntilStable(groups_[gi], s)) return rc;
            reemit = true;
        }
    }
    if (reemit) {
        if (raw_ && anyCartesian_)
            launch_emit_raw(nodeKind_, b, totalWords_, fillP, surf.as<uint32_t>(), ranks.as<WordRank>(), keys.p,
                            keysCap_, s, &launches);
        else if (anyCartesian_)
            launch_emit_cartesian(nodeKind_, b, 0, totalWords_, fin.as<uint32_t>(), fillP, surf.as<uint32_t>(),
                                  ranks.as<WordRank>(), keys.p, keysCap_, shape.emitBlocksPerSm, s, &launches);
        if (nFcc_)
            launch_emit_fcc(nodeKind_, b, reinterpret_cast<const FccMesh*>(tables.as<uint8_t>() + oFcc_),
                            reinterpret_cast<const uint64_t*>(tables.as<uint8_t>() + oGroupBase_), nFcc_,
                            totalGroups_, fillP, surf.as<uint32_t>(), ranks.as<WordRank>(), keys.p, keysCap_, raw_, s,
                            &launches);
        VXB_CUDA(cudaGetLastError());
        VXB_CUDA(cudaStreamSynchronize(s));
        if (hostCopied_) {
            // The chunks already copied predate the re-emission.
            VXB_CUDA(cudaStreamSynchronize(copyStream_));
            VXB_CUDA(cudaMemcpy(hostOut_, units_[0].out, hostBytes_, cudaMemcpyDeviceToHost));
        }
    }
    return 0;
}

}  // namespace vxb
