// The voxelization pipeline of one batch of meshes (a single voxelization is
// a batch of one): plan and tables on the host, one stream-ordered sequence
// of launches for every unit of the batch, and a final check on the host.
#pragma once

#include "vxb.h"
#include "vxb_host.h"
#include "vxb_kernels.cuh"
#include "vxb_plan.h"
#include "vxb_tune.h"

#include <string>

#include <vector>

namespace vxb {

// One mesh of a batch.  The mesh arrays and the output are device memory.
struct MeshJob {
    const float* V;
    const uint32_t* I;
    const uint8_t* M;        // NULL without material output
    uint32_t nV, nT;
    double mn[3], mx[3];     // bounding box of the vertices
    int nodeType;            // VXB_*_NODE
    int nodes;               // 1: node grid, 0: plain bit array
    vxb_request req;
    void* out;
    uint64_t outBytes;
    // Device space: voxelize partition [part[0], part[1]) x [part[2],
    // part[3]) of the yz voxel range as the reference's devices do (space
    // = 1); 0 = the whole grid.
    int space = 0;
    uint32_t part[4] = {0, 0, 0, 0};
    // Node output as it stands before the boundary ids (bid = solid bit,
    // surface material and ratio), no pruning: the first half of a slice
    // along x.  All jobs of a batch share it.
    int raw = 0;
    // The mesh is turned about z (slices along x): FCC sub-lattices take the
    // turned shifts.
    int turned = 0;
};

// Shape of a job's result (vxb_plan).  Returns 0 or a vxb status.
int gridInfo(const Plan& p, int nodeType, int nodes, vxb_grid_info* info);
// Geometry of sub-lattice `lattice` (0 for Cartesian grids).
PassGeom makeGeom(const Plan& p, int lattice);

// Per-stage CUDA events on the launching stream (vxb_set_profiling).
struct StageTimer {
    // 0 solid, 1 surface, 2 prune, 3 emit, 4 material merge, 5 the surface
    // work kernel alone (inside stage 1)
    static constexpr int kStages = 6;
    bool enabled = false;
    // Stages one after another on the call's stream (no second stream), so
    // that each stage's time is its own.
    bool serial = false;
    cudaEvent_t ev[2 * kStages] = {};
    bool used[kStages] = {};
    void reset() {
        for (bool& u : used) u = false;
    }
    void mark(int stage, bool end, cudaStream_t s);
    ~StageTimer();
};

class Pipeline {
public:
    // Plans every job, sizes the buffers and uploads the batch tables.
    int prepare(const std::vector<MeshJob>& jobs, cudaStream_t s);
    // Queues the whole voxelization of the prepared batch.  It neither
    // synchronizes nor allocates, so a CUDA graph can capture it.
    int enqueue(cudaStream_t s, StageTimer* timer);
    // Waits for the queued work, checks the overflow and convergence flags
    // and finishes, on the host's lead, the rare batches that need more
    // work: a hit list that overflowed, or a pruning subspace that needed
    // more passes than were queued.
    int finish(cudaStream_t s);
    // Kernels launched by the last enqueue + finish.
    uint32_t launches = 0;
    // Node output of a one-mesh Cartesian run copied to pinned host memory
    // while it is emitted (in kOutChunks ranges, on `copyStream`): set
    // before enqueue; hostCopied() tells whether the run did it (the caller
    // then waits for copyStream instead of copying).
    void streamOutput(void* host, uint64_t bytes, cudaStream_t copyStream) {
        hostOut_ = host;
        hostBytes_ = bytes;
        copyStream_ = copyStream;
        hostCopied_ = false;
    }
    bool hostCopied() const { return hostCopied_; }
    // Counters of the last finish (vxb_last_stats).
    vxb_stats stats{};

    static constexpr uint32_t kPasses = 8;   // pruning passes queued per subspace
    static constexpr uint32_t kLoopListMax = 32768;   // longest list the one-block passes take
    static constexpr uint32_t kOutChunks = 4;         // emit / host-copy ranges of streamed output

    // Launch shape of the last enqueue (the autotuner's choice).
    LaunchShape shape{};
    ~Pipeline();

private:
    // Autotuner trial of the current run: events around the tuned kernels,
    // reported once finish has waited for them.
    std::string bucket_;
    int trial_ = -1;
    cudaEvent_t tuneEv_[2 * kKnobs] = {};
    void* hostOut_ = nullptr;
    uint64_t hostBytes_ = 0;
    cudaStream_t copyStream_ = nullptr;
    bool hostCopied_ = false;
    cudaEvent_t outEv_[kOutChunks] = {};
    bool tuneUsed_[kKnobs] = {};
    void tuneMark(int knob, bool end, cudaStream_t s);
    void tuneFinish();

    struct Group {            // pruning regions of one subspace index
        uint32_t first, count, words, flagBase;
    };
    Batch batch();
    int pruneGroupUntilStable(const Group& gr, cudaStream_t s);

    std::vector<MeshJob> jobs_;
    std::vector<Unit> units_;
    std::vector<Group> groups_;
    uint32_t nWork_ = 0, nRegions_ = 0, nFcc_ = 0;
    uint64_t totalWords_ = 0, totalRows_ = 0, totalGroups_ = 0;
    int nodeKind_ = 0, nodes_ = 1;
    bool anyMaterials_ = false, anyCartesian_ = false, wide_ = false, aliasFill_ = false, raw_ = false;
    uint32_t listCap_ = 0, keysCap_ = 0, pruneCap_ = 0, mergeEntries_ = 0;
    // table offsets (bytes) in `tables`
    size_t oUnits_ = 0, oWork_ = 0, oRow_ = 0, oWord_ = 0, oSplits_ = 0, oSlices_ = 0, oLater_ = 0, oRegions_ = 0,
           oFcc_ = 0, oGroupBase_ = 0;
    std::vector<uint8_t> blob_;   // host copy of the tables (alive while the upload runs)

    DevBuf tables, status, counts, offsets, tileSums;
    DevBuf fill, surf, fin, ranks, rankTiles, pruneScratch, pruneLists;
    DevBuf codes, unitCounts, buckets, recs, ovl, hitList, keys;
    // The surface pass runs on a second stream beside the solid pass (its
    // own work-list scan buffers), joined before pruning (surface bits) and
    // before emission (merged keys).
    DevBuf sCounts, sOffsets, sTileSums;
    cudaStream_t side_ = nullptr, hi_ = nullptr;
    cudaEvent_t evFork_ = nullptr, evSurfBits_ = nullptr, evSurfDone_ = nullptr, evSolid_ = nullptr,
                evHiDone_ = nullptr;
};

}  // namespace vxb
