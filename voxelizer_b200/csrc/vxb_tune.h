// Launch-shape autotuner.  The shapes below change how the work of a kernel
// is spread over the GPU (grid size, items per warp), never what it computes,
// so every choice gives the same result.  Shapes are chosen per size bucket
// (work triangles, grid words, node kind, material output): in tuning mode a
// bucket's first calls run candidate shapes, each kernel's time is taken with
// CUDA events, and once every candidate has its samples each kernel keeps its
// fastest shape.  Chosen shapes can be saved to and read from a JSON file.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace vxb {

struct LaunchShape {
    uint32_t surfBlocksPerSm = 16;   // surfaceWorkKernel blocks per SM
    uint32_t surfBatch = 8;          // surfaceWorkKernel 32-item chunks per owner search
    // mergeKeysKernel (timed from the surface-bits join to the keys join);
    // 0: one block per 1,024 expected list entries instead of a persistent
    // grid (its blocks retire as they finish, so pruning's blocks get room).
    uint32_t mergeBlocksPerSm = 0;
    uint32_t emitBlocksPerSm = 16;   // emitNarrowKernel
    uint32_t toggleBlocksPerSm = 3;  // solidToggleKernel
    // Work distribution of surfaceWorkKernel / solidToggleKernel: 0 a fixed
    // grid-stride order, 1 a device work queue (persistent warps / blocks
    // take the next batch of items with one atomic each).
    uint32_t surfQueue = 0;
    uint32_t toggleQueue = 0;
    // Material keys of the surface pass: 0 a hit list that mergeKeysKernel
    // merges at the surface ranks, 1 no hit list and a second traversal that
    // merges every hit at its rank.  Tuned after the shapes above are
    // settled, on the time from the first traversal to the merged keys.
    uint32_t surfMerge = 0;
};

// The tuned kernels, in the order of their timing events; kKnobSurfaceSpan
// times the surface pass from its first traversal to its merged keys.
enum TuneKnob { kKnobSurface = 0, kKnobMerge = 1, kKnobEmit = 2, kKnobToggle = 3, kKnobSurfaceSpan = 4, kKnobs = 5 };
constexpr int kTuneCandidates = 3;
constexpr int kMergeCandidates = 2;
constexpr int kTuneSamples = 3;

enum TuneMode { kTuneOff = 0, kTuneOn = 1, kTuneFrozen = 2 };

// Size bucket of a batch.
std::string tuneBucket(uint32_t workTriangles, uint64_t gridWords, int nodeKind, bool materials);

// The shape for the next run of `bucket`.  *trial >= 0 when the run is a
// tuning trial (its kernel times go to tuneReport); -1 otherwise.  Trials
// 0 .. kTuneCandidates-1 try the launch shapes, the later ones the
// material-key strategies on the settled shapes.
LaunchShape tunePick(const std::string& bucket, int* trial, bool allowTrial = true);
// Kernel times (ms, < 0 for a kernel that did not run) of trial `trial`.
void tuneReport(const std::string& bucket, int trial, const float* ms);

int tuneSetMode(int mode, const char* cachePath);
int tuneMode();
// Number of buckets whose shapes are settled, and the JSON text of all of
// them.
uint32_t tuneSettled();
std::string tuneJson();

}  // namespace vxb
