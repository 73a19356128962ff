// Kernel declarations and the plain structs the host engine passes to them.
//
// Every kernel works on a batch of units.  A unit is one mesh voxelized on
// one lattice (a Cartesian mesh is one unit, an FCC mesh four: one per
// shifted sub-lattice).  The batch concatenates what its units need into
// shared arrays: work triangles (the units' triangle lists back to back, so
// an FCC mesh's triangles appear once per sub-lattice), bit-grid words (each
// unit's grids start at a multiple of 32 words), subspace tables and flags.
// Meshes stay in their own device arrays.  A single voxelization is a batch
// of one mesh.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vxb {

// Geometry of one unit.  For FCC lattices each of the four sub-lattices has
// its own shifted minimum corner.
struct PassGeom {
    double mn[3];        // minimum corner (FP64, as the reference's extMinVertex)
    double d;            // voxel length
    float mnf[3];        // float(mn) for the FP32 surface path
    float df;            // float(d)
    uint32_t X;          // voxels along x (padded and rounded to 32 * xSplits)
    uint32_t resY, resZ; // voxels along y / z before the 1-voxel padding
    uint32_t AY, AZ;     // allocated rows: resY + 2, resZ + 2
    uint32_t ipx;        // 32-bit words per row: X / 32
    uint32_t padY, padZ; // allocation row / plane of local voxel row / plane 0 (1, or 0 next to a neighbour)
    uint32_t border;     // zero the allocation's faces in the node output (a device space with neighbours)
    uint32_t pad0;
};

struct SplitYZ { uint32_t y0, y1, z0, z1; };

struct Unit {
    PassGeom g;
    const float* V;       // the mesh: vertices (3 floats each),
    const uint32_t* I;    // indices into V (3 per triangle),
    const uint8_t* M;     // material per triangle (NULL without materials)
    uint32_t nT;          // triangles of the mesh
    uint32_t splitBase;   // solid yz subspaces: SplitYZ entries [splitBase, splitBase + nSplits)
    uint32_t nSplits;
    uint32_t sliceBase;   // material subspace slices: (lo, hi) pairs, x then y then z
    uint32_t sliceN[3];
    uint32_t laterBase;   // AY + AZ flags: row y + 1 / plane z + 1 starts a later pruning subspace
    uint32_t materials;   // surface pass and material output enabled
    uint64_t wordBase;    // first word of the unit's bit grids (a multiple of 32)
    void* out;            // node output (Cartesian units)
};

// A surface word and the rank of its first surface voxel (the exclusive
// popcount prefix of the surface words before it, arena-wide), side by side
// so that one 8-byte load gives both.
struct __align__(8) WordRank {
    uint32_t bits, rank;
};

// Device tables of a batch.  Bases have nUnits + 1 entries (the last one is
// the total), so that the unit of an element is a binary search away.
struct Batch {
    const Unit* units;
    uint32_t nUnits;
    const uint32_t* workBase;   // first work triangle of each unit
    const uint64_t* rowBase;    // first grid row (y, z) of each unit
    const uint64_t* wordBase;   // first grid word of each unit
    const SplitYZ* splits;
    const uint32_t* slices;
    const uint8_t* later;
};

// Work-list scan: exclusive offsets (n + 1 entries) and the grand total.
void launch_scan(const uint32_t* in, uint32_t* offsets, uint32_t n, uint32_t* blockSums, uint32_t* total,
                 uint32_t* overflow, cudaStream_t s, uint32_t* launches);

// ---- Solid (parity) voxelization: src/voxelizer.cu:840-1617 ----
// Candidates per work triangle, the toggles of the listed candidates into
// the `fill` arena, then the row prefix XOR over all rows of the batch.
void launch_solid_count(const Batch& b, uint32_t nWork, uint32_t* counts, cudaStream_t s, uint32_t* launches);
// blocksPerSm: launch shape (the autotuner's choice; results do not depend
// on it), here and in the launchers below that take one.  queue: NULL for
// a fixed grid-stride order, else a device word the launcher zeroes and the
// kernel's persistent blocks take batches of work from.
void launch_solid_toggle(const Batch& b, uint32_t nWork, const uint32_t* offsets, const uint32_t* total,
                         uint32_t* fill, uint32_t blocksPerSm, uint32_t* queue, cudaStream_t s, uint32_t* launches);
void launch_row_fill(const Batch& b, uint64_t nRows, uint32_t* fill, cudaStream_t s, uint32_t* launches);

// ---- Surface voxelization: src/voxelizer.cu:2358-2989, 3040-4201 ----
// Triangles with surface work are partitioned into kSurfaceBuckets buckets
// by (class, axis); each gets a kSurfRecBytes record and a kSurfOvlBytes
// block of projection edge functions.
constexpr uint32_t kSurfaceBuckets = 9;
constexpr size_t kSurfRecBytes = 64;
constexpr size_t kSurfOvlBytes = 112;

// Classify (codes / units in work-triangle order, per-bucket counts in
// buckets[0..9)), then partition (unitsP in partitioned order; buckets[9..18)
// are cursors) and set up (records) the work triangles of units with
// materials.  buckets and unitsP[0..nWork] must be zero on entry.
void launch_surface_prepare(const Batch& b, uint32_t nWork, uint32_t* codes, uint32_t* units, uint32_t* buckets,
                            uint32_t* unitsP, void* recs, void* ovl, cudaStream_t s, uint32_t* launches);
// Surface work over the exclusive scan `offsets` of unitsP (nWork + 1
// entries), one thread per column.  mode 0: set bits in the `surf` arena and
// append (bit position << 24 | key) to `list` (entries past listCap are
// counted, not stored); mode 1: merge every hit's key at its rank (needs
// complete bits and their `ranks`).  wide: 64-bit keys (PartialNode).  kind: the
// node type, whose instantiation of the class kernels the arithmetic
// follows.  queue: as for launch_solid_toggle, per warp.
void launch_surface_work(int kind, int mode, int wide, const Batch& b, const void* recs, const void* ovl,
                         const uint32_t* offsets, uint32_t nWork, const uint32_t* total, const uint32_t* buckets,
                         uint32_t* surf, const WordRank* ranks, void* keys, uint32_t keysCap,
                         unsigned long long* list, uint32_t* listCount, uint32_t listCap, uint32_t blocksPerSm,
                         uint32_t batch, uint32_t* queue, cudaStream_t s, uint32_t* launches);
// Exclusive popcount prefix over `words` surface words, stored beside each
// word; *total = surface voxels.
void launch_surface_rank(const uint32_t* bits, uint64_t words, WordRank* ranks, uint32_t* tileSums, uint32_t* total,
                         cudaStream_t s, uint32_t* launches);
// Zeroes min(*count, cap) keys.
void launch_surface_keys_zero(void* keys, const uint32_t* count, uint32_t cap, int wide, cudaStream_t s,
                              uint32_t* launches);
// Keys at ranks >= keysCap are dropped (the host re-merges after growing).
// blocksPerSm 0 sizes the grid for `entries` entries, a block per 1,024
// (non-persistent).
void launch_surface_merge(const unsigned long long* list, const uint32_t* listCount, uint32_t listCap,
                          const WordRank* ranks, uint32_t* keys, uint32_t keysCap,
                          uint32_t blocksPerSm, uint32_t entries, cudaStream_t s, uint32_t* launches);

// Mesh checks of vxb_create (vxb_meshcheck.cu): hostOut[0..2] / [3..5]
// name the first vertex (after vertex 0) holding the smallest / largest
// non-NaN coordinate per axis as (order code << 32 | vertex), ~0 if none;
// hostOut[6] is the largest index, hostOut[7] the first position of an
// index >= nV (~0 if none).  Synchronizes `s`.
int meshCheck(const float* dV, uint32_t nV, const uint32_t* dI, uint64_t nIdx, unsigned long long* dOut,
              unsigned long long* hostOut, cudaStream_t s);

// ---- Node classification: src/voxelizer.cu:1626-2048 ----
void launch_combine(const uint32_t* a, const uint32_t* b, uint32_t* out, uint64_t n, cudaStream_t s,
                    uint32_t* launches);

// One pruning region: subspace `split` of unit `unit`.  wordStart is the
// exclusive prefix of region words within one launch.
struct PruneRegion {
    uint32_t unit;
    SplitYZ split;
    uint32_t wordStart;
};
// Pruning of one subspace index.  launch_prune: the first pass over every
// word of its `n` regions (groupWords words in all), appending each changed
// word to `list`; launch_prune_list: a later pass over the words next to the
// changes listed in `in`, appending its own changes to `out`.  Lists hold
// (region << 32 | word) entries, at most `cap`; past it *overflow is set and
// the passes are no longer complete.  A region that changed in pass p sets
// flags[(flagBase + region) * passes + p].  Neighbours in later subspaces
// are read from fill | surf (surf may be NULL).
void launch_prune(const Batch& b, const PruneRegion* regions, uint32_t n, uint32_t groupWords, uint32_t* solid,
                  const uint32_t* fill, const uint32_t* surf, uint32_t* flags, uint32_t flagBase, uint32_t passes,
                  unsigned long long* list, uint32_t* count, uint32_t cap, uint32_t* overflow, cudaStream_t s,
                  uint32_t* launches);
// Passes firstPass .. passes - 1 of one subspace index in one block-sized
// launch (lists alternating between list0 and list1, counts[p] the count of
// pass p); it stops at an empty list, and a list longer than escapeAt marks
// all nRegions regions as changed in the last pass (the host then runs full
// passes until stable).
void launch_prune_list_loop(const Batch& b, const PruneRegion* regions, uint32_t nRegions, uint32_t* solid,
                            const uint32_t* fill, const uint32_t* surf, uint32_t* flags, uint32_t flagBase,
                            uint32_t passes, uint32_t firstPass, unsigned long long* list0, unsigned long long* list1,
                            uint32_t* counts, uint32_t cap, uint32_t escapeAt, uint32_t* overflow, cudaStream_t s,
                            uint32_t* launches);
void launch_prune_list(const Batch& b, const PruneRegion* regions, uint32_t* solid, const uint32_t* fill,
                       const uint32_t* surf, uint32_t* flags, uint32_t flagBase, uint32_t passes, uint32_t pass,
                       const unsigned long long* in, const uint32_t* inCount, unsigned long long* out,
                       uint32_t* outCount, uint32_t cap, uint32_t* overflow, cudaStream_t s, uint32_t* launches);
// Slices along x (vxb_xslice.cu): vertex rotation, the node array before
// the boundary ids, un-rotation, one in-place boundary-id pass over a yz
// subspace (sets *changed when a node loses its id) and face zeroing.  The
// node kernels treat nodes as `nodeBytes` bytes with the id in byte 0
// (masked by idMask).
void launch_rotate_vertices(const float* V, float* R, uint32_t n, double a, double b, cudaStream_t s,
                            uint32_t* launches);
void launch_emit_raw(int nodeKind, const Batch& b, uint64_t totalWords, const uint32_t* fill, const uint32_t* surf,
                     const WordRank* ranks, const void* keys, uint32_t keysCap, cudaStream_t s, uint32_t* launches);
void launch_unrotate(const void* in, void* out, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nodeBytes,
                     cudaStream_t s, uint32_t* launches);
void launch_id_pass(void* nodes, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nodeBytes, uint32_t idMask,
                    uint32_t y0, uint32_t y1, uint32_t z0, uint32_t z1, uint32_t* changed, cudaStream_t s,
                    uint32_t* launches);
void launch_zero_faces(void* nodes, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nodeBytes, bool fcc, cudaStream_t s,
                       uint32_t* launches);
// FCC lattices: unRotateNodes' FCC branch (X x Y x Z -> 2Y x X/2 x Z) and
// calculateFCCBoundaries in place.
void launch_unrotate_fcc(const void* in, void* out, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nodeBytes,
                         cudaStream_t s, uint32_t* launches);
void launch_fcc_boundaries(void* nodes, uint32_t X, uint32_t Y, uint32_t Z, uint32_t nodeBytes, cudaStream_t s,
                           uint32_t* launches);
// Keys at ranks >= keysCap read as 0.
// Words [wordBegin, totalWords) of the arena (wordBegin a multiple of 32).
void launch_emit_cartesian(int nodeKind, const Batch& b, uint64_t wordBegin, uint64_t totalWords,
                           const uint32_t* finalSolid,
                           const uint32_t* fill, const uint32_t* surf, const WordRank* ranks, const void* keys,
                           uint32_t keysCap, uint32_t blocksPerSm, cudaStream_t s, uint32_t* launches);

// An FCC mesh: its four sub-lattice units are units [unit0, unit0 + 4).
struct FccMesh {
    uint32_t unit0;
    void* out;
};
// FCC node grids; groupBase[m] is the first 16-byte output group of mesh m
// (nMeshes + 1 entries).  raw: the nodes before calculateFCCBoundaries (id =
// solid bit, the surface material), for slices along x.
void launch_emit_fcc(int nodeKind, const Batch& b, const FccMesh* meshes, const uint64_t* groupBase,
                     uint32_t nMeshes, uint64_t totalGroups, const uint32_t* fill, const uint32_t* surf,
                     const WordRank* ranks, const void* keys, uint32_t keysCap, bool raw, cudaStream_t s,
                     uint32_t* launches);

}  // namespace vxb
