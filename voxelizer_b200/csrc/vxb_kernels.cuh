// Kernel declarations and the plain structs the host engine passes to them.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vxb {

// Geometry of one solid / surface pass.  For FCC lattices each of the four
// sub-lattices is one pass with its own shifted minimum corner.
struct PassGeom {
    double mn[3];        // minimum corner (FP64, as the reference's extMinVertex)
    double d;            // voxel length
    float mnf[3];        // float(mn) for the FP32 surface path
    float df;            // float(d)
    uint32_t X;          // voxels along x (padded and rounded to 32 * xSplits)
    uint32_t resY, resZ; // voxels along y / z before the 1-voxel padding
    uint32_t AY, AZ;     // allocated rows: resY + 2, resZ + 2
    uint32_t ipx;        // 32-bit words per row: X / 32
};

struct SplitYZ { uint32_t y0, y1, z0, z1; };
struct Split3 { uint32_t x0, x1, y0, y1, z0, z1; };

// Work-list scan: exclusive offsets (n + 1 entries) and the grand total.
void launch_scan(const uint32_t* in, uint32_t* offsets, uint32_t n, uint32_t* blockSums, uint32_t* total,
                 uint32_t* overflow, cudaStream_t s, uint32_t* launches);

// ---- Solid (parity) voxelization: src/voxelizer.cu:840-1617 ----
void launch_solid_count(const float* V, const uint32_t* I, uint32_t nT, PassGeom g, const SplitYZ* splits,
                        uint32_t nSplits, uint32_t* counts, cudaStream_t s, uint32_t* launches);
void launch_solid_toggle(const float* V, const uint32_t* I, uint32_t nT, PassGeom g, const SplitYZ* splits,
                         uint32_t nSplits, const uint32_t* offsets, const uint32_t* total, uint32_t* toggles,
                         cudaStream_t s, uint32_t* launches);
void launch_row_fill(uint32_t* words, uint32_t rows, uint32_t ipx, cudaStream_t s, uint32_t* launches);

// ---- Surface voxelization: src/voxelizer.cu:2358-2989, 3040-4201 ----
// Triangles with surface work are partitioned into kSurfaceBuckets buckets
// by (class, axis); each gets a kSurfRecBytes record and a kSurfOvlBytes
// block of projection edge functions.
constexpr uint32_t kSurfaceBuckets = 9;
constexpr size_t kSurfRecBytes = 64;
constexpr size_t kSurfOvlBytes = 112;

// Material subspace slices along each axis: (lo, hi) pairs, axis a at pair
// offset off[a], n[a] of them.
struct SliceTable { uint32_t off[3], n[3]; };

// Classify (codes / units in mesh order, per-bucket counts in buckets[0..9)),
// partition (perm, unitsP in partitioned order; buckets[9..18) are cursors)
// and set up (records).  buckets and unitsP[0..nT] must be zero on entry.
void launch_surface_prepare(const float* V, const uint32_t* I, const uint8_t* M, uint32_t nT, PassGeom g,
                            uint32_t* codes, uint32_t* units, uint32_t* buckets, uint32_t* perm, uint32_t* unitsP,
                            void* recs, void* ovl, cudaStream_t s, uint32_t* launches);
// Surface work over the exclusive scan `offsets` of unitsP (nT + 1 entries),
// one thread per column.  mode 0: set surface bits in `surfBits` and append
// (bit position << 24 | key) to `list` (entries past listCap are counted,
// not stored); mode 1: merge every hit's key at its rank (needs complete
// bits and `ranks`).  posBase is the bit position of surfBits[0] in the rank
// space (FCC sub-lattices are stacked).  wide: 64-bit keys (PartialNode).
void launch_surface_work(int mode, int wide, const void* recs, const void* ovl, const uint32_t* offsets, uint32_t nT,
                         const uint32_t* total, const uint32_t* buckets, PassGeom g, const uint32_t* slices,
                         SliceTable st, uint32_t* surfBits, uint64_t posBase, const uint32_t* ranks, void* keys, unsigned long long* list,
                         uint32_t* listCount, uint32_t listCap, cudaStream_t s, uint32_t* launches);
// Exclusive popcount prefix over `words` surface words; *total = surface voxels.
void launch_surface_rank(const uint32_t* bits, uint64_t words, uint32_t* ranks, uint32_t* tileSums, uint32_t* total,
                         cudaStream_t s, uint32_t* launches);
void launch_surface_keys_zero(void* keys, const uint32_t* count, int wide, cudaStream_t s, uint32_t* launches);
void launch_surface_merge(const unsigned long long* list, const uint32_t* listCount, uint32_t listCap,
                          const uint32_t* bits, const uint32_t* ranks, uint32_t* keys, cudaStream_t s,
                          uint32_t* launches);

// ---- Node classification: src/voxelizer.cu:1626-2048 ----
void launch_combine(const uint32_t* a, const uint32_t* b, uint32_t* out, uint64_t n, cudaStream_t s,
                    uint32_t* launches);
// One in-place pruning pass over `split`; neighbours in later subspaces
// (yLater / zLater) are read from fill | surf.  Sets *changed if any word
// changed.
void launch_prune(uint32_t* solid, const uint32_t* fill, const uint32_t* surf, const uint8_t* yLater,
                  const uint8_t* zLater, PassGeom g, SplitYZ split, uint32_t* changed, cudaStream_t s,
                  uint32_t* launches);
// yLater[y] / zLater[z] are 1 where row y + 1 / plane z + 1 starts a later
// pruning subspace than row y / plane z.  ranks / keys: surface voxel ranks
// and merged material keys (materials only).
void launch_emit_cartesian(int nodeKind, const uint32_t* finalSolid, const uint32_t* fill, const uint32_t* surf,
                           const uint32_t* ranks, const void* keys, PassGeom g, const uint8_t* yLater,
                           const uint8_t* zLater, void* nodes, int materials, cudaStream_t s, uint32_t* launches);
void launch_emit_fcc(int nodeKind, const uint32_t* const* fill, const uint32_t* const* surf,
                     const uint64_t* surfWordBase, const uint32_t* ranks, const void* keys, PassGeom g, void* nodes,
                     int materials, cudaStream_t s, uint32_t* launches);

}  // namespace vxb
