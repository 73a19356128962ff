/* vxb: C ABI of the B200 voxelizer (mesh -> solid bit array / FDTD node grid).
 *
 * This is the drop-in boundary for hakarlss/Voxelizer's single-GPU path.
 * Every entry point below replaces one public member of the reference's
 * `vox::Voxelizer<Node>` (include/voxelizer.h) or, for the device-resident
 * and batched calls, the launcher seam beneath it
 * (include/host_device_interface.h).  Types are plain C: pointers, sizes and
 * POD structs.  Every function returns a vxb_status; on failure
 * vxb_last_error() holds a message (thread-local).
 *
 * Node layouts in output buffers are byte-identical to
 * include/node_types.h of the reference:
 *   VXB_SHORT_NODE      1 byte : bid bits 0-4, material bits 5-7
 *   VXB_LONG_NODE       2 bytes: bid, material
 *   VXB_PARTIAL_NODE    8 bytes: bid, material, 2 padding bytes, float ratio
 *   VXB_SHORT_FCC_NODE  2 bytes: 12-bit neighbour mask, 4-bit material
 *   VXB_LONG_FCC_NODE   4 bytes: uint16 mask, material, 1 padding byte
 * Plain voxelization output is the reference's bit array: uint32 words, row
 * major (z, y, x/32), voxel x = 32*w + b stored in bit (31 - b) of word w.
 */
#ifndef VXB_H
#define VXB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int vxb_status;
#define VXB_OK              0
#define VXB_EINVAL         -1   /* invalid argument */
#define VXB_ENOMEM         -2   /* device or host allocation failed */
#define VXB_ECUDA          -3   /* CUDA runtime error */
#define VXB_EUNSUPPORTED   -4   /* combination the reference rejects (e.g. FCC + plain voxelization) */
#define VXB_ETIMEDOUT      -5   /* a bounded device-side wait ran out */
#define VXB_EOVERFLOW      -6   /* grid or work list exceeds 32-bit indexing (as in the reference) */
#define VXB_ENOMATERIALS   -7   /* material output requested without materials */

typedef enum {
    VXB_SHORT_NODE = 0,
    VXB_LONG_NODE = 1,
    VXB_PARTIAL_NODE = 2,
    VXB_SHORT_FCC_NODE = 3,
    VXB_LONG_FCC_NODE = 4
} vxb_node_type;

typedef struct { uint32_t x, y, z; } vxb_uint3;

/* One voxelization request: the arguments of Voxelizer::voxelize* (either a
 * maxDimension or a cubeLength, plus the internal split sizes). */
typedef struct {
    int by_cube_length;        /* 1: cube_length is used, 0: max_dimension */
    uint32_t max_dimension;    /* voxels along the longest bounding-box side */
    double cube_length;        /* distance between voxel centres */
    vxb_uint3 vox_split_res;   /* reference default (1024, 512, 512) */
    vxb_uint3 mat_split_res;   /* reference default (512, 512, 512) */
} vxb_request;

/* Shape of a result; mirrors NodePointer<Node>::dim plus the plan values. */
typedef struct {
    vxb_uint3 dim;             /* output dims: nodes, or voxels for bit arrays */
    uint64_t bytes;            /* output size in bytes */
    uint64_t count;            /* nodes, or uint32 words for bit arrays */
    double voxel_length;
    double min_vertex[3];
    double max_vertex[3];
    vxb_uint3 resolution;      /* voxel resolution incl. x padding/rounding, before y/z padding */
    uint32_t x_splits;
    /* Device spaces (partitions, slices): NodePointer::loc, the partition's
     * index (0, y, z) among the partitions, and its voxel range [y0, y1) x
     * [z0, z1) of the full grid; (0, 0, 0) and the whole grid otherwise. */
    vxb_uint3 location;
    uint32_t partition[4];
} vxb_grid_info;

typedef struct vxb_voxelizer vxb_voxelizer;

/* Last error message of the calling thread ("" if none). */
const char* vxb_last_error(void);
/* Library version string. */
const char* vxb_version(void);

/* Voxelizer(vertices, indices, nrOfVertices, nrOfTriangles),
 * include/voxelizer.h:712-716.  The arrays are copied; the caller may free
 * them after the call.  `device` selects the CUDA device (reference: 0). */
vxb_status vxb_create(vxb_voxelizer** out, int node_type, const float* vertices, const uint32_t* indices,
                      uint32_t n_vertices, uint32_t n_triangles, int device);
/* ~Voxelizer(): frees the instance.  Its device buffers go to a
 * process-wide cache of idle blocks (at most 16 GiB) that later instances
 * draw from, so that creating one voxelizer per mesh does not pay cudaMalloc
 * / cudaFree every time.  (Calls return with their work complete; after a
 * failed call this waits for the device first.) */
vxb_status vxb_destroy(vxb_voxelizer* v);
/* No reference counterpart: returns every idle cached block to the driver. */
vxb_status vxb_trim_cache(void);

/* setMaterials(materials, nrOfUniqueMaterials), include/voxelizer.h:862,
 * src/host_side.cpp:218-243: one material id per triangle; rejects more
 * unique materials than the node type holds; enables material output. */
vxb_status vxb_set_materials(vxb_voxelizer* v, const uint8_t* materials, uint32_t n_unique_materials);
/* setMaterialOutput(bool), include/voxelizer.h:864. */
vxb_status vxb_set_material_output(vxb_voxelizer* v, int enable);
/* verboseOutput(bool), include/voxelizer.h:866. */
vxb_status vxb_verbose_output(vxb_voxelizer* v, int enable);
/* The mesh's bounding box as the constructor computed it
 * (calculateBoundingBox, src/host_side.cpp:2462-2488: the float vertices'
 * component-wise min / max widened to double). */
vxb_status vxb_bounding_box(const vxb_voxelizer* v, double min_vertex[3], double max_vertex[3]);

/* Dimensions, voxel length and bounds a request produces, without running
 * it (getArrayDimensions, include/voxelizer.h:868-875, plus the getters
 * getVoxelLength / getMinVertex / getMaxVertex / getResolution).
 * `nodes` = 1 for node grids, 0 for the plain bit array. */
vxb_status vxb_plan(vxb_voxelizer* v, int nodes, const vxb_request* req, vxb_grid_info* info);

/* getArrayDimensions(longestSizeInVoxels | cubeLength, maxInternalXSize,
 * sliceAlongX), src/host_side.cpp:3329-3475.  With sliceAlongX: the grid of
 * the mesh turned as for slices along x, with x and y exchanged (FCC
 * lattices: VXB_EUNSUPPORTED). */
vxb_status vxb_get_array_dimensions(vxb_voxelizer* v, int by_cube_length, uint32_t max_dimension,
                                    double cube_length, uint32_t max_internal_x, int slice_along_x,
                                    vxb_uint3* dims);

/* voxelizeToRAM / voxelizeToNodesToRAM, include/voxelizer.h:727-782,
 * src/host_side.cpp:1829-1886 and 2275-2337: runs the whole path and copies
 * the result into `host_out` (>= info.bytes bytes).  Synchronous. */
vxb_status vxb_voxelize_to_host(vxb_voxelizer* v, int nodes, const vxb_request* req, void* host_out,
                                uint64_t host_bytes, vxb_grid_info* info);

/* voxelize / voxelizeToNodes with devConfig (1,1), include/voxelizer.h:718-770:
 * writes the result into the caller's device buffer `dev_out`, stream-ordered
 * on `stream` (a cudaStream_t, NULL for the default stream).  The mesh is
 * uploaded on the first call and stays resident.  Returns when the result is
 * complete (as the reference's calls do); the host reads a few status words
 * once, after all launches. */
vxb_status vxb_voxelize_to_device(vxb_voxelizer* v, int nodes, const vxb_request* req, void* dev_out,
                                  uint64_t dev_bytes, void* stream, vxb_grid_info* info);

/* Partitioned voxelization: voxelize / voxelizeToNodes with devConfig
 * (dev_y, dev_z), include/voxelizer.h:718-770 and src/host_side.cpp:782-1011
 * (voxelizeEntry / voxelizeWorker).  The yz voxel range is split into
 * dev_y x dev_z partitions (splitResolutionByNrOfParts; remainders to the
 * first part) and each is voxelized as the reference voxelizes it on its own
 * device: its box grows by one voxel towards each neighbouring partition,
 * the allocation is the partition plus one row on each side, and in node
 * output the allocation's faces are zeroed (zeroPadding).  The reference
 * hands one NodePointer per device; here every partition is its own output
 * buffer and all of them run as one batch on this voxelizer's GPU.  Arrays
 * hold dev_y * dev_z entries, y fastest; info.location is the partition's
 * (0, y, z).  FCC lattices return VXB_EUNSUPPORTED. */
vxb_status vxb_plan_parts(vxb_voxelizer* v, int nodes, const vxb_request* req, uint32_t dev_y, uint32_t dev_z,
                          vxb_grid_info* infos);
vxb_status vxb_voxelize_parts_to_device(vxb_voxelizer* v, int nodes, const vxb_request* req, uint32_t dev_y,
                                        uint32_t dev_z, void* const* dev_outs, const uint64_t* dev_bytes,
                                        void* stream, vxb_grid_info* infos);
vxb_status vxb_voxelize_parts_to_host(vxb_voxelizer* v, int nodes, const vxb_request* req, uint32_t dev_y,
                                      uint32_t dev_z, void* const* host_outs, const uint64_t* host_bytes,
                                      vxb_grid_info* infos);

/* Slices: voxelizeSlice / voxelizeSliceToRAM with devConfig 1,
 * include/voxelizer.h:765-795, src/host_side.cpp:1927-2262.  `direction`
 * 1 (y) or 2 (z) is the slice normal; `slice` counts grid rows including
 * the padding row, so 1 .. resolution are the voxel rows.  The result is
 * the node array of a partition one voxel thick: three layers along
 * `direction`, the middle one the slice, the outer ones (and all faces)
 * zero; boundary ids see the voxelized neighbour rows.  Slice 0 or past the
 * grid gives the zero array (sliceOOB).  Node output only; the request's
 * split sizes are used as given (the reference's uint2 (a, b) means
 * (a, b, b)).  Direction 0 (x) follows the reference's rotation
 * (src/host_side.cpp:704-718, 1144-1223, 3261-3309): the mesh turned about z
 * (x' = a - y, y' = b + x, from its bounding box) is sliced along y and the
 * node array is turned back before the boundary ids, so the result is
 * (3, X', Z') nodes of the turned grid with the middle x layer the slice;
 * `slice` counts along the turned grid's y.  The voxelizer's own mesh stays
 * as it is (the reference keeps its stored vertices turned after such a
 * call).  FCC lattices return VXB_EUNSUPPORTED. */
vxb_status vxb_plan_slice(vxb_voxelizer* v, const vxb_request* req, int direction, uint32_t slice,
                          vxb_grid_info* info);
vxb_status vxb_voxelize_slice_to_device(vxb_voxelizer* v, const vxb_request* req, int direction, uint32_t slice,
                                        void* dev_out, uint64_t dev_bytes, void* stream, vxb_grid_info* info);
vxb_status vxb_voxelize_slice_to_host(vxb_voxelizer* v, const vxb_request* req, int direction, uint32_t slice,
                                      void* host_out, uint64_t host_bytes, vxb_grid_info* info);

/* Launch-shape autotuner (no reference counterpart).  Several kernels can
 * spread their work over the GPU in different ways (grid size, work items
 * per warp) with identical results; the best shape depends on the size of
 * the job.  mode 0: fixed default shapes; 1: tune online: the first calls of
 * each size bucket (work triangles, grid words, node type, material output)
 * try candidate shapes, timing each tuned kernel with CUDA events, and after
 * two samples per candidate every kernel keeps its fastest shape; calls
 * captured into a CUDA graph never run trials; 2: use the shapes read from
 * `cache_path` and the defaults elsewhere.  With a `cache_path`, settled
 * shapes are read from it when the mode is set and written back (JSON, one
 * bucket per line) as buckets settle.  Process-wide; resets what was
 * learned before. */
vxb_status vxb_set_autotune(int mode, const char* cache_path);
/* Buckets settled so far and their shapes as JSON (truncated to
 * json_bytes - 1 characters; NULL to skip). */
vxb_status vxb_autotune_state(uint32_t* settled, char* json, uint64_t json_bytes);

/* Number of kernels the last voxelize call launched on the device. */
vxb_status vxb_last_launch_count(vxb_voxelizer* v, uint32_t* launches);

/* Work counters of the last voxelize call (no reference counterpart; the
 * reference's verbose mode prints similar sizes). */
typedef struct {
    uint32_t units;                 /* meshes x lattices */
    uint32_t work_triangles;        /* triangles x lattices */
    uint32_t solid_candidates;      /* (triangle, subspace, 4x4 tile) candidates of the solid pass */
    uint32_t surface_columns;       /* work items of the surface pass */
    uint32_t surface_hits;          /* surface voxel hits (with repeats); 0 when no hit list was kept */
    uint32_t surface_voxels;        /* distinct surface voxels */
    uint32_t surface_triangles[3];  /* triangles with surface work by class: 1D, 2D, 3D boxes */
    uint64_t grid_words;            /* 32-bit words of one bit grid */
} vxb_stats;
vxb_status vxb_last_stats(vxb_voxelizer* v, vxb_stats* stats);

/* Stage timing with CUDA events on the call's stream (off by default; no
 * reference counterpart, the reference only prints clock() stamps in verbose
 * mode).  enable: 0 off, 1 on, 2 on with the stages run one after another
 * on the call's stream instead of the surface pass beside the solid pass
 * (each stage's time is then its own; results are the same).  Stages: 0 solid voxelization, 1 surface voxelization, 2 pruning,
 * 3 node emission, 4 material merge, 5 the surface work kernel alone (part
 * of stage 1).  vxb_stage_times waits for the last call and writes the
 * milliseconds of up to n stages (-1 for a stage that did not run). */
vxb_status vxb_set_profiling(vxb_voxelizer* v, int enable);
vxb_status vxb_stage_times(vxb_voxelizer* v, float* ms, uint32_t n);
/* The same stages on one time axis: start_end[2k] and start_end[2k + 1] are
 * the start and end of stage k in milliseconds after the start of stage 0
 * (negative for work queued on the second stream before it), NaN for a
 * stage that did not run.  Shows how the surface stages overlap the solid
 * and pruning stages. */
vxb_status vxb_stage_timeline(vxb_voxelizer* v, float* start_end, uint32_t n);

/* Batches (no reference counterpart; the reference voxelizes one mesh per
 * call).  A batch runs the meshes of several voxelizers through one sequence
 * of launches: every kernel covers all meshes at once, so many small meshes
 * cost about as much as one large one.  All meshes of a batch share the
 * node type and output kind (node grid or plain bit array) and the device;
 * each gets its own request and device output.  Results are identical to
 * vxb_voxelize_to_device on each mesh alone.  The voxelizers must outlive
 * the batch's runs.  vxb_batch_run returns when every result is complete.
 * With VXB_BATCH_GRAPH the launches are captured once into a CUDA graph and
 * replayed on later runs of the same batch (until vxb_batch_add /
 * vxb_batch_clear change it); a NULL stream then means a stream the batch
 * owns, ordered after the default stream. */
typedef struct vxb_batch vxb_batch;
#define VXB_BATCH_GRAPH 1
vxb_status vxb_batch_create(vxb_batch** out, int device);
vxb_status vxb_batch_destroy(vxb_batch* b);
vxb_status vxb_batch_add(vxb_batch* b, vxb_voxelizer* v, int nodes, const vxb_request* req, void* dev_out,
                         uint64_t dev_bytes, vxb_grid_info* info);
vxb_status vxb_batch_clear(vxb_batch* b);
vxb_status vxb_batch_run(vxb_batch* b, void* stream, int flags);
/* Kernels of the last run (graph replays count the captured kernels). */
vxb_status vxb_batch_last_launch_count(vxb_batch* b, uint32_t* launches);

/* No counterpart in the reference.  The plain voxelization of
 * vxb_voxelize_to_device(v, 0, ...) for callers that cannot allocate device
 * memory: solvers that reserve the whole GPU for their own pool, or that
 * cannot let cudaFree / cudaMalloc synchronize the device mid-step.  It
 * allocates nothing: the mesh (dev_vertices: 3 floats per vertex,
 * dev_indices: 3 indices per triangle) and dev_out are the caller's device
 * buffers, and its work lists live in a fixed device array of 20,990,720
 * bytes inside the library, which every GPU that loads the library holds
 * until exit.  min_vertex / max_vertex: the mesh's bounding box, the
 * component-wise min / max of the vertices (vxb_plan reports it).
 * Limits: at most 1,048,576 triangles, 1024 yz subspaces (vox_split_res
 * parts in y times z) and fewer than 2^32 (triangle, yz subspace, 4x4 tile)
 * candidates, bounded by n_triangles * (ceil(Y / 4) + parts in y) *
 * (ceil(Z / 4) + parts in z) over the grid's resolution Y x Z; larger
 * requests return VXB_EINVAL.  Runs on the current device, stream-ordered on
 * `stream`; it neither waits for the GPU nor copies from host memory.  The
 * first call on a device looks up the array's address (one-time set-up);
 * make it before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race and must be serialized by the caller. */
vxb_status vxb_voxelize_bits_noalloc(const float* dev_vertices, const uint32_t* dev_indices, uint32_t n_vertices,
                                     uint32_t n_triangles, const double min_vertex[3], const double max_vertex[3],
                                     const vxb_request* req, void* dev_out, uint64_t dev_bytes, void* stream,
                                     vxb_grid_info* info);

/* No counterpart in the reference.  The errors of the last
 * vxb_voxelize_bits_noalloc call on the current device that only the GPU
 * sees: VXB_EINVAL if an index was >= n_vertices (such indices read vertex
 * 0, so no kernel reads past the vertex buffer, but the bit array is
 * undefined), VXB_EOVERFLOW if the candidate count overflowed, else VXB_OK.
 * Call it once that call's stream has finished; it copies 12 bytes from the
 * device and allocates nothing. */
vxb_status vxb_noalloc_status(void);

/* No counterpart in the reference (the reference sums its tile counts on the
 * host).  The exclusive scan that sizes every work list, exported so that
 * its overflow detection can be tested without a work list of 2^32
 * entries: scans n device counts into offsets (n + 1 device entries) on
 * `stream`, waits, and writes the 32-bit total and the overflow flag (1 when
 * the sum is 2^32 - 1 or more, and the offsets are then not valid).
 * Allocates its tile sums. */
vxb_status vxb_scan_counts(const uint32_t* counts, uint32_t n, uint32_t* offsets, uint32_t* total,
                           uint32_t* overflow, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* VXB_H */
