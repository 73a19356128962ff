/* CPU restatement of hakarlss/Voxelizer's mesh -> node-grid path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * voxelizer_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline may load it.  The product library never links or calls it.
 *
 * It follows the reference files step by step (citations in vox_oracle.cpp):
 * src/host_side.cpp for dimensions, splits and orchestration, and
 * src/voxelizer.cu for the kernels.  Floating-point expressions are evaluated
 * with an explicit fused-multiply-add pattern chosen by `fma_model`
 * (see ORC_FMA_* below), because the reference is built with nvcc's default
 * contraction and that contraction decides results at exact ties.
 */
#ifndef VOX_ORACLE_H
#define VOX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Node layouts (include/node_types.h of the reference). */
enum { ORC_SHORT = 0, ORC_LONG = 1, ORC_PARTIAL = 2, ORC_SHORT_FCC = 3, ORC_LONG_FCC = 4 };

/* Contraction model.  The reference is built with nvcc's default
 * floating-point contraction, which may fuse a multiply and a dependent add
 * into one FMA; the fused form decides results at exact ties.  Each site below
 * is one source expression of the reference; its mode selects how the
 * restatement evaluates it:
 *   p = i*d + m          (P_*, PC_*)   0: mul then add          1: fma(i, d, m)
 *   a*b + c*d + e        (E_*, OT_*)   0: none  1: fma(a,b,c*d)+e  2: fma(c,d,a*b)+e  3: fma(a,b,fma(c,d,e))
 *   -(a*b + c*d)         (D_*, DE_*)   0: none  1: -fma(a,b,c*d)   2: -fma(c,d,a*b)
 *   a*b - c*d            (CR*)         0: none  1: fma(a,b,-(c*d)) 2: fma(-c,d,a*b)
 *   a*b + c*d + e*f      (B_*, TN, DT_*) 0: none 1: fma(e,f,fma(a,b,c*d)) 2: fma(e,f,fma(c,d,a*b))
 *                                      3: fma(a,b,c*d)+e*f  4: fma(e,f,a*b+c*d)  5: fma(c,d,a*b)+e*f
 */
enum {
    /* FP64 solid path, src/voxelizer.cu:840-1617 */
    ORC_S_P_BIN, ORC_S_E_BIN, ORC_S_D_BIN, ORC_S_TN, ORC_S_P_GEN, ORC_S_CR_GEN, ORC_S_D_GEN, ORC_S_E_GEN,
    ORC_S_B_GEN,
    /* FP32 surface path, src/voxelizer.cu:2633-2942, 3040-4119 */
    ORC_S_CRF_CLS, ORC_S_CRF_2D, ORC_S_CRF_3D, ORC_S_PC_2D, ORC_S_PC_3D, ORC_S_PC_3DL,
    ORC_S_DE_2D_YZ, ORC_S_DE_2D_ZX, ORC_S_DE_2D_XY, ORC_S_DE_3D_YZ, ORC_S_DE_3D_ZX, ORC_S_DE_3D_XY,
    ORC_S_OT_2D_YZ, ORC_S_OT_2D_ZX, ORC_S_OT_2D_XY, ORC_S_OT_3D_YZ, ORC_S_OT_3D_ZX, ORC_S_OT_3D_XY,
    ORC_S_OT_3DX_ZX, ORC_S_OT_3DX_XY, ORC_S_OT_3DY_XY, ORC_S_OT_3DY_YZ, ORC_S_OT_3DZ_YZ, ORC_S_OT_3DZ_ZX,
    ORC_S_DT_3DX, ORC_S_DT_3DY, ORC_S_DT_3DZ,
    /* process2DTriangles' inner loop is unrolled: the first (trip count mod
     * UNR_2D) iterations evaluate the edge functions in the OT_2DP_* forms,
     * the rest in the OT_2D_* forms (UNR_2D 0: one form throughout). */
    ORC_S_OT_2DP_YZ, ORC_S_OT_2DP_ZX, ORC_S_OT_2DP_XY, ORC_S_UNR_2D,
    /* The same for the depth loop of process3DTriangles (UNR_3DL, prolog
     * forms OT_3DxP_*). */
    ORC_S_OT_3DXP_ZX, ORC_S_OT_3DXP_XY, ORC_S_OT_3DYP_XY, ORC_S_OT_3DYP_YZ, ORC_S_OT_3DZP_YZ, ORC_S_OT_3DZP_ZX,
    ORC_S_UNR_3DL,
    ORC_NSITES
};

typedef struct {
    int node_type;        /* ORC_* */
    int node_output;      /* 0: plain solid bit array, 1: node grid */
    int materials;        /* surface voxelization with materials */
    int by_cube_length;   /* 1: cube_length given, 0: max_dim given */
    uint32_t max_dim;
    double cube_length;
    uint32_t vox_split[3];
    uint32_t mat_split[3];
    uint8_t fma_sites[64];   /* one mode per ORC_S_* site, for this node type */
    int threads;          /* OpenMP threads (0 = library default) */
    /* Device space (src/host_side.cpp:782-1011): space = 1 voxelizes the
     * yz partition [part[0], part[1]) x [part[2], part[3]) of the grid as
     * the reference's devices do; 0 = the whole grid. */
    int space;
    uint32_t part[4];
    /* Slices along x (src/host_side.cpp:704-718, 1144-1223): the mesh is
     * turned about z as rotateVertices does, the turned grid voxelized (with
     * `part` in its coordinates) and a node result turned back before the
     * boundary ids. */
    int rotate_x;
} orc_params;

typedef struct {
    uint32_t dims[3];         /* output grid dimensions (nodes, or voxels for bit arrays) */
    uint64_t out_bytes;       /* bytes the output occupies */
    double voxel_length;
    double min_vertex[3];
    uint32_t resolution[3];   /* voxel resolution before the y/z padding */
    uint32_t x_splits;
    uint64_t n_conflicts;     /* surface nodes whose winning class saw >1 material */
    uint64_t n_surface;       /* distinct surface nodes */
    uint32_t prune_passes;    /* total pruning passes over all splits */
} orc_info;

/* Computes the output dimensions only (no voxelization). */
int orc_plan(const orc_params* p, const float* verts, uint32_t n_verts, orc_info* info);

/* Full voxelization into `out` (host memory, `out_bytes` >= info.out_bytes).
 * `conflict_out` (optional, one byte per node) receives bit 1 where the
 * surface material of a node was contested inside its winning triangle class
 * and bit 2 where more than one triangle of that class hit the node (the
 * reference's PartialNode ratio then depends on which store landed last);
 * bit 4 marks a PartialNode ratio computed with an edge (nearly) parallel to
 * the plane, where contracted and plain FP32 arithmetic can branch apart. */
int orc_voxelize(const orc_params* p, const float* verts, uint32_t n_verts, const uint32_t* indices,
                 uint32_t n_tris, const uint8_t* materials, uint32_t n_materials, void* out,
                 uint64_t out_bytes, uint8_t* conflict_out, orc_info* info);

/* PartialNode with materials only: orc_voxelize plus, per node, the winning
 * surface triangle (`win_tri`, 0xFFFFFFFF elsewhere; caller fills) and its
 * class 1..3 (`win_cls`). */
int orc_voxelize_winners(const orc_params* p, const float* verts, uint32_t n_verts, const uint32_t* indices,
                         uint32_t n_tris, const uint8_t* materials, uint32_t n_materials, void* out,
                         uint64_t out_bytes, uint8_t* conflict_out, orc_info* info, uint32_t* win_tri,
                         uint8_t* win_cls);

/* The PartialNode ratio triangle `tri` of class `cls` would store at node
 * (x, y, z) of a grid with minimum corner `min_corner` and voxel length d. */
float orc_node_ratio(const orc_params* p, const float* verts, const uint32_t* indices, uint32_t tri, uint32_t cls,
                     int x, int y, int z, const float* min_corner, float d);

#ifdef __cplusplus
}
#endif
#endif
