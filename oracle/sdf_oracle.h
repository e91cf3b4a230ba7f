/* CPU oracle for the SDF -> mesh hot path: TEST INFRASTRUCTURE, not part of the product.
 *
 * A plain-C restatement of the reference's algorithm (mite51/CudaSDF, src/SDFMesh/), used by the
 * tests as the checker and by bench.py as the timed CPU baseline. Only tests/, the smoke check and
 * bench.py's CPU-baseline leg load it. Every function cites the reference lines it restates.
 *
 * Floating point: the reference is compiled by nvcc with FMA contraction on. The oracle is built
 * with -ffp-contract=off and writes each fused multiply-add the reference's compiled code performs
 * as an explicit fmaf(); the pattern is pinned against the reference's own outputs on the GPU
 * (tests/golden/probes.npz, map_probes.npz). Transcendentals (sinf/cosf/atan2f/asinf) come from the
 * host libm and differ from CUDA's by a few ulp; paths using them are compared with a tolerance.
 */
#ifndef SDF_ORACLE_H
#define SDF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Byte-identical to the reference's SDFPrimitive (Commons.cuh:68-102, 160 bytes). */
typedef struct OrPrim {
    float rotation[4];
    float dispParams[4];
    float position[3];
    float blendFactor;
    float scale[3];
    float rounding;
    float color[3];
    float annular;
    float params[6];
    int32_t type, operation, displacement, pad1;
    float uvScale[2];
    float uvOffset[2];
    float uvRotation;
    int32_t uvMode, textureID, atlasIslandID;
    float pad2[2];
} OrPrim;

/* Byte-identical to the reference's BVHNode (Commons.cuh:104-109). */
typedef struct OrNode {
    float mn[3], mx[3];
    int32_t left, right;
} OrNode;

typedef struct OrScene {
    const OrPrim* prims; /* sorted: BVH (union) primitives first */
    int32_t nprims;
    int32_t nbvh;        /* number of primitives in the BVH */
    const OrNode* nodes;
    int32_t nnodes;
} OrScene;

typedef struct OrGridDesc {
    uint32_t width, height, depth; /* samples per axis */
    int32_t bx, by, bz;            /* blocks per axis */
    float origin[3];
    float cell;
} OrGridDesc;

/* output stream mask (same bits as the engine's) */
enum { OR_COLORS = 1, OR_INDICES = 2, OR_UVS = 4, OR_PRIMIDS = 8, OR_NORMALS = 16 };

/* buffer ids for or_result_copy */
enum {
    ORB_ACTIVE = 0, ORB_COUNTS, ORB_OFFSETS, ORB_VERTS, ORB_COLORS, ORB_INDICES, ORB_UVS, ORB_PRIMIDS,
    ORB_NORMALS, ORB_DCMASK, ORB_DCVOFF, ORB_DCVERT, ORB_DCNORM, ORB_SCOUTD
};

typedef struct OrResult OrResult;

/* grid set-up as CudaSDFMesh::Initialize (CudaSDFMesh.cpp:90-129) */
void or_grid_init(OrGridDesc* g, float cell, const float bmin[3], const float bmax[3]);

/* UpdateBVH (CudaSDFMesh.cpp:216-249) + buildBVHRecursive (CudaSDFUtil.h:544-603).
 * sorted_out: n prims; nodes_out: capacity 2n. Returns the number of nodes; *nbvh = unions. */
int or_build_scene(const OrPrim* prims, int n, OrPrim* sorted_out, OrNode* nodes_out, int* nbvh);

/* point queries (batched over n points, 3 floats each) */
void or_map_batch(const OrScene* s, int n, const float* pts, float time, float* out8, int* iters);
void or_normal_batch(const OrScene* s, int n, const float* pts, float time, float cell, float* out3);

/* function-level restatements, batched over records laid out as in the golden probes */
void or_probe(int which, int n, const float* in, int in_stride, float* out, int out_stride);

/* full pipelines: technique 0 = marching cubes, 1 = dual contouring. nthreads <= 0: all. */
OrResult* or_run(const OrScene* s, const OrGridDesc* g, float time, int technique, float qefBlend,
                 uint32_t outMask, uint32_t maxVertices, int nthreads);
void or_result_sizes(const OrResult* r, int64_t out[4]); /* nActive, totalVertices, nDcVerts, scoutCount */
int or_result_copy(const OrResult* r, int buf, void* dst, size_t bytes);
void or_result_free(OrResult* r);

/* scout only, over blocks [b0, b1) (CPU-baseline sampling); returns active count */
int64_t or_scout_range(const OrScene* s, const OrGridDesc* g, float time, int64_t b0, int64_t b1, int nthreads);
/* scout decisions for a list of blocks */
void or_scout_flags(const OrScene* s, const OrGridDesc* g, float time, const int32_t* blocks, int n, uint8_t* flags,
                    int nthreads);
/* marching cubes count+generate over a given list of active blocks (CPU-baseline sampling) */
int64_t or_mc_blocks(const OrScene* s, const OrGridDesc* g, float time, const int32_t* blocks, int nblocks,
                     int nthreads);

/* exclusive prefix sum of uint32 (the reference uses cub::DeviceScan::ExclusiveSum) */
void or_exclusive_scan(const uint32_t* in, uint32_t* out, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
