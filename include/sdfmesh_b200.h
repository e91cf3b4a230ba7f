/* sdfmesh_b200: B200-native (sm_100a) SDF -> mesh engine, C ABI.
 *
 * Drop-in boundary. The library exports, under the same unmangled names, the twelve extern "C"
 * entry points of the reference's src/SDFMesh/Wrappers.cu:19-136 (declared by the reference's
 * caller at CudaSDFMesh.cpp:15-29). The reference passes `SDFGrid&`; a C++ reference is a pointer at
 * the ABI level, so they are declared here as `sdf_grid*`. A project that links this library in
 * place of MarchingCubesKernels.cu + Wrappers.cu keeps its own CudaSDFMesh.cpp unchanged.
 *
 * The data types below are byte-identical to the reference's SDFPrimitive, BVHNode and SDFGrid
 * (Commons.cuh:68-186); their sizes and field offsets are pinned by static assertions.
 *
 * Beside the drop-in launchers, the library has its own entry points (sdf_engine_*, sdf_extract):
 * status codes, an explicit stream, no host synchronisation inside except the final count
 * read-back, and a fused pipeline (scout -> block field -> count -> scan -> emit).
 */
#ifndef SDFMESH_B200_H
#define SDFMESH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#define SDF_ALIGN16 alignas(16)
#else
#define SDF_ALIGN16 _Alignas(16)
#endif

/* ------------------------------------------------------------------------------------------------
 * Data layout (Commons.cuh)
 * ---------------------------------------------------------------------------------------------- */
typedef struct sdf_float2 { float x, y; } sdf_float2;
typedef struct sdf_float4 { SDF_ALIGN16 float x; float y, z, w; } sdf_float4;
typedef struct sdf_ushort4 { uint16_t x, y, z, w; } sdf_ushort4;
typedef struct sdf_short4 { int16_t x, y, z, w; } sdf_short4;

/* PrimitiveType (Commons.cuh:17-34) */
enum {
    SDF_SPHERE = 0, SDF_BOX, SDF_TORUS, SDF_CYLINDER, SDF_CAPSULE, SDF_CONE, SDF_ROUNDED_BOX,
    SDF_ROUNDED_CYLINDER, SDF_ROUNDED_CONE, SDF_ELLIPSOID, SDF_TRIANGULAR_PRISM, SDF_OCTOHEDRON,
    SDF_HEX_PRISM, SDF_SOLID_ANGLE, SDF_CUSTOM_FLOAT, SDF_CUSTOM_VECTOR
};
/* OperationType (Commons.cuh:37-44) */
enum { SDF_UNION = 0, SDF_SUBTRACT, SDF_INTERSECT, SDF_UNION_BLEND, SDF_SUBTRACT_BLEND, SDF_INTERSECT_BLEND };
/* DisplacementType (Commons.cuh:47-57); SINE, TWIST and BEND are the ones map() applies */
enum { DISP_NONE = 0, DISP_SINE, DISP_TWIST, DISP_BEND, DISP_ELONGATE, DISP_ROUND, DISP_ONION, DISP_EXTRUSION,
       DISP_REVOLUTION };

/* SDFPrimitive (Commons.cuh:68-102): 160 bytes */
typedef struct sdf_primitive {
    SDF_ALIGN16 float rotation[4]; /* quaternion x, y, z, w */
    float dispParams[4];
    float position[3];
    float blendFactor;   /* smooth-blend k */
    float scale[3];
    float rounding;
    float color[3];
    float annular;
    float params[6];
    int32_t type;
    int32_t operation;
    int32_t displacement;
    int32_t _pad1;
    float uvScale[2];
    float uvOffset[2];
    float uvRotation;
    int32_t uvMode;
    int32_t textureID;
    int32_t atlasIslandID;
    float _pad2[2];
} sdf_primitive;

/* BVHNode (Commons.cuh:104-109): leaf iff right == -1, then left = primitive index */
typedef struct sdf_bvh_node {
    float min[3];
    float max[3];
    int32_t left;
    int32_t right;
} sdf_bvh_node;

#define SDF_BLOCK_SIZE 8
#define SDF_BLOCK_SIZE_CUBED 512

/* SDFGrid (Commons.cuh:115-186): 232 bytes, passed by reference to every launcher */
typedef struct sdf_grid {
    int32_t* d_activeBlocks;
    int32_t* d_activeBlockCount;
    int32_t maxBlocks;
    int32_t blocksDim[3];
    uint32_t width, height, depth; /* samples per axis */
    float origin[3];
    float cellSize;
    sdf_primitive* d_primitives;
    uint32_t numPrimitives;
    uint32_t numBVHPrimitives;
    sdf_bvh_node* d_bvhNodes;
    uint32_t numBVHNodes;
    uint32_t* d_packetVertexCounts;
    uint32_t* d_packetVertexOffsets;
    int32_t* d_blockToActiveId;
    uint8_t* d_dcCornerMasks;
    uint32_t* d_dcCellVertexOffsets;
    sdf_ushort4* d_dcCellVertices;
    sdf_short4* d_dcCellNormals;
    sdf_short4* d_dcCellNormalsTmp;
    sdf_float4* d_vertices;
    sdf_float4* d_vertexColors;
    uint32_t* d_indices;
    sdf_float2* d_uvCoords;
    int32_t* d_primitiveIDs;  /* holds float bits of the primitive index (MarchingCubesKernels.cu:1093) */
    sdf_float4* d_normals;
    uint32_t maxVertices;
    uint32_t maxIndices;
    uint32_t* d_totalVertices;
    uint32_t* d_totalIndices;
} sdf_grid;

#ifdef __cplusplus
static_assert(sizeof(sdf_primitive) == 160, "SDFPrimitive layout");
static_assert(offsetof(sdf_primitive, position) == 32 && offsetof(sdf_primitive, params) == 80 &&
              offsetof(sdf_primitive, type) == 104 && offsetof(sdf_primitive, uvScale) == 120 &&
              offsetof(sdf_primitive, atlasIslandID) == 148, "SDFPrimitive offsets");
static_assert(sizeof(sdf_bvh_node) == 32, "BVHNode layout");
static_assert(sizeof(sdf_grid) == 232, "SDFGrid layout");
static_assert(offsetof(sdf_grid, cellSize) == 56 && offsetof(sdf_grid, d_primitives) == 64 &&
              offsetof(sdf_grid, d_packetVertexCounts) == 96 && offsetof(sdf_grid, d_vertices) == 160 &&
              offsetof(sdf_grid, maxVertices) == 208 && offsetof(sdf_grid, d_totalIndices) == 224,
              "SDFGrid offsets");
#else
_Static_assert(sizeof(sdf_primitive) == 160, "SDFPrimitive layout");
_Static_assert(sizeof(sdf_bvh_node) == 32, "BVHNode layout");
_Static_assert(sizeof(sdf_grid) == 232, "SDFGrid layout");
#endif

/* ------------------------------------------------------------------------------------------------
 * Drop-in launchers: the reference's Wrappers.cu entry points. Same names, argument meaning and
 * stream (the legacy default stream). Each checks its launch and records the first CUDA error,
 * readable with sdf_last_error(); the reference only printf()s and carries on (Wrappers.cu:26-29).
 * Define SDFMESH_B200_NO_LAUNCHER_DECLS when the reference's own `SDFGrid&` declarations are in
 * scope in the same C++ translation unit.
 * ---------------------------------------------------------------------------------------------- */
#ifndef SDFMESH_B200_NO_LAUNCHER_DECLS
/* Wrappers.cu:19-28  scoutActiveBlocks: active-block list (ascending block index) + count */
void launchScoutActiveBlocks(sdf_grid* grid, float time);
/* Wrappers.cu:30-38  countActiveBlockTriangles: per-cell vertex counts (3 x non-degenerate tris) */
void launchCountActiveBlockTriangles(sdf_grid* grid, int numActiveBlocks, float time);
/* Wrappers.cu:40-48  generateActiveBlockTriangles: triangle-soup emission at the scanned offsets */
void launchGenerateActiveBlockTriangles(sdf_grid* grid, int numActiveBlocks, float time);
/* Wrappers.cu:54-63  buildBlockToActiveMap: dense block -> active-id map (host memsets it to -1) */
void launchBuildBlockToActiveMap(sdf_grid* grid, int numActiveBlocks);
/* Wrappers.cu:65-73  dcMarkCells: 8-bit corner masks + has-vertex counts */
void launchDCMarkCells(sdf_grid* grid, int numActiveBlocks, float time);
/* Wrappers.cu:75-83  dcSolveCellVertices: Hermite data, QEF, quantised vertex + normal */
void launchDCSolveCellVertices(sdf_grid* grid, int numActiveBlocks, float time, unsigned int maxCellVertices,
                               float qefBlend);
/* Wrappers.cu:85-93  dcRecomputeNormalsAtVertices: SDF gradient at the solved vertices */
void launchDCRecomputeNormalsAtVertices(sdf_grid* grid, int numActiveBlocks, float time);
/* Wrappers.cu:95-103 dcSmoothCellNormals: angle-gated 6-neighbour normal smoothing */
void launchDCSmoothCellNormals(sdf_grid* grid, int numActiveBlocks, float cosAngleThreshold);
/* Wrappers.cu:105-113 dcCountQuads: 6 vertices per owned sign-changing edge */
void launchDCCountQuads(sdf_grid* grid, int numActiveBlocks);
/* Wrappers.cu:115-123 dcGenerateQuads: two triangles per quad, soup layout */
void launchDCGenerateQuads(sdf_grid* grid, int numActiveBlocks, float time);
/* Wrappers.cu:125-130 getScanStorageSize: temp bytes for launchScan over num_items */
void getScanStorageSize(unsigned int num_items, size_t* temp_storage_bytes);
/* Wrappers.cu:132-136 launchScan: exclusive prefix sum of uint32 (the reference calls
 * cub::DeviceScan::ExclusiveSum; this one is a single-pass decoupled look-back scan) */
void launchScan(unsigned int* d_input, unsigned int* d_output, unsigned int numItems, void* d_temp_storage,
                size_t temp_storage_bytes);
#endif

/* ------------------------------------------------------------------------------------------------
 * Engine API (no reference counterpart; additive)
 * ---------------------------------------------------------------------------------------------- */
typedef enum sdf_status {
    SDF_OK = 0,
    SDF_ERR_INVALID = 1,   /* bad argument */
    SDF_ERR_CUDA = 2,      /* a CUDA call failed; sdf_last_error() has the cudaError_t */
    SDF_ERR_CAPACITY = 3,  /* output larger than the caller's buffers; counts are still exact */
    SDF_ERR_STACK = 4,     /* BVH deeper than the 64-entry traversal stack */
    SDF_ERR_NOMEM = 5,     /* device allocation failed */
    SDF_ERR_TIMEOUT = 6    /* a bounded device-side wait gave up */
} sdf_status;

/* output stream mask */
enum { SDF_OUT_COLORS = 1, SDF_OUT_INDICES = 2, SDF_OUT_UVS = 4, SDF_OUT_PRIMIDS = 8, SDF_OUT_NORMALS = 16,
       /* indexed mesh (no counterpart in the reference, whose index buffer is the identity):
        * `vertices` receives the shared vertices (stats.welded_vertices of them: one per crossed grid
        * edge for marching cubes, one per surface cell for dual contouring), `indices` (required)
        * three per triangle, the soup's triangles in the soup's order; no colours, UVs, primitive
        * ids or normals; max_vertices bounds both arrays */
       SDF_OUT_WELDED = 32 };
enum { SDF_TECH_MARCHING_CUBES = 0, SDF_TECH_DUAL_CONTOURING = 1 };
/* DC vertex solver: the reference's feature-clustering + regularised QEF, or the mass-point QEF */
enum { SDF_DC_SOLVER_REFERENCE = 0, SDF_DC_SOLVER_MASSPOINT = 1 };

typedef struct sdf_config {
    float cell_size;
    float bounds_min[3];
    float bounds_max[3];
    int32_t technique;          /* SDF_TECH_* */
    float qef_blend;            /* 0 = cell centre, 1 = full QEF solve */
    int32_t dc_solver;          /* SDF_DC_SOLVER_* */
    int32_t projection_iters;   /* mass-point solver: vertex projection iterations (0 = off) */
    int32_t adaptive_diagonal;  /* mass-point solver: split quads along the shorter diagonal */
    float cond_threshold;       /* mass-point solver: pseudo-inverse truncation at lmax / cond_threshold;
                                   cells with condition number above cond_threshold / 16 are solved in FP64 */
    uint32_t out_mask;          /* SDF_OUT_* streams to write (positions are always written) */
} sdf_config;

typedef struct sdf_outputs {
    sdf_float4* vertices;       /* device, capacity max_vertices */
    sdf_float4* colors;         /* optional (SDF_OUT_COLORS) */
    uint32_t* indices;          /* optional (SDF_OUT_INDICES): identity triangle-soup indices */
    sdf_float2* uvs;            /* optional (SDF_OUT_UVS) */
    int32_t* primitive_ids;     /* optional (SDF_OUT_PRIMIDS), float bits as in the reference */
    sdf_float4* normals;        /* optional (SDF_OUT_NORMALS) */
    uint32_t max_vertices;
} sdf_outputs;

typedef struct sdf_stats {
    int64_t total_blocks;
    int64_t active_blocks;
    int64_t total_vertices;     /* exact, even when larger than max_vertices */
    int64_t written_vertices;
    int64_t dc_cell_vertices;
    int64_t bvh_cap_hits;       /* points whose traversal stopped at the 256-visit cap */
    float ms_scout, ms_field, ms_scan, ms_emit, ms_total; /* filled when timing is enabled */
    int64_t scouted_blocks;     /* blocks whose centre the exact scout evaluated (all, unless culled) */
    int64_t dc_fp64_cells;      /* mass-point DC: cells whose QEF was solved in FP64 (condition number) */
    int64_t welded_vertices;    /* SDF_OUT_WELDED: vertices of the indexed mesh (total_vertices = indices) */
    float ms_classify;          /* marching cubes, timing enabled: the part of ms_field that completes the
                                   rows' halos, classifies the cells and counts their triangles */
    float reserved;
} sdf_stats;

typedef struct sdf_engine sdf_engine;

/* Creates an engine on `device` (the current device if < 0). */
sdf_status sdf_engine_create(sdf_engine** out, int device);
void sdf_engine_destroy(sdf_engine* e);
/* Grid as CudaSDFMesh::Initialize (CudaSDFMesh.cpp:90-206). */
sdf_status sdf_engine_configure(sdf_engine* e, const sdf_config* cfg);
/* Scene as CudaSDFMesh::UpdateBVH (CudaSDFMesh.cpp:216-249): unions first, BVH over the unions, built
 * on the host with the reference's node order, then uploaded in the engine's compact device layout. */
sdf_status sdf_engine_set_scene(sdf_engine* e, const sdf_primitive* prims, int count);
/* The scene of sdf_engine_set_scene with the primitives already in device memory (`prims`: a device
 * pointer, 16-byte aligned) and the BVH built on the GPU, on `stream`: the same sorted primitives,
 * nodes and hence meshes as the host build of CudaSDFMesh::UpdateBVH (CudaSDFMesh.cpp:216-249,
 * CudaSDFUtil.h:507-603), which the reference repeats on the host at every Update (:293). Returns
 * after a synchronisation of `stream` (the sizes of the tree are read back). SDF_ERR_STACK when the
 * tree is deeper than the traversal's stack. Drops a trained surrogate. */
sdf_status sdf_engine_set_scene_device(sdf_engine* e, const sdf_primitive* prims, int count, void* stream);
/* One extraction on `stream` (a cudaStream_t, NULL = legacy default stream). The only host
 * synchronisation is the final count read-back into *stats. One stage (the halo samples of the block
 * field) runs on a second, non-blocking stream the engine owns, forked from and joined back into
 * `stream` by events, so the extraction stays ordered on `stream` as a whole. */
sdf_status sdf_engine_extract(sdf_engine* e, float time, const sdf_outputs* out, void* stream, sdf_stats* stats);
/* The extraction of sdf_engine_extract split in two, so that a caller can keep the GPU busy while it
 * reads back earlier results: _async enqueues the whole extraction on `stream` and returns without
 * waiting (a ticket names it); _wait blocks until that extraction has finished and fills `stats`,
 * returning the status sdf_engine_extract would have. Extractions on one stream run one after another;
 * each needs its own output buffers until the caller has read them. Up to four may be pending; a
 * fifth _async first waits for the oldest. Stage times are filled for the most recent one only. No
 * counterpart in the reference, whose Update blocks on its counts (CudaSDFMesh.cpp:466-468). */
sdf_status sdf_engine_extract_async(sdf_engine* e, float time, const sdf_outputs* out, void* stream,
                                    uint64_t* ticket);
sdf_status sdf_engine_extract_wait(sdf_engine* e, uint64_t ticket, sdf_stats* stats);
/* sdf_engine_set_scene with the upload enqueued on `stream` from a pinned copy of the prepared scene
 * (refreshed when the primitives change), so it neither blocks the host nor waits for earlier work.
 * Use the extraction stream. */
sdf_status sdf_engine_set_scene_async(sdf_engine* e, const sdf_primitive* prims, int count, void* stream);
/* Enables per-stage CUDA-event timing inside sdf_engine_extract. */
void sdf_engine_set_timing(sdf_engine* e, int enabled);
/* Debug outputs: bit 0 also writes the per-cell vertex counts/offsets of the drop-in layout in
 * marching-cubes mode (readable through sdf_engine_buffer 1 and 2) and, in dual-contouring mode,
 * the per-cell vertex normals of the reference's dcSolveCellVertices (sdf_engine_buffer 6), which
 * no output of the engine needs; bit 1 keeps, with the mass-point solver, each cell's QEF vertex
 * before its projection steps (sdf_engine_buffer 11: float4 per DC vertex, w = 1 where FP64 solved
 * the cell); bit 2 limits dual contouring's cross-block lists (Hermite normals, projection steps, quad
 * winding normals) to a few hundred entries, so most of the work takes the in-block paths that handle
 * what does not fit (the meshes are the same). */
void sdf_engine_set_debug(sdf_engine* e, int flags);
/* The scene as uploaded: sorted primitives (count = numPrimitives) and BVH nodes. */
int sdf_engine_get_bvh(sdf_engine* e, sdf_bvh_node* nodes_out, int capacity, int* num_bvh_primitives);
/* The host scene build of sdf_engine_set_scene on its own, no GPU involved: CudaSDFMesh::UpdateBVH
 * (CudaSDFMesh.cpp:216-249) with getPrimitiveAABB and buildBVHRecursive (CudaSDFUtil.h:507-603).
 * `sorted_out` (count records) receives the primitives, unions first in their order and then the rest
 * in theirs; `nodes_out` (capacity >= 2 * unions - 1) the BVH over the unions in the reference's node
 * order. Returns the number of nodes (0 without unions), or -1 for a null pointer, a negative count or
 * too small a capacity; *num_bvh_primitives (if set) receives the number of unions. */
int sdf_build_bvh_host(const sdf_primitive* prims, int count, sdf_primitive* sorted_out, sdf_bvh_node* nodes_out,
                       int capacity, int* num_bvh_primitives);
/* Device pointer to the last extraction's internal arrays, for inspection: 0 active block list,
 * 1 per-cell vertex counts (compat layout), 2 per-cell offsets, 3 DC corner masks, 4 DC cell vertex
 * offsets, 5 DC cell vertices, 6 DC cell normals, 7 per-block vertex totals, 8 block field rows; and
 * the scene: 9 sorted primitives, 10 BVH nodes; 11 mass-point QEF vertices (debug bit 1). */
const void* sdf_engine_buffer(sdf_engine* e, int which, size_t* bytes);
/* Copies the first `bytes` bytes of an internal array (ids as for sdf_engine_buffer) to host memory. */
sdf_status sdf_engine_read_buffer(sdf_engine* e, int which, void* host_dst, size_t bytes);

/* The composite SDF of the current scene (the reference's map(), MarchingCubesKernels.cu:570-808) at n
 * device points (x, y, z floats). d_out receives 8 floats per point: distance, colour r g b, primitive
 * index (as a float), local position x y z. Asynchronous on `stream`. */
sdf_status sdf_engine_eval(sdf_engine* e, const float* d_points, int n, float time, float* d_out, void* stream);
/* Distance only (no attributes) at n device points: 1 float per point. */
sdf_status sdf_engine_eval_distance(sdf_engine* e, const float* d_points, int n, float time, float* d_out,
                                    void* stream);
/* The reference's computeNormal (MarchingCubesKernels.cu:814-844) at n device points: 3 floats per
 * point, finite differences of the composite SDF with step 0.001 * cell. */
sdf_status sdf_engine_eval_normals(sdf_engine* e, const float* d_points, int n, float time, float cell,
                                   float* d_out, void* stream);

/* Work counters of one extraction's block-field stage (a separate, slower counting run):
 * out[0] BVH nodes popped per point (summed), out[1] primitive evaluations, out[2] points,
 * out[3] active blocks, out[4] warp-wide stack pops, out[5] of those with a box test,
 * out[6] warp-wide leaf steps, out[7] reserved (0). */
sdf_status sdf_engine_count_work(sdf_engine* e, unsigned long long out[8]);
/* FP32 FMA throughput of the current device in TFLOP/s, measured by a short FMA-loop kernel. */
sdf_status sdf_measure_fp32_peak(double* tflops);

/* One-shot convenience: create, configure, set scene, extract, destroy. */
sdf_status sdf_extract(const sdf_primitive* prims, int count, const sdf_config* cfg, float time,
                       const sdf_outputs* out, void* stream, sdf_stats* stats);

/* The active-block scout of launchScoutActiveBlocks without any device allocation (this entry point
 * has no counterpart in the reference). For callers that must not let a library call cudaMalloc /
 * cudaFree - a per-frame render loop or plugin host that forbids device allocation (both calls
 * synchronise the device and can fail under the host's fixed memory budget), or an application that
 * owns every allocation through its own allocator. Its working memory is one static device array of
 * the library (a little over 4 MiB, held by every device that loads the library until exit).
 * Limit: SDF_SCOUT_STATIC_MAX_BLOCKS 8^3 blocks (1,048,576); larger grids return SDF_ERR_CAPACITY
 * and launch nothing. The first call on a device looks up the array's device address with that
 * device current; make it before any stream capture there. The address is kept for the process's
 * life: after cudaDeviceReset on a device, do not call this entry point there again. Calls share the
 * array and each clears what must start at zero; calls that overlap on the GPU race. A refused launch
 * or memset returns SDF_ERR_CUDA. Runs on the legacy default stream, like launchScoutActiveBlocks;
 * same outputs. */
#define SDF_SCOUT_STATIC_MAX_BLOCKS 1048576u
sdf_status sdf_scout_active_blocks_static(sdf_grid* grid, float time);

/* ---------------------------------------------------------------------------------------------
 * Learned surrogate culling (no counterpart in the reference). A Fourier-feature MLP
 * (3 -> 32 frequencies -> 64 features -> 4 x 64 SiLU -> 1; BF16 weights, FP32 accumulation) is trained
 * on the GPU by the library's own tensor-core forward/backward kernels on samples of the current
 * scene's exact distance (targets clamped to +-clamp). With
 *     K = 16 * sqrt(3) * cell + r_scout + slack_cells * cell,
 * r_scout = (8 * 0.5 * 1.73205 + 2) * cell the scout's own radius (MarchingCubesKernels.cu:874), the
 * certified error eps is the smallest value such that every held-out sample with |f_net| > eps + K
 * has |f_net - clamp(f)| <= eps (errors where the network is near zero never cull anything, so they do
 * not enter), and the cull margin is eps + K.
 * With culling enabled, sdf_engine_extract skips the exact scout inside every coarse block of
 * 32^3 cells (4 x 4 x 4 blocks) whose centre has |f_net| > margin; every kept block runs the exact path, so
 * the mesh is the plain extraction's whenever no culled coarse block holds an active block, which
 * sdf_surrogate_audit checks against a full exact scout.
 * --------------------------------------------------------------------------------------------- */
typedef struct sdf_surrogate_config {
    int32_t samples;            /* training samples (half uniform in the bounds, half near the surface) */
    int32_t validation;         /* held-out samples for the certificate */
    int32_t steps;              /* Adam steps */
    int32_t batch;              /* samples per step */
    float lr;                   /* peak learning rate (cosine decay to 2 %) */
    float freq_sigma;           /* standard deviation of the Fourier frequencies (unit: per half extent) */
    float surface_sigma;        /* standard deviation of the offsets around surface points */
    float clamp;                /* distance targets are clamped to [-clamp, clamp] */
    int32_t surface_res;        /* resolution of the coarse marching-cubes run that supplies surface points */
    float slack_cells;          /* extra cull margin, in cells */
    float time;                 /* scene time the samples are taken at */
    uint32_t seed;
} sdf_surrogate_config;

typedef struct sdf_surrogate_stats {
    float final_loss;           /* mean squared error of the last step */
    float eps_max;              /* max |f_net - clamp(f)| over all held-out samples */
    float eps_cert;             /* the certified error used by the margin (see above) */
    float margin;               /* cull threshold at the configured grid (eps_cert + K) */
    int32_t surface_points;     /* vertices of the coarse run */
    float ms_samples, ms_train, ms_certify;
} sdf_surrogate_stats;

/* Fills *cfg with the defaults (2,000,000 samples, 262,144 held out, 1,500 steps of 65,536, lr 2e-3,
 * frequencies N(0, 2^2), surface offsets N(0, 0.01^2), clamp 0.25, surface run at 128 samples per
 * axis, 2 cells of slack, time 0, seed 1). */
void sdf_surrogate_default_config(sdf_surrogate_config* cfg);
/* Trains the surrogate for the current scene and grid and certifies it; synchronous. */
sdf_status sdf_surrogate_train(sdf_engine* e, const sdf_surrogate_config* cfg, sdf_surrogate_stats* stats);
/* Turns surrogate culling in sdf_engine_extract on or off (SDF_ERR_INVALID if not trained). */
sdf_status sdf_surrogate_enable(sdf_engine* e, int enabled);
/* Coarse-block culling of sdf_engine_extract: SDF_CULL_NONE, SDF_CULL_SURROGATE (f_net with the
 * certified margin eps + K; as sdf_surrogate_enable(e, 1)) or SDF_CULL_EXACT, the method without the
 * network: the exact map() at each coarse centre, one evaluation per 32^3 cells, culled when
 * |f| > K + extra_margin (extra_margin >= 0 is ignored by the other modes). The capped, pruned field
 * of smooth-blended primitives is not 1-Lipschitz (a coarse centre whose search hits the 256-step cap
 * can read far too large a distance), so extra_margin = 0 is not safe in general; the audit below
 * decides whether a margin is. The exact mode needs no training and stays on across scene changes. */
#define SDF_CULL_NONE 0
#define SDF_CULL_SURROGATE 1
#define SDF_CULL_EXACT 2
sdf_status sdf_engine_set_coarse_cull(sdf_engine* e, int mode, float extra_margin);
/* Exact audit of the current culling (surrogate or exact coarse field): a full exact scout at `time`;
 * *violations = exact-active blocks inside culled coarse blocks (0 means the culled extraction equals
 * the plain one), *culled = culled coarse blocks, *coarse = all coarse blocks. Synchronous. */
sdf_status sdf_surrogate_audit(sdf_engine* e, float time, int64_t* violations, int64_t* culled, int64_t* coarse);
/* Number of trainable parameters (hidden W[4][64][64] out x in, b[4][64], w5[64], b5). */
int sdf_surrogate_num_params(void);
/* Parameters: theta (sdf_surrogate_num_params() floats, the order above), freq (32 x 3 floats) and
 * io = {centre x, y, z, scale x, y, z, clamp}; features use (p - centre) * scale. */
sdf_status sdf_surrogate_set_params(sdf_engine* e, const float* theta, const float* freq, const float io[7]);
sdf_status sdf_surrogate_get_params(sdf_engine* e, float* theta, float* freq, float io[7]);
/* f_net at n device points (x, y, z floats) into d_out (n floats). Asynchronous on `stream`. */
sdf_status sdf_surrogate_forward(sdf_engine* e, const float* d_points, int n, float* d_out, void* stream);
/* One forward + backward pass over n device samples (points, targets) without an update: writes the
 * gradient of mean((f_net - clamp(target))^2) into h_grad (num_params floats, host) and the loss into
 * *h_loss. Synchronous. */
sdf_status sdf_surrogate_gradient(sdf_engine* e, const float* d_points, const float* d_targets, int n, float* h_grad,
                                  float* h_loss);

/* ---------------------------------------------------------------------------------------------
 * Batched extraction (no counterpart in the reference, which meshes one scene per Update call).
 * Many independent scenes, each with its own grid, primitives and technique, are meshed together:
 * every stage is one launch over all scenes (the blocks of all marching-cubes scenes form one work
 * queue, those of all dual-contouring scenes another), with per-scene output bases from one scan.
 * sdf_batch_capture records the whole device part of an extraction once as a CUDA graph, after an
 * autotuner has timed the persistent-grid shapes of the heavy kernels on this batch; later
 * sdf_batch_extract calls replay the graph.
 * --------------------------------------------------------------------------------------------- */
typedef struct sdf_batch_scene {
    const sdf_primitive* prims; /* host array, read during sdf_batch_set_scenes */
    int32_t count;
    sdf_config config;          /* grid, technique and DC options of this scene (out_mask: the batch's) */
} sdf_batch_scene;

typedef struct sdf_batch_stats {
    int64_t scenes;
    int64_t total_blocks;
    int64_t active_blocks;
    int64_t mc_vertices;        /* triangle-soup vertices of the marching-cubes scenes */
    int64_t dc_vertices;        /* ... of the dual-contouring scenes */
    float ms_total;             /* host wall time of the call */
    int32_t graph;              /* 1 when the call replayed a captured graph */
    int32_t tuned_ctas[4];      /* CTAs per SM chosen for: block field, emission, DC solve, DC quads */
} sdf_batch_stats;

typedef struct sdf_batch sdf_batch;

sdf_status sdf_batch_create(sdf_batch** out, int device);
void sdf_batch_destroy(sdf_batch* b);
/* Builds every scene's BVH (the engine's order), uploads all scenes and sizes the device buffers.
 * out_mask applies to all scenes. Drops a captured graph. */
sdf_status sdf_batch_set_scenes(sdf_batch* b, const sdf_batch_scene* scenes, int n, uint32_t out_mask);
/* One extraction of all scenes on `stream`. The marching-cubes scenes write one concatenated triangle
 * soup into mc_out, the dual-contouring scenes into dc_out (either may be NULL when no scene uses
 * it); scene i occupies vertices [first_vertex[i], first_vertex[i] + vertex_count[i]) of its
 * technique's buffer (host arrays of n entries, may be NULL), and its identity indices count from
 * the buffer's start. Synchronous (the counts are read back). */
sdf_status sdf_batch_extract(sdf_batch* b, float time, const sdf_outputs* mc_out, const sdf_outputs* dc_out,
                             void* stream, int64_t* first_vertex, int64_t* vertex_count, sdf_batch_stats* stats);
/* Autotunes the CTAs per SM of the heavy kernels on this batch (timing replays), then captures one
 * extraction with the chosen shapes as a CUDA graph for the given outputs and time; later
 * sdf_batch_extract calls with the same outputs replay it (other outputs fall back to direct launches).
 * tune = 0 skips the autotuner (occupancy-limited grids). */
sdf_status sdf_batch_capture(sdf_batch* b, float time, const sdf_outputs* mc_out, const sdf_outputs* dc_out,
                             void* stream, int tune);
/* Copies an internal array of the last extraction of one technique's group to host memory, for
 * inspection (the scenes of a group number their blocks one after another in batch order, scene s
 * owning [base_s, base_s + blocks_s)): 0 active list (int32 global block ids, ascending, so each scene's
 * blocks are one run), 1 per-active-block vertex totals (uint32); dual contouring only: 2 per-cell quad
 * vertex counts (uint32, 512 per active block), 3 corner masks (uint8, 512 per active block), 4 cell
 * vertex offsets (uint32, 512 per active block, counted over the group), 5 cell vertices (ushort4).
 * *bytes: in, the capacity of host_dst; out, the bytes the array holds (host_dst may be NULL to ask). */
sdf_status sdf_batch_read_buffer(sdf_batch* b, int technique, int which, void* host_dst, size_t* bytes);

/* Writes a mesh read back to HOST memory as Wavefront OBJ text, in the format of the reference's
 * ExportMeshToOBJ (src/main.cpp:1043-1115): "# Exported from CudaSDF", "# Generated: <file name>", a
 * blank line, "v x y z" per vertex, a blank line, optionally "vt u v" per vertex and a blank line, then
 * one face line per triangle with 1-based indices ("f a b c", or "f a/a b/b c/c" when uvs is given).
 * Floats are printed as std::ostream prints them by default (%g, six significant digits).
 * indices == NULL: the triangle soup of the reference (face k = vertices 3k, 3k+1, 3k+2);
 * otherwise num_indices / 3 faces from the index buffer (the SDF_OUT_WELDED output).
 * SDF_ERR_INVALID if the file cannot be written, an index is >= num_vertices, or num_vertices == 0
 * (the file then holds the header only, as the reference leaves it). No GPU is used. */
sdf_status sdf_write_obj(const char* path, const sdf_float4* vertices, uint64_t num_vertices, const uint32_t* indices,
                         uint64_t num_indices, const sdf_float2* uvs);

/* ------------------------------------------------------------------------------------------------
 * UV atlas packing: the reference's GridUVPacker (src/SDFMesh/GridUVPacker.{cuh,cu}), which packs the
 * per-primitive UV charts of a mesh (the SDF_OUT_UVS and SDF_OUT_PRIMIDS streams) into one atlas and
 * remaps the UVs into it. The four steps are the reference's ExtractCharts, CreateIslands,
 * PackIslands and RemapUVsToAtlas (GridUVPacker.cuh:186-219, called in that order by main.cpp:1429-1442),
 * with the same results; sdf_uv_atlas_run does all four.
 * ---------------------------------------------------------------------------------------------- */
/* PackingConfig (GridUVPacker.cuh:121-146): the same fields, in the same order, with the same defaults. */
typedef struct sdf_uv_pack_config {
    int32_t grid_size;                 /* board side in cells (square board); at most 16384 */
    int32_t grid_resolution;           /* cells per UV unit */
    int32_t max_iterations;            /* packing attempts; at most 256 run */
    int32_t margin_cells;              /* gutter around each island, in cells (0..1024) */
    int32_t enable_rotation;           /* also try each island rotated by 90 degrees */
    int32_t x_alignment;               /* placement x is a multiple of this */
    int32_t max_candidates_per_island; /* candidate columns per island and rotation (4..64) */
    int32_t max_drop_steps;            /* cap on the downward search (0 = none) */
    int32_t shuffle_order_per_attempt; /* random island order per attempt */
    int32_t random_seed;               /* seed of the attempts' seeds (0 = time()) */
} sdf_uv_pack_config;

/* UVChart (GridUVPacker.cuh:149-157) without its triangle list (sdf_uv_atlas_read 1 has each
 * triangle's chart). */
typedef struct sdf_uv_chart {
    int32_t primitive_id;
    int32_t num_triangles;
    sdf_float2 uv_min, uv_max;
} sdf_uv_chart;

/* A bit grid in the island word arena: 32 cells per word, rows of `stride` words from word_offset. */
typedef struct sdf_uv_grid {
    int32_t width, height, stride, pad;
    int64_t word_offset;
} sdf_uv_grid;

/* Island (GridUVPacker.cuh:68-100), in packing order (the reference's sort by area). */
typedef struct sdf_uv_island {
    int32_t island_index;      /* its chart's index */
    int32_t primitive_id;
    int32_t num_triangles;
    int32_t min_cell_x, min_cell_y;
    int32_t width, height;     /* mask dimensions */
    int32_t pad;
    sdf_uv_grid mask, collision, mask90, collision90;
    int64_t row_bounds, row_bounds90;  /* uint16 arena offsets: first, then last nonzero word of each row */
    int64_t profile, profile90;        /* int32 arena offsets: lowest, then highest set row of each column */
} sdf_uv_island;

/* IslandPlacement (GridUVPacker.cuh:104-111) */
typedef struct sdf_uv_placement {
    int32_t island_index, grid_x, grid_y, rotation;
} sdf_uv_placement;

/* One packing attempt (Solution, GridUVPacker.cuh:114-119). flags bit 0: a candidate loop had fewer
 * aligned columns than its budget and stopped when all were listed (the reference's loop does not end
 * there, GridUVPacker.cu:660-665). */
typedef struct sdf_uv_solution {
    int32_t num_placed, utilized_width, utilized_height, flags;
    float fitness;
    int32_t seed;
} sdf_uv_solution;

/* PackedAtlas (GridUVPacker.cuh:160-170) and the run's counts. */
typedef struct sdf_uv_atlas_info {
    int32_t success;           /* every island placed */
    int32_t atlas_width, atlas_height;  /* squared: both max(utilized width, height) */
    int32_t num_placed;
    float fitness, scaling_factor;
    int32_t num_charts, num_islands, num_solutions;
    int32_t best_solution;     /* -1 when no attempt placed an island */
    int32_t shelf_width;
    int32_t candidate_loop_open;  /* some attempt had a candidate loop the reference could not end */
    float ms_pack;             /* device time of the packing attempts */
    float reserved[3];
} sdf_uv_atlas_info;

typedef struct sdf_uv_atlas sdf_uv_atlas;

void sdf_uv_pack_default_config(sdf_uv_pack_config* c);
sdf_status sdf_uv_atlas_create(sdf_uv_atlas** out);
void sdf_uv_atlas_destroy(sdf_uv_atlas* a);
/* ExtractCharts (GridUVPacker.cu:833-896): one chart per primitive id (the first vertex's float id + 0.5,
 * truncated), in ascending id; d_uvs and d_primitive_ids are num_vertices device entries (the mesh's
 * triangle soup; a partial last triangle is ignored). Synchronises `stream` (the chart table is read
 * back). SDF_ERR_INVALID for ids of 2^24 or more. */
sdf_status sdf_uv_atlas_extract_charts(sdf_uv_atlas* a, const sdf_float2* d_uvs, const float* d_primitive_ids,
                                       int64_t num_vertices, void* stream, int32_t* num_charts);
/* CreateIslands (GridUVPacker.cu:898-1061) for the charts of the last extraction; d_uvs as given to it.
 * Islands wider or taller than 65536 cells (or above 2^30 cells) give SDF_ERR_INVALID. */
sdf_status sdf_uv_atlas_create_islands(sdf_uv_atlas* a, const sdf_float2* d_uvs, int32_t grid_resolution,
                                       int32_t margin_cells, void* stream);
/* PackIslands (GridUVPacker.cu:1063-1439). Synchronises `stream`. info->success as the reference's
 * PackedAtlas.success; SDF_OK also when the atlas is not a success. */
sdf_status sdf_uv_atlas_pack(sdf_uv_atlas* a, const sdf_uv_pack_config* c, void* stream, sdf_uv_atlas_info* info);
/* RemapUVsToAtlas (GridUVPacker.cu:1441-1547): UVs of placed charts into [0, 1] of the atlas; nothing
 * changes when the last packing is not a success. */
sdf_status sdf_uv_atlas_remap(sdf_uv_atlas* a, sdf_float2* d_uvs, const float* d_primitive_ids, int64_t num_vertices,
                              int32_t grid_resolution, void* stream);
/* RemapUVsToAtlas with the atlas given explicitly (the reference's PackedAtlas argument): its
 * placements (host array), squared width and height; the islands of the last sdf_uv_atlas_create_islands.
 * The UVs stay as they are when success is 0 or num_placements is 0. */
sdf_status sdf_uv_atlas_remap_placements(sdf_uv_atlas* a, sdf_float2* d_uvs, const float* d_primitive_ids,
                                         int64_t num_vertices, int32_t grid_resolution,
                                         const sdf_uv_placement* placements, int32_t num_placements,
                                         int32_t success, int32_t atlas_width, int32_t atlas_height, void* stream);
/* The four steps in main.cpp's order (main.cpp:1429-1442). */
sdf_status sdf_uv_atlas_run(sdf_uv_atlas* a, sdf_float2* d_uvs, const float* d_primitive_ids, int64_t num_vertices,
                            const sdf_uv_pack_config* c, void* stream, sdf_uv_atlas_info* info);
/* Copies internal arrays to host memory (after the step that makes them): 0 charts (sdf_uv_chart),
 * 1 chart per triangle (int32, -1 none), 2 islands (sdf_uv_island, packing order), 3 the mask word
 * arena (uint32), 4 row bounds (uint16), 5 column profiles (int32), 6 attempt seeds (int32),
 * 7 attempts (sdf_uv_solution), 8 every attempt's placements (sdf_uv_placement, min(islands, 256) per
 * attempt), 9 the chosen placements. *bytes: in, the capacity of host_dst; out, the bytes the array
 * holds (host_dst may be NULL to ask). Synchronous. */
sdf_status sdf_uv_atlas_read(sdf_uv_atlas* a, int which, void* host_dst, size_t* bytes);
/* For tests: the first `per_seed` values of curand(curand_init(seed, 0, 0)) for each seed, the
 * stream a packing attempt draws from; host arrays. */
sdf_status sdf_uv_pack_random_draws(const int32_t* seeds, int32_t num_seeds, int32_t per_seed, uint32_t* host_out);

/* First CUDA error recorded by a drop-in launcher since the last call (cleared on read). */
int sdf_last_error(void);
/* Library version string. */
const char* sdf_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SDFMESH_B200_H */
