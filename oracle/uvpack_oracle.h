/* CPU oracle for the UV atlas packer: TEST INFRASTRUCTURE, not part of the product.
 *
 * A C++ restatement of the reference's GridUVPacker (mite51/CudaSDF, src/SDFMesh/GridUVPacker.cu),
 * used by the tests as the checker and by bench.py as the timed CPU baseline of the packer. Every
 * function cites the reference lines it restates. It follows the reference's loops literally (one
 * collision test per drop step, per-cell rasterisation); the product's kernels are checked against it.
 *
 * Floating point: the reference's device code is compiled by nvcc with FMA contraction on. This file
 * is built with -ffp-contract=off and writes each contraction of the compiled code as an explicit
 * fmaf(): `u * res - m` -> fmaf(u, res, -m), `a * b - c * d` -> fmaf(a, b, -(c * d)),
 * `area + 0.01f * m` -> fmaf(0.01f, m, area); inside triangleOverlapsCell two of pointInTriangle's
 * areas are not fused (corner_in_triangle). The pattern is pinned against the reference's own
 * compiled helpers (tests/golden/uvpack_probes.npz). The host parts of the reference (ExtractCharts, the
 * island bounds, the shelf width) are plain IEEE float on x86-64 and are restated as such.
 *
 * Random numbers: the reference draws from cuRAND's XORWOW generator (curand_init(seed, 0, 0),
 * curand()). The oracle does not generate them: the caller passes each attempt's draws, recorded on
 * the GPU by the library's own call of curand (sdf_uv_pack_random_draws).
 */
#ifndef UVPACK_ORACLE_H
#define UVPACK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One island: a chart's masks on the packing grid (GridUVPacker.cuh:68-100). The four bit grids are
 * stored row-major in one word arena, 32 cells per word, rows padded to `stride` words (rotated grids:
 * `stride90`, rows = w). Row bounds (computeRowWordBoundsKernel) are uint16: min words then max words. */
typedef struct UvoIsland {
    int32_t island_index;   /* chart index before the sort by area */
    int32_t primitive_id;
    int32_t num_triangles;
    int32_t min_x, min_y;   /* minCell */
    int32_t w, h;           /* mask dimensions (rotation 0) */
    int32_t stride;         /* words per row of the rotation-0 grids: (w + 31) / 32 */
    int32_t stride90;       /* words per row of the rotated grids: (h + 31) / 32 */
    int32_t pad;
    int64_t off_mask, off_coll, off_mask90, off_coll90;   /* word offsets into the arena */
    int64_t off_rb, off_rb90;                             /* uint16 offsets: 2 h entries, 2 w entries */
} UvoIsland;

/* Configuration, the field order of sdf_uv_pack_config (PackingConfig, GridUVPacker.cuh:121-146). */
enum { UVO_GRID_SIZE = 0, UVO_GRID_RES, UVO_MAX_ITER, UVO_MARGIN, UVO_ROTATION, UVO_X_ALIGN, UVO_MAX_CAND,
       UVO_MAX_DROP, UVO_SHUFFLE, UVO_SEED, UVO_NCFG };

/* Per-attempt status bits of uvo_pack. */
enum { UVO_DRAWS_EXHAUSTED = 1, UVO_CANDIDATE_LOOP_OPEN = 2 };

int64_t uvo_extract_charts(const float* uvs, const float* prim_ids, int64_t num_vertices, int32_t* tri_chart,
                           int32_t* chart_prim, int32_t* chart_ntris, float* chart_bounds, int64_t max_charts);
int uvo_island_plan(int num_charts, const int32_t* chart_prim, const int32_t* chart_ntris,
                    const float* chart_bounds, int grid_resolution, int margin_cells, UvoIsland* out,
                    int64_t* total_words, int64_t* total_rb);
int uvo_island_build(const float* uvs, int64_t num_vertices, const int32_t* tri_chart, int num_charts,
                     const UvoIsland* islands, int grid_resolution, int margin_cells, uint32_t* words,
                     uint16_t* rb);
void uvo_probe(const float* rec, const int32_t* cells, int64_t n, float* area, int32_t* pit, int32_t* orient,
               int32_t* seg, int32_t* overlap);
void uvo_island_sort(int n, const UvoIsland* islands, int32_t* order);
void uvo_seeds(int random_seed, int n, int32_t* out);
int uvo_shelf_width(int n, const UvoIsland* sorted, int grid_size);
int uvo_candidate_loops_end(int n, const UvoIsland* sorted, const int32_t* cfg, int shelf_width);
int uvo_pack(int num_islands, const UvoIsland* sorted, const uint32_t* words, const uint16_t* rb,
             const int32_t* cfg, int shelf_width, int num_solutions, const uint32_t* draws,
             int64_t draws_per_solution, int32_t* sol_info, float* sol_fitness, int32_t* placements,
             int nthreads);
int uvo_select(int num_solutions, const int32_t* sol_info, const float* sol_fitness, int num_islands,
               int grid_size, int32_t* atlas_i, float* atlas_f);
void uvo_remap(float* uvs, const float* prim_ids, int64_t num_vertices, int num_charts,
               const int32_t* chart_prim, const UvoIsland* islands_chart_order, const int32_t* placements,
               int num_placements, int atlas_width, int atlas_height, int grid_resolution);

#ifdef __cplusplus
}
#endif
#endif
