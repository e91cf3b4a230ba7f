// Headless driver for the reference's UV atlas packer (test infrastructure only).
//
// Calls the reference's own host API (GridUVPacker.cuh:186-219, compiled from GridUVPacker.cu where it
// lies in the reference tree) in the order of its only caller (main.cpp:1417-1442), on plain device
// buffers instead of mapped GL buffers, and copies every intermediate result back for comparison.
// Two calls: ref_uvpack_islands (ExtractCharts + CreateIslands) and ref_uvpack_pack (PackIslands +
// RemapUVsToAtlas), so the caller can check, between them, that every candidate loop of the
// reference's packing kernel can end (packSolutionKernel draws candidates until its budget is full,
// GridUVPacker.cu:660-665, and never ends when fewer aligned columns exist).
//
// The reference's source file is compiled unchanged as part of this translation unit, so probe
// kernels can also call its __device__ helpers (triangleArea2D, pointInTriangle, orientSign,
// segmentsIntersect, triangleOverlapsCell, GridUVPacker.cu:41-165) on caller-supplied inputs.
#include "GridUVPacker.cu"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {
std::vector<GridUVPacker::UVChart> g_charts;
std::vector<GridUVPacker::Island> g_islands;
float2* g_uvs = nullptr;
float* g_prim = nullptr;
float4* g_verts = nullptr;
int g_n = 0;

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void release() {
    if (!g_islands.empty()) GridUVPacker::FreeIslands(g_islands);
    g_charts.clear();
    cudaFree(g_uvs);
    cudaFree(g_prim);
    cudaFree(g_verts);
    g_uvs = nullptr;
    g_prim = nullptr;
    g_verts = nullptr;
}

int copy_grid(const GridUVPacker::Grid& g, uint32_t* dst, int64_t cap, int64_t* used) {
    int64_t n = (int64_t)g.stride * g.height;
    if (*used + n > cap) return -1;
    if (n > 0 && cudaMemcpy(dst + *used, g.cells, 4 * n, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    *used += n;
    return 0;
}
}  // namespace

extern "C" {

// ExtractCharts + CreateIslands. charts (chart order): prim id, triangle count, uv min/max, and the
// triangle lists concatenated (tri_cap entries). islands (the reference's sorted order), 5 ints each:
// islandIndex, mask width, mask height, minCell x, minCell y; their four grids (mask, collision,
// mask90, collision90) concatenated in words; row bounds (collision min, max, collision90 min, max).
// ms[0] = ExtractCharts, ms[1] = CreateIslands (wall clock, both synchronous). Returns the number
// of charts, or -1 on a CUDA error or a full buffer.
int ref_uvpack_islands(const float* h_uvs, const float* h_prim, int n, int res, int margin, int max_charts,
                       int32_t* chart_prim, int32_t* chart_ntris, float* chart_bounds, uint32_t* tri_lists,
                       int64_t tri_cap, int32_t* island_info, uint32_t* words, int64_t word_cap,
                       int64_t* words_used, uint16_t* rb, int64_t rb_cap, int64_t* rb_used, double* ms) {
    release();
    g_n = n;
    if (cudaMalloc(&g_uvs, sizeof(float2) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) return -1;
    if (cudaMalloc(&g_prim, sizeof(float) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) return -1;
    if (cudaMalloc(&g_verts, sizeof(float4) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) return -1;
    cudaMemcpy(g_uvs, h_uvs, sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(g_prim, h_prim, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemset(g_verts, 0, sizeof(float4) * (size_t)n);
    cudaDeviceSynchronize();
    double t0 = now_ms();
    g_charts = GridUVPacker::ExtractCharts(g_verts, g_uvs, (const int*)g_prim, n);
    double t1 = now_ms();
    g_islands = GridUVPacker::CreateIslands(g_charts, g_uvs, res, margin);
    cudaDeviceSynchronize();
    double t2 = now_ms();
    ms[0] = t1 - t0;
    ms[1] = t2 - t1;
    if (cudaGetLastError() != cudaSuccess) return -1;
    int nc = (int)g_charts.size();
    if (nc > max_charts) return -1;
    int64_t tri_used = 0;
    for (int c = 0; c < nc; c++) {
        const auto& ch = g_charts[c];
        chart_prim[c] = ch.primitiveID;
        chart_ntris[c] = (int32_t)ch.triangleIndices.size();
        chart_bounds[4 * c + 0] = ch.uvMin.x;
        chart_bounds[4 * c + 1] = ch.uvMin.y;
        chart_bounds[4 * c + 2] = ch.uvMax.x;
        chart_bounds[4 * c + 3] = ch.uvMax.y;
        if (tri_used + (int64_t)ch.triangleIndices.size() > tri_cap) return -1;
        memcpy(tri_lists + tri_used, ch.triangleIndices.data(), 4 * ch.triangleIndices.size());
        tri_used += (int64_t)ch.triangleIndices.size();
    }
    *words_used = 0;
    *rb_used = 0;
    for (int i = 0; i < (int)g_islands.size(); i++) {
        const auto& is = g_islands[i];
        island_info[5 * i + 0] = is.islandIndex;
        island_info[5 * i + 1] = is.mask.width;
        island_info[5 * i + 2] = is.mask.height;
        island_info[5 * i + 3] = is.minCell.x;
        island_info[5 * i + 4] = is.minCell.y;
        if (copy_grid(is.mask, words, word_cap, words_used) || copy_grid(is.collisionMask, words, word_cap, words_used) ||
            copy_grid(is.mask90, words, word_cap, words_used) ||
            copy_grid(is.collisionMask90, words, word_cap, words_used))
            return -1;
        int h = is.collisionMask.height, h9 = is.collisionMask90.height;
        if (*rb_used + 2 * (h + h9) > rb_cap) return -1;
        cudaMemcpy(rb + *rb_used, is.d_collMinWord, 2 * h, cudaMemcpyDeviceToHost);
        cudaMemcpy(rb + *rb_used + h, is.d_collMaxWord, 2 * h, cudaMemcpyDeviceToHost);
        cudaMemcpy(rb + *rb_used + 2 * h, is.d_collMinWord90, 2 * h9, cudaMemcpyDeviceToHost);
        cudaMemcpy(rb + *rb_used + 2 * h + h9, is.d_collMaxWord90, 2 * h9, cudaMemcpyDeviceToHost);
        *rb_used += 2 * (h + h9);
    }
    return cudaGetLastError() == cudaSuccess ? nc : -1;
}

// PackIslands + RemapUVsToAtlas on the islands of the last ref_uvpack_islands call. cfg: the ten
// PackingConfig fields in declaration order. atlas_i: success, width, height, placements;
// atlas_f: fitness, scaling factor; placements: 4 ints each (islandIndex, x, y, rotation, at most
// max_placements); uvs_out: the UVs after the remap (unchanged when the atlas is not a success).
// ms[0] = PackIslands, ms[1] = RemapUVsToAtlas. Returns 0, or -1 on a CUDA error.
int ref_uvpack_pack(const int32_t* cfg, int32_t* atlas_i, float* atlas_f, int32_t* placements, int max_placements,
                    float* uvs_out, double* ms) {
    GridUVPacker::PackingConfig c;
    c.gridSize = cfg[0];
    c.gridResolution = cfg[1];
    c.maxIterations = cfg[2];
    c.marginCells = cfg[3];
    c.enableRotation = cfg[4] != 0;
    c.xAlignment = cfg[5];
    c.maxCandidatesPerIsland = cfg[6];
    c.maxDropSteps = cfg[7];
    c.shuffleOrderPerAttempt = cfg[8] != 0;
    c.randomSeed = cfg[9];
    double t0 = now_ms();
    GridUVPacker::PackedAtlas a = GridUVPacker::PackIslands(g_islands, c);
    double t1 = now_ms();
    if (a.success)
        GridUVPacker::RemapUVsToAtlas(g_uvs, (const int*)g_prim, g_n, g_charts, g_islands, a, c.gridResolution);
    cudaDeviceSynchronize();
    double t2 = now_ms();
    ms[0] = t1 - t0;
    ms[1] = t2 - t1;
    atlas_i[0] = a.success ? 1 : 0;
    atlas_i[1] = a.atlasWidth;
    atlas_i[2] = a.atlasHeight;
    atlas_i[3] = (int32_t)a.placements.size();
    atlas_f[0] = a.fitness;
    atlas_f[1] = a.scalingFactor;
    for (int i = 0; i < (int)a.placements.size() && i < max_placements; i++) {
        placements[4 * i + 0] = a.placements[i].islandIndex;
        placements[4 * i + 1] = a.placements[i].gridX;
        placements[4 * i + 2] = a.placements[i].gridY;
        placements[4 * i + 3] = a.placements[i].rotation;
    }
    cudaMemcpy(uvs_out, g_uvs, sizeof(float2) * (size_t)g_n, cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

void ref_uvpack_release(void) { release(); }

}  // extern "C"

namespace uvprobe {
// in: n records of 8 floats (a, b, c, p as float2) and 2 ints (cell x, y)
__global__ void k_probe(const float* in, const int* cells, int n, float* area, int* pit, int* orient, int* seg,
                        int* overlap) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = in + 8 * i;
    float2 a = make_float2(r[0], r[1]), b = make_float2(r[2], r[3]), c = make_float2(r[4], r[5]),
           p = make_float2(r[6], r[7]);
    area[i] = GridUVPacker::triangleArea2D(a, b, c);
    pit[i] = GridUVPacker::pointInTriangle(p, a, b, c) ? 1 : 0;
    orient[i] = GridUVPacker::orientSign(a, b, c);
    seg[i] = GridUVPacker::segmentsIntersect(a, b, c, p) ? 1 : 0;
    overlap[i] = GridUVPacker::triangleOverlapsCell(a, b, c, cells[2 * i], cells[2 * i + 1], 1.0f) ? 1 : 0;
}
}  // namespace uvprobe

extern "C" {

// The helpers on n inputs (host arrays): triangleArea2D(a, b, c), pointInTriangle(p, a, b, c),
// orientSign(a, b, c), segmentsIntersect(a, b, c, p), triangleOverlapsCell(a, b, c, cell).
int ref_uvpack_probe(const float* h_in, const int* h_cells, int n, float* area, int* pit, int* orient, int* seg,
                     int* overlap) {
    if (n <= 0) return 0;
    float *d_in = nullptr, *d_area = nullptr;
    int *d_cells = nullptr, *d_out = nullptr;
    if (cudaMalloc(&d_in, 32 * (size_t)n) != cudaSuccess || cudaMalloc(&d_cells, 8 * (size_t)n) != cudaSuccess ||
        cudaMalloc(&d_area, 4 * (size_t)n) != cudaSuccess || cudaMalloc(&d_out, 16 * (size_t)n) != cudaSuccess)
        return -1;
    cudaMemcpy(d_in, h_in, 32 * (size_t)n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_cells, h_cells, 8 * (size_t)n, cudaMemcpyHostToDevice);
    uvprobe::k_probe<<<(n + 127) / 128, 128>>>(d_in, d_cells, n, d_area, d_out, d_out + n, d_out + 2 * n,
                                                d_out + 3 * n);
    cudaMemcpy(area, d_area, 4 * (size_t)n, cudaMemcpyDeviceToHost);
    cudaMemcpy(pit, d_out, 4 * (size_t)n, cudaMemcpyDeviceToHost);
    cudaMemcpy(orient, d_out + n, 4 * (size_t)n, cudaMemcpyDeviceToHost);
    cudaMemcpy(seg, d_out + 2 * n, 4 * (size_t)n, cudaMemcpyDeviceToHost);
    cudaMemcpy(overlap, d_out + 3 * n, 4 * (size_t)n, cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_cells);
    cudaFree(d_area);
    cudaFree(d_out);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // extern "C"

extern "C" {

// rasterizeIslandKernel (GridUVPacker.cu:171-225) on one island of caller-given triangles: tri_idx holds
// three vertex indices per triangle into h_uvs; the mask (w x h cells, (w + 31) / 32 words per row) is
// copied to out_words. Returns 0, or -1 on a CUDA error.
int ref_uvpack_raster(const float* h_uvs, int nverts, const uint32_t* tri_idx, int ntris, int minx, int miny, int res,
                      int w, int h, uint32_t* out_words) {
    float2* d_uv = nullptr;
    uint32_t* d_idx = nullptr;
    if (cudaMalloc(&d_uv, 8 * (size_t)(nverts > 0 ? nverts : 1)) != cudaSuccess ||
        cudaMalloc(&d_idx, 12 * (size_t)(ntris > 0 ? ntris : 1)) != cudaSuccess)
        return -1;
    cudaMemcpy(d_uv, h_uvs, 8 * (size_t)nverts, cudaMemcpyHostToDevice);
    cudaMemcpy(d_idx, tri_idx, 12 * (size_t)ntris, cudaMemcpyHostToDevice);
    GridUVPacker::Grid g(w, h);
    if (ntris > 0)
        GridUVPacker::rasterizeIslandKernel<<<(ntris + 255) / 256, 256>>>(d_uv, d_idx, ntris, make_int2(minx, miny),
                                                                         res, g);
    cudaMemcpy(out_words, g.cells, 4 * (size_t)g.stride * h, cudaMemcpyDeviceToHost);
    g.free();
    cudaFree(d_uv);
    cudaFree(d_idx);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // extern "C"
