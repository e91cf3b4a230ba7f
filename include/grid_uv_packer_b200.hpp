// GridUVPacker host API on sdfmesh_b200: a header-only C++ mirror of the reference's
// src/SDFMesh/GridUVPacker.cuh:186-219 (ExtractCharts, CreateIslands, PackIslands, RemapUVsToAtlas,
// FreeIslands) over the sdf_uv_atlas_* C entry points, so a caller written against the reference
// (main.cpp:1417-1442) compiles unchanged when it includes this header instead of GridUVPacker.cuh.
//
// Same names, argument meaning and results (charts, island order and masks, placements, remapped UVs).
// Differences: the reference prints its diagnostics to stdout, this prints nothing; the islands'
// device masks are owned by an sdf_uv_atlas that the charts and islands share (FreeIslands drops the
// islands' reference, the last holder frees it); `Island` exposes the reference's host-visible fields
// and its mask dimensions, not the device Grid members. Every call synchronises the device, as the
// reference's do. Errors of the C entry points are reported through the returned values (no charts,
// no islands, PackedAtlas::success = false), as the reference reports its own.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "sdfmesh_b200.h"

namespace GridUVPacker {

// PackingConfig (GridUVPacker.cuh:121-146)
struct PackingConfig {
    int gridSize = 128;
    int gridResolution = 64;
    int maxIterations = 500;
    int marginCells = 2;
    bool enableRotation = true;
    int xAlignment = 8;
    int maxCandidatesPerIsland = 32;
    int maxDropSteps = 0;
    bool shuffleOrderPerAttempt = true;
    int randomSeed = 0;
};

// IslandPlacement (GridUVPacker.cuh:104-111)
struct IslandPlacement {
    int islandIndex = -1;
    int gridX = 0;
    int gridY = 0;
    int rotation = 0;
};

using AtlasHandle = std::shared_ptr<sdf_uv_atlas>;

// UVChart (GridUVPacker.cuh:149-157)
struct UVChart {
    int primitiveID = -1;
    std::vector<uint32_t> triangleIndices;
    float2 uvMin = make_float2(1e10f, 1e10f);
    float2 uvMax = make_float2(-1e10f, -1e10f);
    AtlasHandle atlas;  // the packer state the chart belongs to
};

// Island (GridUVPacker.cuh:68-100): host fields and mask dimensions
struct Island {
    float2 uvMin = make_float2(0.0f, 0.0f);
    float2 uvMax = make_float2(1.0f, 1.0f);
    int2 minCell = make_int2(0, 0);
    int numTriangles = 0;
    int primitiveID = -1;
    int islandIndex = -1;
    int width = 0, height = 0;  // mask.width, mask.height
    AtlasHandle atlas;
};

// PackedAtlas (GridUVPacker.cuh:160-170)
struct PackedAtlas {
    std::vector<IslandPlacement> placements;
    float scalingFactor = 1.0f;
    int atlasWidth = 0;
    int atlasHeight = 0;
    float fitness = 0.0f;
    bool success = false;
};

namespace detail {
inline AtlasHandle make_atlas() {
    sdf_uv_atlas* a = nullptr;
    if (sdf_uv_atlas_create(&a) != SDF_OK) return AtlasHandle();
    return AtlasHandle(a, sdf_uv_atlas_destroy);
}
template <class T>
inline std::vector<T> read(sdf_uv_atlas* a, int which) {
    size_t bytes = 0;
    std::vector<T> out;
    if (sdf_uv_atlas_read(a, which, nullptr, &bytes) != SDF_OK || bytes == 0) return out;
    out.resize(bytes / sizeof(T));
    if (sdf_uv_atlas_read(a, which, out.data(), &bytes) != SDF_OK) out.clear();
    return out;
}
}  // namespace detail

// ExtractCharts (GridUVPacker.cu:833-896). d_vertices is not read (the reference only downloads it).
inline std::vector<UVChart> ExtractCharts(const float4* d_vertices, const float2* d_uvCoords, const int* d_primitiveIDs,
                                          int numVertices) {
    (void)d_vertices;
    std::vector<UVChart> charts;
    AtlasHandle a = detail::make_atlas();
    int32_t n = 0;
    if (!a || sdf_uv_atlas_extract_charts(a.get(), reinterpret_cast<const sdf_float2*>(d_uvCoords),
                                          reinterpret_cast<const float*>(d_primitiveIDs), numVertices, nullptr,
                                          &n) != SDF_OK)
        return charts;
    const std::vector<sdf_uv_chart> table = detail::read<sdf_uv_chart>(a.get(), 0);
    const std::vector<int32_t> tri = detail::read<int32_t>(a.get(), 1);
    charts.resize(table.size());
    for (size_t c = 0; c < table.size(); c++) {
        charts[c].primitiveID = table[c].primitive_id;
        charts[c].uvMin = make_float2(table[c].uv_min.x, table[c].uv_min.y);
        charts[c].uvMax = make_float2(table[c].uv_max.x, table[c].uv_max.y);
        charts[c].triangleIndices.reserve((size_t)table[c].num_triangles);
        charts[c].atlas = a;
    }
    for (size_t t = 0; t < tri.size(); t++)
        if (tri[t] >= 0) charts[(size_t)tri[t]].triangleIndices.push_back((uint32_t)t);
    return charts;
}

// CreateIslands (GridUVPacker.cu:898-1061) for charts returned by ExtractCharts; islands in the
// reference's order (sorted by mask area, largest first).
inline std::vector<Island> CreateIslands(const std::vector<UVChart>& charts, const float2* d_uvCoords,
                                         int gridResolution, int marginCells) {
    std::vector<Island> islands;
    if (charts.empty() || !charts[0].atlas) return islands;
    AtlasHandle a = charts[0].atlas;
    if (sdf_uv_atlas_create_islands(a.get(), reinterpret_cast<const sdf_float2*>(d_uvCoords), gridResolution,
                                    marginCells, nullptr) != SDF_OK ||
        cudaDeviceSynchronize() != cudaSuccess)
        return islands;
    const std::vector<sdf_uv_island> isl = detail::read<sdf_uv_island>(a.get(), 2);
    islands.resize(isl.size());
    for (size_t i = 0; i < isl.size(); i++) {
        const UVChart& c = charts[(size_t)isl[i].island_index];
        islands[i].uvMin = c.uvMin;
        islands[i].uvMax = c.uvMax;
        islands[i].minCell = make_int2(isl[i].min_cell_x, isl[i].min_cell_y);
        islands[i].numTriangles = isl[i].num_triangles;
        islands[i].primitiveID = isl[i].primitive_id;
        islands[i].islandIndex = isl[i].island_index;
        islands[i].width = isl[i].width;
        islands[i].height = isl[i].height;
        islands[i].atlas = a;
    }
    return islands;
}

// PackIslands (GridUVPacker.cu:1063-1439)
inline PackedAtlas PackIslands(const std::vector<Island>& islands, const PackingConfig& config) {
    PackedAtlas r;
    if (islands.empty() || !islands[0].atlas) return r;
    sdf_uv_pack_config c;
    c.grid_size = config.gridSize;
    c.grid_resolution = config.gridResolution;
    c.max_iterations = config.maxIterations;
    c.margin_cells = config.marginCells;
    c.enable_rotation = config.enableRotation ? 1 : 0;
    c.x_alignment = config.xAlignment;
    c.max_candidates_per_island = config.maxCandidatesPerIsland;
    c.max_drop_steps = config.maxDropSteps;
    c.shuffle_order_per_attempt = config.shuffleOrderPerAttempt ? 1 : 0;
    c.random_seed = config.randomSeed;
    sdf_uv_atlas_info info;
    if (sdf_uv_atlas_pack(islands[0].atlas.get(), &c, nullptr, &info) != SDF_OK) return r;
    if (info.best_solution < 0) return r;
    for (const sdf_uv_placement& p : detail::read<sdf_uv_placement>(islands[0].atlas.get(), 9))
        r.placements.push_back(IslandPlacement{p.island_index, p.grid_x, p.grid_y, p.rotation});
    r.scalingFactor = info.scaling_factor;
    r.atlasWidth = info.atlas_width;
    r.atlasHeight = info.atlas_height;
    r.fitness = info.fitness;
    r.success = info.success != 0;
    return r;
}

// RemapUVsToAtlas (GridUVPacker.cu:1441-1547): the placements and size of `atlas`, the islands' cells
inline void RemapUVsToAtlas(float2* d_uvCoords, const int* d_primitiveIDs, int numVertices,
                            const std::vector<UVChart>& charts, const std::vector<Island>& islands,
                            const PackedAtlas& atlas, int gridResolution) {
    (void)charts;
    if (!atlas.success || atlas.placements.empty() || islands.empty() || !islands[0].atlas) return;
    std::vector<sdf_uv_placement> pl;
    for (const IslandPlacement& p : atlas.placements)
        pl.push_back(sdf_uv_placement{p.islandIndex, p.gridX, p.gridY, p.rotation});
    sdf_uv_atlas_remap_placements(islands[0].atlas.get(), reinterpret_cast<sdf_float2*>(d_uvCoords),
                                  reinterpret_cast<const float*>(d_primitiveIDs), numVertices, gridResolution,
                                  pl.data(), (int32_t)pl.size(), 1, atlas.atlasWidth, atlas.atlasHeight, nullptr);
    cudaDeviceSynchronize();
}

// FreeIslands (GridUVPacker.cu:1549-1568)
inline void FreeIslands(std::vector<Island>& islands) { islands.clear(); }

}  // namespace GridUVPacker
