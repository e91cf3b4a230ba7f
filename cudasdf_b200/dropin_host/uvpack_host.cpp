// Headless host for the UV atlas packer through include/grid_uv_packer_b200.hpp: the call sequence of
// the reference's only caller of GridUVPacker (main.cpp:1417-1442: PackingConfig, ExtractCharts,
// CreateIslands, PackIslands, RemapUVsToAtlas when the atlas is a success, FreeIslands), on device
// buffers loaded from files instead of mapped GL buffers.
//
//   uvpack_host <uvs.bin: n float2> <prim.bin: n float> <n> <out_uvs.bin | -> [repeat]
//
// Prints one JSON line: the atlas, its placements and the host wall time per pack (median of `repeat`
// runs, the UVs restored before each).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/grid_uv_packer_b200.hpp"

static bool load(const char* path, void* dst, size_t bytes) {
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    const size_t got = fread(dst, 1, bytes, f);
    fclose(f);
    return got == bytes;
}

int main(int argc, char** argv) {
    if (argc < 5) {
        fprintf(stderr, "usage: %s uvs.bin prim.bin n out_uvs.bin|- [repeat]\n", argv[0]);
        return 2;
    }
    const int n = atoi(argv[3]);
    const int repeat = argc > 5 ? std::max(1, atoi(argv[5])) : 1;
    std::vector<float2> uvs((size_t)n);
    std::vector<float> prim((size_t)n);
    if (!load(argv[1], uvs.data(), sizeof(float2) * (size_t)n) || !load(argv[2], prim.data(), sizeof(float) * (size_t)n)) {
        fprintf(stderr, "cannot read inputs\n");
        return 2;
    }
    float2* d_uv = nullptr;
    int* d_prim = nullptr;
    float4* d_vbo = nullptr;
    if (cudaMalloc(&d_uv, sizeof(float2) * (size_t)std::max(n, 1)) != cudaSuccess ||
        cudaMalloc(&d_prim, sizeof(int) * (size_t)std::max(n, 1)) != cudaSuccess ||
        cudaMalloc(&d_vbo, sizeof(float4) * (size_t)std::max(n, 1)) != cudaSuccess) {
        fprintf(stderr, "cudaMalloc failed\n");
        return 1;
    }
    cudaMemcpy(d_prim, prim.data(), sizeof(float) * (size_t)n, cudaMemcpyHostToDevice);
    GridUVPacker::PackedAtlas atlas;
    std::vector<double> ms;
    for (int r = 0; r < repeat; r++) {
        cudaMemcpy(d_uv, uvs.data(), sizeof(float2) * (size_t)n, cudaMemcpyHostToDevice);
        cudaDeviceSynchronize();
        const auto t0 = std::chrono::steady_clock::now();
        GridUVPacker::PackingConfig cfg;
        cfg.gridSize = 2048;
        cfg.gridResolution = 64;
        cfg.marginCells = 4;
        cfg.enableRotation = true;
        cfg.maxIterations = 256;
        cfg.xAlignment = 8;
        cfg.maxCandidatesPerIsland = 16;
        cfg.maxDropSteps = 256;
        cfg.shuffleOrderPerAttempt = true;
        cfg.randomSeed = 1337;
        auto charts = GridUVPacker::ExtractCharts(d_vbo, d_uv, d_prim, n);
        auto islands = GridUVPacker::CreateIslands(charts, d_uv, cfg.gridResolution, cfg.marginCells);
        atlas = GridUVPacker::PackIslands(islands, cfg);
        if (atlas.success)
            GridUVPacker::RemapUVsToAtlas(d_uv, d_prim, n, charts, islands, atlas, cfg.gridResolution);
        GridUVPacker::FreeIslands(islands);
        cudaDeviceSynchronize();
        ms.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
    std::sort(ms.begin(), ms.end());
    cudaMemcpy(uvs.data(), d_uv, sizeof(float2) * (size_t)n, cudaMemcpyDeviceToHost);
    if (strcmp(argv[4], "-") != 0) {
        FILE* f = fopen(argv[4], "wb");
        if (!f || fwrite(uvs.data(), sizeof(float2), (size_t)n, f) != (size_t)n) {
            fprintf(stderr, "cannot write %s\n", argv[4]);
            return 2;
        }
        fclose(f);
    }
    printf("{\"success\": %d, \"atlas_width\": %d, \"atlas_height\": %d, \"fitness\": %.9g, \"scaling\": %.9g, "
           "\"ms_per_pack\": %.4f, \"repeat\": %d, \"placements\": [",
           atlas.success ? 1 : 0, atlas.atlasWidth, atlas.atlasHeight, atlas.fitness, atlas.scalingFactor,
           ms[ms.size() / 2], repeat);
    for (size_t i = 0; i < atlas.placements.size(); i++) {
        const auto& p = atlas.placements[i];
        printf("%s[%d, %d, %d, %d]", i ? ", " : "", p.islandIndex, p.gridX, p.gridY, p.rotation);
    }
    printf("]}\n");
    cudaFree(d_uv);
    cudaFree(d_prim);
    cudaFree(d_vbo);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
