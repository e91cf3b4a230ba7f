// A headless host application for the reference's own CudaSDFMesh class: CudaSDFMesh.cpp, compiled
// unchanged from the reference tree by the Makefile beside this file, linked against
// libsdfmesh_b200.so in place of the reference's Wrappers.cu + MarchingCubesKernels.cu. It is the
// drop-in as a user of the reference gets it: Initialize, AddPrimitive and Update
// (CudaSDFMesh.cpp:90-206, 281-470) call this library's launch* entry points exactly as they call the
// reference's, with Update's host BVH build, uploads and per-stage synchronisations. The tests compare
// its meshes with the reference's recorded outputs; bench.py times it.
//
// usage: dropin_host <prims.bin> <resolution> <technique 0|1> <out_mask> <repeat> <out_prefix | ->
//   prims.bin   raw SDFPrimitive records (160 bytes each), bounds [-1, 1]^3, cell = 2 / resolution
//   out_mask    bit 0 colours, 1 indices, 2 UVs, 3 primitive ids, 4 normals (positions always)
//   repeat      Update calls after one warm-up call; each is timed on the host (wall, with the
//               host BVH build and uploads Update does every call) and by Update's own kernel timers
//   out_prefix  writes <prefix>.verts, .colors, .indices, .uvs, .primids, .normals (raw, little endian)
// Prints one JSON line with the vertex count and the timings.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "CudaSDFMesh.h"

static void fail(const char* what) {
    fprintf(stderr, "dropin_host: %s\n", what);
    exit(2);
}

template <class T>
static void write_raw(const std::string& path, const T* dev, size_t count) {
    std::vector<T> h(count);
    if (count && cudaMemcpy(h.data(), dev, count * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess)
        fail("read-back failed");
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) fail("cannot write output");
    if (count) fwrite(h.data(), sizeof(T), count, f);
    fclose(f);
}

int main(int argc, char** argv) {
    if (argc != 7) fail("usage: dropin_host prims.bin resolution technique out_mask repeat out_prefix|-");
    const int res = atoi(argv[2]), technique = atoi(argv[3]), mask = atoi(argv[4]), repeat = atoi(argv[5]);
    const std::string prefix = argv[6];
    FILE* f = fopen(argv[1], "rb");
    if (!f) fail("cannot open primitives");
    std::vector<SDFPrimitive> prims;
    SDFPrimitive p;
    while (fread(&p, sizeof(p), 1, f) == 1) prims.push_back(p);
    fclose(f);
    static_assert(sizeof(SDFPrimitive) == 160, "SDFPrimitive layout");

    CudaSDFMesh mesh;
    mesh.Initialize(2.0f / (float)res, make_float3(-1.f, -1.f, -1.f), make_float3(1.f, 1.f, 1.f));
    for (const auto& q : prims) mesh.AddPrimitive(q);

    // output buffers sized for the largest mesh of the workloads this host runs (the caller's job in
    // the reference's application, main.cpp:575-600)
    const size_t cap = (size_t)(res >= 1024 ? 12 : (res >= 512 ? 24 : 4)) << 20;
    float4 *verts = nullptr, *colors = nullptr, *normals = nullptr;
    unsigned* indices = nullptr;
    float2* uvs = nullptr;
    int* primids = nullptr;
    if (cudaMalloc(&verts, cap * sizeof(float4)) != cudaSuccess) fail("cudaMalloc");
    if ((mask & 1) && cudaMalloc(&colors, cap * sizeof(float4)) != cudaSuccess) fail("cudaMalloc");
    if ((mask & 2) && cudaMalloc(&indices, cap * sizeof(unsigned)) != cudaSuccess) fail("cudaMalloc");
    if ((mask & 4) && cudaMalloc(&uvs, cap * sizeof(float2)) != cudaSuccess) fail("cudaMalloc");
    if ((mask & 8) && cudaMalloc(&primids, cap * sizeof(int)) != cudaSuccess) fail("cudaMalloc");
    if ((mask & 16) && cudaMalloc(&normals, cap * sizeof(float4)) != cudaSuccess) fail("cudaMalloc");
    const auto tech = technique ? MeshExtractionTechnique::DualContouring : MeshExtractionTechnique::MarchingCubes;

    mesh.Update(0.f, verts, colors, indices, uvs, primids, normals, tech);  // warm-up
    cudaDeviceSynchronize();
    double wall_ms = 0.0, kernel_ms = 0.0;
    for (int i = 0; i < repeat; ++i) {
        const auto t0 = std::chrono::steady_clock::now();
        mesh.Update(0.f, verts, colors, indices, uvs, primids, normals, tech);
        cudaDeviceSynchronize();
        wall_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        kernel_ms += mesh.GetKernelTimings().totalKernelTime;
    }
    const size_t V = mesh.GetTotalVertexCount();
    if (V > cap) fail("mesh larger than the output buffers");
    if (cudaGetLastError() != cudaSuccess) fail("CUDA error");
    if (prefix != "-") {
        write_raw(prefix + ".verts", verts, V);
        if (colors) write_raw(prefix + ".colors", colors, V);
        if (indices) write_raw(prefix + ".indices", indices, V);
        if (uvs) write_raw(prefix + ".uvs", uvs, V);
        if (primids) write_raw(prefix + ".primids", primids, V);
        if (normals) write_raw(prefix + ".normals", normals, V);
    }
    const CudaSDFMesh::MemStats ms = mesh.GetMemoryStats();
    const CudaSDFMesh::KernelTimings& kt = mesh.GetKernelTimings();
    printf("{\"vertices\": %zu, \"active_blocks\": %d, \"repeat\": %d, \"ms_update_wall\": %.4f, "
           "\"ms_update_kernels\": %.4f, \"ms_scout\": %.4f, \"ms_count\": %.4f, \"ms_scan\": %.4f, "
           "\"ms_generate\": %.4f}\n",
           V, ms.activeBlocks, repeat, repeat ? wall_ms / repeat : 0.0, repeat ? kernel_ms / repeat : 0.0,
           kt.scoutActiveBlocks, kt.mcCountTriangles + kt.dcMarkCells, kt.scan1 + kt.scan2,
           kt.mcGenerateTriangles + kt.dcGenerateQuads);
    cudaFree(verts);
    if (colors) cudaFree(colors);
    if (indices) cudaFree(indices);
    if (uvs) cudaFree(uvs);
    if (primids) cudaFree(primids);
    if (normals) cudaFree(normals);
    return 0;
}
