// Headless driver for the reference CUDA path (test infrastructure only).
//
// Drives the reference's own extern "C" launchers (Wrappers.cu:19-136) in the stage order of
// CudaSDFMesh::Update (CudaSDFMesh.cpp:281-470), with the reference's own host BVH builder
// (CudaSDFUtil.h:501-613, included from the reference tree). It differs from the reference's
// orchestrator only where a headless, comparable run needs it:
//   * output buffers are plain cudaMalloc allocations instead of mapped GL buffers
//     (main.cpp:1324-1372);
//   * the 200000 active-block cap and the 50M vertex cap (CudaSDFMesh.cpp:159,187,352) are
//     parameters, so large grids are not truncated;
//   * after the scout, the active-block list can be sorted by linear block index
//     (the reference appends with atomicAdd, MarchingCubesKernels.cu:883-887, so its order
//     follows the warp schedule); sorting gives one canonical legal order;
//   * cudaGetLastError()/cudaDeviceSynchronize() are checked after every stage
//     (the reference's wrappers only printf, Wrappers.cu:26-29).
#include "CudaSDFUtil.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

extern "C" void launchScoutActiveBlocks(SDFGrid& grid, float time);
extern "C" void launchCountActiveBlockTriangles(SDFGrid& grid, int numActiveBlocks, float time);
extern "C" void launchGenerateActiveBlockTriangles(SDFGrid& grid, int numActiveBlocks, float time);
extern "C" void launchBuildBlockToActiveMap(SDFGrid& grid, int numActiveBlocks);
extern "C" void launchDCMarkCells(SDFGrid& grid, int numActiveBlocks, float time);
extern "C" void launchDCSolveCellVertices(SDFGrid& grid, int numActiveBlocks, float time, unsigned int maxCellVertices, float qefBlend);
extern "C" void launchDCRecomputeNormalsAtVertices(SDFGrid& grid, int numActiveBlocks, float time);
extern "C" void launchDCSmoothCellNormals(SDFGrid& grid, int numActiveBlocks, float cosAngleThreshold);
extern "C" void launchDCCountQuads(SDFGrid& grid, int numActiveBlocks);
extern "C" void launchDCGenerateQuads(SDFGrid& grid, int numActiveBlocks, float time);
extern "C" void getScanStorageSize(unsigned int num_items, size_t* temp_storage_bytes);
extern "C" void launchScan(unsigned int* d_input, unsigned int* d_output, unsigned int numItems, void* d_temp_storage, size_t temp_storage_bytes);

struct RefStats {
    int scoutCount;       // *d_activeBlockCount after the scout
    int activeUsed;       // blocks processed after the cap
    unsigned totalVertices;
    int error;            // first CUDA error seen (cudaError_t), 0 if none
    float msScout, msCount, msScan1, msGenerate;          // MC stages
    float msBlockMap, msMark, msSolve, msCountQuads, msScan2, msQuads;  // DC stages
    float msTotalKernels; // sum of stage event times
    float msWall;         // host wall time of the whole Update-equivalent incl. syncs and readbacks
};

namespace {

enum OutMask { OUT_COLORS = 1, OUT_INDICES = 2, OUT_UVS = 4, OUT_PRIMIDS = 8, OUT_NORMALS = 16 };

struct RefMesh {
    SDFGrid g;
    int packedBlocks = 0;
    void* scanTemp = nullptr;
    size_t scanTempBytes = 0;
    std::vector<SDFPrimitive> prims;
    std::vector<BVHNode> nodes;
    unsigned numBVHPrims = 0;
    unsigned mask = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int err = 0;
};

int check(RefMesh* m) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess && m->err == 0) m->err = (int)e;
    return (int)e;
}

float timeStage(RefMesh* m) {
    float ms = 0.f;
    cudaEventSynchronize(m->e1);
    cudaEventElapsedTime(&ms, m->e0, m->e1);
    check(m);
    return ms;
}

template <class T>
void ensure(T*& p, size_t count) {
    if (!p) cudaMalloc((void**)&p, count * sizeof(T));
}

}  // namespace

extern "C" {

// Mirrors CudaSDFMesh::Initialize (CudaSDFMesh.cpp:90-206) with the two caps as parameters.
void* ref_create(float cellSize, const float* bmin, const float* bmax, int maxActiveBlocks, unsigned maxVertices) {
    RefMesh* m = new RefMesh();
    memset(&m->g, 0, sizeof(SDFGrid));
    SDFGrid& g = m->g;
    g.cellSize = cellSize;
    g.origin = make_float3(bmin[0], bmin[1], bmin[2]);
    float3 size = make_float3(bmax[0] - bmin[0], bmax[1] - bmin[1], bmax[2] - bmin[2]);
    g.width = (unsigned int)ceilf(size.x / cellSize);
    g.height = (unsigned int)ceilf(size.y / cellSize);
    g.depth = (unsigned int)ceilf(size.z / cellSize);
    const int bs = SDF_BLOCK_SIZE;
    g.blocksDim = make_int3((g.width + bs - 1) / bs, (g.height + bs - 1) / bs, (g.depth + bs - 1) / bs);
    g.maxBlocks = g.blocksDim.x * g.blocksDim.y * g.blocksDim.z;
    m->packedBlocks = std::min(g.maxBlocks, maxActiveBlocks > 0 ? maxActiveBlocks : g.maxBlocks);
    const size_t packed = (size_t)m->packedBlocks * SDF_BLOCK_SIZE_CUBED;
    cudaMalloc(&g.d_activeBlocks, (size_t)g.maxBlocks * sizeof(int));
    cudaMalloc(&g.d_activeBlockCount, sizeof(int));
    cudaMalloc(&g.d_packetVertexCounts, packed * sizeof(unsigned));
    cudaMalloc(&g.d_packetVertexOffsets, packed * sizeof(unsigned));
    getScanStorageSize((unsigned)packed, &m->scanTempBytes);
    cudaMalloc(&m->scanTemp, m->scanTempBytes);
    cudaMalloc(&g.d_totalVertices, sizeof(unsigned));
    cudaMalloc(&g.d_totalIndices, sizeof(unsigned));
    g.maxVertices = maxVertices ? maxVertices : 50000000u;
    g.maxIndices = g.maxVertices * 3;
    cudaEventCreate(&m->e0);
    cudaEventCreate(&m->e1);
    check(m);
    return m;
}

void ref_destroy(void* h) {
    RefMesh* m = (RefMesh*)h;
    if (!m) return;
    SDFGrid& g = m->g;
    void* ptrs[] = {g.d_activeBlocks, g.d_activeBlockCount, g.d_packetVertexCounts, g.d_packetVertexOffsets,
                    g.d_blockToActiveId, g.d_dcCornerMasks, g.d_dcCellVertexOffsets, g.d_dcCellVertices,
                    g.d_dcCellNormals, g.d_dcCellNormalsTmp, g.d_primitives, g.d_bvhNodes, g.d_vertices,
                    g.d_vertexColors, g.d_indices, g.d_uvCoords, g.d_primitiveIDs, g.d_normals,
                    g.d_totalVertices, g.d_totalIndices, m->scanTemp};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    cudaEventDestroy(m->e0);
    cudaEventDestroy(m->e1);
    delete m;
}

// Mirrors CudaSDFMesh::UpdateBVH (CudaSDFMesh.cpp:216-249) and the uploads of Update (:293-321):
// union / union-blend primitives first, then the rest; BVH over the unions only.
int ref_set_primitives(void* h, const SDFPrimitive* prims, int n) {
    RefMesh* m = (RefMesh*)h;
    std::vector<int> unionIdx, otherIdx;
    for (int i = 0; i < n; ++i) {
        if (prims[i].operation == SDF_UNION || prims[i].operation == SDF_UNION_BLEND) unionIdx.push_back(i);
        else otherIdx.push_back(i);
    }
    m->prims.clear();
    for (int i : unionIdx) m->prims.push_back(prims[i]);
    for (int i : otherIdx) m->prims.push_back(prims[i]);
    m->nodes.clear();
    if (!unionIdx.empty()) {
        std::vector<int> idx(unionIdx.size());
        for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
        buildBVHRecursive(idx.data(), (int)idx.size(), m->prims, m->nodes);
    }
    m->numBVHPrims = (unsigned)unionIdx.size();
    SDFGrid& g = m->g;
    if (g.d_primitives) cudaFree(g.d_primitives);
    if (g.d_bvhNodes) cudaFree(g.d_bvhNodes);
    g.d_primitives = nullptr;
    g.d_bvhNodes = nullptr;
    cudaMalloc(&g.d_primitives, std::max<size_t>(m->prims.size() * sizeof(SDFPrimitive), 1024));
    cudaMalloc(&g.d_bvhNodes, std::max<size_t>(m->nodes.size() * sizeof(BVHNode), 1024));
    if (!m->prims.empty())
        cudaMemcpy(g.d_primitives, m->prims.data(), m->prims.size() * sizeof(SDFPrimitive), cudaMemcpyHostToDevice);
    if (!m->nodes.empty())
        cudaMemcpy(g.d_bvhNodes, m->nodes.data(), m->nodes.size() * sizeof(BVHNode), cudaMemcpyHostToDevice);
    g.numPrimitives = (unsigned)m->prims.size();
    g.numBVHPrimitives = m->numBVHPrims;
    g.numBVHNodes = (unsigned)m->nodes.size();
    check(m);
    return (int)m->numBVHPrims;
}

int ref_num_nodes(void* h) { return (int)((RefMesh*)h)->nodes.size(); }
void ref_get_nodes(void* h, BVHNode* out) {
    RefMesh* m = (RefMesh*)h;
    if (!m->nodes.empty()) memcpy(out, m->nodes.data(), m->nodes.size() * sizeof(BVHNode));
}
void ref_get_primitives(void* h, SDFPrimitive* out) {
    RefMesh* m = (RefMesh*)h;
    if (!m->prims.empty()) memcpy(out, m->prims.data(), m->prims.size() * sizeof(SDFPrimitive));
}
void ref_get_grid(void* h, SDFGrid* out) { *out = ((RefMesh*)h)->g; }

// Mirrors CudaSDFMesh::Update (CudaSDFMesh.cpp:281-470). technique 0 = marching cubes,
// 1 = dual contouring. outMask selects the optional output streams (vertices are always written).
int ref_run(void* h, float time, int technique, float qefBlend, unsigned outMask, int sortActive, RefStats* st) {
    RefMesh* m = (RefMesh*)h;
    SDFGrid& g = m->g;
    memset(st, 0, sizeof(RefStats));
    m->err = 0;
    const size_t maxV = g.maxVertices;
    ensure(g.d_vertices, maxV);
    if (outMask & OUT_COLORS) ensure(g.d_vertexColors, maxV);
    if (outMask & OUT_INDICES) ensure(g.d_indices, maxV);
    if (outMask & OUT_UVS) ensure(g.d_uvCoords, maxV);
    if (outMask & OUT_PRIMIDS) ensure(g.d_primitiveIDs, maxV);
    if (outMask & OUT_NORMALS) ensure(g.d_normals, maxV);
    // Streams not requested are passed as nullptr, as main.cpp does for indices (main.cpp:1352).
    SDFGrid run = g;
    if (!(outMask & OUT_COLORS)) run.d_vertexColors = nullptr;
    if (!(outMask & OUT_INDICES)) run.d_indices = nullptr;
    if (!(outMask & OUT_UVS)) run.d_uvCoords = nullptr;
    if (!(outMask & OUT_PRIMIDS)) run.d_primitiveIDs = nullptr;
    if (!(outMask & OUT_NORMALS)) run.d_normals = nullptr;
    check(m);

    auto w0 = std::chrono::high_resolution_clock::now();
    cudaMemset(run.d_activeBlockCount, 0, sizeof(int));
    cudaEventRecord(m->e0);
    launchScoutActiveBlocks(run, time);
    cudaEventRecord(m->e1);
    st->msScout = timeStage(m);
    int nActive = 0;
    cudaMemcpy(&nActive, run.d_activeBlockCount, sizeof(int), cudaMemcpyDeviceToHost);
    st->scoutCount = nActive;
    if (nActive > m->packedBlocks) nActive = m->packedBlocks;
    st->activeUsed = nActive;
    if (nActive <= 0) {
        auto w1 = std::chrono::high_resolution_clock::now();
        st->msWall = std::chrono::duration<float, std::milli>(w1 - w0).count();
        st->error = m->err;
        return m->err;
    }
    if (sortActive) {
        std::vector<int> ab(nActive);
        cudaMemcpy(ab.data(), run.d_activeBlocks, nActive * sizeof(int), cudaMemcpyDeviceToHost);
        std::sort(ab.begin(), ab.end());
        cudaMemcpy(run.d_activeBlocks, ab.data(), nActive * sizeof(int), cudaMemcpyHostToDevice);
        if (nActive != st->scoutCount) {
            // Keep the device-side count consistent with the truncated list.
            cudaMemcpy(run.d_activeBlockCount, &nActive, sizeof(int), cudaMemcpyHostToDevice);
        }
    }
    const unsigned totalItems = (unsigned)nActive * SDF_BLOCK_SIZE_CUBED;
    if (technique == 0) {
        cudaEventRecord(m->e0);
        launchCountActiveBlockTriangles(run, nActive, time);
        cudaEventRecord(m->e1);
        st->msCount = timeStage(m);
        cudaEventRecord(m->e0);
        launchScan(run.d_packetVertexCounts, run.d_packetVertexOffsets, totalItems, m->scanTemp, m->scanTempBytes);
        cudaEventRecord(m->e1);
        st->msScan1 = timeStage(m);
        cudaEventRecord(m->e0);
        launchGenerateActiveBlockTriangles(run, nActive, time);
        cudaEventRecord(m->e1);
        st->msGenerate = timeStage(m);
    } else {
        ensure(g.d_blockToActiveId, (size_t)g.maxBlocks);
        ensure(g.d_dcCornerMasks, (size_t)m->packedBlocks * SDF_BLOCK_SIZE_CUBED);
        ensure(g.d_dcCellVertexOffsets, (size_t)m->packedBlocks * SDF_BLOCK_SIZE_CUBED);
        ensure(g.d_dcCellVertices, maxV);
        ensure(g.d_dcCellNormals, maxV);
        ensure(g.d_dcCellNormalsTmp, maxV);
        run.d_blockToActiveId = g.d_blockToActiveId;
        run.d_dcCornerMasks = g.d_dcCornerMasks;
        run.d_dcCellVertexOffsets = g.d_dcCellVertexOffsets;
        run.d_dcCellVertices = g.d_dcCellVertices;
        run.d_dcCellNormals = g.d_dcCellNormals;
        run.d_dcCellNormalsTmp = g.d_dcCellNormalsTmp;
        cudaMemset(run.d_blockToActiveId, 0xFF, (size_t)g.maxBlocks * sizeof(int));
        cudaEventRecord(m->e0);
        launchBuildBlockToActiveMap(run, nActive);
        cudaEventRecord(m->e1);
        st->msBlockMap = timeStage(m);
        cudaEventRecord(m->e0);
        launchDCMarkCells(run, nActive, time);
        cudaEventRecord(m->e1);
        st->msMark = timeStage(m);
        cudaEventRecord(m->e0);
        launchScan(run.d_packetVertexCounts, run.d_dcCellVertexOffsets, totalItems, m->scanTemp, m->scanTempBytes);
        cudaEventRecord(m->e1);
        st->msScan1 = timeStage(m);
        cudaEventRecord(m->e0);
        launchDCSolveCellVertices(run, nActive, time, g.maxVertices, qefBlend);
        cudaEventRecord(m->e1);
        st->msSolve = timeStage(m);
        cudaEventRecord(m->e0);
        launchDCCountQuads(run, nActive);
        cudaEventRecord(m->e1);
        st->msCountQuads = timeStage(m);
        cudaEventRecord(m->e0);
        launchScan(run.d_packetVertexCounts, run.d_packetVertexOffsets, totalItems, m->scanTemp, m->scanTempBytes);
        cudaEventRecord(m->e1);
        st->msScan2 = timeStage(m);
        cudaEventRecord(m->e0);
        launchDCGenerateQuads(run, nActive, time);
        cudaEventRecord(m->e1);
        st->msQuads = timeStage(m);
    }
    unsigned lastOffset = 0, lastCount = 0;
    cudaMemcpy(&lastOffset, &run.d_packetVertexOffsets[totalItems - 1], sizeof(unsigned), cudaMemcpyDeviceToHost);
    cudaMemcpy(&lastCount, &run.d_packetVertexCounts[totalItems - 1], sizeof(unsigned), cudaMemcpyDeviceToHost);
    st->totalVertices = lastOffset + lastCount;
    auto w1 = std::chrono::high_resolution_clock::now();
    st->msWall = std::chrono::duration<float, std::milli>(w1 - w0).count();
    st->msTotalKernels = st->msScout + st->msCount + st->msScan1 + st->msGenerate + st->msBlockMap + st->msMark +
                         st->msSolve + st->msCountQuads + st->msScan2 + st->msQuads;
    check(m);
    st->error = m->err;
    return m->err;
}

// The DC normal passes that the reference's Update never calls (Wrappers.cu:87-105), exposed so that
// their behaviour can be recorded too. Run after ref_run(technique=1).
int ref_dc_normal_passes(void* h, float time, float cosAngle) {
    RefMesh* m = (RefMesh*)h;
    int n = 0;
    cudaMemcpy(&n, m->g.d_activeBlockCount, sizeof(int), cudaMemcpyDeviceToHost);
    n = std::min(n, m->packedBlocks);
    launchDCRecomputeNormalsAtVertices(m->g, n, time);
    check(m);
    launchDCSmoothCellNormals(m->g, n, cosAngle);
    return check(m);
}

// Buffer ids for ref_copy.
enum RefBuf {
    RB_ACTIVE = 0, RB_COUNTS, RB_OFFSETS, RB_VERTS, RB_COLORS, RB_INDICES, RB_UVS, RB_PRIMIDS, RB_NORMALS,
    RB_DCMASK, RB_DCVOFF, RB_DCVERT, RB_DCNORM, RB_B2A, RB_DCNORMTMP
};

int ref_copy(void* h, int buf, void* dst, size_t bytes) {
    RefMesh* m = (RefMesh*)h;
    const SDFGrid& g = m->g;
    const void* src = nullptr;
    switch (buf) {
        case RB_ACTIVE: src = g.d_activeBlocks; break;
        case RB_COUNTS: src = g.d_packetVertexCounts; break;
        case RB_OFFSETS: src = g.d_packetVertexOffsets; break;
        case RB_VERTS: src = g.d_vertices; break;
        case RB_COLORS: src = g.d_vertexColors; break;
        case RB_INDICES: src = g.d_indices; break;
        case RB_UVS: src = g.d_uvCoords; break;
        case RB_PRIMIDS: src = g.d_primitiveIDs; break;
        case RB_NORMALS: src = g.d_normals; break;
        case RB_DCMASK: src = g.d_dcCornerMasks; break;
        case RB_DCVOFF: src = g.d_dcCellVertexOffsets; break;
        case RB_DCVERT: src = g.d_dcCellVertices; break;
        case RB_DCNORM: src = g.d_dcCellNormals; break;
        case RB_B2A: src = g.d_blockToActiveId; break;
        case RB_DCNORMTMP: src = g.d_dcCellNormalsTmp; break;
        default: return -1;
    }
    if (!src) return -2;
    if (bytes == 0) return 0;
    return (int)cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
}

int ref_stats_size() { return (int)sizeof(RefStats); }
int ref_device_count() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

}  // extern "C"
