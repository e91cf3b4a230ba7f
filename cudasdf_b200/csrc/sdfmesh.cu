// libsdfmesh_b200: the C ABI of include/sdfmesh_b200.h for sm_100a.
//
//  * drop-in launchers: the twelve extern "C" entry points of the reference's Wrappers.cu,
//    same names, argument meaning and (legacy default) stream;
//  * sdf_engine_*: a fused pipeline (scout -> compaction -> block field -> block scan -> emission)
//    with no host synchronisation between stages.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <ctime>
#include <new>
#include <mutex>
#include <vector>

#include "../../include/sdfmesh_b200.h"
#include "bvh_host.h"
#include "mc_kernels.cuh"
#include "dc_kernels.cuh"
#include "bvh_device.cuh"
#include "weld.cuh"
#include "surrogate.cuh"
#include "uvpack.cuh"

namespace sdfb {

// ------------------------------------------------------------------------------------------------
// error recording
// ------------------------------------------------------------------------------------------------
static int g_last_error = 0;
static std::mutex g_mutex;

static void record(cudaError_t e) {
    if (e != cudaSuccess && g_last_error == 0) g_last_error = (int)e;
}
static unsigned g_launch_failures = 0;  // launches refused so far (an enqueue compares before / after)
static cudaError_t check_launch() {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        record(e);
        ++g_launch_failures;
    }
    return e;
}

static int num_sms() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

// Static plus dynamic shared memory above 48 KB per block needs the kernel's opt-in.
template <class K>
static void opt_in_smem(K kernel, size_t dyn_smem) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kernel) == cudaSuccess && fa.sharedSizeBytes + dyn_smem > 48 * 1024)
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_smem);
}

template <class K>
static int persistent_grid(K kernel, int threads, int work_items, size_t dyn_smem = 0) {
    int per_sm = 0;
    opt_in_smem(kernel, dyn_smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, dyn_smem);
    if (per_sm < 1) per_sm = 1;
    const int g = num_sms() * per_sm;
    return std::max(1, std::min(g, work_items));
}

static GridView grid_view(const sdf_grid& g) {
    GridView v;
    v.w = (int)g.width;
    v.h = (int)g.height;
    v.d = (int)g.depth;
    v.bx = g.blocksDim[0];
    v.by = g.blocksDim[1];
    v.bz = g.blocksDim[2];
    v.ox = g.origin[0];
    v.oy = g.origin[1];
    v.oz = g.origin[2];
    v.cell = g.cellSize;
    return v;
}

static SceneView scene_view(const sdf_grid& g) {
    SceneView s;
    s.prims = reinterpret_cast<const float4*>(g.d_primitives);
    s.nodes = reinterpret_cast<const float4*>(g.d_bvhNodes);
    s.nprims = (int)g.numPrimitives;
    s.nbvh = (int)std::min(g.numBVHPrimitives, g.numPrimitives);
    s.nnodes = g.d_bvhNodes ? (int)g.numBVHNodes : 0;
    return s;
}

// ------------------------------------------------------------------------------------------------
// device scratch for the drop-in launchers (one set per device, grown on demand). The launchers
// run on the legacy default stream, like the reference's, so one set is enough.
// ------------------------------------------------------------------------------------------------
// What a set of block-field rows was computed for: the grid, the scene, the time and the active list.
struct FieldKey {
    GridView gv;
    SceneView sv;
    float time;
    const int* list;
    const int* count;
    int n;
};
static bool same_key(const FieldKey& a, const FieldKey& b) {
    return a.gv.w == b.gv.w && a.gv.h == b.gv.h && a.gv.d == b.gv.d && a.gv.bx == b.gv.bx && a.gv.by == b.gv.by &&
           a.gv.bz == b.gv.bz && a.gv.ox == b.gv.ox && a.gv.oy == b.gv.oy && a.gv.oz == b.gv.oz &&
           a.gv.cell == b.gv.cell && a.sv.prims == b.sv.prims && a.sv.nodes == b.sv.nodes &&
           a.sv.nprims == b.sv.nprims && a.sv.nbvh == b.sv.nbvh && a.sv.nnodes == b.sv.nnodes && a.time == b.time &&
           a.list == b.list && a.count == b.count && a.n == b.n;
}

struct Scratch {
    int device = -1;
    unsigned* flags = nullptr;
    size_t flags_cap = 0;
    unsigned long long* status = nullptr;  // [0] ticket word, then one status word per scan tile
    size_t status_cap = 0;
    unsigned* tickets = nullptr;           // 8 work tickets
    Diag* diag = nullptr;
    // the shared-halo block field of the counting / marking launchers (k_field_plan / own / miss /
    // gather), kept for the next emission / solve launcher of the same key
    int* b2a = nullptr;
    size_t b2a_cap = 0;
    unsigned* miss = nullptr;
    size_t miss_cap = 0;
    float* rows = nullptr;                 // FIELD_STRIDE floats per active block
    size_t rows_cap = 0;
    bool rows_valid = false;
    FieldKey rows_key{};
};
static Scratch g_scratch[16];

static Scratch& scratch() {
    int dev = 0;
    cudaGetDevice(&dev);
    Scratch& s = g_scratch[dev & 15];
    if (s.device != dev) {
        s.device = dev;
        record(cudaMalloc(&s.tickets, 8 * sizeof(unsigned)));
        record(cudaMalloc(&s.diag, sizeof(Diag)));
        if (s.diag) cudaMemset(s.diag, 0, sizeof(Diag));
    }
    return s;
}

static bool ensure_flags(Scratch& s, size_t n) {
    if (s.flags_cap >= n) return true;
    if (s.flags) cudaFree(s.flags);
    s.flags = nullptr;
    s.flags_cap = 0;
    if (cudaMalloc(&s.flags, n * sizeof(unsigned)) != cudaSuccess) { record(cudaErrorMemoryAllocation); return false; }
    s.flags_cap = n;
    return true;
}
static bool ensure_status(Scratch& s, size_t words) {
    if (s.status_cap >= words) return true;
    if (s.status) cudaFree(s.status);
    s.status = nullptr;
    s.status_cap = 0;
    if (cudaMalloc(&s.status, words * sizeof(unsigned long long)) != cudaSuccess) {
        record(cudaErrorMemoryAllocation);
        return false;
    }
    s.status_cap = words;
    return true;
}

template <class T>
static bool ensure_buffer(T*& p, size_t& cap, size_t n) {
    if (cap >= n) return true;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();  // an allocation that failed leaves no sticky error
        return false;
    }
    cap = n;
    return true;
}

// flags[b] = 1 for every block of the active list (within the grid), the scout's flags for the block
// field's halo ownership
__global__ void k_mark_active(ActiveView av, unsigned* __restrict__ flags, int nblocks) {
    const int n = active_count(av);
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
        const int b = av.list[a];
        if (b >= 0 && b < nblocks) flags[b] = 1u;
    }
}

static FieldKey field_key(const sdf_grid& g, int n, float time) {
    FieldKey k;
    k.gv = grid_view(g);
    k.sv = scene_view(g);
    k.time = time;
    k.list = g.d_activeBlocks;
    k.count = g.d_activeBlockCount;
    k.n = n;
    return k;
}

// The block-field rows of the active list by the engine's shared-halo block field (every sample
// evaluated once: own samples, then the halo samples no active block owns, then the copies), on the
// legacy stream; with packet_counts also the per-cell vertex counts of countActiveBlockTriangles.
// Returns false (nothing launched) when its working memory cannot be allocated; the caller then runs
// the single-kernel field. The rows stay valid for the next launcher with the same key.
static bool dropin_block_field(Scratch& s, const sdf_grid& g, int n, float time, unsigned* packet_counts) {
    const GridView gv = grid_view(g);
    const size_t nblocks = (size_t)gv.bx * gv.by * gv.bz;
    s.rows_valid = false;
    if (!ensure_flags(s, nblocks) || !ensure_buffer(s.b2a, s.b2a_cap, nblocks) ||
        !ensure_buffer(s.miss, s.miss_cap, (size_t)n * HALO_N) ||
        !ensure_buffer(s.rows, s.rows_cap, (size_t)n * FIELD_STRIDE))
        return false;
    const SceneView sv = scene_view(g);
    ActiveView av{g.d_activeBlocks, g.d_activeBlockCount, n};
    record(cudaMemsetAsync(s.flags, 0, nblocks * sizeof(unsigned), 0));
    record(cudaMemsetAsync(s.tickets, 0, 8 * sizeof(unsigned), 0));
    k_mark_active<<<std::max(1, std::min((n + 255) / 256, num_sms() * 8)), 256>>>(av, s.flags, (int)nblocks);
    check_launch();
    // tickets: 0 own samples, 4 listed halo samples, 5 count of listed halo samples
    k_field_plan<<<num_sms() * 8, 256>>>(gv, av, s.flags, s.rows, s.b2a, s.miss, &s.tickets[5]);
    check_launch();
    k_field_own<false><<<persistent_grid(k_field_own<false>, BLK_THREADS, n), BLK_THREADS>>>(gv, sv, time, av, s.rows,
                                                                                          &s.tickets[0], s.diag);
    check_launch();
    k_field_miss<false><<<persistent_grid(k_field_miss<false>, BLK_THREADS, 1 << 30), BLK_THREADS>>>(
        gv, sv, time, av, s.rows, s.miss, &s.tickets[5], &s.tickets[4], s.diag);
    check_launch();
    k_field_gather<<<persistent_grid(k_field_gather, BLK_THREADS, (n + GATHER_WARPS - 1) / GATHER_WARPS), BLK_THREADS>>>(
        gv, av, s.rows, s.b2a, s.flags, nullptr, packet_counts, nullptr);
    check_launch();
    s.rows_valid = true;
    s.rows_key = field_key(g, n, time);
    return true;
}

// the rows of the last dropin_block_field when they were computed for this grid, scene, time and list
static const float* cached_rows(const Scratch& s, const sdf_grid& g, int n, float time) {
    return s.rows_valid && same_key(s.rows_key, field_key(g, n, time)) ? s.rows : nullptr;
}

// ScanState over a caller- or library-owned region: word 0 is the ticket, words 1.. the tiles
static ScanState scan_state(unsigned long long* region) {
    ScanState st;
    st.ticket = reinterpret_cast<unsigned*>(region);
    st.status = region + 1;
    return st;
}

// Returns the first error of its two launches and its memset (each is also recorded).
static cudaError_t run_scout_compact(const GridView& gv, const SceneView& sv, float time, unsigned* flags,
                                     unsigned long long* status, int* list, int* count, Diag* diag,
                                     cudaStream_t stream) {
    const int nblocks = gv.bx * gv.by * gv.bz;
    const int nbricks = scout_pair_bricks(gv);
    const int warps_per_cta = BLK_THREADS / 32;
    k_scout_t<false><<<(nbricks + warps_per_cta - 1) / warps_per_cta, BLK_THREADS, 0, stream>>>(gv, sv, time, flags, diag,
                                                                                          nullptr, 0.f, nullptr);
    cudaError_t err = check_launch();
    const unsigned tiles = scan_tiles((unsigned)nblocks);
    const cudaError_t em = cudaMemsetAsync(status, 0, (tiles + 1) * sizeof(unsigned long long), stream);
    record(em);
    if (err == cudaSuccess) err = em;
    k_compact<<<std::max(1u, tiles), SCAN_THREADS, 0, stream>>>(flags, (unsigned)nblocks, list, count,
                                                                scan_state(status), diag);
    const cudaError_t ec = check_launch();
    return err != cudaSuccess ? err : ec;
}

}  // namespace sdfb

using namespace sdfb;

// ================================================================================================
// Drop-in launchers (Wrappers.cu:19-136)
// ================================================================================================
extern "C" {

void launchScoutActiveBlocks(sdf_grid* grid, float time) {
    std::lock_guard<std::mutex> lk(g_mutex);
    const GridView gv = grid_view(*grid);
    const SceneView sv = scene_view(*grid);
    const size_t nblocks = (size_t)gv.bx * gv.by * gv.bz;
    Scratch& s = scratch();
    s.rows_valid = false;  // the active list is rewritten
    if (!ensure_flags(s, nblocks) || !ensure_status(s, scan_tiles((unsigned)nblocks) + 1)) return;
    run_scout_compact(gv, sv, time, s.flags, s.status, grid->d_activeBlocks, grid->d_activeBlockCount, s.diag, 0);
}

void launchCountActiveBlockTriangles(sdf_grid* grid, int numActiveBlocks, float time) {
    if (numActiveBlocks <= 0) return;
    std::lock_guard<std::mutex> lk(g_mutex);
    Scratch& s = scratch();
    // the shared-halo block field; its rows serve the emission launcher that follows
    if (dropin_block_field(s, *grid, numActiveBlocks, time, grid->d_packetVertexCounts)) return;
    ActiveView av{grid->d_activeBlocks, grid->d_activeBlockCount, numActiveBlocks};
    record(cudaMemsetAsync(s.tickets, 0, sizeof(unsigned), 0));
    k_mc_field<<<persistent_grid(k_mc_field, BLK_THREADS, numActiveBlocks), BLK_THREADS>>>(
        grid_view(*grid), scene_view(*grid), time, av, nullptr, nullptr, grid->d_packetVertexCounts, s.tickets, s.diag);
    check_launch();
}

static unsigned out_mask_of(const sdf_grid& g) {
    unsigned m = 0;
    if (g.d_vertexColors) m |= OUT_COLORS;
    if (g.d_indices) m |= OUT_INDICES;
    if (g.d_uvCoords) m |= OUT_UVS;
    if (g.d_primitiveIDs) m |= OUT_PRIMIDS;
    if (g.d_normals) m |= OUT_NORMALS;
    return m;
}

static MeshOut mesh_out_of(const sdf_grid& g) {
    MeshOut o;
    o.verts = reinterpret_cast<float4*>(g.d_vertices);
    o.colors = reinterpret_cast<float4*>(g.d_vertexColors);
    o.indices = g.d_indices;
    o.uvs = reinterpret_cast<float2*>(g.d_uvCoords);
    o.primids = g.d_primitiveIDs;
    o.normals = reinterpret_cast<float4*>(g.d_normals);
    o.maxV = g.maxVertices;
    return o;
}

void launchGenerateActiveBlockTriangles(sdf_grid* grid, int numActiveBlocks, float time) {
    if (numActiveBlocks <= 0) return;
    std::lock_guard<std::mutex> lk(g_mutex);
    Scratch& s = scratch();
    ActiveView av{grid->d_activeBlocks, grid->d_activeBlockCount, numActiveBlocks};
    record(cudaMemsetAsync(s.tickets, 0, sizeof(unsigned), 0));
    // the rows of the counting launcher when it ran for this grid, scene, time and list (the reference's
    // Update calls count, scan, emission in a row); otherwise the kernel evaluates each block's field
    const float* rows = cached_rows(s, *grid, numActiveBlocks, time);
    k_mc_emit<<<persistent_grid(k_mc_emit, BLK_THREADS, numActiveBlocks), BLK_THREADS>>>(
        grid_view(*grid), scene_view(*grid), time, av, rows, nullptr, grid->d_packetVertexOffsets, nullptr,
        mesh_out_of(*grid), out_mask_of(*grid), s.tickets, s.diag);
    check_launch();
}

void getScanStorageSize(unsigned int num_items, size_t* temp_storage_bytes) {
    *temp_storage_bytes = ((size_t)scan_tiles(num_items) + 1) * sizeof(unsigned long long);
}

void launchScan(unsigned int* d_input, unsigned int* d_output, unsigned int numItems, void* d_temp_storage,
                size_t temp_storage_bytes) {
    if (numItems == 0) return;
    std::lock_guard<std::mutex> lk(g_mutex);
    size_t need = 0;
    getScanStorageSize(numItems, &need);
    if (!d_temp_storage || temp_storage_bytes < need) {
        record(cudaErrorInvalidValue);
        return;
    }
    Scratch& s = scratch();
    unsigned long long* region = static_cast<unsigned long long*>(d_temp_storage);
    record(cudaMemsetAsync(region, 0, need, 0));
    const unsigned tiles = scan_tiles(numItems);
    k_exclusive_scan<<<tiles, SCAN_THREADS>>>(d_input, d_output, numItems, nullptr, 1, scan_state(region), nullptr,
                                              s.diag);
    check_launch();
}

// ------------------------------------------------------------------------------------------------
// dual contouring launchers
// ------------------------------------------------------------------------------------------------
static DcBuffers dc_buffers_of(const sdf_grid& g) {
    DcBuffers b;
    b.block_to_active = g.d_blockToActiveId;
    b.masks = g.d_dcCornerMasks;
    b.vert_offsets = g.d_dcCellVertexOffsets;
    b.cell_verts = reinterpret_cast<ushort4*>(g.d_dcCellVertices);
    b.cell_normals = reinterpret_cast<short4*>(g.d_dcCellNormals);
    b.cell_normals_tmp = reinterpret_cast<short4*>(g.d_dcCellNormalsTmp);
    b.counts = g.d_packetVertexCounts;
    b.offsets = g.d_packetVertexOffsets;
    b.qef_debug = nullptr;
    b.proj = nullptr;
    b.proj_nsum = nullptr;
    b.proj_cap = 0;
    b.hbase = nullptr;
    b.hsample_rep = nullptr;
    b.hnormals = nullptr;
    b.qnormals = nullptr;
    b.qcap = 0;
    return b;
}

void launchBuildBlockToActiveMap(sdf_grid* grid, int numActiveBlocks) {
    if (numActiveBlocks <= 0) return;
    std::lock_guard<std::mutex> lk(g_mutex);
    k_dc_block_map<<<(numActiveBlocks + 255) / 256, 256>>>(grid->d_activeBlocks, grid->d_activeBlockCount,
                                                           numActiveBlocks, grid->maxBlocks, grid->d_blockToActiveId);
    check_launch();
}

void launchDCMarkCells(sdf_grid* grid, int numActiveBlocks, float time) {
    if (numActiveBlocks <= 0) return;
    std::lock_guard<std::mutex> lk(g_mutex);
    Scratch& s = scratch();
    ActiveView av{grid->d_activeBlocks, grid->d_activeBlockCount, numActiveBlocks};
    // the shared-halo block field, then the cells classified from the finished rows (kept for the solve)
    const bool rows = dropin_block_field(s, *grid, numActiveBlocks, time, nullptr);
    record(cudaMemsetAsync(s.tickets, 0, sizeof(unsigned), 0));
    k_dc_mark<<<persistent_grid(k_dc_mark, BLK_THREADS, numActiveBlocks), BLK_THREADS>>>(
        grid_view(*grid), scene_view(*grid), time, av, rows ? s.rows : nullptr, dc_buffers_of(*grid), s.tickets,
        s.diag, rows);
    check_launch();
}

void launchDCSolveCellVertices(sdf_grid* grid, int numActiveBlocks, float time, unsigned int maxCellVertices,
                               float qefBlend) {
    if (numActiveBlocks <= 0) return;
    std::lock_guard<std::mutex> lk(g_mutex);
    Scratch& s = scratch();
    ActiveView av{grid->d_activeBlocks, grid->d_activeBlockCount, numActiveBlocks};
    record(cudaMemsetAsync(s.tickets, 0, sizeof(unsigned), 0));
    DcSolveParams sp;
    sp.max_cell_vertices = maxCellVertices;
    sp.qef_blend = qefBlend;
    sp.solver = SDF_DC_SOLVER_REFERENCE;
    sp.projection_iters = 0;
    sp.cond_threshold = 1e4f;
    const size_t smem = sizeof(SolveSmem);
    const float* rows = cached_rows(s, *grid, numActiveBlocks, time);  // the marking launcher's rows
    k_dc_solve<<<persistent_grid(k_dc_solve, SOLVE_THREADS, numActiveBlocks, smem), SOLVE_THREADS, smem>>>(
        grid_view(*grid), scene_view(*grid), time, av, rows, dc_buffers_of(*grid), sp, s.tickets, s.diag);
    check_launch();
}

void launchDCRecomputeNormalsAtVertices(sdf_grid* grid, int numActiveBlocks, float time) {
    if (numActiveBlocks <= 0 || !grid->d_dcCellNormals) return;
    std::lock_guard<std::mutex> lk(g_mutex);
    Scratch& s = scratch();
    ActiveView av{grid->d_activeBlocks, grid->d_activeBlockCount, numActiveBlocks};
    record(cudaMemsetAsync(s.tickets, 0, sizeof(unsigned), 0));
    k_dc_recompute_normals<<<persistent_grid(k_dc_recompute_normals, BLK_THREADS, numActiveBlocks), BLK_THREADS>>>(
        grid_view(*grid), scene_view(*grid), time, av, dc_buffers_of(*grid), grid->maxVertices, s.tickets, s.diag);
    check_launch();
}

void launchDCSmoothCellNormals(sdf_grid* grid, int numActiveBlocks, float cosAngleThreshold) {
    if (numActiveBlocks <= 0 || !grid->d_dcCellNormals || !grid->d_dcCellNormalsTmp) return;
    std::lock_guard<std::mutex> lk(g_mutex);
    k_dc_smooth_normals<<<numActiveBlocks, 512>>>(grid_view(*grid), ActiveView{grid->d_activeBlocks,
                                                  grid->d_activeBlockCount, numActiveBlocks},
                                                  dc_buffers_of(*grid), grid->maxVertices, cosAngleThreshold);
    check_launch();
}

void launchDCCountQuads(sdf_grid* grid, int numActiveBlocks) {
    if (numActiveBlocks <= 0) return;
    std::lock_guard<std::mutex> lk(g_mutex);
    k_dc_count_quads<<<numActiveBlocks, 512>>>(grid_view(*grid), ActiveView{grid->d_activeBlocks,
                                               grid->d_activeBlockCount, numActiveBlocks}, dc_buffers_of(*grid),
                                               grid->d_packetVertexCounts, nullptr);
    check_launch();
}

void launchDCGenerateQuads(sdf_grid* grid, int numActiveBlocks, float time) {
    if (numActiveBlocks <= 0) return;
    std::lock_guard<std::mutex> lk(g_mutex);
    Scratch& s = scratch();
    ActiveView av{grid->d_activeBlocks, grid->d_activeBlockCount, numActiveBlocks};
    record(cudaMemsetAsync(s.tickets, 0, sizeof(unsigned), 0));
    DcQuadParams qp;
    qp.adaptive_diagonal = 0;
    const size_t smem = sizeof(QuadSmem);
    k_dc_quads<<<persistent_grid(k_dc_quads, BLK_THREADS, numActiveBlocks, smem), BLK_THREADS, smem>>>(
        grid_view(*grid), scene_view(*grid), time, av, dc_buffers_of(*grid), grid->d_packetVertexOffsets,
        grid->d_packetVertexCounts, nullptr, mesh_out_of(*grid), out_mask_of(*grid), qp, s.tickets, s.diag, nullptr,
        nullptr);
    check_launch();
}

int sdf_last_error(void) {
    std::lock_guard<std::mutex> lk(g_mutex);
    const int e = g_last_error;
    g_last_error = 0;
    return e;
}

const char* sdf_version(void) { return "sdfmesh_b200 0.1 (sm_100a)"; }

}  // extern "C"

#include "engine.inl"
#include "surrogate.inl"
#include "batch.inl"
#include "noalloc.inl"
#include "obj_export.inl"
#include "uvpack.inl"
