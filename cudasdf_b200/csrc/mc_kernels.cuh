// Marching-cubes stages for sm_100a: scout, compaction, block field + count, emission.
//
// Work decomposition. One thread block (CTA) owns one active 8^3 block at a time and evaluates
// the block's 9^3 = 729 corner samples once, into shared memory, with warp-coherent map() calls
// (23 warps' worth of 32 samples). The reference evaluates map() 8 times per cell in the count
// kernel and 8 times again in the emit kernel (MarchingCubesKernels.cu:936-950, 987-1001), i.e.
// 8192 evaluations per active block per pass; here a block costs 729. Every sample value equals
// the reference's value at that grid point bit for bit (same point, same arithmetic), so case
// codes, counts and vertex positions are unchanged.
//
// The CTAs are persistent: each claims active blocks from an atomic ticket until the device-side
// active count is exhausted, so no host read-back is needed between stages.
#pragma once

#include "mc_cases.inc"
#include "bulk.cuh"
#include "scan.cuh"
#include "sdf_device.cuh"
#include "uv.cuh"

namespace sdfb {

constexpr int BLK_THREADS = 256;           // 8 warps per CTA
static_assert(BLK_THREADS <= 32 * MAP_WARPS, "one map_warp stack per warp");
constexpr int FIELD_N = 729;               // 9^3 samples of one block incl. the +1 halo
constexpr int FIELD_STRIDE = 736;          // padded to a multiple of 16 floats (64 B rows)
constexpr int FIELD_CHUNKS = (FIELD_N + 31) / 32;
constexpr int MAX_BLOCK_TRIS = 512 * 5;    // upper bound of triangles in one block

// marching-cubes case table (re-encoded reference table, see gen_mc_cases.py)
__constant__ unsigned long long c_mcCases[256] = {SDF_MC_CASE_WORDS};

// One scene of a batched extraction: its grid, its primitives and BVH, and where its blocks start in
// the batch's global block numbering (scene s owns global blocks [block_base, block_base + blocks)).
struct SceneDesc {
    GridView g;
    SceneView sc;
    unsigned block_base;
    unsigned brick_base;   // first global scout brick (4 x 4 x 4 blocks) of the scene
};

struct ActiveView {
    const int* list;       // active block linear indices, ascending
    const int* count_dev;  // device-side active count
    int cap;               // host-side bound (numActiveBlocks of the drop-in launchers)
    const SceneDesc* scenes = nullptr;  // batched extraction: list entries are global block indices
    int nscenes = 0;
};

// the scene owning global block e (the last scene whose block_base is <= e)
__device__ __forceinline__ int scene_of_block(const SceneDesc* s, int n, unsigned e) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s[mid].block_base <= e) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Active-list entry -> the grid and scene it belongs to, its block index inside that scene and the
// scene's first global block (0 and the kernel's own grid / scene outside a batch).
__device__ __forceinline__ void resolve(const ActiveView& av, int entry, GridView& g, SceneView& sc, int& lin,
                                        unsigned& base) {
    if (!av.scenes) {
        lin = entry;
        base = 0u;
        return;
    }
    const SceneDesc& d = av.scenes[scene_of_block(av.scenes, av.nscenes, (unsigned)entry)];
    g = d.g;
    sc = d.sc;
    base = d.block_base;
    lin = entry - (int)base;
}

struct MeshOut {
    float4* verts;
    float4* colors;
    unsigned* indices;
    float2* uvs;
    int* primids;
    float4* normals;
    unsigned maxV;
};

enum { OUT_COLORS = 1, OUT_INDICES = 2, OUT_UVS = 4, OUT_PRIMIDS = 8, OUT_NORMALS = 16, OUT_WELDED = 32 };

__device__ __forceinline__ int active_count(const ActiveView& av) {
    int n = av.count_dev ? *av.count_dev : av.cap;
    return n < av.cap ? n : av.cap;
}

__device__ __forceinline__ void block_coord(const GridView& g, int lin, int& bx, int& by, int& bz) {
    bx = lin % g.bx;
    const int t = lin / g.bx;
    by = t % g.by;
    bz = t / g.by;
}

// claims the next work item for the whole CTA; returns -1 when done
__device__ __forceinline__ int claim(unsigned* ticket, int n, int* s_item) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const int a = (int)atomicAdd(ticket, 1u);
        *s_item = a < n ? a : -1;
    }
    __syncthreads();
    return *s_item;
}

// The block's 729 samples in Morton order of (x, y, z): the first 512 form sixteen 4 x 4 x 2 bricks of
// 32, the +1 faces come as 8 x 4 slabs. Each warp takes 32 consecutive entries, so its points are
// close together and share more of their BVH walks than a run of 32 in row order (9 x 4 x 1).
struct FieldOrder {
    unsigned short idx[FIELD_N];
};
constexpr FieldOrder make_field_order() {
    FieldOrder o{};
    int n = 0;
    for (unsigned m = 0; m < 4096u; ++m) {
        unsigned x = 0, y = 0, z = 0;
        for (int b = 0; b < 4; ++b) {
            x |= ((m >> (3 * b)) & 1u) << b;
            y |= ((m >> (3 * b + 1)) & 1u) << b;
            z |= ((m >> (3 * b + 2)) & 1u) << b;
        }
        if (x < 9 && y < 9 && z < 9) o.idx[n++] = (unsigned short)((z * 9 + y) * 9 + x);
    }
    return o;
}
__device__ const FieldOrder g_field_order = make_field_order();

// 9^3 samples of block `lin` into s_field (index (z*9 + y)*9 + x); samples outside the grid are 0 and
// never read by an in-bounds cell
template <bool COUNT = false>
__device__ __forceinline__ void eval_block_field(const GridView& g, const SceneView& sc, float time, int lin,
                                                 float* s_field, Diag* diag) {
    int bx, by, bz;
    block_coord(g, lin, bx, by, bz);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int chunk = warp; chunk < FIELD_CHUNKS; chunk += nwarps) {
        const int r = chunk * 32 + lane;
        const int s = r < FIELD_N ? (int)g_field_order.idx[r] : r;
        const int sx = s % 9, sy = (s / 9) % 9, sz = s / 81;
        const int gx = bx * 8 + sx, gy = by * 8 + sy, gz = bz * 8 + sz;
        const bool valid = s < FIELD_N && gx < g.w && gy < g.h && gz < g.d;
        const float3 p = grid_loc(g, gx, gy, gz);
        MapState<false> st;
        map_warp<false, COUNT>(sc, p, valid, time, st, diag);
        if (s < FIELD_N) s_field[s] = valid ? st.d : 0.f;
    }
}

__device__ __forceinline__ int fidx(int x, int y, int z) { return (z * 9 + y) * 9 + x; }

// case code and corner values of the cell at local (lx, ly, lz)
__device__ __forceinline__ int cell_case(const float* f, int lx, int ly, int lz, float cv[8]) {
    int code = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        cv[i] = f[fidx(lx + corner_dx(i), ly + corner_dy(i), lz + corner_dz(i))];
        if (cv[i] > 0.f) code |= 1 << i;
    }
    return code;
}

// interpEdgePoint (MarchingCubesKernels.cu:60-81)
__device__ __forceinline__ float3 edge_point(const GridView& g, int x, int y, int z, const float cv[8], int e) {
    const int c1 = edge_c0(e), c2 = edge_c1(e);
    const float t = edge_t(cv[c1], cv[c2]);
    const float3 p1 = grid_loc(g, x + corner_dx(c1), y + corner_dy(c1), z + corner_dz(c1));
    const float3 p2 = grid_loc(g, x + corner_dx(c2), y + corner_dy(c2), z + corner_dz(c2));
    return lerp3(p1, p2, t);
}

__device__ __forceinline__ void tri_points(const GridView& g, int x, int y, int z, const float cv[8],
                                           unsigned long long word, int k, float3 v[3]) {
#pragma unroll
    for (int j = 0; j < 3; ++j) v[j] = edge_point(g, x, y, z, cv, (int)((word >> (4 + 4 * (3 * k + j))) & 0xF));
}

// bit k set iff triangle k of the case is non-degenerate (countActiveBlockTriangles, :952-967)
__device__ __forceinline__ unsigned cell_valid_mask(const GridView& g, int x, int y, int z, const float cv[8],
                                                    unsigned long long word) {
    const int nt = (int)(word & 0xF);
    unsigned m = 0;
    for (int k = 0; k < nt; ++k) {
        float3 v[3];
        tri_points(g, x, y, z, cv, word, k, v);
        if (!degenerate(v[0], v[1], v[2], g.cell)) m |= 1u << k;
    }
    return m;
}

struct CellInfo {
    int x, y, z, lx, ly, lz;
    bool oob;
};

__device__ __forceinline__ CellInfo cell_info(const GridView& g, int bx, int by, int bz, int tid) {
    CellInfo c;
    c.lz = tid >> 6;
    c.ly = (tid >> 3) & 7;
    c.lx = tid & 7;
    c.x = bx * 8 + c.lx;
    c.y = by * 8 + c.ly;
    c.z = bz * 8 + c.lz;
    c.oob = c.x >= g.w - 1 || c.y >= g.h - 1 || c.z >= g.d - 1;  // outOfBounds (Commons.cuh:204-207)
    return c;
}

// ------------------------------------------------------------------------------------------------
// scout (MarchingCubesKernels.cu:850-889). Warps take bricks of blocks (4x4x4 with two centres per
// lane, or 4x4x2 with one) so the block centres of a warp are spatially close and their BVH walks
// coincide; the result is a 0/1 flag per linear block index, compacted in index order afterwards.
// ------------------------------------------------------------------------------------------------
// scoutActiveBlocks (MarchingCubesKernels.cu:850-889) for one brick of 4 x 4 x 2 blocks: one warp,
// one lane per block centre
__device__ __forceinline__ void scout_brick(const GridView& g, const SceneView& sc, float time, int wx, int wy, int wz,
                                            unsigned* flags, Diag* diag) {
    const int lane = threadIdx.x & 31;
    const int bx = wx * 4 + (lane & 3), by = wy * 4 + ((lane >> 2) & 3), bz = wz * 2 + (lane >> 4);
    const bool valid = bx < g.bx && by < g.by && bz < g.bz;
    const float3 c = f3(FMA(ADD((float)(bx * 8), 4.f), g.cell, g.ox), FMA(ADD((float)(by * 8), 4.f), g.cell, g.oy),
                        FMA(ADD((float)(bz * 8), 4.f), g.cell, g.oz));
    MapState<false> st;
    map_warp<false>(sc, c, valid, time, st, diag);
    const float r = MUL(8 * 0.5f * 1.73205f + 2.0f, g.cell);
    if (valid) flags[bx + g.bx * (by + g.by * bz)] = fabsf(st.d) <= r ? 1u : 0u;
}

// scoutActiveBlocks for one brick of 4 x 4 x 4 blocks: one warp, two z-neighbouring block centres per
// lane walked together (map_warp2)
__device__ __forceinline__ void scout_brick_pairs(const GridView& g, const SceneView& sc, float time, int wx, int wy,
                                                  int wz, unsigned* flags, Diag* diag) {
    const int lane = threadIdx.x & 31;
    const int bx = wx * 4 + (lane & 3), by = wy * 4 + ((lane >> 2) & 3), bz0 = wz * 4 + 2 * (lane >> 4), bz1 = bz0 + 1;
    const bool v0 = bx < g.bx && by < g.by && bz0 < g.bz, v1 = bx < g.bx && by < g.by && bz1 < g.bz;
    const float3 c0 = f3(FMA(ADD((float)(bx * 8), 4.f), g.cell, g.ox), FMA(ADD((float)(by * 8), 4.f), g.cell, g.oy),
                         FMA(ADD((float)(bz0 * 8), 4.f), g.cell, g.oz));
    const float z1 = FMA(ADD((float)(bz1 * 8), 4.f), g.cell, g.oz);
    float d0, d1;
    map_warp2<false>(sc, c0, z1, v0, v1, time, d0, d1, diag);
    const float r = MUL(8 * 0.5f * 1.73205f + 2.0f, g.cell);
    if (v0) flags[bx + g.bx * (by + g.by * bz0)] = fabsf(d0) <= r ? 1u : 0u;
    if (v1) flags[bx + g.bx * (by + g.by * bz1)] = fabsf(d1) <= r ? 1u : 0u;
}

// scout bricks of a grid: 4 x 4 x 4 blocks each for the plain scout (two centres per lane), 4 x 4 x 2
// for the culled one (one centre per lane)
__host__ __device__ __forceinline__ int scout_pair_bricks(const GridView& g) {
    return ((g.bx + 3) >> 2) * ((g.by + 3) >> 2) * ((g.bz + 3) >> 2);
}
__host__ __device__ __forceinline__ int scout_single_bricks(const GridView& g) {
    return ((g.bx + 3) >> 2) * ((g.by + 3) >> 2) * ((g.bz + 1) >> 1);
}

// CULL: the brick lies in coarse block (wx, wy, wz / 2) of 4 x 4 x 4 blocks (32^3 cells); when the
// surrogate's value at that coarse block's centre exceeds `margin` in magnitude, the brick's blocks
// are marked inactive without evaluating the scene. The culled scout is a persistent grid whose warps
// claim one brick at a time (ticket): a culled brick only writes its zero flags, so the resident warps
// keep walking kept bricks instead of idling in CTAs whose other warps were culled; it keeps one centre
// per lane, since its few kept bricks are about one wave of warps, which pairs would halve while
// lengthening each. The plain scout is one warp per 4 x 4 x 4 brick, two centres per lane.
template <bool CULL>
__global__ void __launch_bounds__(BLK_THREADS) k_scout_t(GridView g, SceneView sc, float time, unsigned* flags,
                                                         Diag* diag, const float* __restrict__ coarse_f,
                                                         float margin, unsigned* ticket) {
    const int lane = threadIdx.x & 31;
    const int nbx = (g.bx + 3) >> 2, nby = (g.by + 3) >> 2;
    if (!CULL) {
        const int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
        if (w >= scout_pair_bricks(g)) return;
        const int wx = w % nbx, t = w / nbx, wy = t % nby, wz = t / nby;
        scout_brick_pairs(g, sc, time, wx, wy, wz, flags, diag);
        return;
    }
    const int nbricks = scout_single_bricks(g);
    for (;;) {
        int w = 0;
        if (lane == 0) w = (int)atomicAdd(ticket, 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        if (w >= nbricks) break;
        const int wx = w % nbx, t = w / nbx, wy = t % nby, wz = t / nby;
        const int bx = wx * 4 + (lane & 3), by = wy * 4 + ((lane >> 2) & 3), bz = wz * 2 + (lane >> 4);
        const bool valid = bx < g.bx && by < g.by && bz < g.bz;
        const float fc = coarse_f[wx + nbx * (wy + nby * (wz >> 1))];
        if (fabsf(fc) > margin) {
            if (valid) flags[bx + g.bx * (by + g.by * bz)] = 0u;
            continue;
        }
        const unsigned v = __ballot_sync(0xffffffffu, valid);
        if (lane == 0) atomicAdd(&diag->scouted, (unsigned long long)__popc(v));
        scout_brick(g, sc, time, wx, wy, wz, flags, diag);
    }
}

// the scout of every scene of a batch in one launch: global brick -> scene -> brick of that scene;
// flags are in the batch's global block numbering
__global__ void __launch_bounds__(BLK_THREADS) k_scout_batch(const SceneDesc* __restrict__ scenes, int nscenes,
                                                             unsigned total_bricks, float time, unsigned* flags,
                                                             Diag* diag) {
    const unsigned w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= total_bricks) return;
    int lo = 0, hi = nscenes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (scenes[mid].brick_base <= w) lo = mid; else hi = mid - 1;
    }
    const SceneDesc& d = scenes[lo];
    const GridView g = d.g;
    const int local = (int)(w - d.brick_base);
    const int nbx = (g.bx + 3) >> 2, nby = (g.by + 3) >> 2;
    const int wx = local % nbx, t = local / nbx, wy = t % nby, wz = t / nby;
    scout_brick_pairs(g, d.sc, time, wx, wy, wz, flags + d.block_base, diag);
}

// first output vertex of every scene of a batch: the offset of its first active block (the active
// list is ascending in global block numbering, so each scene's blocks are one run of it)
__global__ void k_batch_scene_first(const SceneDesc* __restrict__ scenes, int nscenes, ActiveView av,
                                    const unsigned* __restrict__ block_offsets, const unsigned* __restrict__ total,
                                    unsigned* __restrict__ first) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s > nscenes) return;
    const int n = active_count(av);
    if (s == nscenes) {
        first[s] = *total;
        return;
    }
    const unsigned b = scenes[s].block_base;
    int lo = 0, hi = n;  // first active entry with a global block index >= b
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((unsigned)av.list[mid] < b) lo = mid + 1; else hi = mid;
    }
    first[s] = lo < n ? block_offsets[lo] : *total;
}

// ------------------------------------------------------------------------------------------------
// block field + per-cell counts
// ------------------------------------------------------------------------------------------------
// per-cell vertex counts of the block whose 9^3 field is in s_field (countActiveBlockTriangles,
// MarchingCubesKernels.cu:914-970): optionally the whole field to fields_out, the per-cell counts in the
// drop-in layout, the block total, and one word per cell for the flat emission (cell_words):
// case code (bits 0-7), mask of the non-degenerate triangles (bits 8-12), first vertex of the cell
// inside its block (bits 13-31)
__device__ __forceinline__ void block_counts(const GridView& g, int a, int lin, float* s_field, unsigned* s_red,
                                             float* __restrict__ fields_out, unsigned* __restrict__ block_totals,
                                             unsigned* __restrict__ packet_counts,
                                             unsigned* __restrict__ cell_words = nullptr) {
    if (threadIdx.x < FIELD_STRIDE - FIELD_N) s_field[FIELD_N + threadIdx.x] = 0.f;
    __syncthreads();
    if (fields_out) {
        float4* dst = reinterpret_cast<float4*>(fields_out + (size_t)a * FIELD_STRIDE);
        const float4* src = reinterpret_cast<const float4*>(s_field);
        for (int i = threadIdx.x; i < FIELD_STRIDE / 4; i += blockDim.x) dst[i] = src[i];
    }
    int bx, by, bz;
    block_coord(g, lin, bx, by, bz);
    unsigned cnt[2], code[2], vm[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int tid = 2 * threadIdx.x + h;
        const CellInfo c = cell_info(g, bx, by, bz, tid);
        cnt[h] = 0;
        code[h] = 0;
        vm[h] = 0;
        if (!c.oob) {
            float cv[8];
            code[h] = (unsigned)cell_case(s_field, c.lx, c.ly, c.lz, cv);
            const unsigned long long word = c_mcCases[code[h]];
            vm[h] = cell_valid_mask(g, c.x, c.y, c.z, cv, word);
            cnt[h] = 3u * __popc(vm[h]);
        }
    }
    if (packet_counts)
        *reinterpret_cast<uint2*>(packet_counts + (size_t)a * 512 + 2 * threadIdx.x) = make_uint2(cnt[0], cnt[1]);
    if (cell_words) {
        unsigned total;
        const unsigned pre = block_exclusive<BLK_THREADS>(cnt[0] + cnt[1], s_red, &total);
        *reinterpret_cast<uint2*>(cell_words + (size_t)a * 512 + 2 * threadIdx.x) =
            make_uint2(code[0] | (vm[0] << 8) | (pre << 13), code[1] | (vm[1] << 8) | ((pre + cnt[0]) << 13));
        if (block_totals && threadIdx.x == 0) block_totals[a] = total;
        __syncthreads();  // s_red is free again
    } else if (block_totals) {
        unsigned v = cnt[0] + cnt[1];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned s = 0;
            for (int w = 0; w < BLK_THREADS / 32; ++w) s += s_red[w];
            block_totals[a] = s;
        }
    }
}

template <bool COUNT>
__global__ void __launch_bounds__(BLK_THREADS) k_mc_field_t(GridView g, SceneView sc, float time, ActiveView av,
                                                          float* __restrict__ fields_out,
                                                          unsigned* __restrict__ block_totals,
                                                          unsigned* __restrict__ packet_counts, unsigned* ticket,
                                                          Diag* diag) {
    __shared__ __align__(16) float s_field[FIELD_STRIDE];
    __shared__ unsigned s_red[BLK_THREADS / 32];
    __shared__ int s_item;
    const int n = active_count(av);
    for (;;) {
        const int a = claim(ticket, n, &s_item);
        if (a < 0) break;
        const int lin = av.list[a];
        eval_block_field<COUNT>(g, sc, time, lin, s_field, diag);
        block_counts(g, a, lin, s_field, s_red, fields_out, block_totals, packet_counts);
    }
}

// ------------------------------------------------------------------------------------------------
// block field with shared halos (engine path). Sample (x, y, z) of the grid belongs to block
// (x / 8, y / 8, z / 8); the 9^3 field of a block is its own 8^3 samples plus the 217 samples of its
// +x / +y / +z faces, edges and corner, which are their neighbours' own samples. Every sample is the
// same map() call at the same grid point as in k_mc_field, so the rows are identical; each sample
// is evaluated once per extraction when its block is active, and only halo samples whose block is
// not active are evaluated for the block that needs them.
//   k_field_plan    block-to-active map; the halo samples whose block is not active, as a list
//   k_field_own     every active block's own samples
//   k_field_miss    the listed halo samples, 32 per warp task
//   k_field_gather  completes each row with the halo copied from the active neighbours' rows, then
//                   the per-cell counts and the block total
// A row's own entries are written only by k_field_own, its listed halo entries only by k_field_miss
// and its other halo entries only by k_field_gather of the same block.
// ------------------------------------------------------------------------------------------------
constexpr int OWN_N = 512;
constexpr int HALO_N = FIELD_N - OWN_N;  // 81 + 72 + 64

// halo sample h (0 <= h < 217) of a block in 9^3-local coordinates: the x = 8 face, then the y = 8
// face without x = 8, then the z = 8 face without x = 8 and y = 8
__device__ __forceinline__ void halo_coord(int h, int& x, int& y, int& z) {
    if (h < 81) {
        x = 8; y = h % 9; z = h / 9;
    } else if (h < 153) {
        h -= 81; y = 8; x = h & 7; z = h >> 3;
    } else {
        h -= 153; z = 8; x = h & 7; y = h >> 3;
    }
}

// linear index of the block owning halo sample (hx, hy, hz) of block (bx, by, bz), -1 outside the grid
__device__ __forceinline__ int halo_owner(const GridView& g, int bx, int by, int bz, int hx, int hy, int hz) {
    const int ox = bx + (hx >> 3), oy = by + (hy >> 3), oz = bz + (hz >> 3);
    if (ox >= g.bx || oy >= g.by || oz >= g.bz) return -1;
    return ox + g.bx * (oy + g.by * oz);
}

// one thread per (active block, halo sample); missing samples are listed as (a << 8) | h
__global__ void __launch_bounds__(256) k_field_plan(GridView g0, ActiveView av, const unsigned* __restrict__ flags,
                                                    float* __restrict__ fields, int* __restrict__ block_to_active,
                                                    unsigned* __restrict__ miss, unsigned* __restrict__ miss_count) {
    const int n = active_count(av);
    const long long total = (long long)n * HALO_N;
    const int lane = threadIdx.x & 31;
    for (long long i0 = (long long)blockIdx.x * blockDim.x; i0 < total; i0 += (long long)gridDim.x * blockDim.x) {
        const long long i = i0 + threadIdx.x;
        bool m = false;
        int a = 0, h = 0;
        if (i < total) {
            a = (int)(i / HALO_N);
            h = (int)(i - (long long)a * HALO_N);
            GridView g = g0;
            SceneView unused;
            int lin;
            unsigned bbase;
            resolve(av, av.list[a], g, unused, lin, bbase);
            if (h == 0) block_to_active[bbase + lin] = a;
            int bx, by, bz, hx, hy, hz;
            block_coord(g, lin, bx, by, bz);
            halo_coord(h, hx, hy, hz);
            const int olin = halo_owner(g, bx, by, bz, hx, hy, hz);
            if (olin < 0)
                fields[(size_t)a * FIELD_STRIDE + (hz * 9 + hy) * 9 + hx] = 0.f;  // outside the grid
            else
                m = flags[bbase + olin] == 0u;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, m);
        unsigned base = 0;
        if (lane == 0 && bal) base = atomicAdd(miss_count, (unsigned)__popc(bal));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (m) miss[base + __popc(bal & ((1u << lane) - 1u))] = ((unsigned)a << 8) | (unsigned)h;
    }
}

// one task of the listed halo samples: entries [32 t, 32 t + 32) of the list (all lanes of a warp)
template <bool COUNT>
__device__ __forceinline__ void miss_task(const GridView& g0, const SceneView& sc0, float time, const ActiveView& av,
                                          float* __restrict__ fields, const unsigned* __restrict__ miss, int nmiss,
                                          int t, Diag* diag) {
    const int lane = threadIdx.x & 31;
    const int e = t * 32 + lane;
    const bool live = e < nmiss;
    const unsigned m = live ? miss[e] : miss[t * 32];
    const int a = (int)(m >> 8);
    GridView g = g0;
    SceneView sc = sc0;
    int lin;
    unsigned bbase;
    resolve(av, av.list[a], g, sc, lin, bbase);
    int sx, sy, sz, bx, by, bz;
    halo_coord((int)(m & 255u), sx, sy, sz);
    block_coord(g, lin, bx, by, bz);
    const int gx = bx * 8 + sx, gy = by * 8 + sy, gz = bz * 8 + sz;
    const bool inside = live && gx < g.w && gy < g.h && gz < g.d;
    const float3 p = grid_loc(g, gx, gy, gz);
    // the warp walks one scene's BVH at a time (a batch's tasks can straddle two scenes)
    unsigned pending = __ballot_sync(0xffffffffu, live);
    while (pending) {
        const unsigned lead_base = __shfl_sync(0xffffffffu, bbase, __ffs(pending) - 1);
        const bool mine = live && bbase == lead_base && ((pending >> lane) & 1u);
        SceneView scw = sc;
        if (av.scenes) scw = av.scenes[scene_of_block(av.scenes, av.nscenes, lead_base)].sc;
        MapState<false> st;
        map_warp<false, COUNT>(scw, p, mine && inside, time, st, diag);
        if (mine) fields[(size_t)a * FIELD_STRIDE + (sz * 9 + sy) * 9 + sx] = inside ? st.d : 0.f;
        pending &= ~__ballot_sync(0xffffffffu, mine);
    }
}

// own samples: eight 4 x 4 x 4 bricks of 64 samples per active block, two z-neighbours per lane; each
// warp claims one brick at a time in (active block, brick) order, so the warps of an SM walk the BVH
// near the same few blocks (the nodes they read stay in L1) and no warp waits for a block's slowest
// brick (measured 11.6 ms against 12.3 ms with one CTA per block at 1024^3)
template <bool COUNT>
__global__ void __launch_bounds__(BLK_THREADS) k_field_own(GridView g0, SceneView sc0, float time, ActiveView av,
                                                         float* __restrict__ fields, unsigned* ticket, Diag* diag) {
    const int n = active_count(av);
    const int lane = threadIdx.x & 31;
    for (;;) {
        int t = 0;
        if (lane == 0) t = (int)atomicAdd(ticket, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= n * (OWN_N / 64)) break;
        const int a = t / (OWN_N / 64), brick = t % (OWN_N / 64);
        GridView g = g0;
        SceneView sc = sc0;
        int lin;
        unsigned bbase;
        resolve(av, av.list[a], g, sc, lin, bbase);
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        {
            const int sx = (brick & 1) * 4 + (lane & 3), sy = ((brick >> 1) & 1) * 4 + ((lane >> 2) & 3);
            const int sz0 = (brick >> 2) * 4 + 2 * (lane >> 4), sz1 = sz0 + 1;
            const int gx = bx * 8 + sx, gy = by * 8 + sy, gz0 = bz * 8 + sz0, gz1 = gz0 + 1;
            const bool v0 = gx < g.w && gy < g.h && gz0 < g.d, v1 = gx < g.w && gy < g.h && gz1 < g.d;
            float d0, d1;
            map_warp2<COUNT>(sc, grid_loc(g, gx, gy, gz0), grid_loc(g, gx, gy, gz1).z, v0, v1, time, d0, d1, diag);
            float* row = fields + (size_t)a * FIELD_STRIDE;
            row[(sz0 * 9 + sy) * 9 + sx] = v0 ? d0 : 0.f;
            row[(sz1 * 9 + sy) * 9 + sx] = v1 ? d1 : 0.f;
        }
    }
}

// listed halo samples, 32 per warp task, tasks claimed one at a time by each warp
template <bool COUNT>
__global__ void __launch_bounds__(BLK_THREADS) k_field_miss(GridView g0, SceneView sc0, float time, ActiveView av,
                                                          float* __restrict__ fields,
                                                          const unsigned* __restrict__ miss,
                                                          const unsigned* __restrict__ miss_count, unsigned* ticket,
                                                          Diag* diag) {
    const int nmiss = (int)*miss_count;
    const int tasks = (nmiss + 31) / 32;
    const int lane = threadIdx.x & 31;
    for (;;) {
        int t = 0;
        if (lane == 0) t = (int)atomicAdd(ticket, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= tasks) break;
        miss_task<COUNT>(g0, sc0, time, av, fields, miss, nmiss, t, diag);
    }
}

// k_field_gather: one warp per active block (static stride over the active list), no CTA barriers,
// so 32 blocks per SM are in flight (four CTAs of eight warps) instead of one per CTA. The warp stages
// the block's row in its own shared memory and fetches the halo entries owned by active neighbours
// (their loads issued together with the row's); with counts requested it classifies the 512 cells:
// case codes first, then the triangle validity of the surface cells only (compacted, one cell per
// lane), then a warp scan in cell order gives each cell's first vertex inside the block. The words and
// totals are those of block_counts (countActiveBlockTriangles, MarchingCubesKernels.cu:914-970).
constexpr int GATHER_WARPS = BLK_THREADS / 32;
constexpr int HALO_PER_LANE = (HALO_N + 31) / 32;          // 7
constexpr int ROW_VEC = FIELD_STRIDE / 4;                  // 184 float4 per row
constexpr int ROW_VEC_PER_LANE = (ROW_VEC + 31) / 32;      // 6

struct GatherWarpSmem {
    float row[FIELD_STRIDE];          // the block's 9^3 row; reused for the 512 cell words at the end
    unsigned char code[512];          // case code per cell (0 for cells outside the grid)
    unsigned char vm[512];            // non-degenerate triangle mask per cell
    unsigned short list[512];         // the block's surface cells (a case with triangles)
};

__global__ void __launch_bounds__(BLK_THREADS, 4) k_field_gather(GridView g0, ActiveView av, float* __restrict__ fields,
                                                            const int* __restrict__ block_to_active,
                                                            const unsigned* __restrict__ flags,
                                                            unsigned* __restrict__ block_totals,
                                                            unsigned* __restrict__ packet_counts,
                                                            unsigned* __restrict__ cell_words = nullptr) {
    __shared__ __align__(16) GatherWarpSmem s_warp[GATHER_WARPS];
    __shared__ unsigned long long s_cases[256];
    const bool classify = block_totals || packet_counts || cell_words;  // dual contouring classifies itself
    if (classify) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) s_cases[i] = c_mcCases[i];
        __syncthreads();
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    GatherWarpSmem& W = s_warp[warp];
    const int n = active_count(av);
    for (int a = blockIdx.x * GATHER_WARPS + warp; a < n; a += gridDim.x * GATHER_WARPS) {
        GridView g = g0;
        SceneView unused;
        int lin;
        unsigned bbase;
        resolve(av, av.list[a], g, unused, lin, bbase);
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        float* row = fields + (size_t)a * FIELD_STRIDE;
#pragma unroll
        for (int k = 0; k < ROW_VEC_PER_LANE; ++k) {
            const int i = lane + 32 * k;
            if (i < ROW_VEC) reinterpret_cast<float4*>(W.row)[i] = reinterpret_cast<const float4*>(row)[i];
        }
        // halo entries owned by active neighbours: flag -> owner's row -> value
        int src[HALO_PER_LANE];
#pragma unroll
        for (int k = 0; k < HALO_PER_LANE; ++k) {
            const int h = lane + 32 * k;
            src[k] = -1;
            if (h < HALO_N) {
                int hx, hy, hz;
                halo_coord(h, hx, hy, hz);
                const int olin = halo_owner(g, bx, by, bz, hx, hy, hz);
                if (olin >= 0 && flags[bbase + olin]) src[k] = olin;
            }
        }
        float hv[HALO_PER_LANE];
#pragma unroll
        for (int k = 0; k < HALO_PER_LANE; ++k) {
            if (src[k] < 0) continue;
            int hx, hy, hz;
            halo_coord(lane + 32 * k, hx, hy, hz);
            const int b = block_to_active[bbase + src[k]];
            // an owner past the rows the buffers hold (the engine then grows them and runs again) has no
            // row this extraction: the entry is left as it is
            if (b < 0 || b >= n) {
                src[k] = -1;
                continue;
            }
            hv[k] = fields[(size_t)b * FIELD_STRIDE + ((hz & 7) * 9 + (hy & 7)) * 9 + (hx & 7)];
        }
        __syncwarp();  // the row is in place before the copied halo entries overwrite their slots
#pragma unroll
        for (int k = 0; k < HALO_PER_LANE; ++k) {
            if (src[k] < 0) continue;
            int hx, hy, hz;
            halo_coord(lane + 32 * k, hx, hy, hz);
            const int h = (hz * 9 + hy) * 9 + hx;
            W.row[h] = hv[k];
            row[h] = hv[k];
        }
        __syncwarp();
        if (!classify) continue;
        // case codes of all cells; the surface cells listed
        int nlist = 0;
#pragma unroll 4
        for (int j = 0; j < 16; ++j) {
            const int tid = lane + 32 * j;
            const CellInfo c = cell_info(g, bx, by, bz, tid);
            int code = 0;
            if (!c.oob) {
                float cv[8];
                code = cell_case(W.row, c.lx, c.ly, c.lz, cv);
            }
            const bool surf = (s_cases[code] & 0xF) != 0;
            W.code[tid] = (unsigned char)code;
            W.vm[tid] = 0;
            const unsigned bal = __ballot_sync(0xffffffffu, surf);
            if (surf) W.list[nlist + __popc(bal & ((1u << lane) - 1u))] = (unsigned short)tid;
            nlist += __popc(bal);
        }
        __syncwarp();
        // triangle validity of the surface cells, one per lane
        for (int i = lane; i < nlist; i += 32) {
            const int tid = W.list[i];
            const CellInfo c = cell_info(g, bx, by, bz, tid);
            float cv[8];
            const int code = cell_case(W.row, c.lx, c.ly, c.lz, cv);
            W.vm[tid] = (unsigned char)cell_valid_mask(g, c.x, c.y, c.z, cv, s_cases[code]);
        }
        __syncwarp();
        // cells 16 lane .. 16 lane + 15: counts, warp scan in cell order, words
        const uint4 vm4 = reinterpret_cast<const uint4*>(W.vm)[lane];
        const uint4 cd4 = reinterpret_cast<const uint4*>(W.code)[lane];
        const unsigned vmw[4] = {vm4.x, vm4.y, vm4.z, vm4.w}, cdw[4] = {cd4.x, cd4.y, cd4.z, cd4.w};
        // the vm bytes hold at most 5 bits each, so the popcount of a word is that of its four cells
        const unsigned sum = 3u * (__popc(vmw[0]) + __popc(vmw[1]) + __popc(vmw[2]) + __popc(vmw[3]));
        unsigned incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
        if (packet_counts) {
            uint4* dst = reinterpret_cast<uint4*>(packet_counts + (size_t)a * 512 + 16 * lane);
#pragma unroll
            for (int q = 0; q < 4; ++q)
                dst[q] = make_uint4(3u * __popc(vmw[q] & 0xFFu), 3u * __popc((vmw[q] >> 8) & 0xFFu),
                                    3u * __popc((vmw[q] >> 16) & 0xFFu), 3u * __popc(vmw[q] >> 24));
        }
        if (cell_words) {
            unsigned* words = reinterpret_cast<unsigned*>(W.row);  // the row is no longer read
            unsigned pre = incl - sum;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const unsigned code = (cdw[j >> 2] >> (8 * (j & 3))) & 0xFFu;
                const unsigned vm = (vmw[j >> 2] >> (8 * (j & 3))) & 0xFFu;
                words[16 * lane + j] = code | (vm << 8) | (pre << 13);
                pre += 3u * __popc(vm);
            }
            __syncwarp();
            uint4* dst = reinterpret_cast<uint4*>(cell_words + (size_t)a * 512);
#pragma unroll
            for (int q = 0; q < 4; ++q) dst[lane + 32 * q] = reinterpret_cast<const uint4*>(words)[lane + 32 * q];
        }
        if (block_totals && lane == 0) block_totals[a] = total;
        __syncwarp();  // the warp's shared memory is free for the next block
    }
}

// the single-kernel block field of the drop-in launcher (no block-to-active map is at hand there)
static constexpr auto k_mc_field = k_mc_field_t<false>;

// FP32 FMA throughput probe: 8 independent FMA chains per thread, no memory traffic in the loop
__global__ void __launch_bounds__(256) k_fma_peak(float* out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-7f, x2 = x0 + 2e-7f, x3 = x0 + 3e-7f;
    float x4 = x0 + 4e-7f, x5 = x0 + 5e-7f, x6 = x0 + 6e-7f, x7 = x0 + 7e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = __fmaf_rn(x0, a, b); x1 = __fmaf_rn(x1, a, b); x2 = __fmaf_rn(x2, a, b); x3 = __fmaf_rn(x3, a, b);
            x4 = __fmaf_rn(x4, a, b); x5 = __fmaf_rn(x5, a, b); x6 = __fmaf_rn(x6, a, b); x7 = __fmaf_rn(x7, a, b);
        }
    }
    const float r = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (r == 12345.f) out[threadIdx.x] = r;  // keeps the chains live
}

// ------------------------------------------------------------------------------------------------
// flat emission (generateActiveBlockTriangles, MarchingCubesKernels.cu:972-1110, positions and
// identity indices only): one warp per active block (static stride over the active list). The warp
// loads the block's 512 cell words (coalesced) into its shared memory, lists the cells that emit
// (about 4 % of them), and each lane then takes one listed cell: its eight corner values from the
// block's row, its case's non-degenerate triangles, written from the cell's first vertex. The words
// come from the gather kernel; the vertex order is the block emission's: block offset, then cells in
// order, then the case's triangles in order.
// ------------------------------------------------------------------------------------------------
constexpr int EMIT_WARPS = 8;

// A warp's staging: the 512 cell words of two blocks (the one it emits and the next one it will emit,
// filled by a bulk copy while the current one is processed), the emitting cells, the copies' barriers.
struct EmitWarpSmem {
    unsigned words[2][512];
    unsigned short list[512];
    uint64_t bar[2];
};

__global__ void __launch_bounds__(EMIT_WARPS * 32, 5) k_mc_emit_cells(GridView g0, ActiveView av,
                                                                  const float* __restrict__ fields,
                                                                  const unsigned* __restrict__ cell_words,
                                                                  const unsigned* __restrict__ block_offsets,
                                                                  MeshOut out, unsigned mask, Diag* diag) {
    __shared__ unsigned long long s_cases[256];
    __shared__ __align__(16) EmitWarpSmem s_warp[EMIT_WARPS];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s_cases[i] = c_mcCases[i];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    EmitWarpSmem& W = s_warp[warp];
    if (lane == 0) {
        bar_init(&W.bar[0], 1);
        bar_init(&W.bar[1], 1);
    }
    __syncthreads();
    const int n = active_count(av);
    const int stride = gridDim.x * EMIT_WARPS;
    // the cell words of block a into staging buffer b (lane 0; 2 KB, 16-byte aligned rows)
    auto stage = [&](int a, int b) {
        bar_expect_tx(&W.bar[b], 512 * sizeof(unsigned));
        bulk_g2s(W.words[b], cell_words + (size_t)a * 512, 512 * sizeof(unsigned), &W.bar[b]);
    };
    int a = blockIdx.x * EMIT_WARPS + warp;
    if (a < n && lane == 0) stage(a, 0);
    unsigned parity[2] = {0u, 0u};
    int buf = 0;
    bool pending_other = false;  // a copy into the other buffer is in flight
    for (; a < n; a += stride) {
        const int next = a + stride;
        if (next < n && lane == 0) stage(next, buf ^ 1);  // that buffer was released at the end of the last block
        pending_other = next < n;
        if (!__all_sync(0xffffffffu, bar_wait(&W.bar[buf], parity[buf]))) {
            if (lane == 0 && diag) atomicExch(&diag->timeout, 1);
            break;
        }
        parity[buf] ^= 1u;
        const unsigned* words = W.words[buf];
        GridView g = g0;
        SceneView unused;
        int lin;
        unsigned bbase;
        resolve(av, av.list[a], g, unused, lin, bbase);
        const unsigned long long base = block_offsets[a];
        int nlist = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint4 w4 = reinterpret_cast<const uint4*>(words)[lane + 32 * q];
            const unsigned wq[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const bool emits = ((wq[r] >> 8) & 31u) != 0;
                const unsigned bal = __ballot_sync(0xffffffffu, emits);
                if (emits)
                    W.list[nlist + __popc(bal & ((1u << lane) - 1u))] = (unsigned short)(4 * (lane + 32 * q) + r);
                nlist += __popc(bal);
            }
        }
        __syncwarp();
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        const float* f = fields + (size_t)a * FIELD_STRIDE;
        for (int i = lane; i < nlist; i += 32) {
            const int tid = W.list[i];
            const unsigned w = words[tid];
            const unsigned vm = (w >> 8) & 31u;
            const CellInfo c = cell_info(g, bx, by, bz, tid);
            float cv[8];
#pragma unroll
            for (int k = 0; k < 8; ++k)
                cv[k] = __ldg(f + fidx(c.lx + corner_dx(k), c.ly + corner_dy(k), c.lz + corner_dz(k)));
            const unsigned long long word = s_cases[w & 255u];
            unsigned long long v = base + (w >> 13);
            const int nt = (int)(word & 0xF);
            for (int k = 0; k < nt; ++k) {
                if (!((vm >> k) & 1u)) continue;
                if (v + 2 >= out.maxV) break;  // the reference's capacity stop (:1020)
                float3 p[3];
                tri_points(g, c.x, c.y, c.z, cv, word, k, p);
#pragma unroll
                for (int j = 0; j < 3; ++j) out.verts[v + j] = make_float4(p[j].x, p[j].y, p[j].z, 1.f);
                if ((mask & OUT_INDICES) && out.indices) {
                    out.indices[v] = (unsigned)v;
                    out.indices[v + 1] = (unsigned)v + 1;
                    out.indices[v + 2] = (unsigned)v + 2;
                }
                v += 3;
            }
        }
        __syncwarp();  // the buffer and the list are free for the next block
        buf ^= 1;
        pending_other = false;
    }
    // after a timeout, the copy already issued into the other buffer is waited for (bounded) before
    // the CTA's shared memory goes away
    if (pending_other) (void)bar_wait(&W.bar[buf ^ 1], parity[buf ^ 1]);
}

// ------------------------------------------------------------------------------------------------
// emission (generateActiveBlockTriangles, MarchingCubesKernels.cu:972-1110)
// ------------------------------------------------------------------------------------------------
struct EmitSmem {
    float field[FIELD_STRIDE];
    unsigned long long cases[256];            // the case table, staged from constant memory
    unsigned warp_sums[BLK_THREADS / 32];
    unsigned short tri_cell[MAX_BLOCK_TRIS];  // (cell << 3) | triangle slot
    unsigned tri_out[MAX_BLOCK_TRIS];         // first output vertex of the triangle
    int ntri;
    int item;
};

// writes the triangle-list attributes: colour / primitive id / uv from map() at the triangle
// centre (one warp-coherent call per 32 triangles), normals from computeNormal at each vertex
__device__ void emit_attributes(const GridView& g, const SceneView& sc, float time, int bx, int by, int bz,
                                EmitSmem& S, const MeshOut& out, unsigned mask, Diag* diag) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int ntri = S.ntri;
    if (mask & (OUT_COLORS | OUT_PRIMIDS | OUT_UVS)) {
        for (int base = warp * 32; base < ntri; base += nwarps * 32) {
            const int i = base + lane;
            const bool valid = i < ntri;
            float3 v[3] = {f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f)};
            unsigned w = 0;
            if (valid) {
                const int tid = S.tri_cell[i] >> 3, k = S.tri_cell[i] & 7;
                const CellInfo c = cell_info(g, bx, by, bz, tid);
                float cv[8];
                const int code = cell_case(S.field, c.lx, c.ly, c.lz, cv);
                tri_points(g, c.x, c.y, c.z, cv, c_mcCases[code], k, v);
                w = S.tri_out[i];
            }
            const float3 ctr = f3(DIV(ADD(ADD(v[0].x, v[1].x), v[2].x), 3.f), DIV(ADD(ADD(v[0].y, v[1].y), v[2].y), 3.f),
                                  DIV(ADD(ADD(v[0].z, v[1].z), v[2].z), 3.f));
            MapState<true> st;
            map_warp<true>(sc, ctr, valid, time, st, diag);
            if (valid) {
                if ((mask & OUT_COLORS) && out.colors) {
                    const float4 c4 = make_float4(st.color.x, st.color.y, st.color.z, 1.f);
                    out.colors[w] = c4;
                    out.colors[w + 1] = c4;
                    out.colors[w + 2] = c4;
                }
                if ((mask & OUT_PRIMIDS) && out.primids) {
                    const int bits = __float_as_int((float)st.id);
                    out.primids[w] = bits;
                    out.primids[w + 1] = bits;
                    out.primids[w + 2] = bits;
                }
                if ((mask & OUT_UVS) && out.uvs) {
                    float2 uv[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
                    if (st.id >= 0 && st.id < sc.nprims) {
                        const float4* pr = sc.prims + (size_t)st.id * PRIM_ROWS;
                        const float4 rot = __ldg(pr + 0), pos = __ldg(pr + 2), scl = __ldg(pr + 3);
                        float3 lp[3];
#pragma unroll
                        for (int j = 0; j < 3; ++j) lp[j] = to_local(v[j], rot, pos, scl);
                        triangle_uvs(lp, load_uv_params(pr), uv);
                    }
                    out.uvs[w] = uv[0];
                    out.uvs[w + 1] = uv[1];
                    out.uvs[w + 2] = uv[2];
                }
            }
        }
    }
    if ((mask & OUT_NORMALS) && out.normals) {
        const int nv = ntri * 3;
        for (int base = warp * 32; base < nv; base += nwarps * 32) {
            const int i = base + lane;
            const bool valid = i < nv;
            float3 p = f3(0.f, 0.f, 0.f);
            unsigned w = 0;
            if (valid) {
                const int t = i / 3, j = i - 3 * t;
                const int tid = S.tri_cell[t] >> 3, k = S.tri_cell[t] & 7;
                const CellInfo c = cell_info(g, bx, by, bz, tid);
                float cv[8];
                const int code = cell_case(S.field, c.lx, c.ly, c.lz, cv);
                float3 v[3];
                tri_points(g, c.x, c.y, c.z, cv, c_mcCases[code], k, v);
                p = v[j];
                w = S.tri_out[t] + j;
            }
            const float3 nrm = normal_warp(sc, p, valid, time, g.cell, diag);
            if (valid) out.normals[w] = make_float4(nrm.x, nrm.y, nrm.z, 0.f);
        }
    }
}

// Modes: FIELD_FROM (fields_in != nullptr: load the stored field; else evaluate it) and OFFSETS_FROM
// (packet_offsets_in != nullptr: per-cell offsets of the drop-in layout; else block_offsets + an
// in-block scan).
__global__ void __launch_bounds__(BLK_THREADS) k_mc_emit(GridView g0, SceneView sc0, float time, ActiveView av,
                                                         const float* __restrict__ fields_in,
                                                         const unsigned* __restrict__ block_offsets,
                                                         const unsigned* __restrict__ packet_offsets_in,
                                                         unsigned* __restrict__ packet_offsets_out, MeshOut out,
                                                         unsigned mask, unsigned* ticket, Diag* diag) {
    __shared__ __align__(16) EmitSmem S;
    const int n = active_count(av);
    const bool attrs = (mask & (OUT_COLORS | OUT_PRIMIDS | OUT_UVS | OUT_NORMALS)) != 0;
    for (int i = threadIdx.x; i < 256; i += blockDim.x) S.cases[i] = c_mcCases[i];
    for (;;) {
        const int a = claim(ticket, n, &S.item);
        if (a < 0) break;
        GridView g = g0;
        SceneView sc = sc0;
        int lin;
        unsigned bbase;
        resolve(av, av.list[a], g, sc, lin, bbase);
        if (fields_in) {
            const float4* src = reinterpret_cast<const float4*>(fields_in + (size_t)a * FIELD_STRIDE);
            float4* dst = reinterpret_cast<float4*>(S.field);
            for (int i = threadIdx.x; i < FIELD_STRIDE / 4; i += blockDim.x) dst[i] = __ldcs(src + i);
        } else {
            eval_block_field(g, sc, time, lin, S.field, diag);
        }
        __syncthreads();
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        CellInfo c[2];
        float cv[2][8];
        unsigned long long word[2];
        unsigned vm[2], cnt[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            c[h] = cell_info(g, bx, by, bz, 2 * threadIdx.x + h);
            vm[h] = 0;
            word[h] = 0;
            if (!c[h].oob) {
                const int code = cell_case(S.field, c[h].lx, c[h].ly, c[h].lz, cv[h]);
                word[h] = S.cases[code];
                vm[h] = cell_valid_mask(g, c[h].x, c[h].y, c[h].z, cv[h], word[h]);
            }
            cnt[h] = 3u * __popc(vm[h]);
        }
        unsigned local_total;
        const unsigned local = block_exclusive<BLK_THREADS>(cnt[0] + cnt[1], S.warp_sums, &local_total);
        unsigned off[2];
        if (packet_offsets_in) {
            const uint2 o = *reinterpret_cast<const uint2*>(packet_offsets_in + (size_t)a * 512 + 2 * threadIdx.x);
            off[0] = o.x;
            off[1] = o.y;
        } else {
            off[0] = block_offsets[a] + local;
            off[1] = off[0] + cnt[0];
        }
        if (packet_offsets_out)
            *reinterpret_cast<uint2*>(packet_offsets_out + (size_t)a * 512 + 2 * threadIdx.x) = make_uint2(off[0], off[1]);
        // the block's triangle list in output order: slot s writes vertices base + 3 s .. + 2
        unsigned tslot = local / 3;  // this thread's first slot
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (c[h].oob) continue;
            const int nt = (int)(word[h] & 0xF);
            for (int k = 0; k < nt; ++k)
                if ((vm[h] >> k) & 1u) S.tri_cell[tslot++] = (unsigned short)(((2 * threadIdx.x + h) << 3) | k);
        }
        const unsigned base = packet_offsets_in ? 0u : block_offsets[a];
        const unsigned ntri_all = local_total / 3;
        // the reference stops a block's output at the first triangle that would reach maxV (:1020)
        unsigned ntri = 0;
        if (!packet_offsets_in && (unsigned long long)base + 3 <= out.maxV)
            ntri = min(ntri_all, (unsigned)(((unsigned long long)out.maxV - base - 3) / 3 + 1));
        if (threadIdx.x == 0) S.ntri = (int)ntri;
        __syncthreads();
        if (packet_offsets_in) {
            // drop-in path: the cells' offsets come from the caller's scan, one run per thread
            unsigned slot = local / 3;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (c[h].oob) continue;
                unsigned w = off[h];
                const int nt = (int)(word[h] & 0xF);
                for (int k = 0; k < nt; ++k) {
                    if (!((vm[h] >> k) & 1u)) continue;
                    if ((unsigned long long)w + 2 >= out.maxV) break;
                    if (attrs) {
                        S.tri_out[slot] = w;
                        atomicAdd(&S.ntri, 1);
                    }
                    ++slot;
                    float3 v[3];
                    tri_points(g, c[h].x, c[h].y, c[h].z, cv[h], word[h], k, v);
#pragma unroll
                    for (int j = 0; j < 3; ++j) out.verts[w + j] = make_float4(v[j].x, v[j].y, v[j].z, 1.f);
                    if ((mask & OUT_INDICES) && out.indices) {
                        out.indices[w] = w;
                        out.indices[w + 1] = w + 1;
                        out.indices[w + 2] = w + 2;
                    }
                    w += 3;
                }
            }
        } else {
            // one output vertex per thread: consecutive threads write consecutive float4s
            const unsigned nv = 3 * ntri;
            for (unsigned v = threadIdx.x; v < nv; v += blockDim.x) {
                const unsigned slot = v / 3, j = v - 3 * slot;
                const int cell = S.tri_cell[slot] >> 3, k = S.tri_cell[slot] & 7;
                const CellInfo ci = cell_info(g, bx, by, bz, cell);
                float cvv[8];
                const int code = cell_case(S.field, ci.lx, ci.ly, ci.lz, cvv);
                const unsigned long long wd = S.cases[code];
                const float3 p = edge_point(g, ci.x, ci.y, ci.z, cvv, (int)((wd >> (4 + 4 * (3 * k + j))) & 0xF));
                out.verts[base + v] = make_float4(p.x, p.y, p.z, 1.f);
                if ((mask & OUT_INDICES) && out.indices) out.indices[base + v] = base + v;
            }
            if (attrs)
                for (unsigned t = threadIdx.x; t < ntri; t += blockDim.x) S.tri_out[t] = base + 3 * t;
        }
        if (attrs) {
            __syncthreads();
            // slots are dense except when the capacity stop dropped triangles; S.ntri counts them,
            // and dropped slots only occur at the end of the output, i.e. the tail of the list
            emit_attributes(g, sc, time, bx, by, bz, S, out, mask, diag);
        }
    }
}

// map() at arbitrary points: out[8*i ..] = distance, colour xyz, primitive id (as float), local xyz.
// Points are taken 32 per warp in input order, so spatially sorted input keeps the walks coherent.
__global__ void __launch_bounds__(BLK_THREADS) k_eval_points(SceneView sc, const float* __restrict__ pts, int n,
                                                             float time, float* __restrict__ out, Diag* diag) {
    const int warps_total = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n; base += warps_total * 32) {
        const int i = base + lane;
        const bool valid = i < n;
        const float3 p = valid ? f3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]) : f3(0.f, 0.f, 0.f);
        MapState<true> st;
        map_warp<true>(sc, p, valid, time, st, diag);
        if (valid) {
            float* o = out + 8 * (size_t)i;
            o[0] = st.d; o[1] = st.color.x; o[2] = st.color.y; o[3] = st.color.z;
            o[4] = (float)st.id; o[5] = st.local.x; o[6] = st.local.y; o[7] = st.local.z;
        }
    }
}

// distance only (no colour / id / local position tracking) at arbitrary points
__global__ void __launch_bounds__(BLK_THREADS) k_eval_distance(SceneView sc, const float* __restrict__ pts, int n,
                                                               float time, float* __restrict__ out, Diag* diag) {
    const int warps_total = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n; base += warps_total * 32) {
        const int i = base + lane;
        const bool valid = i < n;
        const float3 p = valid ? f3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]) : f3(0.f, 0.f, 0.f);
        MapState<false> st;
        map_warp<false>(sc, p, valid, time, st, diag);
        if (valid) out[i] = st.d;
    }
}

// computeNormal at arbitrary points: out[3*i ..] = unit gradient (central differences of map(),
// step 0.001 cell, as the reference's computeNormal)
__global__ void __launch_bounds__(BLK_THREADS) k_eval_normals(SceneView sc, const float* __restrict__ pts, int n,
                                                              float time, float cell, float* __restrict__ out,
                                                              Diag* diag) {
    const int warps_total = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < n; base += warps_total * 32) {
        const int i = base + lane;
        const bool valid = i < n;
        const float3 p = valid ? f3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]) : f3(0.f, 0.f, 0.f);
        const float3 nrm = normal_warp(sc, p, valid, time, cell, diag);
        if (valid) {
            out[3 * (size_t)i] = nrm.x;
            out[3 * (size_t)i + 1] = nrm.y;
            out[3 * (size_t)i + 2] = nrm.z;
        }
    }
}

// active list from the 0/1 flags: out[prefix(i)] = i where flags[i] != 0 (same look-back scan)
__global__ void __launch_bounds__(SCAN_THREADS) k_compact(const unsigned* __restrict__ flags, unsigned n,
                                                          int* __restrict__ list, int* __restrict__ count,
                                                          ScanState st, Diag* diag) {
    __shared__ unsigned s_warp[SCAN_THREADS / 32];
    __shared__ unsigned s_pfx;
    __shared__ int s_tile;
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(st.ticket, 1u);
    __syncthreads();
    const int tile = s_tile;
    const unsigned base = (unsigned)tile * SCAN_TILE;
    if (base >= n && tile != 0) return;
    uint4 v[SCAN_ROUNDS];
    unsigned tsum[SCAN_ROUNDS], pre[SCAN_ROUNDS], rtot[SCAN_ROUNDS];
#pragma unroll
    for (int r = 0; r < SCAN_ROUNDS; ++r) {
        const unsigned i0 = base + (unsigned)r * (SCAN_THREADS * 4) + threadIdx.x * 4;
        if (i0 + 3 < n) {
            v[r] = *reinterpret_cast<const uint4*>(flags + i0);
        } else {
            v[r].x = i0 < n ? flags[i0] : 0u;
            v[r].y = i0 + 1 < n ? flags[i0 + 1] : 0u;
            v[r].z = i0 + 2 < n ? flags[i0 + 2] : 0u;
            v[r].w = i0 + 3 < n ? flags[i0 + 3] : 0u;
        }
        tsum[r] = v[r].x + v[r].y + v[r].z + v[r].w;
    }
#pragma unroll
    for (int r = 0; r < SCAN_ROUNDS; ++r) pre[r] = block_exclusive<SCAN_THREADS>(tsum[r], s_warp, &rtot[r]);
    unsigned agg = 0;
#pragma unroll
    for (int r = 0; r < SCAN_ROUNDS; ++r) agg += rtot[r];
    const unsigned tile_pfx = tile_lookback(st, tile, agg, &s_pfx, diag);
    unsigned carry = tile_pfx;
#pragma unroll
    for (int r = 0; r < SCAN_ROUNDS; ++r) {
        const unsigned i0 = base + (unsigned)r * (SCAN_THREADS * 4) + threadIdx.x * 4;
        unsigned p = carry + pre[r];
        if (v[r].x) list[p++] = (int)i0;
        if (v[r].y) list[p++] = (int)(i0 + 1);
        if (v[r].z) list[p++] = (int)(i0 + 2);
        if (v[r].w) list[p++] = (int)(i0 + 3);
        carry += rtot[r];
    }
    if (threadIdx.x == 0 && base + SCAN_TILE >= n) *count = (int)(tile_pfx + agg);
}

}  // namespace sdfb
