// Welded (indexed) marching-cubes output: one vertex per crossed grid edge, shared by every triangle
// on that edge, and three indices per triangle. The reference only writes a triangle soup (its index
// buffer is the identity and its index count stays 0, CudaSDFMesh.cpp:466-469); welding by edge is
// the step its plan names next (CUDA_Parallelization_Plan.md, "Mesh Welding"). Two cells that share an
// edge compute its soup vertex in opposite directions for 4 of the 12 cell edges, so the soup's copies
// can differ in the last bits; here each edge has one vertex, computed from its lower to its upper
// sample with the reference's interpolation (interpEdgePoint, MarchingCubesKernels.cu:60-81), which is
// the soup vertex itself for the 8 edges a cell walks in that direction.
//
// Ownership: an edge belongs to the active block with the smallest linear index among the blocks of
// its (up to four) adjacent in-grid cells. Every block that emits a triangle on the edge reaches the
// same owner from the scout flags alone. Per active block a bitmap over its 2,187 edge slots
// (lower endpoint (lx, ly, lz) in [0, 8]^3, axis) marks the owned crossed edges; word prefixes give
// each owned edge its rank, and a scan over blocks the block's first vertex.
#pragma once

#include "mc_kernels.cuh"

namespace sdfb {

constexpr int WELD_SLOTS = 9 * 9 * 9 * 3;          // 2187
constexpr int WELD_WORDS = (WELD_SLOTS + 31) / 32;  // 69 bit words
constexpr int WELD_STRIDE = 72;                     // words (and prefixes) per active block

struct WeldBuffers {
    unsigned* bits;             // WELD_STRIDE words per active block
    unsigned short* prefix;     // WELD_STRIDE exclusive popcounts per active block
    unsigned* totals;           // owned vertices per active block
    unsigned* base;             // first welded vertex per active block (exclusive scan of totals)
    const unsigned* flags;      // scout flags per linear block
    const int* block_to_active; // active id per linear block (valid where the flag is set)
};

__device__ __forceinline__ int weld_slot(int lx, int ly, int lz, int axis) { return ((lz * 9 + ly) * 9 + lx) * 3 + axis; }

// Linear index of the block that owns the edge from sample (X, Y, Z) along `axis`, or -1 when no
// adjacent in-grid cell lies in an active block. Candidates are visited from the smallest linear
// block index up (z offset first, then y, then x), so the first active one is the owner.
__device__ __forceinline__ int edge_owner(const GridView& g, int X, int Y, int Z, int axis, const unsigned* flags) {
    // adjacent cells: the edge's lower sample minus 0 or 1 along each of the two other axes, a (the
    // lower of them: y for an x edge, else x) and b (the higher: y for a z edge, else z)
    int best = -1;
#pragma unroll
    for (int db = 1; db >= 0; --db) {      // the higher axis (b) minus 1 first: smaller block index
#pragma unroll
        for (int da = 1; da >= 0; --da) {
            const int cx = X - (axis != 0 ? da : 0);
            const int cy = Y - (axis == 0 ? da : 0) - (axis == 2 ? db : 0);
            const int cz = Z - (axis != 2 ? db : 0);
            if (cx < 0 || cy < 0 || cz < 0 || cx > g.w - 2 || cy > g.h - 2 || cz > g.d - 2) continue;
            const int lin = (cx >> 3) + g.bx * ((cy >> 3) + g.by * (cz >> 3));
            if (flags[lin] != 0u && (best < 0 || lin < best)) best = lin;
        }
    }
    return best;
}

// Whether this block owns the crossed edge at local lower sample (lx, ly, lz) along `axis`. An edge
// off the block's lower faces (both other coordinates >= 1) has no adjacent cell in a block of smaller
// linear index, so it is this block's when one of its adjacent cells here lies in the grid; edges on
// the lower faces ask edge_owner.
__device__ __forceinline__ bool weld_owns(const GridView& g, int lin, int bx, int by, int bz, int lx, int ly, int lz,
                                          int axis, const unsigned* flags) {
    const int la = axis == 0 ? ly : lx, lb = axis == 2 ? ly : lz;       // the two other axes
    if (la >= 1 && lb >= 1) {
        const int ga = 8 * (axis == 0 ? by : bx) + la, na = axis == 0 ? g.h : g.w;
        const int gb = 8 * (axis == 2 ? by : bz) + lb, nb = axis == 2 ? g.h : g.d;
        const int ge = axis == 0 ? 8 * bx + lx : (axis == 1 ? 8 * by + ly : 8 * bz + lz);
        const int ne = axis == 0 ? g.w : (axis == 1 ? g.h : g.d);
        return ga - 1 <= na - 2 && gb - 1 <= nb - 2 && ge <= ne - 2;
    }
    return edge_owner(g, 8 * bx + lx, 8 * by + ly, 8 * bz + lz, axis, flags) == lin;
}

// The three kernels below run one warp per active block (static stride over the active list): no
// CTA barriers, 32 to 64 blocks per SM in flight (as their registers allow).
constexpr int WELD_WARPS = 8;

// whether the edge of slot s (lower sample, axis) is crossed, from the block's row in shared memory
__device__ __forceinline__ bool weld_crossed(const float* row, int s, int& lx, int& ly, int& lz, int& axis) {
    axis = s % 3;
    const int cell = s / 3;
    lx = cell % 9;
    ly = (cell / 9) % 9;
    lz = cell / 81;
    const int ux = lx + (axis == 0), uy = ly + (axis == 1), uz = lz + (axis == 2);
    return ux <= 8 && uy <= 8 && uz <= 8 && ((row[fidx(lx, ly, lz)] > 0.f) != (row[fidx(ux, uy, uz)] > 0.f));
}

// Marks the owned crossed edges of every active block and counts them: word w of the bitmap is the
// ballot of slots 32 w .. 32 w + 31; lane l keeps words l, l + 32 and l + 64, whose exclusive
// popcount prefixes come from three warp scans.
__global__ void __launch_bounds__(WELD_WARPS * 32) k_weld_mark(GridView g, ActiveView av,
                                                               const float* __restrict__ fields, WeldBuffers wb) {
    __shared__ __align__(16) float s_rows[WELD_WARPS][FIELD_STRIDE];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* row = s_rows[warp];
    const int n = active_count(av);
    for (int a = blockIdx.x * WELD_WARPS + warp; a < n; a += gridDim.x * WELD_WARPS) {
        const int lin = av.list[a];
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        const float4* f = reinterpret_cast<const float4*>(fields + (size_t)a * FIELD_STRIDE);
        for (int i = lane; i < FIELD_STRIDE / 4; i += 32) reinterpret_cast<float4*>(row)[i] = f[i];
        __syncwarp();
        unsigned keep[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            unsigned acc = 0;
            for (int j = 0; j < 32; ++j) {
                const int w = 32 * k + j;
                if (w >= WELD_STRIDE) break;  // warp-uniform
                const int s = 32 * w + lane;
                bool own = false;
                int lx, ly, lz, axis;
                if (s < WELD_SLOTS && weld_crossed(row, s, lx, ly, lz, axis))
                    own = weld_owns(g, lin, bx, by, bz, lx, ly, lz, axis, wb.flags);
                const unsigned word = __ballot_sync(0xffffffffu, own);
                if (j == lane) acc = word;
            }
            keep[k] = acc;
        }
        unsigned carry = 0;
        unsigned* bits = wb.bits + (size_t)a * WELD_STRIDE;
        unsigned short* pre = wb.prefix + (size_t)a * WELD_STRIDE;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int w = 32 * k + lane;
            const unsigned c = w < WELD_STRIDE ? (unsigned)__popc(keep[k]) : 0u;
            unsigned x = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (w < WELD_STRIDE) {
                bits[w] = keep[k];
                pre[w] = (unsigned short)(carry + x - c);
            }
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        if (lane == 0) wb.totals[a] = carry;
        __syncwarp();  // the warp's row is free for the next block
    }
}

// Rank of an owned slot among its block's owned edges.
__device__ __forceinline__ unsigned weld_rank(const WeldBuffers& wb, int a, int slot) {
    const unsigned w = wb.bits[(size_t)a * WELD_STRIDE + (slot >> 5)];
    return wb.prefix[(size_t)a * WELD_STRIDE + (slot >> 5)] + (unsigned)__popc(w & ((1u << (slot & 31)) - 1u));
}

// The welded vertices: each owned edge's point from its lower to its upper sample. Lane l walks the
// set bits of words l, l + 32 and l + 64; the row is staged in the warp's shared memory.
__global__ void __launch_bounds__(WELD_WARPS * 32) k_weld_vertices(GridView g, ActiveView av,
                                                                   const float* __restrict__ fields, WeldBuffers wb,
                                                                   float4* __restrict__ verts, unsigned max_verts) {
    __shared__ __align__(16) float s_rows[WELD_WARPS][FIELD_STRIDE];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* row = s_rows[warp];
    const int n = active_count(av);
    for (int a = blockIdx.x * WELD_WARPS + warp; a < n; a += gridDim.x * WELD_WARPS) {
        const float4* f = reinterpret_cast<const float4*>(fields + (size_t)a * FIELD_STRIDE);
        for (int i = lane; i < FIELD_STRIDE / 4; i += 32) reinterpret_cast<float4*>(row)[i] = f[i];
        const int lin = av.list[a];
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        const unsigned base = wb.base[a];
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int w = 32 * k + lane;
            if (w >= WELD_WORDS) continue;
            unsigned bitsw = wb.bits[(size_t)a * WELD_STRIDE + w];
            unsigned rank = base + wb.prefix[(size_t)a * WELD_STRIDE + w];
            while (bitsw) {
                const int b = __ffs(bitsw) - 1;
                bitsw &= bitsw - 1u;
                int lx, ly, lz, axis;
                (void)weld_crossed(row, 32 * w + b, lx, ly, lz, axis);
                const int ux = lx + (axis == 0), uy = ly + (axis == 1), uz = lz + (axis == 2);
                const float t = edge_t(row[fidx(lx, ly, lz)], row[fidx(ux, uy, uz)]);
                const float3 p = lerp3(grid_loc(g, bx * 8 + lx, by * 8 + ly, bz * 8 + lz),
                                       grid_loc(g, bx * 8 + ux, by * 8 + uy, bz * 8 + uz), t);
                if (rank < max_verts) verts[rank] = make_float4(p.x, p.y, p.z, 1.f);
                ++rank;
            }
        }
        __syncwarp();  // the warp's row is free for the next block
    }
}

// The index buffer: the soup's triangles in the soup's order (the same degenerate-triangle test on the
// same soup points, read from the gather's cell words), each corner replaced by its edge's welded
// vertex. One warp per block lists the cells that emit and gives each lane one of them.
__global__ void __launch_bounds__(WELD_WARPS * 32) k_weld_indices(GridView g, ActiveView av,
                                                                  const unsigned* __restrict__ cell_words,
                                                                  const unsigned* __restrict__ block_offsets,
                                                                  WeldBuffers wb, unsigned* __restrict__ indices,
                                                                  unsigned max_indices) {
    __shared__ unsigned long long s_cases[256];
    __shared__ __align__(16) unsigned s_words[WELD_WARPS][512];
    __shared__ unsigned short s_list[WELD_WARPS][512];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s_cases[i] = c_mcCases[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned* words = s_words[warp];
    unsigned short* list = s_list[warp];
    const int n = active_count(av);
    for (int a = blockIdx.x * WELD_WARPS + warp; a < n; a += gridDim.x * WELD_WARPS) {
        const uint4* src = reinterpret_cast<const uint4*>(cell_words + (size_t)a * 512);
#pragma unroll
        for (int q = 0; q < 4; ++q) reinterpret_cast<uint4*>(words)[lane + 32 * q] = __ldcs(src + lane + 32 * q);
        const int lin = av.list[a];
        const unsigned long long block_v = block_offsets[a];
        int nlist = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint4 w4 = reinterpret_cast<const uint4*>(words)[lane + 32 * q];
            const unsigned wq[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const bool emits = ((wq[r] >> 8) & 31u) != 0;
                const unsigned bal = __ballot_sync(0xffffffffu, emits);
                if (emits) list[nlist + __popc(bal & ((1u << lane) - 1u))] = (unsigned short)(4 * (lane + 32 * q) + r);
                nlist += __popc(bal);
            }
        }
        __syncwarp();
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        for (int i = lane; i < nlist; i += 32) {
            const int tid = list[i];
            const unsigned w = words[tid];
            const unsigned vm = (w >> 8) & 31u;
            const CellInfo c = cell_info(g, bx, by, bz, tid);
            const unsigned long long word = s_cases[w & 255u];
            unsigned long long v = block_v + (w >> 13);
            const int nt = (int)(word & 0xF);
            for (int k = 0; k < nt; ++k) {
                if (!((vm >> k) & 1u)) continue;
                if (v + 2 >= max_indices) break;  // the soup's capacity stop
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const int e = (int)((word >> (4 + 4 * (3 * k + j))) & 0xF);
                    const int c0 = edge_c0(e), c1 = edge_c1(e);
                    const int X = c.x + min(corner_dx(c0), corner_dx(c1)), Y = c.y + min(corner_dy(c0), corner_dy(c1)),
                              Z = c.z + min(corner_dz(c0), corner_dz(c1));
                    const int axis = corner_dx(c0) != corner_dx(c1) ? 0 : (corner_dy(c0) != corner_dy(c1) ? 1 : 2);
                    const int lx = X - 8 * bx, ly = Y - 8 * by, lz = Z - 8 * bz;
                    // off this block's lower faces the edge is this block's (its cell here is in the grid)
                    const bool inner = (axis == 0 || lx >= 1) && (axis == 1 || ly >= 1) && (axis == 2 || lz >= 1);
                    int oa = a, slot = weld_slot(lx, ly, lz, axis);
                    if (!inner) {
                        const int olin = edge_owner(g, X, Y, Z, axis, wb.flags);
                        oa = wb.block_to_active[olin];
                        int obx, oby, obz;
                        block_coord(g, olin, obx, oby, obz);
                        slot = weld_slot(X - 8 * obx, Y - 8 * oby, Z - 8 * obz, axis);
                    }
                    // an owner past the rows the buffers hold has no bitmap this extraction (the engine
                    // grows them and runs again)
                    indices[v + j] = (oa >= 0 && oa < n) ? wb.base[oa] + weld_rank(wb, oa, slot) : 0u;
                }
                v += 3;
            }
        }
        __syncwarp();  // the warp's shared memory is free for the next block
    }
}

}  // namespace sdfb
