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
    // adjacent cells: the edge's lower sample minus 0 or 1 along each of the two other axes
    const int ua = axis == 0 ? 1 : 0, ub = axis == 2 ? 1 : 2;  // the two other axes (ua < ub)
    int best = -1;
#pragma unroll
    for (int db = 1; db >= 0; --db) {      // the higher axis (ub) minus 1 first: smaller block index
#pragma unroll
        for (int da = 1; da >= 0; --da) {
            int c[3] = {X, Y, Z};
            c[ua] -= da;
            c[ub] -= db;
            if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] > g.w - 2 || c[1] > g.h - 2 || c[2] > g.d - 2) continue;
            const int lin = (c[0] >> 3) + g.bx * ((c[1] >> 3) + g.by * (c[2] >> 3));
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
    const int l[3] = {lx, ly, lz};
    const int b[3] = {bx, by, bz};
    const int dims[3] = {g.w, g.h, g.d};
    const int ua = axis == 0 ? 1 : 0, ub = axis == 2 ? 1 : 2;
    if (l[ua] >= 1 && l[ub] >= 1)
        return 8 * b[ua] + l[ua] - 1 <= dims[ua] - 2 && 8 * b[ub] + l[ub] - 1 <= dims[ub] - 2 &&
               8 * b[axis] + l[axis] <= dims[axis] - 2;
    return edge_owner(g, 8 * bx + lx, 8 * by + ly, 8 * bz + lz, axis, flags) == lin;
}

// Marks the owned crossed edges of every active block (one CTA per block, its row staged in shared
// memory) and counts them.
__global__ void __launch_bounds__(256) k_weld_mark(GridView g, ActiveView av, const float* __restrict__ fields,
                                                   WeldBuffers wb) {
    __shared__ float s_row[FIELD_N];
    __shared__ unsigned s_bits[WELD_STRIDE];
    const int n = active_count(av);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int a = blockIdx.x; a < n; a += gridDim.x) {
        const int lin = av.list[a];
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        const float* f = fields + (size_t)a * FIELD_STRIDE;
        for (int i = threadIdx.x; i < FIELD_N; i += blockDim.x) s_row[i] = f[i];
        __syncthreads();
        for (int s0 = 0; s0 < WELD_STRIDE * 32; s0 += blockDim.x) {
            const int s = s0 + (int)threadIdx.x;
            bool own = false;
            if (s < WELD_SLOTS) {
                const int axis = s % 3, cell = s / 3;
                const int lx = cell % 9, ly = (cell / 9) % 9, lz = cell / 81;
                const int ux = lx + (axis == 0), uy = ly + (axis == 1), uz = lz + (axis == 2);
                if (ux <= 8 && uy <= 8 && uz <= 8 && ((s_row[fidx(lx, ly, lz)] > 0.f) != (s_row[fidx(ux, uy, uz)] > 0.f)))
                    own = weld_owns(g, lin, bx, by, bz, lx, ly, lz, axis, wb.flags);
            }
            const unsigned word = __ballot_sync(0xffffffffu, own);
            if (lane == 0) s_bits[s0 / 32 + warp] = word;
        }
        __syncthreads();
        // word prefixes (72 words: three per lane of warp 0) and the block's count
        if (warp == 0) {
            const int k0 = 3 * lane;
            const unsigned c0 = k0 < WELD_STRIDE ? (unsigned)__popc(s_bits[k0]) : 0u;
            const unsigned c1 = k0 + 1 < WELD_STRIDE ? (unsigned)__popc(s_bits[k0 + 1]) : 0u;
            const unsigned c2 = k0 + 2 < WELD_STRIDE ? (unsigned)__popc(s_bits[k0 + 2]) : 0u;
            const unsigned tsum = c0 + c1 + c2;
            unsigned x = tsum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            const unsigned e = x - tsum;
            unsigned* bits = wb.bits + (size_t)a * WELD_STRIDE;
            unsigned short* pre = wb.prefix + (size_t)a * WELD_STRIDE;
            if (k0 < WELD_STRIDE) { bits[k0] = s_bits[k0]; pre[k0] = (unsigned short)e; }
            if (k0 + 1 < WELD_STRIDE) { bits[k0 + 1] = s_bits[k0 + 1]; pre[k0 + 1] = (unsigned short)(e + c0); }
            if (k0 + 2 < WELD_STRIDE) { bits[k0 + 2] = s_bits[k0 + 2]; pre[k0 + 2] = (unsigned short)(e + c0 + c1); }
            if (lane == 31) wb.totals[a] = x;
        }
        __syncthreads();
    }
}

// Rank of an owned slot among its block's owned edges.
__device__ __forceinline__ unsigned weld_rank(const WeldBuffers& wb, int a, int slot) {
    const unsigned w = wb.bits[(size_t)a * WELD_STRIDE + (slot >> 5)];
    return wb.prefix[(size_t)a * WELD_STRIDE + (slot >> 5)] + (unsigned)__popc(w & ((1u << (slot & 31)) - 1u));
}

// The welded vertices: each owned edge's point from its lower to its upper sample.
__global__ void __launch_bounds__(256) k_weld_vertices(GridView g, ActiveView av, const float* __restrict__ fields,
                                                       WeldBuffers wb, float4* __restrict__ verts, unsigned max_verts) {
    const int n = active_count(av);
    for (int a = blockIdx.x; a < n; a += gridDim.x) {
        const int lin = av.list[a];
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        const float* f = fields + (size_t)a * FIELD_STRIDE;
        const unsigned base = wb.base[a];
        for (int s = threadIdx.x; s < WELD_SLOTS; s += blockDim.x) {
            const unsigned w = wb.bits[(size_t)a * WELD_STRIDE + (s >> 5)];
            if (!((w >> (s & 31)) & 1u)) continue;
            const int axis = s % 3, cell = s / 3;
            const int lx = cell % 9, ly = (cell / 9) % 9, lz = cell / 81;
            const int ux = lx + (axis == 0), uy = ly + (axis == 1), uz = lz + (axis == 2);
            const float t = edge_t(f[fidx(lx, ly, lz)], f[fidx(ux, uy, uz)]);
            const float3 p = lerp3(grid_loc(g, bx * 8 + lx, by * 8 + ly, bz * 8 + lz),
                                   grid_loc(g, bx * 8 + ux, by * 8 + uy, bz * 8 + uz), t);
            const unsigned v = base + weld_rank(wb, a, s);
            if (v < max_verts) verts[v] = make_float4(p.x, p.y, p.z, 1.f);
        }
    }
}

// The index buffer: the soup's triangles in the soup's order (the same degenerate-triangle test on the
// same soup points), each corner replaced by its edge's welded vertex.
__global__ void __launch_bounds__(256) k_weld_indices(GridView g, ActiveView av, const float* __restrict__ fields,
                                                      const unsigned* __restrict__ cell_words,
                                                      const unsigned* __restrict__ block_offsets, WeldBuffers wb,
                                                      unsigned* __restrict__ indices, unsigned max_indices) {
    __shared__ unsigned long long s_cases[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s_cases[i] = c_mcCases[i];
    __syncthreads();
    const long long n = (long long)active_count(av) * 512;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned w = cell_words[i];
        const unsigned vm = (w >> 8) & 31u;
        if (!vm) continue;
        const int a = (int)(i >> 9), tid = (int)(i & 511);
        const int lin = av.list[a];
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        const CellInfo c = cell_info(g, bx, by, bz, tid);
        const unsigned long long word = s_cases[w & 255u];
        unsigned long long v = (unsigned long long)block_offsets[a] + (w >> 13);
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
                indices[v + j] = wb.base[oa] + weld_rank(wb, oa, slot);
            }
            v += 3;
        }
    }
}

}  // namespace sdfb
