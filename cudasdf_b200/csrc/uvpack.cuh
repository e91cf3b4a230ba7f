// UV atlas packing for sm_100a: charts, island masks and the packing attempts of the reference's
// GridUVPacker (src/SDFMesh/GridUVPacker.cu), which packs the per-primitive UV charts of a mesh into
// one atlas after meshing.
//
// Layout differences from the reference, which change no result:
//  * charts are found on the GPU (a max pass, a per-primitive histogram with UV bounds as ordered
//    integer minima and maxima, a compaction in primitive order) instead of a host std::map over a
//    download of the whole mesh;
//  * every island's masks live in one word arena, and each mask stage is one launch over all islands
//    (the reference launches six kernels per island, each followed by a device synchronisation);
//  * one CTA of 256 threads runs each packing attempt (the reference runs each on one thread of a
//    256-thread block). Thread 0 draws the random numbers in the reference's order; the candidate
//    columns are evaluated one warp each; the drop search uses the board's column heights: with
//    `pf = max over island columns c of (height(x + c) - lowest cell of c)`, every position
//    y >= pf is free (each island cell lies above every board cell of its column) and, when pf > 0,
//    position pf - 1 collides (the column that attains pf touches). A drop that starts at or above
//    pf therefore ends at max(pf, 0, start - cap) without testing a position; positions below pf
//    are tested cell by cell as in the reference.
#pragma once

#include <curand_kernel.h>
#include <stdint.h>

#include "../../include/sdfmesh_b200.h"

namespace uvp {

constexpr int kMaxOrder = 256;      // islands one attempt orders and places (GridUVPacker.cu:617)
constexpr int kMaxCand = 64;        // candidate columns per rotation (GridUVPacker.cu:612)
constexpr int kPackThreads = 256;
constexpr int kPackWarps = kPackThreads / 32;
constexpr unsigned kFull = 0xffffffffu;

// (int)f as x86-64 host code converts it: NaN and out-of-range give INT_MIN (the reference's
// ExtractCharts runs on the host, GridUVPacker.cu:852-855)
__device__ __forceinline__ int host_f2i(float f) {
    return (f >= -2147483648.0f && f < 2147483648.0f) ? __float2int_rz(f) : (int)0x80000000;
}
// primitive id of a vertex as ExtractCharts reads it: (int)(f + 0.5f)
__device__ __forceinline__ int chart_prim_id(float f) { return host_f2i(__fadd_rn(f, 0.5f)); }

// float -> unsigned key with the float order (-0 below +0)
__device__ __forceinline__ unsigned fkey(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// ------------------------------------------------------------------------------------------------
// charts (ExtractCharts, GridUVPacker.cu:833-896)
// ------------------------------------------------------------------------------------------------
__global__ void k_uv_max_id(const float* __restrict__ prim, int64_t T, int* __restrict__ max_id) {
    int m = -1;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < T; t += (int64_t)gridDim.x * blockDim.x)
        m = max(m, chart_prim_id(prim[3 * t]));
    m = __reduce_max_sync(kFull, m);
    if ((threadIdx.x & 31) == 0 && m >= 0) atomicMax(max_id, m);
}

__global__ void k_uv_hist_init(unsigned* __restrict__ cnt, unsigned* __restrict__ keys, int R) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < R; i += gridDim.x * blockDim.x) {
        cnt[i] = 0u;
        keys[4 * i + 0] = fkey(1e10f);   // uvMin starts at 1e10, uvMax at -1e10 (GridUVPacker.cu:875-876)
        keys[4 * i + 1] = fkey(1e10f);
        keys[4 * i + 2] = fkey(-1e10f);
        keys[4 * i + 3] = fkey(-1e10f);
    }
}

// triangles per primitive and the UV bounds of their vertices; lanes that share an id are reduced
// first, so an id sees one group of atomics per warp
__global__ void k_uv_hist(const sdf_float2* __restrict__ uvs, const float* __restrict__ prim, int64_t T, int R,
                          unsigned* __restrict__ cnt, unsigned* __restrict__ keys) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * blockDim.x / 32;
    for (int64_t base = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x - lane); base < T; base += warps * 32) {
        const int64_t t = base + lane;
        int id = -1;
        unsigned mnx = 0xffffffffu, mny = 0xffffffffu, mxx = 0u, mxy = 0u;
        if (t < T) {
            id = chart_prim_id(prim[3 * t]);
            if (id >= R) id = -1;
            if (id >= 0)
                for (int v = 0; v < 3; v++) {
                    const sdf_float2 uv = uvs[3 * t + v];
                    if (uv.x == uv.x) { mnx = min(mnx, fkey(uv.x)); mxx = max(mxx, fkey(uv.x)); }   // fminf skips NaN
                    if (uv.y == uv.y) { mny = min(mny, fkey(uv.y)); mxy = max(mxy, fkey(uv.y)); }
                }
        }
        unsigned pending = __ballot_sync(kFull, id >= 0);
        while (pending) {
            const int leader = __ffs(pending) - 1;
            const int lid = __shfl_sync(kFull, id, leader);
            const bool mine = id == lid;
            const unsigned grp = __ballot_sync(kFull, mine);
            const unsigned a = __reduce_min_sync(kFull, mine ? mnx : 0xffffffffu);
            const unsigned b = __reduce_min_sync(kFull, mine ? mny : 0xffffffffu);
            const unsigned c = __reduce_max_sync(kFull, mine ? mxx : 0u);
            const unsigned d = __reduce_max_sync(kFull, mine ? mxy : 0u);
            if (lane == leader) {
                atomicAdd(&cnt[lid], (unsigned)__popc(grp));
                atomicMin(&keys[4 * lid + 0], a);
                atomicMin(&keys[4 * lid + 1], b);
                atomicMax(&keys[4 * lid + 2], c);
                atomicMax(&keys[4 * lid + 3], d);
            }
            pending &= ~grp;
        }
    }
}

// charts in ascending primitive id (the std::map order), one CTA of 1024 threads over the id range
__global__ void __launch_bounds__(1024) k_uv_chart_compact(const unsigned* __restrict__ cnt,
                                                           const unsigned* __restrict__ keys, int R,
                                                           int* __restrict__ chart_of_id,
                                                           sdf_uv_chart* __restrict__ charts,
                                                           int* __restrict__ num_charts) {
    __shared__ int warp_sum[32];
    __shared__ int base_s;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) base_s = 0;
    __syncthreads();
    for (int start = 0; start < R; start += 1024) {
        const int id = start + threadIdx.x;
        const int present = (id < R && cnt[id] > 0u) ? 1 : 0;
        const unsigned bal = __ballot_sync(kFull, present);
        if (lane == 0) warp_sum[warp] = __popc(bal);
        __syncthreads();
        int before = 0;
        for (int w = 0; w < warp; w++) before += warp_sum[w];
        const int base = base_s;
        const int rank = base + before + __popc(bal & ((1u << lane) - 1u));
        if (id < R) chart_of_id[id] = present ? rank : -1;
        if (present) {
            sdf_uv_chart c;
            c.primitive_id = id;
            c.num_triangles = (int32_t)cnt[id];
            c.uv_min.x = fkey_inv(keys[4 * id + 0]);
            c.uv_min.y = fkey_inv(keys[4 * id + 1]);
            c.uv_max.x = fkey_inv(keys[4 * id + 2]);
            c.uv_max.y = fkey_inv(keys[4 * id + 3]);
            charts[rank] = c;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int w = 0; w < 32; w++) tot += warp_sum[w];
            base_s = base + tot;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *num_charts = base_s;
}

__global__ void k_uv_tri_chart(const float* __restrict__ prim, int64_t T, int R, const int* __restrict__ chart_of_id,
                               int* __restrict__ tri_chart) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < T; t += (int64_t)gridDim.x * blockDim.x) {
        const int id = chart_prim_id(prim[3 * t]);
        tri_chart[t] = (id >= 0 && id < R) ? chart_of_id[id] : -1;
    }
}

// ------------------------------------------------------------------------------------------------
// island masks (CreateIslands, GridUVPacker.cu:898-1061)
// ------------------------------------------------------------------------------------------------
struct F2 { float x, y; };

// triangleArea2D (GridUVPacker.cu:41-43) with the reference's compiled rounding: where the difference
// of products is fused it is fma(t1, t2, -(t3 * t4)); otherwise both products are rounded
template <bool kFused>
__device__ __forceinline__ float area2d(F2 a, F2 b, F2 c) {
    const float t1 = __fsub_rn(b.x, a.x), t2 = __fsub_rn(c.y, a.y);
    const float t3 = __fsub_rn(c.x, a.x), t4 = __fsub_rn(b.y, a.y);
    const float v = kFused ? __fmaf_rn(t1, t2, -__fmul_rn(t3, t4)) : __fsub_rn(__fmul_rn(t1, t2), __fmul_rn(t3, t4));
    return __fmul_rn(0.5f, fabsf(v));
}
// pointInTriangle (GridUVPacker.cu:56-64) for a cell corner, as the reference's triangleOverlapsCell
// computes it: each product of area(a, p, c) and area(a, b, p) involves only the corner's x or only its
// y, the four corner tests share those products, and the compiled code rounds them on their own; the
// total and area(p, b, c) are fused. The test |total - sum| < 1e-6 decides large triangles by their
// rounding alone, so the rounding has to be the reference's.
__device__ __forceinline__ bool corner_in_triangle(F2 p, F2 a, F2 b, F2 c) {
    const float total = area2d<true>(a, b, c);
    const float s = __fadd_rn(__fadd_rn(area2d<true>(p, b, c), area2d<false>(a, p, c)), area2d<false>(a, b, p));
    return fabsf(__fsub_rn(total, s)) < 1e-6f;
}
__device__ __forceinline__ int orient_sign(F2 a, F2 b, F2 c) {
    const float ux = __fsub_rn(b.x, a.x), uy = __fsub_rn(b.y, a.y);
    const float wx = __fsub_rn(c.x, a.x), wy = __fsub_rn(c.y, a.y);
    const float v = __fmaf_rn(ux, wy, -__fmul_rn(uy, wx));
    return v > 1e-6f ? 1 : (v < -1e-6f ? -1 : 0);
}
__device__ __forceinline__ bool on_segment(F2 a, F2 b, F2 p) {
    return p.x >= __fsub_rn(fminf(a.x, b.x), 1e-6f) && p.x <= __fadd_rn(fmaxf(a.x, b.x), 1e-6f) &&
           p.y >= __fsub_rn(fminf(a.y, b.y), 1e-6f) && p.y <= __fadd_rn(fmaxf(a.y, b.y), 1e-6f);
}
__device__ __forceinline__ bool segments_intersect(F2 a, F2 b, F2 c, F2 d) {
    const int o1 = orient_sign(a, b, c), o2 = orient_sign(a, b, d), o3 = orient_sign(c, d, a), o4 = orient_sign(c, d, b);
    if (o1 != o2 && o3 != o4) return true;
    return (o1 == 0 && on_segment(a, b, c)) || (o2 == 0 && on_segment(a, b, d)) || (o3 == 0 && on_segment(c, d, a)) ||
           (o4 == 0 && on_segment(c, d, b));
}
__device__ __forceinline__ bool in_cell(F2 v, float x0, float y0, float x1, float y1) {
    return v.x >= x0 && v.x <= x1 && v.y >= y0 && v.y <= y1;
}
// triangleOverlapsCell (GridUVPacker.cu:107-165), same tests in the same order
__device__ bool triangle_overlaps_cell(F2 v0, F2 v1, F2 v2, int cx, int cy) {
    const float x0 = (float)cx, y0 = (float)cy, x1 = (float)(cx + 1), y1 = (float)(cy + 1);
    if (in_cell(v0, x0, y0, x1, y1) || in_cell(v1, x0, y0, x1, y1) || in_cell(v2, x0, y0, x1, y1)) return true;
    const F2 k[4] = {{x0, y0}, {x1, y0}, {x1, y1}, {x0, y1}};
#pragma unroll
    for (int i = 0; i < 4; i++)
        if (corner_in_triangle(k[i], v0, v1, v2)) return true;
    const F2 ta[3] = {v0, v1, v2}, tb[3] = {v1, v2, v0};
#pragma unroll
    for (int e = 0; e < 3; e++)
#pragma unroll
        for (int r = 0; r < 4; r++)
            if (segments_intersect(ta[e], tb[e], k[r], k[(r + 1) & 3])) return true;
    const F2 ctr{__fdiv_rn(__fadd_rn(__fadd_rn(v0.x, v1.x), v2.x), 3.0f),
                 __fdiv_rn(__fadd_rn(__fadd_rn(v0.y, v1.y), v2.y), 3.0f)};
    return in_cell(ctr, x0, y0, x1, y1);
}

// rasterizeIslandKernel (GridUVPacker.cu:171-225) for every triangle of every chart in one launch. A lane
// tests the cells of its own triangle when its box has at most 32 cells; a larger box (UV triangles can
// span hundreds of cells) is tested by the whole warp, one cell per lane. Cells are set with atomicOr,
// so the order of the tests changes nothing.
__global__ void k_uv_raster(const sdf_float2* __restrict__ uvs, int64_t T, const int* __restrict__ tri_chart,
                            const int* __restrict__ slot_of_chart, const sdf_uv_island* __restrict__ isl,
                            uint32_t* __restrict__ words, int res) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * blockDim.x / 32;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x + threadIdx.x - lane; base < T; base += warps * 32) {
        const int64_t t = base + lane;
        const int c = t < T ? tri_chart[t] : -1;
        F2 p[3] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
        int xMin = 0, xMax = 0, yMin = 0, yMax = 0, stride = 0;
        int64_t off = 0;
        if (c >= 0) {
            const sdf_uv_island& I = isl[slot_of_chart[c]];
            const float fr = (float)res, mx0 = (float)I.min_cell_x, my0 = (float)I.min_cell_y;
#pragma unroll
            for (int v = 0; v < 3; v++) {
                const sdf_float2 uv = uvs[3 * t + v];
                p[v] = F2{__fmaf_rn(uv.x, fr, -mx0), __fmaf_rn(uv.y, fr, -my0)};
            }
            const float minU = fminf(fminf(p[0].x, p[1].x), p[2].x), maxU = fmaxf(fmaxf(p[0].x, p[1].x), p[2].x);
            const float minV = fminf(fminf(p[0].y, p[1].y), p[2].y), maxV = fmaxf(fmaxf(p[0].y, p[1].y), p[2].y);
            const int W = I.width, H = I.height;
            xMin = max(0, min(__float2int_rz(floorf(minU)), W - 1));
            xMax = max(0, min(__float2int_rz(ceilf(maxU)), W));
            yMin = max(0, min(__float2int_rz(floorf(minV)), H - 1));
            yMax = max(0, min(__float2int_rz(ceilf(maxV)), H));
            stride = I.mask.stride;
            off = I.mask.word_offset;
        }
        const int wx = max(xMax - xMin, 0), ncell = wx * max(yMax - yMin, 0);
        const bool big = ncell > 32;
        if (c >= 0 && !big) {
            uint32_t* m = words + off;
            for (int y = yMin; y < yMax; y++)
                for (int x = xMin; x < xMax; x++)
                    if (triangle_overlaps_cell(p[0], p[1], p[2], x, y))
                        atomicOr(&m[(int64_t)y * stride + (x >> 5)], 1u << (x & 31));
        }
        unsigned todo = __ballot_sync(kFull, c >= 0 && big);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            F2 q[3];
#pragma unroll
            for (int v = 0; v < 3; v++) q[v] = F2{__shfl_sync(kFull, p[v].x, src), __shfl_sync(kFull, p[v].y, src)};
            const int qx = __shfl_sync(kFull, xMin, src), qy = __shfl_sync(kFull, yMin, src);
            const int qw = __shfl_sync(kFull, wx, src), qn = __shfl_sync(kFull, ncell, src);
            const int qs = __shfl_sync(kFull, stride, src);
            uint32_t* m = words + __shfl_sync(kFull, off, src);
            for (int k = lane; k < qn; k += 32) {
                const int x = qx + k % qw, y = qy + k / qw;
                if (triangle_overlaps_cell(q[0], q[1], q[2], x, y))
                    atomicOr(&m[(int64_t)y * qs + (x >> 5)], 1u << (x & 31));
            }
        }
    }
}

// index of the island whose item range [pre[i], pre[i + 1]) holds `item`
__device__ __forceinline__ int find_island(const int64_t* __restrict__ pre, int n, int64_t item) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// 32 cells of a grid row starting at cell `start` (cells outside the row read as empty)
__device__ __forceinline__ uint32_t row_bits(const uint32_t* __restrict__ row, int stride, int start) {
    const int q = start >> 5, sh = start & 31;
    const uint32_t w0 = (q >= 0 && q < stride) ? row[q] : 0u;
    const uint32_t w1 = (q + 1 >= 0 && q + 1 < stride) ? row[q + 1] : 0u;
    return (uint32_t)((((uint64_t)w1 << 32) | w0) >> sh);
}

// dilateGridKernel (GridUVPacker.cu:227-257), one output word per item: a cell is set when an input
// cell within the disc dx^2 + dy^2 <= r^2 is set; margin <= 0 copies the mask (GridUVPacker.cu:977-982)
__global__ void k_uv_dilate(const sdf_uv_island* __restrict__ isl, int n, const int64_t* __restrict__ pre,
                            uint32_t* __restrict__ words, int r) {
    const int64_t total = pre[n];
    for (int64_t item = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; item < total;
         item += (int64_t)gridDim.x * blockDim.x) {
        const int i = find_island(pre, n, item);
        const sdf_uv_island& I = isl[i];
        const int64_t local = item - pre[i];
        const int s = I.mask.stride, y = (int)(local / s), k = (int)(local % s);
        const uint32_t* mask = words + I.mask.word_offset;
        uint32_t out = 0u;
        if (r <= 0) {
            out = mask[local];
        } else {
            for (int dy = -r; dy <= r; dy++) {
                const int yy = y + dy;
                if (yy < 0 || yy >= I.height) continue;
                int span = r;
                while (span * span > r * r - dy * dy) span--;
                const uint32_t* row = mask + (int64_t)yy * s;
                for (int dx = -span; dx <= span; dx++) out |= row_bits(row, s, 32 * k + dx);
            }
            const int valid = I.width - 32 * k;
            if (valid < 32) out &= (1u << valid) - 1u;
        }
        words[I.collision.word_offset + local] = out;
    }
}

// rotateGridKernel with rotation 1 (90 degrees clockwise, GridUVPacker.cu:273-277) for the mask and
// the collision mask: out(x, y) = in(y, h - 1 - x); one output word per item
__global__ void k_uv_rotate(const sdf_uv_island* __restrict__ isl, int n, const int64_t* __restrict__ pre,
                            uint32_t* __restrict__ words) {
    const int64_t total = pre[n];
    for (int64_t item = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; item < total;
         item += (int64_t)gridDim.x * blockDim.x) {
        const int i = find_island(pre, n, item);
        const sdf_uv_island& I = isl[i];
        int64_t local = item - pre[i];
        const int s9 = I.mask90.stride;
        const int64_t per = (int64_t)s9 * I.width;
        const bool coll = local >= per;
        if (coll) local -= per;
        const uint32_t* src = words + (coll ? I.collision.word_offset : I.mask.word_offset);
        const int y = (int)(local / s9), k = (int)(local % s9);
        uint32_t out = 0u;
        for (int b = 0; b < 32; b++) {
            const int x = 32 * k + b;
            if (x >= I.height) break;
            const int sy = I.height - 1 - x;
            out |= ((src[(int64_t)sy * I.mask.stride + (y >> 5)] >> (y & 31)) & 1u) << b;
        }
        words[(coll ? I.collision90.word_offset : I.mask90.word_offset) + local] = out;
    }
}

// computeRowWordBoundsKernel (GridUVPacker.cu:300-339) for both collision masks, and the column
// profiles the drop search uses (lowest and highest set row of each column, -1 when empty).
// Items per island: h + w rows, then w + h columns.
__global__ void k_uv_bounds(const sdf_uv_island* __restrict__ isl, int n, const int64_t* __restrict__ pre,
                            const uint32_t* __restrict__ words, uint16_t* __restrict__ rb,
                            int32_t* __restrict__ prof) {
    const int64_t total = pre[n];
    for (int64_t item = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; item < total;
         item += (int64_t)gridDim.x * blockDim.x) {
        const int i = find_island(pre, n, item);
        const sdf_uv_island& I = isl[i];
        int q = (int)(item - pre[i]);
        const int w = I.width, h = I.height;
        if (q < h + w) {
            const bool rot = q >= h;
            const int row = rot ? q - h : q;
            const sdf_uv_grid& g = rot ? I.collision90 : I.collision;
            const uint32_t* p = words + g.word_offset + (int64_t)row * g.stride;
            int lo = -1, hi = -1;
            for (int k = 0; k < g.stride; k++)
                if (p[k] != 0u) {
                    if (lo < 0) lo = k;
                    hi = k;
                }
            uint16_t* mn = rb + (rot ? I.row_bounds90 : I.row_bounds);
            const int rows = rot ? w : h;
            mn[row] = lo < 0 ? (uint16_t)0xFFFF : (uint16_t)lo;
            mn[rows + row] = lo < 0 ? (uint16_t)0 : (uint16_t)hi;
        } else {
            q -= h + w;
            const bool rot = q >= w;
            const int col = rot ? q - w : q;
            const sdf_uv_grid& g = rot ? I.collision90 : I.collision;
            const uint32_t* p = words + g.word_offset + (col >> 5);
            const uint32_t bit = 1u << (col & 31);
            int lo = -1, hi = -1;
            for (int r = 0; r < g.height; r++)
                if (p[(int64_t)r * g.stride] & bit) {
                    if (lo < 0) lo = r;
                    hi = r;
                }
            int32_t* pr = prof + (rot ? I.profile90 : I.profile);
            const int cols = g.width;
            pr[col] = lo;
            pr[cols + col] = hi;
        }
    }
}

// ------------------------------------------------------------------------------------------------
// packing attempts (packSolutionKernel, GridUVPacker.cu:585-777)
// ------------------------------------------------------------------------------------------------
struct PackArgs {
    int G, bs;          // board side in cells, words per board row
    int align;          // X_ALIGNMENT (>= 1)
    int shelf_max;      // shelfMaxWidth
    int budget;         // candBudget
    int drop_cap;       // maxDropSteps (0 = none)
    int n;              // islands ordered per attempt: min(num_islands, 256)
    int num_islands;
    int rotation, shuffle;
};

enum { UVP_CANDIDATE_LOOP_OPEN = 1 };

struct PackGrid {
    const uint32_t* w;
    const uint16_t* mn;
    const uint16_t* mx;
    const int32_t* lowest;
    const int32_t* highest;
    int gw, gh, gs;
};

__device__ __forceinline__ PackGrid pack_grid(const sdf_uv_island& I, int rot, const uint32_t* words,
                                              const uint16_t* rb, const int32_t* prof) {
    PackGrid g;
    const sdf_uv_grid& c = rot ? I.collision90 : I.collision;
    g.w = words + c.word_offset;
    g.gw = c.width;
    g.gh = c.height;
    g.gs = c.stride;
    g.mn = rb + (rot ? I.row_bounds90 : I.row_bounds);
    g.mx = g.mn + g.gh;
    g.lowest = prof + (rot ? I.profile90 : I.profile);
    g.highest = g.lowest + g.gw;
    return g;
}

__host__ __device__ __forceinline__ int align_down(int v, int a) { return a <= 1 ? v : v - v % a; }

// checkIslandCollisionBitsAlignedRanged (GridUVPacker.cu:341-386), the rows split over the warp
__device__ bool warp_collides(const uint32_t* __restrict__ board, int bs, int G, const PackGrid& g, int ox, int oy,
                              int lane) {
    if (ox < 0 || oy < 0 || ox + g.gw > G || oy + g.gh > G) return true;
    const int ws = ox >> 5, bsh = ox & 31;
    bool hit = false;
    for (int r = lane; r < g.gh && !hit; r += 32) {
        const int lo = g.mn[r];
        if (lo == 0xFFFF) continue;
        const int wc = (int)g.mx[r] - lo + 1;
        const uint32_t* ir = g.w + (int64_t)r * g.gs + lo;
        const uint32_t* br = board + (int64_t)(oy + r) * bs + ws + lo;
        if (bsh == 0) {
            for (int k = 0; k < wc; k++)
                if (br[k] & ir[k]) { hit = true; break; }
        } else {
            uint32_t carry = 0u;
            for (int k = 0; k < wc && !hit; k++) {
                const uint32_t cur = ir[k];
                hit = (br[k] & ((cur << bsh) | carry)) != 0u;
                carry = cur >> (32 - bsh);
            }
            if (!hit && carry != 0u && ws + lo + wc < bs) hit = (br[wc] & carry) != 0u;
        }
    }
    return __any_sync(kFull, hit);
}

// final y of one candidate column (the up-scan and drop of GridUVPacker.cu:676-698), -1 when the
// column has no fit
__device__ int drop_position(const uint32_t* __restrict__ board, const PackArgs& a, const PackGrid& g,
                             const unsigned short* __restrict__ heights, int x, int uH, int lane) {
    const int y0 = min(uH, a.G - g.gh);
    if (y0 < 0) return -1;
    int pf = INT_MIN;
    for (int c = lane; c < g.gw; c += 32) {
        const int lo = g.lowest[c];
        if (lo >= 0) pf = max(pf, (int)heights[x + c] - lo);
    }
    pf = __reduce_max_sync(kFull, pf);
    if (y0 >= pf) {
        int y = max(pf, 0);
        if (a.drop_cap > 0) y = max(y, y0 - a.drop_cap);
        return y;
    }
    int y = y0;
    while (y <= a.G - g.gh && y < pf && warp_collides(board, a.bs, a.G, g, x, y, lane)) y++;
    if (y > a.G - g.gh) return -1;
    int steps = 0;
    while (y > 0) {
        if (a.drop_cap > 0 && steps >= a.drop_cap) break;
        if (y - 1 < pf && warp_collides(board, a.bs, a.G, g, x, y - 1, lane)) break;
        y--;
        steps++;
    }
    return y;
}

// writeIslandToMaskBitsAlignedRanged (GridUVPacker.cu:388-425), one row per thread
__device__ __forceinline__ void write_row(uint32_t* __restrict__ board, int bs, const PackGrid& g, int r, int ox,
                                          int oy) {
    const int lo = g.mn[r];
    if (lo == 0xFFFF) return;
    const int wc = (int)g.mx[r] - lo + 1;
    const int ws = ox >> 5, bsh = ox & 31;
    const uint32_t* ir = g.w + (int64_t)r * g.gs + lo;
    uint32_t* br = board + (int64_t)(oy + r) * bs + ws + lo;
    if (bsh == 0) {
        for (int k = 0; k < wc; k++) br[k] |= ir[k];
    } else {
        uint32_t carry = 0u;
        for (int k = 0; k < wc; k++) {
            const uint32_t cur = ir[k];
            br[k] |= (cur << bsh) | carry;
            carry = cur >> (32 - bsh);
        }
        if (carry != 0u && ws + lo + wc < bs) br[wc] |= carry;
    }
}

// One packing attempt per CTA. Dynamic shared memory: the board's column heights (G u16).
__global__ void __launch_bounds__(kPackThreads) k_uv_pack(const sdf_uv_island* __restrict__ isl, PackArgs a,
                                                           const int32_t* __restrict__ seeds,
                                                           const uint32_t* __restrict__ words,
                                                           const uint16_t* __restrict__ rb,
                                                           const int32_t* __restrict__ prof,
                                                           uint32_t* __restrict__ boards,
                                                           sdf_uv_solution* __restrict__ sols,
                                                           sdf_uv_placement* __restrict__ placements) {
    extern __shared__ unsigned short heights[];
    __shared__ int order[kMaxOrder];
    __shared__ int cand_x[2 * kMaxCand];
    __shared__ int cand_y[2 * kMaxCand];
    __shared__ int cand_n[2], cand_rot[2];
    __shared__ unsigned long long warp_best[kPackWarps];
    __shared__ int s_uW, s_uH, s_placed, s_go, s_bx, s_by, s_brot, s_flags;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int sol = blockIdx.x;
    uint32_t* board = boards + (size_t)sol * a.G * a.bs;
    sdf_uv_placement* pl = placements + (size_t)sol * a.n;

    curandState rng;  // thread 0 only
    if (tid == 0) {
        curand_init(seeds[sol], 0, 0, &rng);
        s_uW = 0;
        s_uH = 0;
        s_placed = 0;
        s_flags = 0;
    }
    for (int i = tid; i < a.G; i += kPackThreads) heights[i] = 0;
    for (int i = tid; i < a.n; i += kPackThreads) order[i] = i;
    __syncthreads();
    if (tid == 0 && a.shuffle && a.n > 1)
        for (int i = a.n - 1; i > 0; i--) {   // Fisher-Yates (GridUVPacker.cu:621-629)
            const int j = (int)(curand(&rng) % (unsigned)(i + 1));
            const int t = order[i];
            order[i] = order[j];
            order[j] = t;
        }
    __syncthreads();

    for (int oi = 0; oi < a.n; oi++) {
        const sdf_uv_island& I = isl[order[oi]];
        if (tid == 0) {
            // candidate columns for each rotation, in the reference's draw order (GridUVPacker.cu:636-665)
            const int nrot = a.rotation ? 2 : 1;
            const int rotOrder = a.rotation ? (int)(curand(&rng) & 1u) : 0;
            for (int rr = 0; rr < 2; rr++) {
                cand_n[rr] = 0;
                cand_rot[rr] = rr ^ rotOrder;
                if (rr >= nrot) continue;
                const int rot = rr ^ rotOrder;
                const int gw = rot ? I.height : I.width, gh = rot ? I.width : I.height;
                if (gw > a.G || gh > a.G) continue;
                const int maxX = min(a.shelf_max, a.G) - gw;
                if (maxX < 0) continue;
                int* cx = cand_x + rr * kMaxCand;
                int cc = 0;
                auto push = [&](int x) {
                    if (cc >= a.budget) return;
                    x = align_down(max(0, min(maxX, x)), a.align);
                    for (int k = 0; k < cc; k++)
                        if (cx[k] == x) return;
                    cx[cc++] = x;
                };
                push(0);
                push(align_down(s_uW - gw, a.align));
                push(align_down(maxX, a.align));
                // the reference draws until the budget is full; with fewer aligned columns than the
                // budget its loop never ends, here it stops once every column is listed
                const int columns = maxX / a.align + 1;
                while (cc < a.budget) {
                    if (cc >= columns) {
                        s_flags |= UVP_CANDIDATE_LOOP_OPEN;
                        break;
                    }
                    const unsigned r = curand(&rng);
                    push((int)(r % (unsigned)(maxX + 1)));
                }
                cand_n[rr] = cc;
            }
        }
        __syncthreads();
        const int n0 = cand_n[0], total = cand_n[0] + cand_n[1];
        const int uW = s_uW, uH = s_uH;
        unsigned long long best = ~0ull;
        for (int j = warp; j < total; j += kPackWarps) {
            const int rr = j < n0 ? 0 : 1;
            const int ci = rr ? j - n0 : j;
            const int idx = rr * kMaxCand + ci;
            const PackGrid g = pack_grid(I, cand_rot[rr], words, rb, prof);
            const int x = cand_x[idx];
            const int y = drop_position(board, a, g, heights, x, uH, lane);
            if (y >= 0) {
                const int newW = max(uW, x + g.gw), newH = max(uH, y + g.gh);
                const int maxDim = max(newW, newH);
                // score = area + 0.01 * maxDim^2 as the reference's compiled code rounds it (one fma)
                const float score = __fmaf_rn(0.01f, (float)(maxDim * maxDim), (float)(newW * newH));
                const unsigned long long key = ((unsigned long long)__float_as_uint(score) << 32) | (unsigned)idx;
                if (lane == 0) cand_y[idx] = y;
                best = min(best, key);
            }
        }
        if (lane == 0) warp_best[warp] = best;
        __syncthreads();
        if (tid == 0) {
            unsigned long long b = warp_best[0];
            for (int w = 1; w < kPackWarps; w++) b = min(b, warp_best[w]);
            s_go = b != ~0ull;
            if (s_go) {
                const int idx = (int)(b & 0xffffffffu);
                const int rr = idx >= kMaxCand ? 1 : 0;
                s_bx = cand_x[idx];
                s_by = cand_y[idx];
                s_brot = cand_rot[rr];
                const PackGrid g = pack_grid(I, s_brot, words, rb, prof);
                sdf_uv_placement p;
                p.island_index = I.island_index;
                p.grid_x = s_bx;
                p.grid_y = s_by;
                p.rotation = s_brot;
                pl[s_placed] = p;
                s_placed = s_placed + 1;
                s_uW = max(s_uW, s_bx + g.gw);
                s_uH = max(s_uH, s_by + g.gh);
            }
        }
        __syncthreads();
        if (!s_go) break;
        {
            const PackGrid g = pack_grid(I, s_brot, words, rb, prof);
            for (int r = tid; r < g.gh; r += kPackThreads) write_row(board, a.bs, g, r, s_bx, s_by);
            for (int c = tid; c < g.gw; c += kPackThreads) {
                const int hi = g.highest[c];
                if (hi >= 0) {
                    const int v = s_by + hi + 1;
                    if (v > heights[s_bx + c]) heights[s_bx + c] = (unsigned short)v;
                }
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        // fitness (GridUVPacker.cu:765-776)
        float fit = 0.0f;
        const int placed = s_placed, uW = s_uW, uH = s_uH;
        if (placed > 0 && uW > 0 && uH > 0) {
            const float ratio = __fdiv_rn((float)placed, (float)a.num_islands);
            const int m = max(uW, uH);
            fit = __fmul_rn(ratio, __fdiv_rn((float)(uW * uH), (float)(m * m)));
        }
        sdf_uv_solution s;
        s.num_placed = placed;
        s.utilized_width = uW;
        s.utilized_height = uH;
        s.flags = s_flags;
        s.fitness = fit;
        s.seed = seeds[sol];
        sols[sol] = s;
    }
}

// the atlas PackIslands returns (GridUVPacker.cu:1188-1214, 1403-1420)
struct AtlasResult {
    int32_t success, width, height, placed, best, open;
    float fitness, scaling;
};

// The choice of the attempt, one warp. The reference's loop keeps the first attempt with the most islands placed and replaces it
// only by a later one with as many and a strictly higher fitness: the maximum of
// (placed, fitness, -index), which the warp reduces in one 64-bit key (fitness >= 0, so its bits order).
__global__ void k_uv_select(const sdf_uv_solution* __restrict__ sols, int nsol, int num_islands, int G,
                            const sdf_uv_placement* __restrict__ placements, int n,
                            sdf_uv_placement* __restrict__ best_pl, AtlasResult* __restrict__ out) {
    const int lane = threadIdx.x;
    unsigned long long key = 0ull;
    unsigned open = 0u;
    for (int i = lane; i < nsol; i += 32) {
        const sdf_uv_solution s = sols[i];
        open |= (unsigned)(s.flags & UVP_CANDIDATE_LOOP_OPEN);
        if (s.num_placed > 0) {
            const unsigned long long k = ((unsigned long long)s.num_placed << 40) |
                                         ((unsigned long long)__float_as_uint(s.fitness) << 8) |
                                         (unsigned long long)(255 - i);
            key = max(key, k);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) key = max(key, __shfl_xor_sync(kFull, key, o));
    open = __reduce_or_sync(kFull, open);
    const int best = key ? 255 - (int)(key & 255ull) : -1;
    if (lane == 0) {
        AtlasResult r;
        r.success = 0; r.width = 0; r.height = 0; r.placed = 0; r.best = best; r.open = open ? 1 : 0;
        r.fitness = 0.0f; r.scaling = 1.0f;
        if (best >= 0) {
            const sdf_uv_solution s = sols[best];
            const int m = max(s.utilized_width, s.utilized_height);
            r.success = s.num_placed == num_islands;
            r.width = m;
            r.height = m;
            r.placed = s.num_placed;
            r.fitness = s.fitness;
            r.scaling = m > 0 ? __fdiv_rn((float)G, (float)m) : 1.0f;
        }
        *out = r;
    }
    if (best >= 0)
        for (int i = lane; i < sols[best].num_placed && i < n; i += 32) best_pl[i] = placements[(size_t)best * n + i];
}

// ------------------------------------------------------------------------------------------------
// remap (RemapUVsToAtlas + remapUVsKernel, GridUVPacker.cu:779-831, 1441-1547)
// ------------------------------------------------------------------------------------------------
struct ChartPlace {
    int32_t island_index, grid_x, grid_y, rotation;
    int32_t min_x, min_y, width, height;
};

__global__ void k_uv_remap_init(const sdf_uv_island* __restrict__ isl, int n, ChartPlace* __restrict__ cp) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const sdf_uv_island& I = isl[i];
        ChartPlace c;
        c.island_index = -1;
        c.grid_x = 0;
        c.grid_y = 0;
        c.rotation = 0;
        c.min_x = I.min_cell_x;
        c.min_y = I.min_cell_y;
        c.width = I.width;
        c.height = I.height;
        cp[I.island_index] = c;
    }
}

__global__ void k_uv_remap_place(const sdf_uv_placement* __restrict__ pl, int np, int num_charts,
                                 ChartPlace* __restrict__ cp) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        const sdf_uv_placement p = pl[i];
        if (p.island_index >= 0 && p.island_index < num_charts) {
            cp[p.island_index].island_index = p.island_index;
            cp[p.island_index].grid_x = p.grid_x;
            cp[p.island_index].grid_y = p.grid_y;
            cp[p.island_index].rotation = p.rotation;
        }
    }
}

__global__ void k_uv_remap(sdf_float2* __restrict__ uvs, const float* __restrict__ prim, int64_t nv,
                           const int* __restrict__ chart_of_id, int R, const ChartPlace* __restrict__ cp, int res,
                           float denom) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const int id = __float2int_rz(__fadd_rn(prim[v], 0.5f));   // device conversion (GridUVPacker.cu:798)
        if (id < 0) continue;
        const int c = id < R ? chart_of_id[id] : -1;
        if (c < 0) continue;
        const ChartPlace p = cp[c];
        if (p.island_index < 0) continue;
        const sdf_float2 uv = uvs[v];
        float cx = __fmaf_rn(uv.x, (float)res, -(float)p.min_x);
        float cy = __fmaf_rn(uv.y, (float)res, -(float)p.min_y);
        if (p.rotation == 1) {
            const float t = cx;
            cx = cy;
            cy = __fsub_rn((float)(p.width - 1), t);
        }
        const float ax = __fadd_rn((float)p.grid_x, cx), ay = __fadd_rn((float)p.grid_y, cy);
        if (denom <= 0.0f) continue;
        sdf_float2 o;
        o.x = __fdiv_rn(ax, denom);
        o.y = __fdiv_rn(ay, denom);
        uvs[v] = o;
    }
}

// curand(seed, 0, 0) draws for tests: the stream each packing attempt consumes
__global__ void k_uv_draws(const int32_t* __restrict__ seeds, int n, int per, uint32_t* __restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    curandState st;
    curand_init(seeds[s], 0, 0, &st);
    for (int k = 0; k < per; k++) out[(size_t)s * per + k] = curand(&st);
}

}  // namespace uvp
