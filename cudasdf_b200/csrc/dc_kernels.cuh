// Dual-contouring stages for sm_100a (MarchingCubesKernels.cu:1112-2044).
//
// The mark, solve and quad stages run one CTA per active block at a time, with the block's 9^3 field
// (from the shared-halo block field of marching cubes) in shared memory. The per-cell map() work of the reference (4 evaluations per Hermite point for
// its normal, 4 at the solved vertex, 4 + 1 per quad, 24 per quad for output normals) is irregular,
// so it is first compacted into per-block lists in shared memory and then evaluated 32 points per
// warp-coherent call. Every arithmetic step follows the reference's order (see sdf_device.cuh).
#pragma once

#include "mc_kernels.cuh"

namespace sdfb {

struct DcBuffers {
    int* block_to_active;     // dense block index -> active id, -1 if inactive
    unsigned char* masks;     // per packed cell: corner sign mask
    unsigned* vert_offsets;   // per packed cell: exclusive scan of has-vertex
    ushort4* cell_verts;      // per DC vertex: quantised position in its cell
    short4* cell_normals;     // per DC vertex: quantised normal
    short4* cell_normals_tmp; // smoothing output
    unsigned* counts;         // per packed cell: has-vertex (mark) / quad vertex count (count quads)
    unsigned* offsets;        // per packed cell: scanned counts
    float4* qef_debug;        // optional, per DC vertex: mass-point QEF vertex before projection, w = 1 if FP64
    // optional, mass-point projection: per DC vertex below proj_cap, two float4 (start point in cell-local
    // coordinates, active block; mean Hermite normal, cell | has-direction << 16) for k_dc_project, and
    // the raw Hermite normal sum when cell normals are written
    float4* proj;
    float4* proj_nsum;
    unsigned proj_cap;
    // optional, Hermite normals evaluated across blocks (k_dc_hermite_reps / k_dc_hermite_normals): per
    // active block its first sample, first representative and their counts (x < 0: not listed, k_dc_solve
    // evaluates its normals itself), per sample its representative, per representative the normal
    int4* hbase;
    const unsigned* hsample_rep;
    const float4* hnormals;
    // optional, the quads' winding normals evaluated across blocks (k_dc_quad_list / k_dc_quad_normals),
    // per counted quad in emission order (quad q = its first vertex / 6), q < qcap
    const float4* qnormals;
    unsigned qcap;
};

struct DcSolveParams {
    unsigned max_cell_vertices;
    float qef_blend;
    int solver;             // SDF_DC_SOLVER_REFERENCE / SDF_DC_SOLVER_MASSPOINT
    int projection_iters;   // mass-point solver only
    float cond_threshold;   // mass-point solver only: FP64 eigensolve above this condition number
};

struct DcQuadParams {
    int adaptive_diagonal;  // split along the shorter diagonal (0 = the reference's fixed (0,1,2),(0,2,3))
};

__device__ __forceinline__ bool surface_mask(unsigned char m) { return m != 0x00 && m != 0xFF; }

// buildBlockToActiveMap (:1303-1310)
__global__ void k_dc_block_map(const int* __restrict__ list, const int* __restrict__ count_dev, int cap,
                               int max_blocks, int* __restrict__ b2a) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = min(*count_dev, cap);
    if (a >= n) return;
    const int b = list[a];
    if (b >= 0 && b < max_blocks) b2a[b] = a;
}

// dcMarkCells (:1312-1346): corner masks + has-vertex counts. With fields_out the block field is
// also stored for the solve pass.
// rows_ready: the block rows in fields_out are already complete (the engine's shared-halo block field);
// the kernel then only classifies the cells
__global__ void __launch_bounds__(BLK_THREADS) k_dc_mark(GridView g0, SceneView sc0, float time, ActiveView av,
                                                         float* __restrict__ fields_out, DcBuffers B, unsigned* ticket,
                                                         Diag* diag, bool rows_ready = false) {
    __shared__ __align__(16) float s_field[FIELD_STRIDE];
    __shared__ int s_item;
    const int n = active_count(av);
    for (;;) {
        const int a = claim(ticket, n, &s_item);
        if (a < 0) break;
        GridView g = g0;
        SceneView sc = sc0;
        int lin;
        unsigned bbase;
        resolve(av, av.list[a], g, sc, lin, bbase);
        if (rows_ready) {
            const float4* src = reinterpret_cast<const float4*>(fields_out + (size_t)a * FIELD_STRIDE);
            float4* dst = reinterpret_cast<float4*>(s_field);
            for (int i = threadIdx.x; i < FIELD_STRIDE / 4; i += blockDim.x) dst[i] = src[i];
        } else {
            eval_block_field(g, sc, time, lin, s_field, diag);
        }
        if (threadIdx.x < FIELD_STRIDE - FIELD_N) s_field[FIELD_N + threadIdx.x] = 0.f;
        __syncthreads();
        if (fields_out && !rows_ready) {
            float4* dst = reinterpret_cast<float4*>(fields_out + (size_t)a * FIELD_STRIDE);
            const float4* src = reinterpret_cast<const float4*>(s_field);
            for (int i = threadIdx.x; i < FIELD_STRIDE / 4; i += blockDim.x) dst[i] = src[i];
        }
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        unsigned char m2[2];
        unsigned c2[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const CellInfo c = cell_info(g, bx, by, bz, 2 * threadIdx.x + h);
            unsigned char m = 0;
            if (!c.oob) {
                float cv[8];
                m = (unsigned char)cell_case(s_field, c.lx, c.ly, c.lz, cv);
            }
            m2[h] = m;
            c2[h] = surface_mask(m) ? 1u : 0u;
        }
        *reinterpret_cast<uchar2*>(B.masks + (size_t)a * 512 + 2 * threadIdx.x) = make_uchar2(m2[0], m2[1]);
        *reinterpret_cast<uint2*>(B.counts + (size_t)a * 512 + 2 * threadIdx.x) = make_uint2(c2[0], c2[1]);
    }
}

// ------------------------------------------------------------------------------------------------
// QEF solvers (MarchingCubesKernels.cu:1185-1301)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ bool solve3x3(const float A[9], const float b[3], float x[3]) {
    const float a00 = A[0], a01 = A[1], a02 = A[2], a10 = A[3], a11 = A[4], a12 = A[5], a20 = A[6], a21 = A[7],
                a22 = A[8];
    const float det = FMA(a02, det2(a10, a21, a11, a20), FMA(a00, det2(a11, a22, a12, a21), -MUL(a01, det2(a10, a22, a12, a20))));
    if (fabsf(det) < 1e-12f) return false;
    const float inv = DIV(1.f, det);
    const float bx = b[0], by = b[1], bz = b[2];
    const float dX = FMA(a02, det2(by, a21, a11, bz), FMA(bx, det2(a11, a22, a12, a21), -MUL(a01, det2(by, a22, a12, bz))));
    const float dY = FMA(a02, det2(a10, bz, by, a20), FMA(a00, det2(by, a22, a12, bz), -MUL(bx, det2(a10, a22, a12, a20))));
    const float dZ = FMA(bx, det2(a10, a21, a11, a20), FMA(a00, FMA(-by, a21, MUL(a11, bz)), -MUL(a01, det2(a10, bz, by, a20))));
    x[0] = MUL(dX, inv);
    x[1] = MUL(dY, inv);
    x[2] = MUL(dZ, inv);
    return true;
}

// ------------------------------------------------------------------------------------------------
// codecs (MarchingCubesKernels.cu:1133-1182)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ float3 normalize_or_up(float3 n) {
    const float len = SQRT(dot3(n, n));
    if (len > 1e-6f) return f3(DIV(n.x, len), DIV(n.y, len), DIV(n.z, len));
    return f3(0.f, 1.f, 0.f);
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ short4 encode_normal(float3 n) {
    n = normalize_or_up(n);
    short4 o;
    o.x = (short)clampi((int)lrintf(MUL(CLAMP(n.x, -1.f, 1.f), 32767.f)), -32767, 32767);
    o.y = (short)clampi((int)lrintf(MUL(CLAMP(n.y, -1.f, 1.f), 32767.f)), -32767, 32767);
    o.z = (short)clampi((int)lrintf(MUL(CLAMP(n.z, -1.f, 1.f), 32767.f)), -32767, 32767);
    o.w = 0;
    return o;
}
__device__ __forceinline__ float3 decode_normal(short4 q) {
    const float inv = 1.0f / 32767.0f;
    return normalize_or_up(f3(MUL((float)q.x, inv), MUL((float)q.y, inv), MUL((float)q.z, inv)));
}
__device__ __forceinline__ ushort4 encode_vertex(float3 p, float3 cmin, float cell) {
    const float tx = CLAMP(DIV(SUB(p.x, cmin.x), cell), 0.f, 1.f);
    const float ty = CLAMP(DIV(SUB(p.y, cmin.y), cell), 0.f, 1.f);
    const float tz = CLAMP(DIV(SUB(p.z, cmin.z), cell), 0.f, 1.f);
    ushort4 o;
    o.x = (unsigned short)clampi((int)lrintf(MUL(tx, 65535.f)), 0, 65535);
    o.y = (unsigned short)clampi((int)lrintf(MUL(ty, 65535.f)), 0, 65535);
    o.z = (unsigned short)clampi((int)lrintf(MUL(tz, 65535.f)), 0, 65535);
    o.w = 0;
    return o;
}
__device__ __forceinline__ float3 decode_vertex(ushort4 q, float3 cmin, float cell) {
    const float inv = 1.0f / 65535.0f;
    return f3(FMA(MUL((float)q.x, inv), cell, cmin.x), FMA(MUL((float)q.y, inv), cell, cmin.y),
              FMA(MUL((float)q.z, inv), cell, cmin.z));
}

}  // namespace sdfb
#include "qef_masspoint.cuh"
namespace sdfb {

// ------------------------------------------------------------------------------------------------
// dcSolveCellVertices (:1348-1597)
// ------------------------------------------------------------------------------------------------
// threads of a k_dc_solve CTA (measured at 512^3: 23 ms; 31 ms with 128, 49 ms with 64)
constexpr int SOLVE_THREADS = 256;
constexpr int DC_CELL_CAP = 2 * SOLVE_THREADS;            // cells per pass (two per thread)
constexpr int DC_HERMITE_CAP = 6 * SOLVE_THREADS;         // Hermite samples staged per pass
constexpr int DC_EDGE_KEYS = 729 * 6;   // start corner in the 9^3 lattice x axis x direction

struct SolveSmem {
    float field[FIELD_STRIDE];
    unsigned warp_sums[SOLVE_THREADS / 32];
    // solve cells of the current pass
    unsigned short cell_tid[DC_CELL_CAP];
    unsigned cell_vidx[DC_CELL_CAP];
    unsigned short cell_h0[DC_CELL_CAP];   // first Hermite entry of the cell
    unsigned char cell_m[DC_CELL_CAP];
    float3 cell_x[DC_CELL_CAP];
    // Hermite samples of the current pass
    unsigned short h_cell[DC_HERMITE_CAP];  // (cell tid << 4) | edge
    float3 h_n[DC_HERMITE_CAP];
    // one normal per (edge, direction) of the pass: the sample that claimed the key evaluates it
    unsigned short edge_rep[DC_EDGE_KEYS];  // key -> representative sample, 0xFFFF if unclaimed
    unsigned short h_rep[DC_HERMITE_CAP];   // sample -> its representative
    unsigned short rep_list[DC_HERMITE_CAP];
    // computeNormal stencils spread over all warps: map() at (p, p + h x, p + h y, p + h z) of up to
    // STENCIL_CHUNK centres at a time, one point per lane
    float st_d[4 * 256];
    int nrep;
    int next_cursor;
    int item;
};
constexpr int STENCIL_CHUNK = 256;

// The four-point stencil (MarchingCubesKernels.cu:814-844) of n centres, spread over all warps of the
// CTA (lane i of the pass takes centre i / 4, offset i % 4), STENCIL_CHUNK centres per round; `use`
// receives (centre, d0, d1, d2, d3) from one thread per centre. Called by all threads.
template <class Centre, class Use>
__device__ __forceinline__ void stencil_all_warps(const SceneView& sc, int n, float cell, float time, float* st_d,
                                                  Centre centre, Use use, Diag* diag) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const float h = MUL(cell, 0.001f);
    for (int c0 = 0; c0 < n; c0 += STENCIL_CHUNK) {
        const int cn = min(STENCIL_CHUNK, n - c0);
        for (int base = warp * 32; base < 4 * cn; base += nwarps * 32) {
            const int i = base + lane;
            const bool valid = i < 4 * cn;
            float3 p = f3(0.f, 0.f, 0.f);
            if (valid) {
                const float3 c = centre(c0 + (i >> 2));
                const int k = i & 3;
                p = k == 0 ? c : (k == 1 ? f3(ADD(c.x, h), c.y, c.z) : (k == 2 ? f3(c.x, ADD(c.y, h), c.z)
                                                                               : f3(c.x, c.y, ADD(c.z, h))));
            }
            MapState<false> st;
            map_warp<false>(sc, p, valid, time, st, diag);
            if (valid) st_d[i] = st.d;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < cn; j += blockDim.x)
            use(c0 + j, st_d[4 * j], st_d[4 * j + 1], st_d[4 * j + 2], st_d[4 * j + 3]);
        __syncthreads();
    }
}

__device__ __forceinline__ float3 hermite_point(const GridView& g, const CellInfo& c, const float cv[8], int e) {
    return edge_point(g, c.x, c.y, c.z, cv, e);
}

// the reference solver for one cell: feature clustering, plane intersections, regularised QEF
__device__ float3 solve_reference(const GridView& g, const CellInfo& c, const float cv[8], const SolveSmem& S,
                                  int h0, int m) {
    const float3 cmin = grid_loc(g, c.x, c.y, c.z);
    float3 xs = f3(FMA(0.5f, g.cell, cmin.x), FMA(0.5f, g.cell, cmin.y), FMA(0.5f, g.cell, cmin.z));
    float3 centroid = xs;
    if (m > 0) {
        float3 sum = f3(0.f, 0.f, 0.f);
        for (int i = 0; i < m; ++i) sum = add3(sum, hermite_point(g, c, cv, S.h_cell[h0 + i] & 15));
        centroid = scl3(sum, DIV(1.f, (float)m));
    }
    float3 cN[3] = {f3(0, 0, 0), f3(0, 0, 0), f3(0, 0, 0)}, cP[3] = {f3(0, 0, 0), f3(0, 0, 0), f3(0, 0, 0)};
    int cC[3] = {0, 0, 0}, k = 0;
    for (int i = 0; i < m; ++i) {
        float3 n = S.h_n[h0 + i];
        const float len = SQRT(dot3(n, n));
        if (len < 1e-6f) continue;
        n = f3(DIV(n.x, len), DIV(n.y, len), DIV(n.z, len));
        const float3 p = hermite_point(g, c, cv, S.h_cell[h0 + i] & 15);
        int best = -1;
        float bestDot = -1.f;
        for (int ci = 0; ci < k; ++ci) {
            float3 cn = cN[ci];
            const float cl = SQRT(dot3(cn, cn));
            if (cl > 1e-6f) cn = f3(DIV(cn.x, cl), DIV(cn.y, cl), DIV(cn.z, cl));
            const float d = fabsf(dot3(cn, n));
            if (d > bestDot) { bestDot = d; best = ci; }
        }
        if (best >= 0 && bestDot > 0.92f) {
            cN[best] = add3(cN[best], n); cP[best] = add3(cP[best], p); cC[best]++;
        } else if (k < 3) {
            cN[k] = n; cP[k] = p; cC[k] = 1; k++;
        } else {
            cN[best] = add3(cN[best], n); cP[best] = add3(cP[best], p); cC[best]++;
        }
    }
    bool solved = false;
    float3 xsol = xs;
    if (k >= 2) {
        float3 n1 = cN[0], n2 = cN[1], n3 = cN[2];
        const float l1 = SQRT(dot3(n1, n1)), l2 = SQRT(dot3(n2, n2)), l3 = SQRT(dot3(n3, n3));
        if (l1 > 1e-6f && l2 > 1e-6f) {
            n1 = f3(DIV(n1.x, l1), DIV(n1.y, l1), DIV(n1.z, l1));
            n2 = f3(DIV(n2.x, l2), DIV(n2.y, l2), DIV(n2.z, l2));
            if (l3 > 1e-6f) n3 = f3(DIV(n3.x, l3), DIV(n3.y, l3), DIV(n3.z, l3));
            const float d12 = fabsf(dot3(n1, n2));
            const float d13 = (k >= 3 && l3 > 1e-6f) ? fabsf(dot3(n1, n3)) : 1.f;
            const float d23 = (k >= 3 && l3 > 1e-6f) ? fabsf(dot3(n2, n3)) : 1.f;
            const bool c01 = cC[0] >= 2 && cC[1] >= 2;
            const bool c012 = c01 && k >= 3 && cC[2] >= 2 && l3 > 1e-6f;
            const bool doEdge = k == 2 && c01 && d12 < 0.75f;
            const bool doCorner = k >= 3 && c012 && d12 < 0.80f && d13 < 0.80f && d23 < 0.80f;
            if (doEdge || doCorner) {
                const float i0 = DIV(1.f, (float)(cC[0] > 0 ? cC[0] : 1)), i1 = DIV(1.f, (float)(cC[1] > 0 ? cC[1] : 1));
                const float3 p1 = scl3(cP[0], i0), p2 = scl3(cP[1], i1);
                float A[9], b[3], sol[3];
                if (doEdge) {
                    float3 ne = cross_ff(n1, n2);
                    const float le = SQRT(dot3(ne, ne));
                    if (le > 1e-6f) {
                        ne = f3(DIV(ne.x, le), DIV(ne.y, le), DIV(ne.z, le));
                        float3 pa = f3(0.f, 0.f, 0.f);
                        for (int i = 0; i < m; ++i) pa = add3(pa, hermite_point(g, c, cv, S.h_cell[h0 + i] & 15));
                        pa = scl3(pa, DIV(1.f, (float)(m > 0 ? m : 1)));
                        A[0] = n1.x; A[1] = n1.y; A[2] = n1.z; A[3] = n2.x; A[4] = n2.y; A[5] = n2.z;
                        A[6] = ne.x; A[7] = ne.y; A[8] = ne.z;
                        b[0] = dot3(n1, p1); b[1] = dot3(n2, p2); b[2] = dot3(ne, pa);
                        if (solve3x3(A, b, sol)) { xsol = f3(sol[0], sol[1], sol[2]); solved = true; }
                    }
                } else {
                    const float i2 = DIV(1.f, (float)(cC[2] > 0 ? cC[2] : 1));
                    const float3 p3 = scl3(cP[2], i2);
                    A[0] = n1.x; A[1] = n1.y; A[2] = n1.z; A[3] = n2.x; A[4] = n2.y; A[5] = n2.z;
                    A[6] = n3.x; A[7] = n3.y; A[8] = n3.z;
                    b[0] = dot3(n1, p1); b[1] = dot3(n2, p2); b[2] = dot3(n3, p3);
                    if (solve3x3(A, b, sol)) { xsol = f3(sol[0], sol[1], sol[2]); solved = true; }
                }
            }
        }
    }
    if (!solved && m > 0) {
        // solveQEFRegularized (alpha 0.05, lambda 1e-6), then solveQEF (lambda 1e-5) as fallback
        float M[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, rhs[3] = {0, 0, 0};
        for (int i = 0; i < m; ++i) {
            float3 n = S.h_n[h0 + i];
            const float len = SQRT(dot3(n, n));
            if (len < 1e-6f) continue;
            n = f3(DIV(n.x, len), DIV(n.y, len), DIV(n.z, len));
            const float d = dot3(n, hermite_point(g, c, cv, S.h_cell[h0 + i] & 15));
            M[0] = FMA(n.x, n.x, M[0]); M[1] = FMA(n.x, n.y, M[1]); M[2] = FMA(n.x, n.z, M[2]);
            M[3] = FMA(n.y, n.x, M[3]); M[4] = FMA(n.y, n.y, M[4]); M[5] = FMA(n.y, n.z, M[5]);
            M[6] = FMA(n.z, n.x, M[6]); M[7] = FMA(n.z, n.y, M[7]); M[8] = FMA(n.z, n.z, M[8]);
            rhs[0] = FMA(n.x, d, rhs[0]); rhs[1] = FMA(n.y, d, rhs[1]); rhs[2] = FMA(n.z, d, rhs[2]);
        }
        float Mr[9], rr[3], x[3];
        for (int q = 0; q < 9; ++q) Mr[q] = M[q];
        const float a = 0.05f;
        Mr[0] = ADD(Mr[0], a); Mr[4] = ADD(Mr[4], a); Mr[8] = ADD(Mr[8], a);
        rr[0] = FMA(a, centroid.x, rhs[0]); rr[1] = FMA(a, centroid.y, rhs[1]); rr[2] = FMA(a, centroid.z, rhs[2]);
        Mr[0] = ADD(Mr[0], 1e-6f); Mr[4] = ADD(Mr[4], 1e-6f); Mr[8] = ADD(Mr[8], 1e-6f);
        if (solve3x3(Mr, rr, x)) {
            xsol = f3(x[0], x[1], x[2]);
        } else {
            M[0] = ADD(M[0], 1e-5f); M[4] = ADD(M[4], 1e-5f); M[8] = ADD(M[8], 1e-5f);
            if (solve3x3(M, rhs, x)) xsol = f3(x[0], x[1], x[2]);
        }
    }
    return xsol;
}

// the (edge, direction) key of Hermite sample (cell tid, edge e) in the block's 9^3 lattice: the cells
// around an edge that name it with the same direction share the key, the edge point and the normal
__device__ __forceinline__ int hermite_key(int tid, int e) {
    const int c0 = edge_c0(e), c1 = edge_c1(e);
    const int d0 = corner_dx(c0) + 2 * corner_dy(c0) + 4 * corner_dz(c0);
    const int d1 = corner_dx(c1) + 2 * corner_dy(c1) + 4 * corner_dz(c1);
    const int lo = d0 < d1 ? c0 : c1;  // the edge's lower corner
    const int axis = (d0 ^ d1) == 1 ? 0 : ((d0 ^ d1) == 2 ? 1 : 2);
    const int sx = (tid & 7) + corner_dx(lo), sy = ((tid >> 3) & 7) + corner_dy(lo), sz = (tid >> 6) + corner_dz(lo);
    return ((sz * 9 + sy) * 9 + sx) * 6 + axis * 2 + (d0 < d1 ? 0 : 1);
}

// the edge mask of a solved cell (sign-changing edges), 0 for a cell k_dc_solve does not solve
__device__ __forceinline__ unsigned solved_cell_edges(const GridView& g, const DcBuffers& B, const DcSolveParams& P,
                                                      const float* field, int a, int bx, int by, int bz, int tid,
                                                      CellInfo& c, float (&cv)[8]) {
    const size_t pk = (size_t)a * 512 + tid;
    if (B.counts[pk] == 0) return 0u;
    c = cell_info(g, bx, by, bz, tid);
    if (c.oob) return 0u;
    if (B.vert_offsets[pk] >= P.max_cell_vertices) return 0u;
    const int mask = cell_case(field, c.lx, c.ly, c.lz, cv);
    unsigned em = 0;
    for (int e = 0; e < 12; ++e)
        if (((mask >> edge_c0(e)) & 1) != ((mask >> edge_c1(e)) & 1)) em |= 1u << e;
    return em;
}

// Lists every active block's Hermite samples in k_dc_solve's order (cells in order, edges in order)
// with the representative of each (edge, direction): its first sample in that order. Each block
// reserves a range of samples and representatives in the global lists; writes each sample's
// representative index and each representative's edge point (w: the active block). A block whose range
// does not fit keeps hbase.x = -1 and k_dc_solve evaluates its normals itself.
struct HermSmem {
    float field[FIELD_STRIDE];
    unsigned key_tab[DC_EDGE_KEYS];  // first sample of each key, then its representative number
    unsigned warp_sums[SOLVE_THREADS / 32];
    int base_s, base_r, item;
};

__global__ void __launch_bounds__(SOLVE_THREADS) k_dc_hermite_reps(GridView g0, ActiveView av,
                                                                  const float* __restrict__ fields, DcBuffers B,
                                                                  DcSolveParams P, unsigned* __restrict__ counters,
                                                                  unsigned* __restrict__ sample_rep, float4* __restrict__ reps,
                                                                  unsigned sample_cap, unsigned rep_cap, unsigned* ticket) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    HermSmem& S = *reinterpret_cast<HermSmem*>(dyn_smem);
    const int n = active_count(av);
    for (;;) {
        const int a = claim(ticket, n, &S.item);
        if (a < 0) break;
        GridView g = g0;
        SceneView unused;
        int lin;
        unsigned bbase;
        resolve(av, av.list[a], g, unused, lin, bbase);
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        const float4* src = reinterpret_cast<const float4*>(fields + (size_t)a * FIELD_STRIDE);
        for (int i = threadIdx.x; i < FIELD_STRIDE / 4; i += blockDim.x) reinterpret_cast<float4*>(S.field)[i] = src[i];
        for (int k = threadIdx.x; k < DC_EDGE_KEYS; k += blockDim.x) S.key_tab[k] = 0xFFFFFFFFu;
        __syncthreads();
        // this thread's two cells: their edge masks and sample counts
        unsigned em[2];
        CellInfo ci[2];
        float cvs[2][8];
#pragma unroll
        for (int h = 0; h < 2; ++h) em[h] = solved_cell_edges(g, B, P, S.field, a, bx, by, bz, 2 * threadIdx.x + h, ci[h], cvs[h]);
        const unsigned mine = __popc(em[0]) + __popc(em[1]);
        unsigned total = 0;
        const unsigned k0 = block_exclusive<SOLVE_THREADS>(mine, S.warp_sums, &total);
        // the first sample of every key
        unsigned k = k0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
            for (int e = 0; e < 12; ++e)
                if ((em[h] >> e) & 1u) atomicMin(&S.key_tab[hermite_key(2 * threadIdx.x + h, e)], k++);
        __syncthreads();
        unsigned nr = 0;
        k = k0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
            for (int e = 0; e < 12; ++e)
                if ((em[h] >> e) & 1u) nr += S.key_tab[hermite_key(2 * threadIdx.x + h, e)] == k++ ? 1u : 0u;
        unsigned rtotal = 0;
        const unsigned r0 = block_exclusive<SOLVE_THREADS>(nr, S.warp_sums, &rtotal);
        if (threadIdx.x == 0) {
            const unsigned bs = total ? atomicAdd(&counters[0], total) : 0u;
            const unsigned br = rtotal ? atomicAdd(&counters[1], rtotal) : 0u;
            const bool fits = (unsigned long long)bs + total <= sample_cap && (unsigned long long)br + rtotal <= rep_cap;
            S.base_s = fits ? (int)bs : -1;
            S.base_r = fits ? (int)br : -1;
            B.hbase[a] = make_int4(S.base_s, S.base_r, (int)total, (int)rtotal);
        }
        __syncthreads();  // key_tab holds first samples until every thread has tested its own
        const int bs = S.base_s, br = S.base_r;
        if (bs >= 0) {
            // representatives: their number replaces the key's first sample, and their edge point is listed
            unsigned r = r0;
            k = k0;
            int rep_keys[24];
            int nrk = 0;
#pragma unroll
            for (int h = 0; h < 2; ++h)
                for (int e = 0; e < 12; ++e)
                    if ((em[h] >> e) & 1u) {
                        const int key = hermite_key(2 * threadIdx.x + h, e);
                        if (S.key_tab[key] == k) {
                            const float3 pt = edge_point(g, ci[h].x, ci[h].y, ci[h].z, cvs[h], e);
                            reps[(size_t)br + r] = make_float4(pt.x, pt.y, pt.z, __int_as_float(a));
                            rep_keys[nrk++] = key;
                            ++r;
                        }
                        ++k;
                    }
            __syncthreads();  // every first-sample test is done before the table is overwritten
            r = r0;
            for (int q = 0; q < nrk; ++q) S.key_tab[rep_keys[q]] = r++;
            __syncthreads();
            k = k0;
#pragma unroll
            for (int h = 0; h < 2; ++h)
                for (int e = 0; e < 12; ++e)
                    if ((em[h] >> e) & 1u)
                        sample_rep[(size_t)bs + k++] = (unsigned)br + S.key_tab[hermite_key(2 * threadIdx.x + h, e)];
        }
    }
}

// computeNormal (:814-844) at centre c, its four stencil points held by two neighbouring lanes (even lane:
// c and c + h z; odd lane: c + h x and c + h y) and walked two per lane by map_pair, one scene's BVH at a
// time (bbase: the lane's scene block base). The normal is returned on the even lane of each pair.
__device__ __forceinline__ float3 stencil_normal_pairs(const ActiveView& av, const SceneView& sc, unsigned bbase,
                                                       float3 c, float cell, bool live, float time, Diag* diag) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool odd = (lane & 1) != 0;
    const float h = MUL(cell, 0.001f);
    const float3 pa = odd ? f3(ADD(c.x, h), c.y, c.z) : c;
    const float3 pb = odd ? f3(c.x, ADD(c.y, h), c.z) : f3(c.x, c.y, ADD(c.z, h));
    float da = 0.f, db = 0.f;
    unsigned pending = __ballot_sync(FULL, live);
    while (pending) {
        const unsigned lead = __shfl_sync(FULL, bbase, __ffs(pending) - 1);
        const bool mine = live && bbase == lead && ((pending >> lane) & 1u);
        SceneView scw = sc;
        if (av.scenes) scw = av.scenes[scene_of_block(av.scenes, av.nscenes, lead)].sc;
        float a, b;
        map_pair<false, false>(scw, pa, pb, mine, mine, time, a, b, diag);
        if (mine) {
            da = a;
            db = b;
        }
        pending &= ~__ballot_sync(FULL, mine);
    }
    const float d1 = __shfl_xor_sync(FULL, da, 1), d2 = __shfl_xor_sync(FULL, db, 1);  // the odd lane's points
    const float3 gr = f3(SUB(d1, da), SUB(d2, da), SUB(db, da));
    const float len = SQRT(dot3(gr, gr));
    return len > 1e-6f ? f3(DIV(gr.x, len), DIV(gr.y, len), DIV(gr.z, len)) : f3(0.f, 1.f, 0.f);
}

// computeNormal at every listed representative's edge point, 16 per warp task with two stencil points
// per lane on two lanes (measured faster than four lanes of one point, and than 32 representatives
// with their four points walked together per lane)
__global__ void __launch_bounds__(BLK_THREADS) k_dc_hermite_normals(GridView g0, SceneView sc0, float time,
                                                                   ActiveView av, const float4* __restrict__ reps,
                                                                   const unsigned* __restrict__ counters, unsigned rep_cap,
                                                                   float4* __restrict__ normals, unsigned* ticket,
                                                                   Diag* diag) {
    const unsigned n = min(counters[1], rep_cap);
    const int nact = active_count(av);
    const int tasks = nact > 0 ? (int)((n + 15u) / 16u) : 0;
    const int lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;
    for (;;) {
        int t = 0;
        if (lane == 0) t = (int)atomicAdd(ticket, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= tasks) break;
        const unsigned r = (unsigned)t * 16u + (unsigned)(lane >> 1);
        const bool in = r < n;
        const float4 rec = reps[in ? r : (unsigned)t * 16u];
        const int ra = __float_as_int(rec.w);
        const bool live = in && ra >= 0 && ra < nact;
        GridView g = g0;
        SceneView sc = sc0;
        int lin;
        unsigned bbase;
        resolve(av, av.list[live ? ra : 0], g, sc, lin, bbase);
        const float3 nn = stencil_normal_pairs(av, sc, bbase, f3(rec.x, rec.y, rec.z), g.cell, live, time, diag);
        if (live && (lane & 1) == 0) normals[r] = make_float4(nn.x, nn.y, nn.z, 0.f);
    }
}

// value and normalised gradient (computeNormal's differences) at the 32 points of a warp
__device__ __forceinline__ float3 value_gradient_warp(const SceneView& sc, float3 p, bool valid, float time,
                                                      float cell, float& d, Diag* diag) {
    float dd[4];
    stencil4_warp(sc, p, valid, time, cell, dd, diag);
    d = dd[0];
    const float3 gr = f3(SUB(dd[1], dd[0]), SUB(dd[2], dd[0]), SUB(dd[3], dd[0]));
    const float len = SQRT(dot3(gr, gr));
    if (len > 1e-6f) return f3(DIV(gr.x, len), DIV(gr.y, len), DIV(gr.z, len));
    return f3(0.f, 0.f, 0.f);
}

// three CTAs per SM (80 registers): measured 23 ms for the 512^3 solve against 29 ms at 116 registers
__global__ void __launch_bounds__(SOLVE_THREADS, 3) k_dc_solve(GridView g0, SceneView sc0, float time, ActiveView av,
                                                          const float* __restrict__ fields_in, DcBuffers B,
                                                          DcSolveParams P, unsigned* ticket, Diag* diag) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    SolveSmem& S = *reinterpret_cast<SolveSmem*>(dyn_smem);
    const int n = active_count(av);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
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
        // the block's samples listed by k_dc_hermite_reps (their normals already evaluated), if any
        const int4 hbase = B.hbase ? B.hbase[a] : make_int4(-1, -1, 0, 0);
        const int hb = hbase.x;
        unsigned hk0 = 0;  // samples of the earlier passes
        // The cells that get a vertex are processed in cell order, in passes bounded by the Hermite
        // staging capacity (a cell has at most 12 samples, so every pass makes progress).
        int cursor = 0;
        while (cursor < 512) {
            unsigned want[2] = {0, 0}, hm[2] = {0, 0}, vi[2] = {0, 0};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int tid = cursor + 2 * threadIdx.x + h;
                if (tid >= 512) continue;
                const size_t pk = (size_t)a * 512 + tid;
                if (B.counts[pk] == 0) continue;
                const CellInfo c = cell_info(g, bx, by, bz, tid);
                if (c.oob) continue;
                const unsigned v = B.vert_offsets[pk];
                if (v >= P.max_cell_vertices) continue;
                float cv[8];
                const int mask = cell_case(S.field, c.lx, c.ly, c.lz, cv);
                unsigned m = 0;
                for (int e = 0; e < 12; ++e) m += ((mask >> edge_c0(e)) & 1) != ((mask >> edge_c1(e)) & 1);
                want[h] = 1;
                hm[h] = m;
                vi[h] = v;
            }
            unsigned tot_h;
            const unsigned h_pre = block_exclusive<SOLVE_THREADS>(hm[0] + hm[1], S.warp_sums, &tot_h);
            const bool fit0 = h_pre + hm[0] <= (unsigned)DC_HERMITE_CAP;
            const bool fit1 = h_pre + hm[0] + hm[1] <= (unsigned)DC_HERMITE_CAP;
            const unsigned take = (want[0] && fit0 ? 1u : 0u) + (want[1] && fit1 ? 1u : 0u);
            unsigned ncells;
            const unsigned c_pre = block_exclusive<SOLVE_THREADS>(take, S.warp_sums, &ncells);
            int last = -1;  // the last cell (fitting or not wanted) this thread's pair covers
            if (cursor + 2 * (int)threadIdx.x < 512 && fit0) last = cursor + 2 * threadIdx.x;
            if (cursor + 2 * (int)threadIdx.x + 1 < 512 && fit1) last = cursor + 2 * threadIdx.x + 1;
            if (threadIdx.x == 0) S.next_cursor = cursor;
            __syncthreads();
            atomicMax(&S.next_cursor, last + 1);
            unsigned slot = c_pre, hslot = h_pre;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int tid = cursor + 2 * threadIdx.x + h;
                if (!want[h] || !(h == 0 ? fit0 : fit1)) continue;
                S.cell_tid[slot] = (unsigned short)tid;
                S.cell_vidx[slot] = vi[h];
                S.cell_h0[slot] = (unsigned short)hslot;
                S.cell_m[slot] = (unsigned char)hm[h];
                const CellInfo c = cell_info(g, bx, by, bz, tid);
                float cv[8];
                const int mask = cell_case(S.field, c.lx, c.ly, c.lz, cv);
                for (int e = 0; e < 12; ++e)
                    if (((mask >> edge_c0(e)) & 1) != ((mask >> edge_c1(e)) & 1))
                        S.h_cell[hslot++] = (unsigned short)((tid << 4) | e);
                ++slot;
            }
            __syncthreads();
            const int next = S.next_cursor;
            const unsigned nh = ncells ? (unsigned)S.cell_h0[ncells - 1] + S.cell_m[ncells - 1] : 0u;
            // Hermite normals: computeNormal at each edge point (:1383-1411). The cells around an
            // edge that name it with the same direction compute the same float edge point from the
            // same two samples, hence the same normal: it is evaluated once per (edge, direction),
            // by k_dc_hermite_normals for a listed block, here otherwise.
            if (hb >= 0) {
                // the listing enumerates the same samples; an index past its count is not followed
                for (int i = threadIdx.x; i < (int)nh; i += blockDim.x) {
                    float3 nn = f3(0.f, 1.f, 0.f);
                    if (hk0 + (unsigned)i < (unsigned)hbase.z) {
                        const float4 v = B.hnormals[B.hsample_rep[(size_t)hb + hk0 + i]];
                        nn = f3(v.x, v.y, v.z);
                    } else if (diag) {
                        atomicExch(&diag->inconsistent, 1);
                    }
                    S.h_n[i] = nn;
                }
                hk0 += nh;
                __syncthreads();
            } else {
            for (int k = threadIdx.x; k < DC_EDGE_KEYS; k += blockDim.x) S.edge_rep[k] = 0xFFFF;
            if (threadIdx.x == 0) S.nrep = 0;
            __syncthreads();
            for (int i = threadIdx.x; i < (int)nh; i += blockDim.x) {
                const int tid = S.h_cell[i] >> 4, e = S.h_cell[i] & 15;
                const int c0 = edge_c0(e), c1 = edge_c1(e);
                const int d0 = corner_dx(c0) + 2 * corner_dy(c0) + 4 * corner_dz(c0);
                const int d1 = corner_dx(c1) + 2 * corner_dy(c1) + 4 * corner_dz(c1);
                const int lo = d0 < d1 ? c0 : c1;  // the edge's lower corner
                const int axis = (d0 ^ d1) == 1 ? 0 : ((d0 ^ d1) == 2 ? 1 : 2);
                const int sx = (tid & 7) + corner_dx(lo), sy = ((tid >> 3) & 7) + corner_dy(lo),
                          sz = (tid >> 6) + corner_dz(lo);
                const int key = ((sz * 9 + sy) * 9 + sx) * 6 + axis * 2 + (d0 < d1 ? 0 : 1);
                const unsigned short prev = atomicCAS(&S.edge_rep[key], (unsigned short)0xFFFF, (unsigned short)i);
                if (prev == 0xFFFF) {
                    S.h_rep[i] = (unsigned short)i;
                    S.rep_list[atomicAdd(&S.nrep, 1)] = (unsigned short)i;
                } else {
                    S.h_rep[i] = prev;
                }
            }
            __syncthreads();
            const int nrep = S.nrep;
            stencil_all_warps(
                sc, nrep, g.cell, time, S.st_d,
                [&](int r) {
                    const int i = S.rep_list[r];
                    const CellInfo c = cell_info(g, bx, by, bz, S.h_cell[i] >> 4);
                    float cv[8];
                    (void)cell_case(S.field, c.lx, c.ly, c.lz, cv);
                    return edge_point(g, c.x, c.y, c.z, cv, S.h_cell[i] & 15);
                },
                [&](int r, float d0, float d1, float d2, float d3) {
                    const float3 gr = f3(SUB(d1, d0), SUB(d2, d0), SUB(d3, d0));
                    const float len = SQRT(dot3(gr, gr));
                    S.h_n[S.rep_list[r]] = len > 1e-6f ? f3(DIV(gr.x, len), DIV(gr.y, len), DIV(gr.z, len))
                                                       : f3(0.f, 1.f, 0.f);
                },
                diag);
            for (int i = threadIdx.x; i < (int)nh; i += blockDim.x)
                if (S.h_rep[i] != i) S.h_n[i] = S.h_n[S.h_rep[i]];
            __syncthreads();
            }
            // per-cell solve
            for (int i = threadIdx.x; i < (int)ncells; i += blockDim.x) {
                const CellInfo c = cell_info(g, bx, by, bz, S.cell_tid[i]);
                float cv[8];
                (void)cell_case(S.field, c.lx, c.ly, c.lz, cv);
                if (P.solver == SDF_DC_SOLVER_MASSPOINT) {
                    int fp64 = 0;
                    S.cell_x[i] = solve_masspoint(g, c, cv, S.h_n + S.cell_h0[i], S.h_cell + S.cell_h0[i], S.cell_m[i],
                                                  P.cond_threshold, &fp64);
                    if (fp64 && diag) atomicAdd(&diag->fp64_cells, 1ull);
                    if (B.qef_debug)
                        B.qef_debug[S.cell_vidx[i]] = make_float4(S.cell_x[i].x, S.cell_x[i].y, S.cell_x[i].z,
                                                                  fp64 ? 1.f : 0.f);
                } else {
                    S.cell_x[i] = solve_reference(g, c, cv, S, S.cell_h0[i], S.cell_m[i]);
                }
            }
            __syncthreads();
            // mass-point mode: project the vertex onto the surface, x <- x - f(x) n, along the cell's mean
            // Hermite normal n (the normalised sum of its unit Hermite normals; no step where that sum is
            // shorter than 1e-6). The steps run in cell-local coordinates y = x - cell corner, starting
            // from the vertex clamped to the cell widened by 0.1 cell and kept in that box; each step
            // evaluates map() at the float point corner + y. A fixed direction per cell keeps the step
            // independent of finite differences of the field at the vertex, and every operation is
            // rounded on its own, so a float32 restatement on the host reproduces the steps.
            // The steps of a block's few cells leave most warps of the CTA idle at the next barrier, so
            // every cell whose vertex slot has a projection record is handed to k_dc_project (64 cells
            // per warp over all blocks) with its start point and direction; the others finish here.
            const bool handoff = P.solver == SDF_DC_SOLVER_MASSPOINT && P.projection_iters > 0 && B.proj;
            if (P.solver == SDF_DC_SOLVER_MASSPOINT && P.projection_iters > 0) {
                const float margin = MUL(0.10f, g.cell), hi = ADD(g.cell, margin);
                for (int i = threadIdx.x; i < (int)ncells; i += blockDim.x) {
                    const CellInfo c = cell_info(g, bx, by, bz, S.cell_tid[i]);
                    const float3 y = sub3(S.cell_x[i], grid_loc(g, c.x, c.y, c.z));
                    S.cell_x[i] = f3(CLAMP(y.x, -margin, hi), CLAMP(y.y, -margin, hi), CLAMP(y.z, -margin, hi));
                }
                __syncthreads();
                if (handoff)
                    for (int i = threadIdx.x; i < (int)ncells; i += blockDim.x) {
                        const unsigned v = S.cell_vidx[i];
                        if (v >= B.proj_cap) continue;
                        float3 nsum = f3(0.f, 0.f, 0.f), nbar = f3(0.f, 0.f, 0.f);
                        const int h0 = S.cell_h0[i], m = S.cell_m[i];
                        for (int q = 0; q < m; ++q) {
                            float3 nq;
                            if (unit_normal_rn(S.h_n[h0 + q], nq)) nsum = add3(nsum, nq);
                        }
                        const bool has_dir = unit_normal_rn(nsum, nbar);
                        const float3 y = S.cell_x[i];
                        B.proj[2 * (size_t)v] = make_float4(y.x, y.y, y.z, __int_as_float(a));
                        B.proj[2 * (size_t)v + 1] =
                            make_float4(nbar.x, nbar.y, nbar.z, __uint_as_float(S.cell_tid[i] | (has_dir ? 0x10000u : 0u)));
                        if (B.cell_normals && B.proj_nsum) {
                            float3 raw = f3(0.f, 0.f, 0.f);
                            for (int q = 0; q < m; ++q) raw = add3(raw, S.h_n[h0 + q]);
                            B.proj_nsum[v] = make_float4(raw.x, raw.y, raw.z, 0.f);
                        }
                    }
                // each remaining cell stays with one lane of one warp for all steps
                for (int base = warp * 32; base < (int)ncells; base += nwarps * 32) {
                    const int i = base + lane;
                    const bool valid = i < (int)ncells && !(handoff && S.cell_vidx[i] < B.proj_cap);
                    float3 cm = f3(0.f, 0.f, 0.f), nbar = f3(0.f, 0.f, 0.f), y = f3(0.f, 0.f, 0.f);
                    bool has_dir = false;
                    if (valid) {
                        const CellInfo c = cell_info(g, bx, by, bz, S.cell_tid[i]);
                        cm = grid_loc(g, c.x, c.y, c.z);
                        y = S.cell_x[i];
                        float3 nsum = f3(0.f, 0.f, 0.f);
                        const int h0 = S.cell_h0[i], m = S.cell_m[i];
                        for (int q = 0; q < m; ++q) {
                            float3 n;
                            if (unit_normal_rn(S.h_n[h0 + q], n)) nsum = add3(nsum, n);
                        }
                        has_dir = unit_normal_rn(nsum, nbar);
                    }
                    for (int it = 0; it < P.projection_iters; ++it) {
                        MapState<false> st;
                        map_warp<false>(sc, add3(cm, y), valid && has_dir, time, st, diag);
                        if (valid && has_dir && isfinite(st.d)) {
                            const float3 yn = sub3(y, scl3(nbar, st.d));
                            y = f3(CLAMP(yn.x, -margin, hi), CLAMP(yn.y, -margin, hi), CLAMP(yn.z, -margin, hi));
                        }
                    }
                    if (valid) S.cell_x[i] = add3(cm, y);
                }
                __syncthreads();
            }
            // soft clamp, hard clamp to the cell, blend towards the cell centre (:1556-1577)
            for (int i = threadIdx.x; i < (int)ncells; i += blockDim.x) {
                if (handoff && S.cell_vidx[i] < B.proj_cap) continue;  // k_dc_project finishes it
                const CellInfo c = cell_info(g, bx, by, bz, S.cell_tid[i]);
                float3 x = S.cell_x[i];
                const float3 cmin = grid_loc(g, c.x, c.y, c.z);
                const float3 cmax = f3(ADD(cmin.x, g.cell), ADD(cmin.y, g.cell), ADD(cmin.z, g.cell));
                const float margin = MUL(0.10f, g.cell);
                x = f3(CLAMP(x.x, SUB(cmin.x, margin), ADD(cmax.x, margin)),
                       CLAMP(x.y, SUB(cmin.y, margin), ADD(cmax.y, margin)),
                       CLAMP(x.z, SUB(cmin.z, margin), ADD(cmax.z, margin)));
                x = f3(CLAMP(x.x, cmin.x, cmax.x), CLAMP(x.y, cmin.y, cmax.y), CLAMP(x.z, cmin.z, cmax.z));
                const float3 ctr = f3(FMA(0.5f, g.cell, cmin.x), FMA(0.5f, g.cell, cmin.y), FMA(0.5f, g.cell, cmin.z));
                x = lerp3(ctr, x, P.qef_blend);
                S.cell_x[i] = x;
                B.cell_verts[S.cell_vidx[i]] = encode_vertex(x, cmin, g.cell);
            }
            __syncthreads();
            // vertex normal: averaged Hermite normals, oriented by the SDF gradient at the vertex
            if (B.cell_normals) {
                for (int base = warp * 32; base < (int)ncells; base += nwarps * 32) {
                    const int i = base + lane;
                    const bool valid = i < (int)ncells && !(handoff && S.cell_vidx[i] < B.proj_cap);
                    const float3 x = valid ? S.cell_x[i] : f3(0.f, 0.f, 0.f);
                    const float3 nref = normal_warp(sc, x, valid, time, g.cell, diag);
                    if (valid) {
                        float3 nsum = f3(0.f, 0.f, 0.f);
                        const int h0 = S.cell_h0[i], m = S.cell_m[i];
                        for (int q = 0; q < m; ++q) nsum = add3(nsum, S.h_n[h0 + q]);
                        const float len = SQRT(dot3(nsum, nsum));
                        float3 nout = (len > 1e-6f) ? f3(DIV(nsum.x, len), DIV(nsum.y, len), DIV(nsum.z, len)) : nref;
                        if (dot3(nout, nref) < 0.f) nout = f3(-nout.x, -nout.y, -nout.z);
                        B.cell_normals[S.cell_vidx[i]] = encode_normal(nout);
                    }
                }
            }
            __syncthreads();
            cursor = next > cursor ? next : 512;
        }
    }
}

// one vertex of k_dc_project: its record's cell corner, mean Hermite normal and cell-local point
struct ProjVertex {
    unsigned v;
    bool live, has_dir;
    unsigned bbase;
    float cell;
    float3 cm, nbar, y;
};

__device__ __forceinline__ ProjVertex proj_vertex(const GridView& g0, const ActiveView& av, const DcBuffers& B,
                                                  unsigned v, unsigned n, unsigned first, int nact) {
    ProjVertex V;
    V.v = v;
    const unsigned vv = v < n ? v : first;  // vertices past the end read the task's first record
    const float4 r0 = B.proj[2 * (size_t)vv], r1 = B.proj[2 * (size_t)vv + 1];
    const int ra = __float_as_int(r0.w);
    const unsigned cw = __float_as_uint(r1.w);
    // every vertex below n has a record from k_dc_solve; a record that names no active block or cell
    // is skipped rather than followed
    const bool ok = ra >= 0 && ra < nact && (cw & 0xFFFFu) < 512u;
    V.live = v < n && ok;
    V.has_dir = V.live && ((cw >> 16) & 1u);
    GridView g = g0;
    SceneView unused;
    int lin;
    resolve(av, av.list[ok ? ra : 0], g, unused, lin, V.bbase);
    int bx, by, bz;
    block_coord(g, lin, bx, by, bz);
    const CellInfo c = cell_info(g, bx, by, bz, ok ? (int)(cw & 0xFFFFu) : 0);
    V.cm = grid_loc(g, c.x, c.y, c.z);
    V.cell = g.cell;
    V.nbar = f3(r1.x, r1.y, r1.z);
    V.y = f3(r0.x, r0.y, r0.z);
    return V;
}

// one projection step: y <- y - f n, kept in the cell widened by 0.1 cell
__device__ __forceinline__ void proj_step(ProjVertex& V, bool mine, float d) {
    if (mine && V.has_dir && isfinite(d)) {
        const float margin = MUL(0.10f, V.cell), hi = ADD(V.cell, margin);
        const float3 yn = sub3(V.y, scl3(V.nbar, d));
        V.y = f3(CLAMP(yn.x, -margin, hi), CLAMP(yn.y, -margin, hi), CLAMP(yn.z, -margin, hi));
    }
}

// soft clamp, hard clamp to the cell, blend towards the cell centre (:1556-1577)
__device__ __forceinline__ float3 proj_finish(const ProjVertex& V, float qef_blend) {
    const float3 cm = V.cm;
    const float margin = MUL(0.10f, V.cell);
    float3 x = add3(cm, V.y);
    const float3 cmax = f3(ADD(cm.x, V.cell), ADD(cm.y, V.cell), ADD(cm.z, V.cell));
    x = f3(CLAMP(x.x, SUB(cm.x, margin), ADD(cmax.x, margin)), CLAMP(x.y, SUB(cm.y, margin), ADD(cmax.y, margin)),
           CLAMP(x.z, SUB(cm.z, margin), ADD(cmax.z, margin)));
    x = f3(CLAMP(x.x, cm.x, cmax.x), CLAMP(x.y, cm.y, cmax.y), CLAMP(x.z, cm.z, cmax.z));
    const float3 ctr = f3(FMA(0.5f, V.cell, cm.x), FMA(0.5f, V.cell, cm.y), FMA(0.5f, V.cell, cm.z));
    return lerp3(ctr, x, qef_blend);
}

// vertex normal: averaged Hermite normals, oriented by the SDF gradient at the vertex
__device__ __forceinline__ void proj_normal(const ActiveView& av, const SceneView& sc0, const DcBuffers& B,
                                            const ProjVertex& V, float3 x, float time, Diag* diag) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned pending = __ballot_sync(FULL, V.live);
    while (pending) {
        const unsigned lead = __shfl_sync(FULL, V.bbase, __ffs(pending) - 1);
        const bool mine = V.live && V.bbase == lead && ((pending >> lane) & 1u);
        SceneView scw = sc0;
        if (av.scenes) scw = av.scenes[scene_of_block(av.scenes, av.nscenes, lead)].sc;
        const float3 nref = normal_warp(scw, x, mine, time, V.cell, diag);
        if (mine) {
            const float4 r = B.proj_nsum[V.v];
            const float3 nsum = f3(r.x, r.y, r.z);
            const float len = SQRT(dot3(nsum, nsum));
            float3 nout = (len > 1e-6f) ? f3(DIV(nsum.x, len), DIV(nsum.y, len), DIV(nsum.z, len)) : nref;
            if (dot3(nout, nref) < 0.f) nout = f3(-nout.x, -nout.y, -nout.z);
            B.cell_normals[V.v] = encode_normal(nout);
        }
        pending &= ~__ballot_sync(FULL, mine);
    }
}

// The mass-point projection steps and the finishing of the DC vertices handed off by k_dc_solve: 64
// vertices per warp task in vertex order (so a warp's cells are neighbours from one or two blocks), two
// consecutive vertices per lane walked together by map_pair (each point its own walk), each taking
// x <- x - f(x) n along its cell's mean Hermite normal, in cell-local coordinates kept in the cell
// widened by 0.1 cell, then the clamps, the blend and the encoding of k_dc_solve. The same operations
// as there, so the vertices are the same; a warp walks one scene's BVH at a time.
__global__ void __launch_bounds__(BLK_THREADS) k_dc_project(GridView g0, SceneView sc0, float time, ActiveView av,
                                                           DcBuffers B, DcSolveParams P,
                                                           const unsigned* __restrict__ nverts, unsigned* ticket,
                                                           Diag* diag) {
    const unsigned n = min(min(*nverts, B.proj_cap), P.max_cell_vertices);
    const int nact = active_count(av);
    const int tasks = nact > 0 ? (int)((n + 63u) / 64u) : 0;
    const int lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;
    for (;;) {
        int t = 0;
        if (lane == 0) t = (int)atomicAdd(ticket, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= tasks) break;
        const unsigned first = (unsigned)t * 64u, v0 = first + 2u * (unsigned)lane;
        ProjVertex V0 = proj_vertex(g0, av, B, v0, n, first, nact);
        ProjVertex V1 = proj_vertex(g0, av, B, v0 + 1u, n, first, nact);
        for (int it = 0; it < P.projection_iters; ++it) {
            unsigned pend0 = __ballot_sync(FULL, V0.live), pend1 = __ballot_sync(FULL, V1.live);
            while (pend0 | pend1) {
                // the scene of the first pending point (every point of a lane in it walks now)
                const unsigned lead = pend0 ? __shfl_sync(FULL, V0.bbase, __ffs(pend0) - 1)
                                            : __shfl_sync(FULL, V1.bbase, __ffs(pend1) - 1);
                const bool mine0 = V0.live && V0.bbase == lead && ((pend0 >> lane) & 1u);
                const bool mine1 = V1.live && V1.bbase == lead && ((pend1 >> lane) & 1u);
                SceneView scw = sc0;
                if (av.scenes) scw = av.scenes[scene_of_block(av.scenes, av.nscenes, lead)].sc;
                float d0, d1;
                map_pair<false, false>(scw, add3(V0.cm, V0.y), add3(V1.cm, V1.y), mine0 && V0.has_dir,
                                       mine1 && V1.has_dir, time, d0, d1, diag);
                proj_step(V0, mine0, d0);
                proj_step(V1, mine1, d1);
                pend0 &= ~__ballot_sync(FULL, mine0);
                pend1 &= ~__ballot_sync(FULL, mine1);
            }
        }
        const float3 x0 = proj_finish(V0, P.qef_blend), x1 = proj_finish(V1, P.qef_blend);
        if (V0.live) B.cell_verts[V0.v] = encode_vertex(x0, V0.cm, V0.cell);
        if (V1.live) B.cell_verts[V1.v] = encode_vertex(x1, V1.cm, V1.cell);
        if (B.cell_normals && B.proj_nsum) {
            proj_normal(av, sc0, B, V0, x0, time, diag);
            proj_normal(av, sc0, B, V1, x1, time, diag);
        }
    }
}

// dcRecomputeNormalsAtVertices (:1602-1630): the gradient at each decoded vertex
__global__ void __launch_bounds__(BLK_THREADS) k_dc_recompute_normals(GridView g, SceneView sc, float time,
                                                                      ActiveView av, DcBuffers B, unsigned maxV,
                                                                      unsigned* ticket, Diag* diag) {
    __shared__ int s_item;
    const int n = active_count(av);
    for (;;) {
        const int a = claim(ticket, n, &s_item);
        if (a < 0) break;
        const int lin = av.list[a];
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        for (int h = 0; h < 2; ++h) {
            const int tid = 2 * threadIdx.x + h;
            const size_t pk = (size_t)a * 512 + tid;
            const CellInfo c = cell_info(g, bx, by, bz, tid);
            bool valid = B.counts[pk] != 0 && !c.oob;
            const unsigned vi = valid ? B.vert_offsets[pk] : 0u;
            valid = valid && vi < maxV;
            float3 p = f3(0.f, 0.f, 0.f);
            if (valid) p = decode_vertex(B.cell_verts[vi], grid_loc(g, c.x, c.y, c.z), g.cell);
            const float3 nrm = normal_warp(sc, p, valid, time, g.cell, diag);
            if (valid) B.cell_normals[vi] = encode_normal(nrm);
        }
    }
}

// lookupPackedCell (:1633-1657)
__device__ __forceinline__ bool lookup_packed(const GridView& g, const int* __restrict__ b2a, int cx, int cy, int cz,
                                              int& out) {
    if (cx < 0 || cy < 0 || cz < 0) return false;
    if (cx >= g.w - 1 || cy >= g.h - 1 || cz >= g.d - 1) return false;
    const int bx = cx >> 3, by = cy >> 3, bz = cz >> 3;
    if (bx >= g.bx || by >= g.by || bz >= g.bz) return false;
    const int a = __ldg(b2a + bx + by * g.bx + bz * g.bx * g.by);
    if (a < 0) return false;
    out = a * 512 + (cx - bx * 8) + (cy - by * 8) * 8 + (cz - bz * 8) * 64;
    return true;
}

// dcSmoothCellNormals (:1659-1712): 6-neighbour angle-gated smoothing into the tmp buffer
__global__ void k_dc_smooth_normals(GridView g, ActiveView av, DcBuffers B, unsigned maxV, float cosT) {
    const int a = blockIdx.x;
    if (a >= active_count(av)) return;
    const int tid = threadIdx.x;
    int bx, by, bz;
    block_coord(g, av.list[a], bx, by, bz);
    const size_t pk = (size_t)a * 512 + tid;
    const CellInfo c = cell_info(g, bx, by, bz, tid);
    if (c.oob) return;
    if (!surface_mask(B.masks[pk])) return;
    const unsigned vi = B.vert_offsets[pk];
    if (vi >= maxV) return;
    const float3 self = decode_normal(B.cell_normals[vi]);
    float3 sum = self;
    const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (int i = 0; i < 6; ++i) {
        int pn;
        if (!lookup_packed(g, B.block_to_active, c.x + off[i][0], c.y + off[i][1], c.z + off[i][2], pn)) continue;
        if (!surface_mask(B.masks[pn])) continue;
        const unsigned vn = B.vert_offsets[pn];
        if (vn >= maxV) continue;
        const float3 nb = decode_normal(B.cell_normals[vn]);
        const float d = dot3(nb, self);
        if (d >= cosT) {
            const float w = DIV(SUB(d, cosT), fmaxf(1e-6f, SUB(1.f, cosT)));
            // nSum + w * nNbr (:1697), the product fused into the sum
            sum = f3(FMA(w, nb.x, sum.x), FMA(w, nb.y, sum.y), FMA(w, nb.z, sum.z));
        }
    }
    const float len = SQRT(dot3(sum, sum));
    const float3 o = (len > 1e-6f) ? f3(DIV(sum.x, len), DIV(sum.y, len), DIV(sum.z, len)) : self;
    B.cell_normals_tmp[vi] = encode_normal(o);
}

// the four cells around the edge of `axis` leaving corner 0 of cell (x, y, z), in the order the
// reference's quad uses them (:1981-2043)
__device__ __forceinline__ bool quad_cells(const GridView& g, const int* b2a, int axis, int x, int y, int z,
                                           int q[4]) {
    int pa, pb, pc, pd;
    if (axis == 0) {
        if (!(y > 0 && z > 0)) return false;
        if (!(lookup_packed(g, b2a, x, y, z, pa) && lookup_packed(g, b2a, x, y - 1, z, pb) &&
              lookup_packed(g, b2a, x, y, z - 1, pc) && lookup_packed(g, b2a, x, y - 1, z - 1, pd)))
            return false;
        q[0] = pa; q[1] = pb; q[2] = pd; q[3] = pc;
    } else if (axis == 1) {
        if (!(x > 0 && z > 0)) return false;
        if (!(lookup_packed(g, b2a, x, y, z, pa) && lookup_packed(g, b2a, x - 1, y, z, pb) &&
              lookup_packed(g, b2a, x, y, z - 1, pc) && lookup_packed(g, b2a, x - 1, y, z - 1, pd)))
            return false;
        q[0] = pa; q[1] = pc; q[2] = pd; q[3] = pb;
    } else {
        if (!(x > 0 && y > 0)) return false;
        if (!(lookup_packed(g, b2a, x, y, z, pa) && lookup_packed(g, b2a, x - 1, y, z, pb) &&
              lookup_packed(g, b2a, x, y - 1, z, pc) && lookup_packed(g, b2a, x - 1, y - 1, z, pd)))
            return false;
        q[0] = pa; q[1] = pb; q[2] = pd; q[3] = pc;
    }
    return true;
}

__device__ __forceinline__ int edge_corner(int axis) { return axis == 0 ? 1 : (axis == 1 ? 3 : 4); }

// dcCountQuads (:1714-1784); block_totals (optional) gets the per-block sum
__global__ void k_dc_count_quads(GridView g0, ActiveView av, DcBuffers B, unsigned* __restrict__ counts,
                                 unsigned* __restrict__ block_totals) {
    __shared__ unsigned s_red[16];
    const int n = active_count(av);
    const int tid = threadIdx.x;
    for (int a = blockIdx.x; a < n; a += gridDim.x) {
        GridView g = g0;
        SceneView unused;
        int lin;
        unsigned bbase;
        resolve(av, av.list[a], g, unused, lin, bbase);
        const int* b2a = B.block_to_active + bbase;  // this scene's block-to-active map
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        const size_t pk = (size_t)a * 512 + tid;
        const CellInfo c = cell_info(g, bx, by, bz, tid);
        unsigned cnt = 0;
        if (!c.oob) {
            const unsigned char mask = B.masks[pk];
            const unsigned s0 = mask & 1u;
            for (int axis = 0; axis < 3; ++axis) {
                if (((mask >> edge_corner(axis)) & 1u) == s0) continue;
                int q[4];
                if (quad_cells(g, b2a, axis, c.x, c.y, c.z, q) && surface_mask(B.masks[q[0]]) &&
                    surface_mask(B.masks[q[1]]) && surface_mask(B.masks[q[2]]) && surface_mask(B.masks[q[3]]))
                    cnt += 6;
            }
        }
        counts[pk] = cnt;
        if (block_totals) {
            unsigned v = cnt;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if ((tid & 31) == 0) s_red[tid >> 5] = v;
            __syncthreads();
            if (tid == 0) {
                unsigned s = 0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += s_red[w];
                block_totals[a] = s;
            }
            __syncthreads();  // s_red is free for the next block
        }
    }
}

// ------------------------------------------------------------------------------------------------
// dcGenerateQuads (:1806-2044)
// ------------------------------------------------------------------------------------------------
constexpr int DC_QUAD_CAP = 1024;  // quads staged per pass

struct QuadSmem {
    unsigned q_cell[DC_QUAD_CAP];   // (cell tid << 2) | axis
    unsigned q_out[DC_QUAD_CAP];    // first output vertex
    unsigned char q_flags[DC_QUAD_CAP];  // 1 flipped, 2 not written (capacity), 4 alternate diagonal
    float3 q_fn[DC_QUAD_CAP][2];    // face normals of the two triangles (normals output); [1] holds the
                                    // winding normal until the quad is written
    float st_d[4 * STENCIL_CHUNK];  // the winding normals' stencils (stencil_all_warps)
    unsigned warp_sums[BLK_THREADS / 32];
    int item;
};

struct QuadVerts {
    float3 v[4];
    float3 qc;
    unsigned vi[4];  // the four cell vertex indices (the indexed output's corners)
};

__device__ __forceinline__ float3 cell_min_of_packet(const GridView& g, const int* list, unsigned base, int packet) {
    const int ab = packet >> 9, t = packet & 511;
    int bx, by, bz;
    block_coord(g, list[ab] - (int)base, bx, by, bz);
    const CellInfo c = cell_info(g, bx, by, bz, t);
    return grid_loc(g, c.x, c.y, c.z);
}

// decodes the quad's four vertices (:1851-1875); false when a vertex index is out of range (the
// reference then skips the quad without advancing its write cursor)
__device__ __forceinline__ bool quad_vertices(const GridView& g, const int* list, unsigned base, const DcBuffers& B,
                                              const int q[4], unsigned maxV, QuadVerts& Q) {
    unsigned vi[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) vi[j] = B.vert_offsets[q[j]];
    if (vi[0] >= maxV || vi[1] >= maxV || vi[2] >= maxV || vi[3] >= maxV) return false;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        Q.vi[j] = vi[j];
        Q.v[j] = decode_vertex(B.cell_verts[vi[j]], cell_min_of_packet(g, list, base, q[j]), g.cell);
    }
    Q.qc = f3(MUL(0.25f, ADD(ADD(ADD(Q.v[0].x, Q.v[1].x), Q.v[2].x), Q.v[3].x)),
              MUL(0.25f, ADD(ADD(ADD(Q.v[0].y, Q.v[1].y), Q.v[2].y), Q.v[3].y)),
              MUL(0.25f, ADD(ADD(ADD(Q.v[0].z, Q.v[1].z), Q.v[2].z), Q.v[3].z)));
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (!finite3(Q.v[j])) Q.v[j] = Q.qc;
    return true;
}

__device__ __forceinline__ bool quad_indices_ok(const DcBuffers& B, const int q[4], unsigned maxV) {
    return B.vert_offsets[q[0]] < maxV && B.vert_offsets[q[1]] < maxV && B.vert_offsets[q[2]] < maxV &&
           B.vert_offsets[q[3]] < maxV;
}

// The quads can be emitted from the quad list (by k_dc_quad_normals, which holds each quad's corners and
// winding normal) instead of per block (k_dc_quads) when nothing overflows: every counted quad listed,
// every cell vertex index and every output vertex within the output's capacity, so every counted quad
// is emitted, at six times its list index; and no output needs map() at the quad or per-face normals.
// Both kernels take the decision from the same counts, so exactly one of them emits.
__device__ __forceinline__ bool quads_from_list(const DcBuffers& B, const unsigned* offsets,
                                                const unsigned* total_vertices, const unsigned* dc_vertices,
                                                unsigned maxV, unsigned mask) {
    if (!B.qnormals || offsets || !total_vertices || !dc_vertices || B.qcap == 0) return false;
    if (mask & (OUT_COLORS | OUT_PRIMIDS | OUT_UVS | OUT_NORMALS)) return false;
    const unsigned total = *total_vertices;
    return total / 6u <= B.qcap && total <= maxV && *dc_vertices <= maxV;
}

// one emitted quad without per-quad attributes, as k_dc_quads writes it: winding against the normal at
// the centre, the split diagonal, then the six vertices with identity indices at w, or (indexed output)
// the corners' cell vertex indices
__device__ __forceinline__ void emit_quad_plain(QuadVerts& Q, float3 nref, unsigned w, unsigned mask,
                                                const DcQuadParams& QP, const MeshOut& out) {
    const int order_a[6] = {0, 1, 2, 0, 2, 3}, order_b[6] = {1, 2, 3, 1, 3, 0};
    const float3 nt = cross_ff(sub3(Q.v[1], Q.v[0]), sub3(Q.v[2], Q.v[0]));
    if (dot3(nt, nref) < 0.f) {
        const float3 t = Q.v[1]; Q.v[1] = Q.v[3]; Q.v[3] = t;
        const unsigned u = Q.vi[1]; Q.vi[1] = Q.vi[3]; Q.vi[3] = u;
    }
    bool alt = false;
    if (QP.adaptive_diagonal) {
        const float3 e02 = sub3(Q.v[2], Q.v[0]), e13 = sub3(Q.v[3], Q.v[1]);
        alt = dot3_rn(e13, e13) < dot3_rn(e02, e02);
    }
    if (mask & OUT_WELDED) {
#pragma unroll
        for (int j = 0; j < 6; ++j) out.indices[w + j] = Q.vi[alt ? order_b[j] : order_a[j]];
        return;
    }
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        const int vj = alt ? order_b[j] : order_a[j];
        out.verts[w + j] = make_float4(Q.v[vj].x, Q.v[vj].y, Q.v[vj].z, 1.f);
        if ((mask & OUT_INDICES) && out.indices) out.indices[w + j] = w + j;
    }
}

// Every counted quad of every active block, in emission order: quad q = (block offset + in-block count
// prefix) / 6 gets (active block, cell << 2 | axis). The enumeration is k_dc_quads' own.
__global__ void __launch_bounds__(BLK_THREADS) k_dc_quad_list(GridView g0, ActiveView av, DcBuffers B,
                                                             const unsigned* __restrict__ counts,
                                                             const unsigned* __restrict__ block_offsets,
                                                             uint2* __restrict__ recs, unsigned cap) {
    __shared__ unsigned s_warp[BLK_THREADS / 32];
    const int n = active_count(av);
    for (int a = blockIdx.x; a < n; a += gridDim.x) {
        GridView g = g0;
        SceneView unused;
        int lin;
        unsigned bbase;
        resolve(av, av.list[a], g, unused, lin, bbase);
        const int* b2a = B.block_to_active + bbase;
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        unsigned cnt[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) cnt[h] = counts[(size_t)a * 512 + 2 * threadIdx.x + h];
        unsigned tot;
        const unsigned local = block_exclusive<BLK_THREADS>(cnt[0] + cnt[1], s_warp, &tot);
        const unsigned q0 = block_offsets[a] / 6u;
        unsigned q = q0 + local / 6u;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int tid = 2 * threadIdx.x + h;
            if (cnt[h] == 0) continue;
            const CellInfo c = cell_info(g, bx, by, bz, tid);
            if (c.oob) continue;
            const unsigned char m = B.masks[(size_t)a * 512 + tid];
            const unsigned s0 = m & 1u;
            for (int axis = 0; axis < 3; ++axis) {
                if (((m >> edge_corner(axis)) & 1u) == s0) continue;
                int qc[4];
                if (!quad_cells(g, b2a, axis, c.x, c.y, c.z, qc)) continue;
                if (!surface_mask(B.masks[qc[0]]) || !surface_mask(B.masks[qc[1]]) || !surface_mask(B.masks[qc[2]]) ||
                    !surface_mask(B.masks[qc[3]]))
                    continue;
                if (q < cap) recs[q] = make_uint2((unsigned)a, (unsigned)((tid << 2) | axis));
                ++q;
            }
        }
        __syncthreads();  // s_warp is free for the next block
    }
}

// computeNormal (:814-844) at the centre of every listed quad (its four decoded cell vertices), 16 quads
// per warp task with two stencil points per lane on two lanes, one scene's BVH at a time
__global__ void __launch_bounds__(BLK_THREADS) k_dc_quad_normals(GridView g0, SceneView sc0, float time,
                                                                ActiveView av, DcBuffers B,
                                                                const uint2* __restrict__ recs,
                                                                const unsigned* __restrict__ total_vertices,
                                                                unsigned cap, unsigned maxV,
                                                                float4* __restrict__ normals, unsigned* ticket,
                                                                Diag* diag, const unsigned* __restrict__ dc_vertices,
                                                                MeshOut out, unsigned mask, DcQuadParams QP) {
    const unsigned n = min(*total_vertices / 6u, cap);
    const bool emit = quads_from_list(B, nullptr, total_vertices, dc_vertices, out.maxV, mask);
    const int nact = active_count(av);
    const int tasks = nact > 0 ? (int)((n + 15u) / 16u) : 0;
    const int lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;
    for (;;) {
        int t = 0;
        if (lane == 0) t = (int)atomicAdd(ticket, 1u);
        t = __shfl_sync(FULL, t, 0);
        if (t >= tasks) break;
        const unsigned qi = (unsigned)t * 16u + (unsigned)(lane >> 1);
        const bool in = qi < n;
        const uint2 rec = recs[in ? qi : (unsigned)t * 16u];
        const int ra = (int)rec.x, tid = (int)(rec.y >> 2), axis = (int)(rec.y & 3u);
        bool live = in && ra < nact && tid < 512 && axis < 3;
        GridView g = g0;
        SceneView sc = sc0;
        int lin;
        unsigned bbase;
        resolve(av, av.list[live ? ra : 0], g, sc, lin, bbase);
        const int* b2a = B.block_to_active + bbase;
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        float3 qc = f3(0.f, 0.f, 0.f);
        QuadVerts Q;
        bool ok = false;
        if (live) {
            const CellInfo c = cell_info(g, bx, by, bz, tid);
            int q[4];
            if (quad_cells(g, b2a, axis, c.x, c.y, c.z, q)) {
                Q.qc = f3(0.f, 0.f, 0.f);
                ok = quad_vertices(g, av.list, bbase, B, q, maxV, Q);  // a skipped quad's normal stays unused
                qc = Q.qc;
            }
        }
        const float3 nn = stencil_normal_pairs(av, sc, bbase, qc, g.cell, live, time, diag);
        if (live && (lane & 1) == 0) {
            normals[qi] = make_float4(nn.x, nn.y, nn.z, 0.f);
            if (emit && ok) emit_quad_plain(Q, nn, 6u * qi, mask, QP, out);  // k_dc_quads stands aside
            // a listed quad always has its cells and corners when nothing overflows; one without them
            // would be written by neither kernel
            if (emit && !ok && diag) atomicExch(&diag->inconsistent, 1);
        }
    }
}

// three CTAs per SM (80 registers): measured 4.2 ms for the 512^3 quads against 7.8 ms at 128 registers
__global__ void __launch_bounds__(BLK_THREADS, 3) k_dc_quads(GridView g0, SceneView sc0, float time, ActiveView av,
                                                          DcBuffers B, const unsigned* __restrict__ offsets,
                                                          const unsigned* __restrict__ counts,
                                                          const unsigned* __restrict__ block_offsets, MeshOut out,
                                                          unsigned mask, DcQuadParams QP, unsigned* ticket,
                                                          Diag* diag, const unsigned* __restrict__ total_vertices,
                                                          const unsigned* __restrict__ dc_vertices) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    QuadSmem& S = *reinterpret_cast<QuadSmem*>(dyn_smem);
    // k_dc_quad_normals emitted every quad from the quad list
    if (quads_from_list(B, offsets, total_vertices, dc_vertices, out.maxV, mask)) return;
    const int n = active_count(av);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int order_a[6] = {0, 1, 2, 0, 2, 3}, order_b[6] = {1, 2, 3, 1, 3, 0};
    for (;;) {
        const int a = claim(ticket, n, &S.item);
        if (a < 0) break;
        GridView g = g0;
        SceneView sc = sc0;
        int lin;
        unsigned bbase;
        resolve(av, av.list[a], g, sc, lin, bbase);
        const int* b2a = B.block_to_active + bbase;  // this scene's block-to-active map
        int bx, by, bz;
        block_coord(g, lin, bx, by, bz);
        // cell offsets: per-cell (drop-in layout) or block offset + in-block scan of the counts
        unsigned cnt[2], off[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) cnt[h] = counts[(size_t)a * 512 + 2 * threadIdx.x + h];
        unsigned tot;
        const unsigned local = block_exclusive<BLK_THREADS>(cnt[0] + cnt[1], S.warp_sums, &tot);
        if (offsets) {
            off[0] = offsets[(size_t)a * 512 + 2 * threadIdx.x];
            off[1] = offsets[(size_t)a * 512 + 2 * threadIdx.x + 1];
        } else {
            off[0] = block_offsets[a] + local;
            off[1] = off[0] + cnt[0];
        }
        // the quads of this thread's two cells, in the reference's emission order; quad slot numbers
        // follow the in-block count prefix (each counted quad is 6 vertices)
        const unsigned slot0 = local / 6;
        const unsigned nslots_total = tot / 6;
        for (unsigned pass0 = 0; pass0 < nslots_total; pass0 += DC_QUAD_CAP) {
            unsigned slot = slot0;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int tid = 2 * threadIdx.x + h;
                if (cnt[h] == 0) continue;
                const CellInfo c = cell_info(g, bx, by, bz, tid);
                if (c.oob) continue;
                const unsigned char m = B.masks[(size_t)a * 512 + tid];
                const unsigned s0 = m & 1u;
                unsigned w = off[h];
                for (int axis = 0; axis < 3; ++axis) {
                    if (((m >> edge_corner(axis)) & 1u) == s0) continue;
                    int q[4];
                    if (!quad_cells(g, b2a, axis, c.x, c.y, c.z, q)) continue;
                    if (!surface_mask(B.masks[q[0]]) || !surface_mask(B.masks[q[1]]) || !surface_mask(B.masks[q[2]]) ||
                        !surface_mask(B.masks[q[3]]))
                        continue;
                    const bool emit = quad_indices_ok(B, q, out.maxV);
                    const bool fits = (unsigned long long)w + 5 < out.maxV;
                    if (slot >= pass0 && slot < pass0 + DC_QUAD_CAP) {
                        const unsigned i = slot - pass0;
                        S.q_cell[i] = (unsigned)((tid << 2) | axis);
                        S.q_out[i] = w;
                        S.q_flags[i] = (emit && fits) ? 0 : 2;
                    }
                    ++slot;
                    if (emit && fits) w += 6;
                }
            }
            const unsigned nq = min(nslots_total - pass0, (unsigned)DC_QUAD_CAP);
            __syncthreads();
            // the winding normal of every staged quad: computeNormal at the quad centre, listed by
            // k_dc_quad_normals (quad = block offset / 6 + slot) or the four points of each stencil
            // spread over all warps here
            const unsigned qfirst = offsets ? 0u : block_offsets[a] / 6u + pass0;
            if (B.qnormals && !offsets && qfirst + nq <= B.qcap) {
                for (int i = threadIdx.x; i < (int)nq; i += blockDim.x) {
                    const float4 v = B.qnormals[qfirst + i];
                    S.q_fn[i][1] = f3(v.x, v.y, v.z);
                }
                __syncthreads();
            } else
            stencil_all_warps(
                sc, (int)nq, g.cell, time, S.st_d,
                [&](int i) {
                    const int tid = S.q_cell[i] >> 2, axis = S.q_cell[i] & 3;
                    const CellInfo c = cell_info(g, bx, by, bz, tid);
                    int q[4];
                    quad_cells(g, b2a, axis, c.x, c.y, c.z, q);
                    QuadVerts Q;
                    Q.qc = f3(0.f, 0.f, 0.f);
                    quad_vertices(g, av.list, bbase, B, q, out.maxV, Q);  // a skipped quad's stays unused
                    return Q.qc;
                },
                [&](int i, float d0, float d1, float d2, float d3) {
                    const float3 gr = f3(SUB(d1, d0), SUB(d2, d0), SUB(d3, d0));
                    const float len = SQRT(dot3(gr, gr));
                    S.q_fn[i][1] = len > 1e-6f ? f3(DIV(gr.x, len), DIV(gr.y, len), DIV(gr.z, len)) : f3(0.f, 1.f, 0.f);
                },
                diag);
            // per quad: winding against the gradient at the centre, attributes from map() at the centre
            for (int base = warp * 32; base < (int)nq; base += nwarps * 32) {
                const int i = base + lane;
                bool valid = i < (int)nq;
                QuadVerts Q;
                Q.qc = f3(0.f, 0.f, 0.f);
                unsigned w = 0;
                if (valid) {
                    const int tid = S.q_cell[i] >> 2, axis = S.q_cell[i] & 3;
                    const CellInfo c = cell_info(g, bx, by, bz, tid);
                    int q[4];
                    quad_cells(g, b2a, axis, c.x, c.y, c.z, q);
                    valid = quad_vertices(g, av.list, bbase, B, q, out.maxV, Q);
                    w = S.q_out[i];
                }
                // map() at the centre with attributes, only when an output needs them
                MapState<true> st;
                if (mask & (OUT_COLORS | OUT_PRIMIDS | OUT_UVS))
                    map_warp<true>(sc, Q.qc, valid, time, st, diag);
                else
                    st.init();
                if (!valid) continue;
                const float3 nref = S.q_fn[i][1];
                const float3 nt = cross_ff(sub3(Q.v[1], Q.v[0]), sub3(Q.v[2], Q.v[0]));
                const bool flip = dot3(nt, nref) < 0.f;
                if (flip) {
                    const float3 t = Q.v[1]; Q.v[1] = Q.v[3]; Q.v[3] = t;
                    const unsigned u = Q.vi[1]; Q.vi[1] = Q.vi[3]; Q.vi[3] = u;
                }
                unsigned char fl = S.q_flags[i] | (flip ? 1 : 0);
                bool alt = false;
                if (QP.adaptive_diagonal) {
                    // split along the shorter diagonal: (1,2,3),(1,3,0) instead of (0,1,2),(0,2,3); squared
                    // lengths with every operation rounded on its own (a float32 restatement reproduces the choice)
                    const float3 e02 = sub3(Q.v[2], Q.v[0]), e13 = sub3(Q.v[3], Q.v[1]);
                    const float d02 = dot3_rn(e02, e02), d13 = dot3_rn(e13, e13);
                    alt = d13 < d02;
                    if (alt) fl |= 4;
                }
                S.q_flags[i] = fl;
                if (!(fl & 2)) {
                    float2 quv[4] = {make_float2(0, 0), make_float2(0, 0), make_float2(0, 0), make_float2(0, 0)};
                    if ((mask & OUT_UVS) && out.uvs && st.id >= 0 && st.id < sc.nprims) {
                        const float4* pr = sc.prims + (size_t)st.id * PRIM_ROWS;
                        const float4 rot = __ldg(pr + 0), pos = __ldg(pr + 2), scl = __ldg(pr + 3);
                        float3 lp[4];
#pragma unroll
                        for (int j = 0; j < 4; ++j) lp[j] = to_local(Q.v[j], rot, pos, scl);
                        const UvParams up = load_uv_params(pr);
                        const float3 t0[3] = {lp[0], lp[1], lp[2]}, t1[3] = {lp[0], lp[2], lp[3]};
                        float2 u0[3], u1[3];
                        triangle_uvs(t0, up, u0);
                        triangle_uvs(t1, up, u1);
                        quv[0] = make_float2(MUL(ADD(u0[0].x, u1[0].x), 0.5f), MUL(ADD(u0[0].y, u1[0].y), 0.5f));
                        quv[1] = u0[1];
                        quv[2] = make_float2(MUL(ADD(u0[2].x, u1[1].x), 0.5f), MUL(ADD(u0[2].y, u1[1].y), 0.5f));
                        quv[3] = u1[2];
                    }
                    if (mask & OUT_WELDED) {  // indexed output: the corners' cell vertices
#pragma unroll
                        for (int j = 0; j < 6; ++j) out.indices[w + j] = Q.vi[alt ? order_b[j] : order_a[j]];
                        continue;
                    }
#pragma unroll
                    for (int j = 0; j < 6; ++j) {
                        const int vj = alt ? order_b[j] : order_a[j];
                        out.verts[w + j] = make_float4(Q.v[vj].x, Q.v[vj].y, Q.v[vj].z, 1.f);
                        if ((mask & OUT_COLORS) && out.colors)
                            out.colors[w + j] = make_float4(st.color.x, st.color.y, st.color.z, 1.f);
                        if ((mask & OUT_PRIMIDS) && out.primids) out.primids[w + j] = __float_as_int((float)st.id);
                        if ((mask & OUT_UVS) && out.uvs) out.uvs[w + j] = quv[vj];
                        if ((mask & OUT_INDICES) && out.indices) out.indices[w + j] = w + j;
                    }
                }
                if ((mask & OUT_NORMALS) && out.normals) {
                    // face normal of each triangle; a degenerate face uses the gradient at the centre
#pragma unroll
                    for (int t = 0; t < 2; ++t) {
                        const int i0 = alt ? order_b[3 * t] : order_a[3 * t];
                        const int i1 = alt ? order_b[3 * t + 1] : order_a[3 * t + 1];
                        const int i2 = alt ? order_b[3 * t + 2] : order_a[3 * t + 2];
                        float3 fn = cross_ff(sub3(Q.v[i1], Q.v[i0]), sub3(Q.v[i2], Q.v[i0]));
                        const float len = SQRT(dot3(fn, fn));
                        fn = len > 1e-6f ? f3(DIV(fn.x, len), DIV(fn.y, len), DIV(fn.z, len)) : nref;
                        S.q_fn[i][t] = fn;
                    }
                }
            }
            __syncthreads();
            if ((mask & OUT_NORMALS) && out.normals) {
                // six offset samples per quad, each a computeNormal (:1918-1966)
                const float offs = MUL(g.cell, 0.25f);
                const int nv = (int)nq * 6;
                for (int base = warp * 32; base < nv; base += nwarps * 32) {
                    const int i = base + lane;
                    bool valid = i < nv;
                    float3 sp = f3(0.f, 0.f, 0.f);
                    unsigned w = 0;
                    bool write = false;
                    if (valid) {
                        const int qi = i / 6, j = i - 6 * qi;
                        const int tid = S.q_cell[qi] >> 2, axis = S.q_cell[qi] & 3;
                        const CellInfo c = cell_info(g, bx, by, bz, tid);
                        int q[4];
                        quad_cells(g, b2a, axis, c.x, c.y, c.z, q);
                        QuadVerts Q;
                        valid = quad_vertices(g, av.list, bbase, B, q, out.maxV, Q);
                        if (valid) {
                            const unsigned char fl = S.q_flags[qi];
                            if (fl & 1) { const float3 t = Q.v[1]; Q.v[1] = Q.v[3]; Q.v[3] = t; }
                            const int vj = (fl & 4) ? order_b[j] : order_a[j];
                            const float3 fn = S.q_fn[qi][j / 3];
                            sp = f3(FMA(fn.x, offs, Q.v[vj].x), FMA(fn.y, offs, Q.v[vj].y), FMA(fn.z, offs, Q.v[vj].z));
                            w = S.q_out[qi] + j;
                            write = !(fl & 2);
                        }
                    }
                    const float3 nrm = normal_warp(sc, sp, valid, time, g.cell, diag);
                    if (valid && write) out.normals[w] = make_float4(nrm.x, nrm.y, nrm.z, 0.f);
                }
            }
            __syncthreads();
        }
    }
}

// Indexed dual-contouring output: every surface cell's vertex, decoded as the quads decode it
// (:1851-1875), at its cell vertex index; the quads then write indices instead of positions.
__global__ void __launch_bounds__(256) k_dc_weld_vertices(GridView g, ActiveView av, DcBuffers B, unsigned max_cells,
                                                          float4* __restrict__ verts, unsigned max_verts) {
    const long long n = (long long)active_count(av) * 512;
    for (long long pk = blockIdx.x * (long long)blockDim.x + threadIdx.x; pk < n; pk += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(pk >> 9), tid = (int)(pk & 511);
        int bx, by, bz;
        block_coord(g, av.list[a], bx, by, bz);
        const CellInfo c = cell_info(g, bx, by, bz, tid);
        if (c.oob || !surface_mask(B.masks[pk])) continue;
        const unsigned vi = B.vert_offsets[pk];
        if (vi >= max_verts || vi >= max_cells) continue;
        const float3 p = decode_vertex(B.cell_verts[vi], grid_loc(g, c.x, c.y, c.z), g.cell);
        verts[vi] = make_float4(p.x, p.y, p.z, 1.f);
    }
}

}  // namespace sdfb
