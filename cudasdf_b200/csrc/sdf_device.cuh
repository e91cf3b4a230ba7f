// Device-side SDF evaluation for sm_100a.
//
// Arithmetic: every floating-point operation on the parity path is written as an explicit
// round-to-nearest intrinsic (__fmul_rn, __fadd_rn, __fsub_rn, __fmaf_rn, __fdiv_rn, __fsqrt_rn), so
// no result depends on the compiler's contraction choices. The sequence of operations - including
// which products are fused into adds - is the one the reference's compiled code performs, pinned
// against the reference's own outputs on the GPU. The functions restate, in that exact order:
//   SDF primitives        MarchingCubesKernels.cu:129-219
//   displacements         MarchingCubesKernels.cu:229-243, 604-606
//   world -> local        MarchingCubesKernels.cu:597-599, Commons.cuh:264-278
//   CSG combine           MarchingCubesKernels.cu:631-694
//   map()                 MarchingCubesKernels.cu:570-808
//   computeNormal         MarchingCubesKernels.cu:814-844
//
// Traversal: map() is evaluated for 32 points at once by one warp. The reference runs an
// independent depth-first search per point (64-entry stack, right child pushed first, at most 256
// popped nodes, a node is skipped when its box is not closer than the running distance). Here the
// warp walks ONE stack whose entries are (node, mask of lanes that pushed it). Lane L's own stack is
// exactly the subsequence of warp entries whose mask holds L, in the same LIFO order, so each lane
// visits the same nodes in the same order, pops the same number of nodes before the cap, and folds
// the same primitives in the same order: results are identical to the per-point search, while node
// and primitive loads are warp-uniform (one broadcast load instead of 32 divergent ones).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sdfb {

// ------------------------------------------------------------------------------------------------
// exact-operation helpers
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ float MUL(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float ADD(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float SUB(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float FMA(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float DIV(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float SQRT(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ float CLAMP(float v, float lo, float hi) { return fmaxf(lo, fminf(v, hi)); }

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return f3(ADD(a.x, b.x), ADD(a.y, b.y), ADD(a.z, b.z)); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return f3(SUB(a.x, b.x), SUB(a.y, b.y), SUB(a.z, b.z)); }
__device__ __forceinline__ float3 scl3(float3 a, float s) { return f3(MUL(s, a.x), MUL(s, a.y), MUL(s, a.z)); }
// a.x*b.x + a.y*b.y + a.z*b.z
__device__ __forceinline__ float dot3(float3 a, float3 b) { return FMA(a.z, b.z, FMA(a.x, b.x, MUL(a.y, b.y))); }
__device__ __forceinline__ float len3(float3 a) { return SQRT(dot3(a, a)); }
// length(float2) with the first square fused (len2) or the second (len2b)
__device__ __forceinline__ float len2(float x, float y) { return SQRT(FMA(x, x, MUL(y, y))); }
__device__ __forceinline__ float len2b(float x, float y) { return SQRT(FMA(y, y, MUL(x, x))); }
// a*b - c*d with the first product fused
__device__ __forceinline__ float det2(float a, float b, float c, float d) { return FMA(a, b, -MUL(c, d)); }
// cross3 (MarchingCubesKernels.cu:21-27) as the DC kernels compute it: first product fused
__device__ __forceinline__ float3 cross_ff(float3 a, float3 b) {
    return f3(det2(a.y, b.z, a.z, b.y), det2(a.z, b.x, a.x, b.z), det2(a.x, b.y, a.y, b.x));
}
__device__ __forceinline__ bool finite3(float3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// ------------------------------------------------------------------------------------------------
// scene view: primitives in the reference layout (10 float4 rows of 160 bytes), nodes in the
// reference layout (2 float4 rows of 32 bytes)
// ------------------------------------------------------------------------------------------------
enum { P_SPHERE = 0, P_BOX, P_TORUS, P_CYLINDER, P_CAPSULE, P_CONE, P_RBOX, P_RCYL, P_RCONE, P_ELLIPSOID,
       P_TRIPRISM, P_OCTA, P_HEXPRISM };
enum { OP_UNION = 0, OP_SUB, OP_INT, OP_UNION_BLEND, OP_SUB_BLEND, OP_INT_BLEND };
enum { DSP_NONE = 0, DSP_SINE, DSP_TWIST, DSP_BEND };

struct SceneView {
    const float4* prims;  // 10 rows per primitive
    const float4* nodes;  // 2 rows per node
    int nprims;
    int nbvh;             // primitives [0, nbvh) are in the BVH, the rest form the linear pass
    int nnodes;
};

constexpr int PRIM_ROWS = 10;
constexpr int MAP_STACK = 64;   // the reference's per-point stack (MarchingCubesKernels.cu:577)
constexpr int MAP_CAP = 256;    // the reference's popped-node cap (:582)
constexpr int MAP_WARPS = 8;    // warps per CTA of every kernel that calls map_warp (one stack each)

// row 0 rotation | 1 dispParams | 2 position, blend | 3 scale, rounding | 4 color, annular |
// 5 params[0..3] | 6 params[4..5], type, operation | 7 displacement, pad, uvScale |
// 8 uvOffset, uvRotation, uvMode | 9 textureID, atlasIslandID, pad
struct Leaf {
    float4 rot, pos, scale, prm;
    float annular, rounding;
    int type, op, disp;
    float dp0, dp1;
};

__device__ __forceinline__ Leaf load_leaf(const float4* __restrict__ pr) {
    Leaf L;
    L.rot = __ldg(pr + 0);
    L.pos = __ldg(pr + 2);
    L.scale = __ldg(pr + 3);
    const float4 r4 = __ldg(pr + 4);
    L.prm = __ldg(pr + 5);
    const float4 r6 = __ldg(pr + 6);
    const float4 r7 = __ldg(pr + 7);
    L.annular = r4.w;
    L.rounding = L.scale.w;
    L.type = __float_as_int(r6.z);
    L.op = __float_as_int(r6.w);
    L.disp = __float_as_int(r7.x);
    L.dp0 = 0.f;
    L.dp1 = 0.f;
    if (L.disp == DSP_SINE || L.disp == DSP_TWIST || L.disp == DSP_BEND) {
        const float4 r1 = __ldg(pr + 1);
        L.dp0 = r1.x;
        L.dp1 = r1.y;
    }
    return L;
}

// rotateVector with u = q.xyz, s = q.w (Commons.cuh:264-273):
// 2*dot(u,v)*u + (s*s - dot(u,u))*v + 2*s*cross(u,v); the inline cross fuses its second product
__device__ __forceinline__ float3 rotate(float3 v, float ux, float uy, float uz, float s) {
    const float3 u = f3(ux, uy, uz);
    const float a = MUL(2.0f, FMA(u.z, v.z, FMA(u.y, v.y, MUL(u.x, v.x))));
    const float b = FMA(s, s, -dot3(u, u));
    const float c = MUL(2.0f, s);
    const float3 cr = f3(FMA(-u.z, v.y, MUL(u.y, v.z)), FMA(-u.x, v.z, MUL(u.z, v.x)), FMA(-u.y, v.x, MUL(u.x, v.y)));
    return f3(FMA(c, cr.x, FMA(b, v.x, MUL(a, u.x))), FMA(c, cr.y, FMA(b, v.y, MUL(a, u.y))),
              FMA(c, cr.z, FMA(b, v.z, MUL(a, u.z))));
}
// world -> primitive local: subtract position, conjugate rotation, divide by scale
__device__ __forceinline__ float3 to_local(float3 pw, float4 rot, float4 pos, float4 scale) {
    float3 p = f3(SUB(pw.x, pos.x), SUB(pw.y, pos.y), SUB(pw.z, pos.z));
    p = rotate(p, -rot.x, -rot.y, -rot.z, rot.w);
    return f3(DIV(p.x, scale.x), DIV(p.y, scale.y), DIV(p.z, scale.z));
}

// ---------------------------------------------------------------- primitive distance functions
__device__ __forceinline__ float sd_sphere(float3 p, float r) { return SUB(len3(p), r); }
__device__ __forceinline__ float sd_box(float3 p, float bx, float by, float bz) {
    const float qx = SUB(fabsf(p.x), bx), qy = SUB(fabsf(p.y), by), qz = SUB(fabsf(p.z), bz);
    return ADD(len3(f3(fmaxf(qx, 0.f), fmaxf(qy, 0.f), fmaxf(qz, 0.f))), fminf(fmaxf(qx, fmaxf(qy, qz)), 0.f));
}
__device__ __forceinline__ float sd_torus(float3 p, float r1, float r2) {
    return SUB(len2b(SUB(len2(p.x, p.z), r1), p.y), r2);
}
__device__ __forceinline__ float sd_cylinder(float3 p, float h, float r) {
    const float dx = SUB(fabsf(len2(p.x, p.z)), r), dy = SUB(fabsf(p.y), h);
    return ADD(fminf(fmaxf(dx, dy), 0.f), len2b(fmaxf(dx, 0.f), fmaxf(dy, 0.f)));
}
__device__ __forceinline__ float sd_capsule(float3 p, float h, float r) {
    p.y = SUB(p.y, CLAMP(p.y, 0.f, h));
    return SUB(len3(p), r);
}
__device__ __forceinline__ float sd_cone(float3 p, float h, float angle) {
    const float cx = sinf(MUL(angle, 0.0174533f)), cy = cosf(MUL(angle, 0.0174533f));
    const float qx = MUL(h, DIV(cx, cy)), qy = -h;
    const float wx = len2(p.x, p.z), wy = p.y;
    const float dwq = FMA(wx, qx, MUL(wy, qy));
    const float dqq = FMA(qx, qx, MUL(qy, qy));
    const float t = CLAMP(DIV(dwq, dqq), 0.f, 1.f);
    const float ax = FMA(-qx, t, wx), ay = FMA(-qy, t, wy);
    const float tb = CLAMP(DIV(wx, qx), 0.f, 1.f);
    const float bx = FMA(-qx, tb, wx), by = SUB(wy, qy);
    const float k = (qy > 0.f) ? 1.f : -1.f;
    const float d = fminf(FMA(ax, ax, MUL(ay, ay)), FMA(bx, bx, MUL(by, by)));
    const float s = fmaxf(MUL(k, det2(wx, qy, wy, qx)), MUL(k, SUB(wy, qy)));
    return MUL(SQRT(d), (s > 0.f ? 1.f : -1.f));
}
__device__ __forceinline__ float sd_ellipsoid(float3 p, float rx, float ry, float rz) {
    const float k0 = len3(f3(DIV(p.x, rx), DIV(p.y, ry), DIV(p.z, rz)));
    const float k1 = len3(f3(DIV(p.x, MUL(rx, rx)), DIV(p.y, MUL(ry, ry)), DIV(p.z, MUL(rz, rz))));
    return DIV(MUL(k0, SUB(k0, 1.f)), k1);
}
__device__ __forceinline__ float sd_octahedron(float3 p, float s) {
    return MUL(SUB(ADD(ADD(fabsf(p.x), fabsf(p.y)), fabsf(p.z)), s), 0.57735027f);
}
__device__ __forceinline__ float sd_triprism(float3 p, float hx, float hy) {
    const float qx = fabsf(p.x), qz = fabsf(p.z);
    return fmaxf(SUB(qz, hy), FMA(-hx, 0.5f, fmaxf(FMA(qx, 0.866025f, MUL(p.y, 0.5f)), -p.y)));
}
__device__ __forceinline__ float sd_rounded_cone(float3 p, float h, float r1, float r2) {
    const float qx = len2(p.x, p.z), qy = p.y;
    const float b = DIV(SUB(r1, r2), h);
    const float a = SQRT(FMA(-b, b, 1.f));
    const float k = FMA(qx, -b, MUL(qy, a));
    if (k < 0.f) return SUB(len2b(qx, qy), r1);
    if (k > MUL(a, h)) return SUB(len2b(qx, SUB(qy, h)), r2);
    return SUB(FMA(qy, b, MUL(qx, a)), r1);
}
__device__ __forceinline__ float sd_rounded_cylinder(float3 p, float h, float r1, float r2) {
    const float dx = ADD(FMA(-2.f, r1, len2(p.x, p.z)), r2), dy = SUB(fabsf(p.y), h);
    return SUB(ADD(fminf(fmaxf(dx, dy), 0.f), len2b(fmaxf(dx, 0.f), fmaxf(dy, 0.f))), r2);
}
__device__ __forceinline__ float sd_hexprism(float3 p, float hx, float hy) {
    const float kx = -0.8660254f, ky = 0.5f, kz = 0.57735027f;
    p = f3(fabsf(p.x), fabsf(p.y), fabsf(p.z));
    const float m = fminf(FMA(ky, p.z, MUL(kx, p.x)), 0.f);
    const float px = FMA(-MUL(kx, 2.f), m, p.x), pz = FMA(-MUL(ky, 2.f), m, p.z);
    const float ex = SUB(px, CLAMP(px, MUL(-kz, hx), MUL(kz, hx))), ez = SUB(pz, hx);
    const float dx = MUL(len2b(ex, ez), copysignf(1.f, SUB(pz, hx))), dy = SUB(p.y, hy);
    return ADD(fminf(fmaxf(dx, dy), 0.f), len2b(fmaxf(dx, 0.f), fmaxf(dy, 0.f)));
}

__device__ __forceinline__ float sd_eval(int type, float3 p, float4 pm) {
    switch (type) {
        case P_SPHERE: return sd_sphere(p, pm.x);
        case P_BOX: return sd_box(p, pm.x, pm.y, pm.z);
        case P_TORUS: return sd_torus(p, pm.x, pm.y);
        case P_CYLINDER: return sd_cylinder(p, pm.x, pm.y);
        case P_CAPSULE: return sd_capsule(p, pm.x, pm.y);
        case P_CONE: return sd_cone(p, pm.x, pm.y);
        case P_RBOX: return SUB(sd_box(p, pm.x, pm.y, pm.z), pm.w);
        case P_ELLIPSOID: return sd_ellipsoid(p, pm.x, pm.y, pm.z);
        case P_OCTA: return sd_octahedron(p, pm.x);
        case P_TRIPRISM: return sd_triprism(p, pm.x, pm.y);
        case P_RCYL: return sd_rounded_cylinder(p, pm.x, pm.y, pm.z);
        case P_RCONE: return sd_rounded_cone(p, pm.x, pm.y, pm.z);
        case P_HEXPRISM: return sd_hexprism(p, pm.x, pm.y);
        default: return SUB(len3(p), 1.f);
    }
}

// leaf: local transform, displacement, distance, min-scale, annular, rounding (:594-629)
__device__ __forceinline__ float leaf_distance(const Leaf& L, float3 pw, float time, float3& pre) {
    float3 p = to_local(pw, L.rot, L.pos, L.scale);
    pre = p;
    if (L.disp == DSP_TWIST) {
        const float c = cosf(MUL(L.dp0, p.y)), s = sinf(MUL(L.dp0, p.y));
        p = f3(det2(c, p.x, s, p.z), p.y, FMA(c, p.z, MUL(s, p.x)));
    } else if (L.disp == DSP_BEND) {
        const float c = cosf(MUL(L.dp0, p.x)), s = sinf(MUL(L.dp0, p.x));
        p = f3(det2(c, p.x, s, p.y), FMA(c, p.y, MUL(s, p.x)), p.z);
    } else if (L.disp == DSP_SINE) {
        p.y = FMA(sinf(FMA(p.x, L.dp0, time)), L.dp1, p.y);
    }
    float d = sd_eval(L.type, p, L.prm);
    d = MUL(d, fminf(L.scale.x, fminf(L.scale.y, L.scale.z)));
    if (L.annular > 0.f) d = SUB(fabsf(d), L.annular);
    if (L.rounding > 0.f) d = SUB(d, L.rounding);
    return d;
}

// mix(x, y, a) = x*(1-a) + y*a (Commons.cuh:247). Inside map()'s blends the union / intersect
// blends and the colour mix fuse y*a, the subtract blend fuses x*(1-a).
__device__ __forceinline__ float mix_fy(float x, float y, float a) { return FMA(y, a, MUL(x, SUB(1.f, a))); }
__device__ __forceinline__ float mix_fx(float x, float y, float a) { return FMA(x, SUB(1.f, a), MUL(y, a)); }

// running state of one point's map(); colour/id/local only tracked when ATTR
template <bool ATTR>
struct MapState {
    float d;
    float3 color;
    int id;
    float3 local;
    __device__ __forceinline__ void init() {
        d = 1e10f;
        if (ATTR) {
            color = f3(0.f, 0.f, 0.f);
            id = -1;
            local = f3(0.f, 0.f, 0.f);
        }
    }
};

// CSG combine (MarchingCubesKernels.cu:631-694)
template <bool ATTR>
__device__ __forceinline__ void combine(MapState<ATTR>& st, int op, float k, const float4* __restrict__ pr, int i,
                                        float dp, float3 pre) {
    float3 pc = f3(0.f, 0.f, 0.f);
    if (ATTR) {
        const float4 c4 = __ldg(pr + 4);
        pc = f3(c4.x, c4.y, c4.z);
    }
    if (st.d == 1e10f) {
        st.d = dp;
        if (ATTR) { st.color = pc; st.id = i; st.local = pre; }
        return;
    }
    float h;
    switch (op) {
        case OP_UNION:
            if (dp < st.d) {
                st.d = dp;
                if (ATTR) { st.color = pc; st.id = i; st.local = pre; }
            }
            break;
        case OP_SUB: {
            const float old = st.d;
            st.d = fmaxf(st.d, -dp);
            if (ATTR && st.d > old) { st.color = pc; st.id = i; st.local = pre; }
        } break;
        case OP_INT:
            if (dp > st.d) {
                st.d = dp;
                if (ATTR) { st.color = pc; st.id = i; st.local = pre; }
            }
            break;
        case OP_UNION_BLEND:
            h = CLAMP(ADD(0.5f, DIV(MUL(0.5f, SUB(st.d, dp)), k)), 0.f, 1.f);
            st.d = FMA(-MUL(k, h), SUB(1.f, h), mix_fy(st.d, dp, h));
            if (ATTR) {
                st.color = f3(mix_fy(st.color.x, pc.x, h), mix_fy(st.color.y, pc.y, h), mix_fy(st.color.z, pc.z, h));
                if (dp < st.d || h > 0.5f) { st.id = i; st.local = pre; }
            }
            break;
        case OP_SUB_BLEND:
            h = CLAMP(SUB(0.5f, DIV(MUL(0.5f, ADD(st.d, dp)), k)), 0.f, 1.f);
            st.d = FMA(MUL(k, h), SUB(1.f, h), mix_fx(st.d, -dp, h));
            if (ATTR) {
                st.color = f3(mix_fy(st.color.x, pc.x, h), mix_fy(st.color.y, pc.y, h), mix_fy(st.color.z, pc.z, h));
                if (h > 0.5f) { st.id = i; st.local = pre; }
            }
            break;
        case OP_INT_BLEND:
            h = CLAMP(SUB(0.5f, DIV(MUL(0.5f, SUB(st.d, dp)), k)), 0.f, 1.f);
            st.d = FMA(MUL(k, h), SUB(1.f, h), mix_fy(st.d, dp, h));
            if (ATTR) {
                st.color = f3(mix_fy(st.color.x, pc.x, h), mix_fy(st.color.y, pc.y, h), mix_fy(st.color.z, pc.z, h));
                if (dp > st.d || h > 0.5f) { st.id = i; st.local = pre; }
            }
            break;
        default: break;
    }
}

// ---------------------------------------------------------------- two points of one lane, one primitive
// The two points of a map_pair lane folding the same primitive: the same operations as two
// leaf_distance / combine<false> calls, with the type and operation dispatched once and, for points
// (x, y, z0) and (x, y, z1), the parts of the transform that depend on x and y alone computed once.

// the primitive-local points of to_local for both points (rotate's operations, shared terms once)
__device__ __forceinline__ void to_local2(float3 pw, float z1, float4 rot, float4 pos, float4 scale, float3& q0,
                                          float3& q1) {
    const float ux = -rot.x, uy = -rot.y, uz = -rot.z, s = rot.w;
    const float vx = SUB(pw.x, pos.x), vy = SUB(pw.y, pos.y);
    const float vz0 = SUB(pw.z, pos.z), vz1 = SUB(z1, pos.z);
    const float axy = FMA(uy, vy, MUL(ux, vx));                         // dot(u, v) without its z term
    const float b = FMA(s, s, -FMA(uz, uz, FMA(ux, ux, MUL(uy, uy))));  // s*s - dot3(u, u)
    const float c = MUL(2.0f, s);
    const float crz = FMA(-uy, vx, MUL(ux, vy));
    const float cyx = MUL(uz, vx);
    const float a0 = MUL(2.0f, FMA(uz, vz0, axy)), a1 = MUL(2.0f, FMA(uz, vz1, axy));
    const float crx0 = FMA(-uz, vy, MUL(uy, vz0)), crx1 = FMA(-uz, vy, MUL(uy, vz1));
    const float cry0 = FMA(-ux, vz0, cyx), cry1 = FMA(-ux, vz1, cyx);
    q0 = f3(DIV(FMA(c, crx0, FMA(b, vx, MUL(a0, ux))), scale.x), DIV(FMA(c, cry0, FMA(b, vy, MUL(a0, uy))), scale.y),
            DIV(FMA(c, crz, FMA(b, vz0, MUL(a0, uz))), scale.z));
    q1 = f3(DIV(FMA(c, crx1, FMA(b, vx, MUL(a1, ux))), scale.x), DIV(FMA(c, cry1, FMA(b, vy, MUL(a1, uy))), scale.y),
            DIV(FMA(c, crz, FMA(b, vz1, MUL(a1, uz))), scale.z));
}

// the displacement of leaf_distance for one local point
__device__ __forceinline__ float3 displace(const Leaf& L, float3 p, float time) {
    if (L.disp == DSP_TWIST) {
        const float c = cosf(MUL(L.dp0, p.y)), s = sinf(MUL(L.dp0, p.y));
        p = f3(det2(c, p.x, s, p.z), p.y, FMA(c, p.z, MUL(s, p.x)));
    } else if (L.disp == DSP_BEND) {
        const float c = cosf(MUL(L.dp0, p.x)), s = sinf(MUL(L.dp0, p.x));
        p = f3(det2(c, p.x, s, p.y), FMA(c, p.y, MUL(s, p.x)), p.z);
    } else if (L.disp == DSP_SINE) {
        p.y = FMA(sinf(FMA(p.x, L.dp0, time)), L.dp1, p.y);
    }
    return p;
}

// sd_eval for two points of the same primitive
__device__ __forceinline__ void sd_eval2(int type, float3 p0, float3 p1, float4 pm, float& d0, float& d1) {
    switch (type) {
        case P_SPHERE: d0 = sd_sphere(p0, pm.x); d1 = sd_sphere(p1, pm.x); break;
        case P_BOX: d0 = sd_box(p0, pm.x, pm.y, pm.z); d1 = sd_box(p1, pm.x, pm.y, pm.z); break;
        case P_TORUS: d0 = sd_torus(p0, pm.x, pm.y); d1 = sd_torus(p1, pm.x, pm.y); break;
        case P_CAPSULE: d0 = sd_capsule(p0, pm.x, pm.y); d1 = sd_capsule(p1, pm.x, pm.y); break;
        default: d0 = sd_eval(type, p0, pm); d1 = sd_eval(type, p1, pm); break;
    }
}

// leaf_distance at p0 and p1 (SAME_XY: p1 differs from p0 only in z, and the transform shares terms)
template <bool SAME_XY>
__device__ __forceinline__ void leaf_distance2(const Leaf& L, float3 p0, float3 p1, float time, float& d0, float& d1) {
    float3 q0, q1;
    if (SAME_XY) {
        to_local2(p0, p1.z, L.rot, L.pos, L.scale, q0, q1);
    } else {
        q0 = to_local(p0, L.rot, L.pos, L.scale);
        q1 = to_local(p1, L.rot, L.pos, L.scale);
    }
    if (L.disp != DSP_NONE) {
        q0 = displace(L, q0, time);
        q1 = displace(L, q1, time);
    }
    sd_eval2(L.type, q0, q1, L.prm, d0, d1);
    const float ms = fminf(L.scale.x, fminf(L.scale.y, L.scale.z));
    d0 = MUL(d0, ms);
    d1 = MUL(d1, ms);
    if (L.annular > 0.f) {
        d0 = SUB(fabsf(d0), L.annular);
        d1 = SUB(fabsf(d1), L.annular);
    }
    if (L.rounding > 0.f) {
        d0 = SUB(d0, L.rounding);
        d1 = SUB(d1, L.rounding);
    }
}

// combine<false>'s new running distance for one point
template <int OP>
__device__ __forceinline__ float fold_d(float d, float dp, float k) {
    if (d == 1e10f) return dp;
    float h;
    switch (OP) {
        case OP_UNION: return dp < d ? dp : d;
        case OP_SUB: return fmaxf(d, -dp);
        case OP_INT: return dp > d ? dp : d;
        case OP_UNION_BLEND:
            h = CLAMP(ADD(0.5f, DIV(MUL(0.5f, SUB(d, dp)), k)), 0.f, 1.f);
            return FMA(-MUL(k, h), SUB(1.f, h), mix_fy(d, dp, h));
        case OP_SUB_BLEND:
            h = CLAMP(SUB(0.5f, DIV(MUL(0.5f, ADD(d, dp)), k)), 0.f, 1.f);
            return FMA(MUL(k, h), SUB(1.f, h), mix_fx(d, -dp, h));
        case OP_INT_BLEND:
            h = CLAMP(SUB(0.5f, DIV(MUL(0.5f, SUB(d, dp)), k)), 0.f, 1.f);
            return FMA(MUL(k, h), SUB(1.f, h), mix_fy(d, dp, h));
        default: return d;
    }
}

// combine<false> for both points, the operation dispatched once
__device__ __forceinline__ void combine_d2(int op, float k, float& d0, float& d1, float dp0, float dp1) {
    switch (op) {
        case OP_UNION: d0 = fold_d<OP_UNION>(d0, dp0, k); d1 = fold_d<OP_UNION>(d1, dp1, k); break;
        case OP_SUB: d0 = fold_d<OP_SUB>(d0, dp0, k); d1 = fold_d<OP_SUB>(d1, dp1, k); break;
        case OP_INT: d0 = fold_d<OP_INT>(d0, dp0, k); d1 = fold_d<OP_INT>(d1, dp1, k); break;
        case OP_UNION_BLEND: d0 = fold_d<OP_UNION_BLEND>(d0, dp0, k); d1 = fold_d<OP_UNION_BLEND>(d1, dp1, k); break;
        case OP_SUB_BLEND: d0 = fold_d<OP_SUB_BLEND>(d0, dp0, k); d1 = fold_d<OP_SUB_BLEND>(d1, dp1, k); break;
        case OP_INT_BLEND: d0 = fold_d<OP_INT_BLEND>(d0, dp0, k); d1 = fold_d<OP_INT_BLEND>(d1, dp1, k); break;
        default: d0 = fold_d<-1>(d0, dp0, k); d1 = fold_d<-1>(d1, dp1, k); break;
    }
}

// intersectAABB (MarchingCubesKernels.cu:564-568): sqrt_rn(|p - box|^2) < running d.
// The same decision without the square root in all but boundary cases: with D = dmin^2 rounded,
// dd < D(1 - 2^-20) implies sqrt_rn(dd) < dmin, and dd > D(1 + 2^-20) implies sqrt_rn(dd) > dmin
// (the two roundings of D and of the square root are each within 2^-24 relative, far inside the
// 2^-20 margin); in between, and when dmin^2 could under- or overflow, the square root decides.
__device__ __forceinline__ bool box_closer(float3 p, float4 a, float4 b, float dmin) {
    const float dx = fmaxf(fmaxf(SUB(a.x, p.x), SUB(p.x, a.w)), 0.f);
    const float dy = fmaxf(fmaxf(SUB(a.y, p.y), SUB(p.y, b.x)), 0.f);
    const float dz = fmaxf(fmaxf(SUB(a.z, p.z), SUB(p.z, b.y)), 0.f);
    const float dd = FMA(dz, dz, FMA(dx, dx, MUL(dy, dy)));
    if (!(dmin > 0.f)) return false;  // sqrt_rn(dd) >= 0; NaN compares false
    if (dmin >= 1e-18f && dmin <= 1e18f) {
        const float d2 = MUL(dmin, dmin);
        if (dd < MUL(d2, 0x1.ffffep-1f)) return true;   // 1 - 2^-20
        if (dd > MUL(d2, 0x1.00001p+0f)) return false;  // 1 + 2^-20
    }
    return SQRT(dd) < dmin;
}

// The decision of box_closer for one running distance dmin, with the parts that depend on dmin alone
// computed once per change of dmin: lo / hi are the two fast-path thresholds (lo = hi = -1 when
// dmin > 0 fails, so every box is rejected; lo = -1, hi = +inf when dmin^2 could under- or overflow,
// so the square root decides).
struct PruneBound {
    float lo, hi, dmin;
    __device__ __forceinline__ void set(float d) {
        dmin = d;
        if (!(d > 0.f)) {
            lo = -1.f;
            hi = -1.f;
        } else if (d >= 1e-18f && d <= 1e18f) {
            const float d2 = MUL(d, d);
            lo = MUL(d2, 0x1.ffffep-1f);
            hi = MUL(d2, 0x1.00001p+0f);
        } else {
            lo = -1.f;
            hi = __int_as_float(0x7f800000);
        }
    }
    __device__ __forceinline__ bool alive() const { return hi >= 0.f; }
    // sqrt(dd) < dmin for the dmin of the last set()
    __device__ __forceinline__ bool closer_dd(float dd) const {
        if (dd < lo) return true;
        if (dd > hi) return false;
        return SQRT(dd) < dmin;
    }
    // box_closer(p, a, b, dmin) for the dmin of the last set()
    __device__ __forceinline__ bool closer(float3 p, float4 a, float4 b) const {
        return closer_dd(box_dd_z(p.z, a, b, box_dd_xy(p, a, b)));
    }
    // the squared box distance of box_closer in its rounding order, dz^2 + (dx^2 + dy^2): the
    // bracket depends on x and y only, so points that differ only in z share it
    __device__ __forceinline__ static float box_dd_xy(float3 p, float4 a, float4 b) {
        const float dx = fmaxf(fmaxf(SUB(a.x, p.x), SUB(p.x, a.w)), 0.f);
        const float dy = fmaxf(fmaxf(SUB(a.y, p.y), SUB(p.y, b.x)), 0.f);
        return FMA(dx, dx, MUL(dy, dy));
    }
    __device__ __forceinline__ static float box_dd_z(float z, float4 a, float4 b, float xy) {
        const float dz = fmaxf(fmaxf(SUB(a.z, z), SUB(z, b.y)), 0.f);
        return FMA(dz, dz, xy);
    }
};

// Per-launch diagnostics shared by all kernels of an extraction.
struct Diag {
    unsigned long long cap_hits;    // points whose search was cut by the 256-pop cap
    unsigned long long fp64_cells;  // mass-point DC cells solved with the FP64 eigensolve
    unsigned long long node_pops;   // work counters (counting runs only): per-point popped nodes,
    unsigned long long leaf_evals;  //   per-point primitive evaluations,
    unsigned long long points;      //   evaluated points
    unsigned long long scouted;     // blocks the surrogate-culled scout evaluated exactly
    unsigned long long warp_pops;   // counting runs: warp-wide stack pops,
    unsigned long long warp_tests;  //   of which with a box test (some lane alive),
    unsigned long long warp_leaves; //   and leaf steps (some lane evaluates the primitive)
    int stack_overflow;             // a search needed more than 64 stack entries
    int timeout;                    // a bounded wait gave up
    int inconsistent;               // a kernel found another's list disagreeing with its own work (a bug)
};

// The stacks of map_multi (every point count shares them: a warp runs one walk at a time), 2 KB per
// warp of the CTA.
constexpr int MULTI_STACK_UINT4 = MAP_STACK * 2;  // uint4 per warp
__shared__ uint4 s_multi_stack[MAP_WARPS * MULTI_STACK_UINT4];

// The first pops of every walk. While no primitive has been folded, every running distance is 1e10,
// and a box whose six coordinates are below 1e8 in magnitude passes the prune test for every point
// below 1e8 (squared distance under 1.2e17, square root under 3.5e8 < 1e10). So every walk starts by
// popping the root and descending along left children, each point hitting every node, each right
// child pushed with the live masks, down to the first leaf. first_descent replays that without the
// box tests: push(sp, right) stores one entry (lane 0), and the return value is the number of
// internal nodes popped (each live point's pop count). It stops at a leaf, at a box outside the bound
// and where the ordinary walk would overflow the stack; the ordinary walk then pops `node` next.
constexpr float DESCENT_BOUND = 1e8f;
__device__ __forceinline__ bool below_descent_bound(float x) { return fabsf(x) < DESCENT_BOUND; }  // NaN fails
template <class Push>
__device__ __forceinline__ int first_descent(const SceneView& sc, int& node, int& sp, Push push) {
    int depth = 0;
    for (;;) {
        const float4 nb = __ldg(sc.nodes + 2 * node + 1);
        const int right = __float_as_int(nb.w);
        if (right == -1 || sp + 2 > MAP_STACK) break;
        const float4 na = __ldg(sc.nodes + 2 * node);
        if (!(below_descent_bound(na.x) && below_descent_bound(na.y) && below_descent_bound(na.z) &&
              below_descent_bound(na.w) && below_descent_bound(nb.x) && below_descent_bound(nb.y)))
            break;
        push(sp, right);
        ++sp;
        node = __float_as_int(nb.z);
        ++depth;
    }
    __syncwarp();  // the pushed entries are visible to the warp's pops
    return depth;
}

// map() for the 32 points of a warp. Must be called by all 32 lanes together (warp-uniform control
// flow); lanes with valid == false take part in the walk but own no point.
template <bool ATTR, bool COUNT = false>
__device__ __forceinline__ void map_warp(const SceneView& sc, float3 p, bool valid, float time, MapState<ATTR>& st,
                                         Diag* diag) {
    unsigned long long cnt_pops = 0, cnt_leaves = 0, cnt_wpops = 0, cnt_wtests = 0, cnt_wleaves = 0;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    st.init();
    const unsigned live = __ballot_sync(FULL, valid);
    int iter = 0;
    // the warp's stack of (node, mask of the lanes that pushed it) in shared memory; a CTA with more
    // warps than stacks is refused (reported as a stack overflow)
    __shared__ uint2 s_map_stack[MAP_WARPS][MAP_STACK];
    bool overflow = blockDim.x > 32 * MAP_WARPS;
    if (sc.nnodes > 0 && live && !overflow) {
        PruneBound pb;
        pb.set(st.d);
        uint2* stk = s_map_stack[threadIdx.x >> 5];
        // The reference pushes right then left and pops the left child next; here the left child is
        // kept as the next node (same mask) and only the right one goes on the stack: the same pop
        // sequence with one stack entry less per internal node.
        int sp = 0;
        int node = 0;
        unsigned mask = live;
        bool have = true;
        // counting runs walk every pop, so the work counters count the descent's tests too
        if (!COUNT && __all_sync(FULL, !valid || (below_descent_bound(p.x) && below_descent_bound(p.y) &&
                                                  below_descent_bound(p.z)))) {
            const int depth = first_descent(sc, node, sp, [&](int s, int right) {
                if (lane == 0) stk[s] = make_uint2((unsigned)right, live);
            });
            if (valid) iter = depth;
        }
        for (;;) {
            if (!have) {
                if (sp == 0) break;
                --sp;
                const uint2 e = stk[sp];
                node = (int)e.x;
                mask = e.y;
            }
            have = false;
            // a lane pops this node iff it pushed it and has popped fewer than MAP_CAP nodes
            const bool pops = ((mask >> lane) & 1u) && iter < MAP_CAP;
            if (pops) iter++;
            if (COUNT) {
                cnt_pops += __popc(__ballot_sync(FULL, pops));
                ++cnt_wpops;
            }
            // a node can only pass the prune test for a lane whose running distance is > 0
            const bool lane_alive = pops && pb.alive();
            if (!__any_sync(FULL, lane_alive)) continue;
            if (COUNT) ++cnt_wtests;
            const float4 na = __ldg(sc.nodes + 2 * node);
            const float4 nb = __ldg(sc.nodes + 2 * node + 1);
            const bool hit = lane_alive && pb.closer(p, na, nb);
            const unsigned hm = __ballot_sync(FULL, hit);
            if (hm == 0) continue;
            const int left = __float_as_int(nb.z), right = __float_as_int(nb.w);
            if (right == -1) {
                const float4* pr = sc.prims + (size_t)left * PRIM_ROWS;
                const Leaf L = load_leaf(pr);
                if (COUNT) {
                    cnt_leaves += __popc(hm);
                    ++cnt_wleaves;
                }
                if (hit) {
                    float3 pre;
                    const float dp = leaf_distance(L, p, time, pre);
                    combine<ATTR>(st, L.op, L.pos.w, pr, left, dp, pre);
                    pb.set(st.d);
                }
            } else {
                if (sp + 2 > MAP_STACK) { overflow = true; break; }  // the reference's stack holds both
                __syncwarp();  // every lane has read stk[sp] (popped above) before it is overwritten
                if (lane == 0) stk[sp] = make_uint2((unsigned)right, hm);
                __syncwarp();
                ++sp;
                node = left;
                mask = hm;
                have = true;
            }
        }
        if (diag) {
            const unsigned capped = __ballot_sync(FULL, valid && iter >= MAP_CAP);
            if (lane == 0 && capped) atomicAdd(&diag->cap_hits, (unsigned long long)__popc(capped));
        }
    }
    if (diag && overflow && lane == 0) atomicExch(&diag->stack_overflow, 1);
    if (COUNT && diag && lane == 0) {
        const unsigned nlive = __popc(live);
        atomicAdd(&diag->node_pops, cnt_pops);
        atomicAdd(&diag->leaf_evals, cnt_leaves + (unsigned long long)nlive * (sc.nprims - sc.nbvh));
        atomicAdd(&diag->points, (unsigned long long)nlive);
        atomicAdd(&diag->warp_pops, cnt_wpops);
        atomicAdd(&diag->warp_tests, cnt_wtests);
        atomicAdd(&diag->warp_leaves, cnt_wleaves);
    }
    // non-union primitives: a linear pass in scene order (:703-803)
    for (int i = sc.nbvh; i < sc.nprims; ++i) {
        const float4* pr = sc.prims + (size_t)i * PRIM_ROWS;
        const Leaf L = load_leaf(pr);
        if (valid) {
            float3 pre;
            const float dp = leaf_distance(L, p, time, pre);
            combine<ATTR>(st, L.op, L.pos.w, pr, i, dp, pre);
        }
    }
}

// map() distance for 64 points per warp, two per lane (points 0 and 1 of a lane are usually
// neighbours). One stack entry carries the two lane masks of its pushers, so the pop, the node loads,
// the ballots and the push are shared by the two walks while every point still makes its own prune
// decision at every node it pops: each point's sequence of pops is its own depth-first walk with the
// 64-entry stack and the 256-pop cap, exactly as in map_warp. Must be called by all 32 lanes.
// SAME_XY: the two points of every lane differ only in z (p1.x == p0.x, p1.y == p0.y), so the x and y
// part of each box distance and of each primitive transform is computed once for both.
template <bool COUNT, bool SAME_XY>
__device__ __forceinline__ void map_pair(const SceneView& sc, float3 p0, float3 p1, bool v0, bool v1, float time,
                                         float& d0, float& d1, Diag* diag) {
    const float z1 = p1.z;
    unsigned long long cnt_pops = 0, cnt_leaves = 0, cnt_wpops = 0, cnt_wtests = 0, cnt_wleaves = 0;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    MapState<false> s0, s1;
    s0.init();
    s1.init();
    const unsigned live0 = __ballot_sync(FULL, v0), live1 = __ballot_sync(FULL, v1);
    int it0 = 0, it1 = 0;
    __shared__ uint4 s_map_stack2[MAP_WARPS][MAP_STACK];
    bool overflow = blockDim.x > 32 * MAP_WARPS;
    if (sc.nnodes > 0 && (live0 | live1) && !overflow) {
        PruneBound b0, b1;
        b0.set(s0.d);
        b1.set(s1.d);
        uint4* stk = s_map_stack2[threadIdx.x >> 5];
        int sp = 0;
        int node = 0;
        unsigned m0 = live0, m1 = live1;
        bool have = true;
        const bool ok0 = below_descent_bound(p0.x) && below_descent_bound(p0.y) && below_descent_bound(p0.z);
        const bool ok1 = below_descent_bound(p1.x) && below_descent_bound(p1.y) && below_descent_bound(p1.z);
        if (!COUNT && __all_sync(FULL, (!v0 || ok0) && (!v1 || ok1))) {
            const int depth = first_descent(sc, node, sp, [&](int s, int right) {
                if (lane == 0) stk[s] = make_uint4((unsigned)right, live0, live1, 0u);
            });
            if (v0) it0 = depth;
            if (v1) it1 = depth;
        }
        for (;;) {
            if (!have) {
                if (sp == 0) break;
                --sp;
                const uint4 e = stk[sp];
                node = (int)e.x;
                m0 = e.y;
                m1 = e.z;
            }
            have = false;
            const bool pops0 = ((m0 >> lane) & 1u) && it0 < MAP_CAP;
            const bool pops1 = ((m1 >> lane) & 1u) && it1 < MAP_CAP;
            if (pops0) it0++;
            if (pops1) it1++;
            if (COUNT) {
                cnt_pops += __popc(__ballot_sync(FULL, pops0)) + __popc(__ballot_sync(FULL, pops1));
                cnt_wpops += 2;
            }
            const bool a0 = pops0 && b0.alive(), a1 = pops1 && b1.alive();
            if (!__any_sync(FULL, a0 || a1)) continue;
            if (COUNT) cnt_wtests += 2;
            const float4 na = __ldg(sc.nodes + 2 * node);
            const float4 nb = __ldg(sc.nodes + 2 * node + 1);
            const float xy = PruneBound::box_dd_xy(p0, na, nb);
            const float xy1 = SAME_XY ? xy : PruneBound::box_dd_xy(p1, na, nb);
            const bool h0 = a0 && b0.closer_dd(PruneBound::box_dd_z(p0.z, na, nb, xy));
            const bool h1 = a1 && b1.closer_dd(PruneBound::box_dd_z(z1, na, nb, xy1));
            const unsigned hm0 = __ballot_sync(FULL, h0), hm1 = __ballot_sync(FULL, h1);
            if ((hm0 | hm1) == 0) continue;
            const int left = __float_as_int(nb.z), right = __float_as_int(nb.w);
            if (right == -1) {
                const float4* pr = sc.prims + (size_t)left * PRIM_ROWS;
                const Leaf L = load_leaf(pr);
                if (COUNT) {
                    cnt_leaves += __popc(hm0) + __popc(hm1);
                    cnt_wleaves += (__any_sync(FULL, h0 || h1) ? 1 : 0) + (__any_sync(FULL, h0 && h1) ? 1 : 0);
                }
                if (__any_sync(FULL, h0 && h1)) {
                    // some lane folds the primitive into both its points: one pass evaluates both
                    // points of every lane that hit with either, and each point keeps the fold only
                    // where it hit (an unchanged distance leaves its prune bound unchanged)
                    if (h0 || h1) {
                        float dp0, dp1;
                        leaf_distance2<SAME_XY>(L, p0, p1, time, dp0, dp1);
                        float n0 = s0.d, n1 = s1.d;
                        combine_d2(L.op, L.pos.w, n0, n1, dp0, dp1);
                        s0.d = h0 ? n0 : s0.d;
                        s1.d = h1 ? n1 : s1.d;
                        b0.set(s0.d);
                        b1.set(s1.d);
                    }
                } else if (h0 || h1) {
                    // each lane folds the primitive into one point
                    const bool use0 = h0;
                    MapState<false> t;
                    t.d = use0 ? s0.d : s1.d;
                    float3 pre;
                    const float dp = leaf_distance(L, use0 ? p0 : p1, time, pre);
                    combine<false>(t, L.op, L.pos.w, pr, left, dp, pre);
                    if (use0) {
                        s0.d = t.d;
                        b0.set(t.d);
                    } else {
                        s1.d = t.d;
                        b1.set(t.d);
                    }
                }
            } else {
                if (sp + 2 > MAP_STACK) { overflow = true; break; }  // the reference's stack holds both
                __syncwarp();  // every lane has read stk[sp] (popped above) before it is overwritten
                if (lane == 0) stk[sp] = make_uint4((unsigned)right, hm0, hm1, 0u);
                __syncwarp();
                ++sp;
                node = left;
                m0 = hm0;
                m1 = hm1;
                have = true;
            }
        }
        if (diag) {
            const unsigned c0 = __ballot_sync(FULL, v0 && it0 >= MAP_CAP), c1 = __ballot_sync(FULL, v1 && it1 >= MAP_CAP);
            if (lane == 0 && (c0 | c1)) atomicAdd(&diag->cap_hits, (unsigned long long)(__popc(c0) + __popc(c1)));
        }
    }
    if (diag && overflow && lane == 0) atomicExch(&diag->stack_overflow, 1);
    if (COUNT && diag && lane == 0) {
        const unsigned nlive = __popc(live0) + __popc(live1);
        atomicAdd(&diag->node_pops, cnt_pops);
        atomicAdd(&diag->leaf_evals, cnt_leaves + (unsigned long long)nlive * (sc.nprims - sc.nbvh));
        atomicAdd(&diag->points, (unsigned long long)nlive);
        atomicAdd(&diag->warp_pops, cnt_wpops);
        atomicAdd(&diag->warp_tests, cnt_wtests);
        atomicAdd(&diag->warp_leaves, cnt_wleaves);
    }
    // non-union primitives: a linear pass in scene order (:703-803)
    for (int i = sc.nbvh; i < sc.nprims; ++i) {
        const float4* pr = sc.prims + (size_t)i * PRIM_ROWS;
        const Leaf L = load_leaf(pr);
        if (v0) {
            float3 pre;
            const float dp = leaf_distance(L, p0, time, pre);
            combine<false>(s0, L.op, L.pos.w, pr, i, dp, pre);
        }
        if (v1) {
            float3 pre;
            const float dp = leaf_distance(L, p1, time, pre);
            combine<false>(s1, L.op, L.pos.w, pr, i, dp, pre);
        }
    }
    d0 = s0.d;
    d1 = s1.d;
}

// map_pair for two points per lane that differ only in z: (p0.x, p0.y, p0.z) and (p0.x, p0.y, z1)
template <bool COUNT = false>
__device__ __forceinline__ void map_warp2(const SceneView& sc, float3 p0, float z1, bool v0, bool v1, float time,
                                          float& d0, float& d1, Diag* diag) {
    map_pair<COUNT, true>(sc, p0, f3(p0.x, p0.y, z1), v0, v1, time, d0, d1, diag);
}

// map() distance for NP points per lane (32 x NP per warp) that are close together, such as the four
// points of computeNormal's stencil: one shared stack whose entries carry NP lane masks, so the pop,
// the node loads, the ballots and the push are shared by the NP walks, while every point makes its
// own prune decision at every node it pops: each point's sequence of pops is its own depth-first walk
// with the 64-entry stack and the 256-pop cap, as in map_warp. Leaf steps evaluate a lane's hit
// points one after another. Must be called by all 32 lanes.
template <int NP>
__device__ __forceinline__ void map_multi(const SceneView& sc, const float3 (&p)[NP], bool valid, float time,
                                          float (&d)[NP], Diag* diag) {
    static_assert(NP >= 1 && NP <= 7, "a stack entry holds the node and NP masks in two uint4");
    constexpr int W4 = (NP + 1 + 3) / 4;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned live = __ballot_sync(FULL, valid);
    int it[NP];
    PruneBound b[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) {
        d[i] = 1e10f;
        it[i] = 0;
    }
    bool overflow = blockDim.x > 32 * MAP_WARPS;
    if (sc.nnodes > 0 && live && !overflow) {
#pragma unroll
        for (int i = 0; i < NP; ++i) b[i].set(d[i]);
        uint4(*stk)[W4] = reinterpret_cast<uint4(*)[W4]>(s_multi_stack + (threadIdx.x >> 5) * MULTI_STACK_UINT4);
        int sp = 0;
        int node = 0;
        unsigned m[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) m[i] = live;
        bool have = true;
        bool in_bound = true;
#pragma unroll
        for (int i = 0; i < NP; ++i)
            in_bound = in_bound && below_descent_bound(p[i].x) && below_descent_bound(p[i].y) &&
                       below_descent_bound(p[i].z);
        if (__all_sync(FULL, !valid || in_bound)) {
            const int depth = first_descent(sc, node, sp, [&](int s, int right) {
                if (lane == 0) {
                    unsigned w[4 * W4];
                    w[0] = (unsigned)right;
#pragma unroll
                    for (int i = 0; i < NP; ++i) w[i + 1] = live;
#pragma unroll
                    for (int i = NP + 1; i < 4 * W4; ++i) w[i] = 0u;
#pragma unroll
                    for (int k = 0; k < W4; ++k) stk[s][k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
                }
            });
            if (valid) {
#pragma unroll
                for (int i = 0; i < NP; ++i) it[i] = depth;
            }
        }
        for (;;) {
            if (!have) {
                if (sp == 0) break;
                --sp;
                unsigned w[4 * W4];
#pragma unroll
                for (int k = 0; k < W4; ++k) {
                    const uint4 e = stk[sp][k];
                    w[4 * k] = e.x;
                    w[4 * k + 1] = e.y;
                    w[4 * k + 2] = e.z;
                    w[4 * k + 3] = e.w;
                }
                node = (int)w[0];
#pragma unroll
                for (int i = 0; i < NP; ++i) m[i] = w[i + 1];
            }
            have = false;
            bool alive[NP];
            bool any = false;
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                const bool pops = ((m[i] >> lane) & 1u) && it[i] < MAP_CAP;
                if (pops) it[i]++;
                alive[i] = pops && b[i].alive();
                any |= alive[i];
            }
            if (!__any_sync(FULL, any)) continue;
            const float4 na = __ldg(sc.nodes + 2 * node);
            const float4 nb = __ldg(sc.nodes + 2 * node + 1);
            unsigned hits = 0;
            unsigned hm[NP];
#pragma unroll
            for (int i = 0; i < NP; ++i) {
                const bool h = alive[i] && b[i].closer(p[i], na, nb);
                hits |= (h ? 1u : 0u) << i;
                hm[i] = __ballot_sync(FULL, h);
            }
            if (!__any_sync(FULL, hits != 0u)) continue;
            const int left = __float_as_int(nb.z), right = __float_as_int(nb.w);
            if (right == -1) {
                const float4* pr = sc.prims + (size_t)left * PRIM_ROWS;
                const Leaf L = load_leaf(pr);
                // the lane's hit points in turn, selected by unrolled compares (state stays in registers)
                while (__any_sync(FULL, hits != 0u)) {
                    if (hits) {
                        const int sel = __ffs(hits) - 1;
                        hits &= hits - 1u;
                        float3 ps = p[0];
                        MapState<false> t;
                        t.d = d[0];
#pragma unroll
                        for (int i = 1; i < NP; ++i)
                            if (sel == i) {
                                ps = p[i];
                                t.d = d[i];
                            }
                        float3 pre;
                        const float dp = leaf_distance(L, ps, time, pre);
                        combine<false>(t, L.op, L.pos.w, pr, left, dp, pre);
#pragma unroll
                        for (int i = 0; i < NP; ++i)
                            if (sel == i) {
                                d[i] = t.d;
                                b[i].set(t.d);
                            }
                    }
                }
            } else {
                if (sp + 2 > MAP_STACK) { overflow = true; break; }  // the reference's stack holds both
                __syncwarp();  // every lane has read stk[sp] (popped above) before it is overwritten
                if (lane == 0) {
                    unsigned w[4 * W4];
                    w[0] = (unsigned)right;
#pragma unroll
                    for (int i = 0; i < NP; ++i) w[i + 1] = hm[i];
#pragma unroll
                    for (int i = NP + 1; i < 4 * W4; ++i) w[i] = 0u;
#pragma unroll
                    for (int k = 0; k < W4; ++k) stk[sp][k] = make_uint4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
                }
                __syncwarp();
                ++sp;
                node = left;
#pragma unroll
                for (int i = 0; i < NP; ++i) m[i] = hm[i];
                have = true;
            }
        }
        if (diag) {
            unsigned ncap = 0;
#pragma unroll
            for (int i = 0; i < NP; ++i) ncap += __popc(__ballot_sync(FULL, valid && it[i] >= MAP_CAP));
            if (lane == 0 && ncap) atomicAdd(&diag->cap_hits, (unsigned long long)ncap);
        }
    }
    if (diag && overflow && lane == 0) atomicExch(&diag->stack_overflow, 1);
    // non-union primitives: a linear pass in scene order (:703-803), one point at a time
    if (valid) {
        for (int j = sc.nbvh; j < sc.nprims; ++j) {
            const float4* pr = sc.prims + (size_t)j * PRIM_ROWS;
            const Leaf L = load_leaf(pr);
#pragma unroll 1
            for (int sel = 0; sel < NP; ++sel) {
                float3 ps = p[0];
                MapState<false> t;
                t.d = d[0];
#pragma unroll
                for (int i = 1; i < NP; ++i)
                    if (sel == i) {
                        ps = p[i];
                        t.d = d[i];
                    }
                float3 pre;
                const float dp = leaf_distance(L, ps, time, pre);
                combine<false>(t, L.op, L.pos.w, pr, j, dp, pre);
#pragma unroll
                for (int i = 0; i < NP; ++i)
                    if (sel == i) d[i] = t.d;
            }
        }
    }
}

// computeNormal (MarchingCubesKernels.cu:814-844) for the 32 points of a warp, with the distance at
// p itself already known (map() at p, with or without attributes: the distance is the same); the
// three offset points walk the BVH together (map_multi).
__device__ __forceinline__ float3 normal_warp_at(const SceneView& sc, float3 p, float d0, bool valid, float time,
                                                 float cell, Diag* diag) {
    const float h = MUL(cell, 0.001f);
    const float3 pts[3] = {f3(ADD(p.x, h), p.y, p.z), f3(p.x, ADD(p.y, h), p.z), f3(p.x, p.y, ADD(p.z, h))};
    float d[3];
    map_multi<3>(sc, pts, valid, time, d, diag);
    const float3 g = f3(SUB(d[0], d0), SUB(d[1], d0), SUB(d[2], d0));
    const float len = SQRT(dot3(g, g));
    if (len > 1e-6f) return f3(DIV(g.x, len), DIV(g.y, len), DIV(g.z, len));
    return f3(0.f, 1.f, 0.f);
}

// map() at computeNormal's four points (p, then p + h along x, y, z), walked together.
__device__ __forceinline__ void stencil4_warp(const SceneView& sc, float3 p, bool valid, float time, float cell,
                                              float (&d)[4], Diag* diag) {
    const float h = MUL(cell, 0.001f);
    const float3 pts[4] = {p, f3(ADD(p.x, h), p.y, p.z), f3(p.x, ADD(p.y, h), p.z), f3(p.x, p.y, ADD(p.z, h))};
    map_multi<4>(sc, pts, valid, time, d, diag);
}

// computeNormal (MarchingCubesKernels.cu:814-844) for the 32 points of a warp.
__device__ __forceinline__ float3 normal_warp(const SceneView& sc, float3 p, bool valid, float time, float cell,
                                              Diag* diag) {
    float d[4];
    stencil4_warp(sc, p, valid, time, cell, d, diag);
    const float3 g = f3(SUB(d[1], d[0]), SUB(d[2], d[0]), SUB(d[3], d[0]));
    const float len = SQRT(dot3(g, g));
    if (len > 1e-6f) return f3(DIV(g.x, len), DIV(g.y, len), DIV(g.z, len));
    return f3(0.f, 1.f, 0.f);
}

// ------------------------------------------------------------------------------------------------
// grid geometry (Commons.cuh:190-215) and marching-cubes helpers (MarchingCubesKernels.cu:33-103)
// ------------------------------------------------------------------------------------------------
struct GridView {
    int w, h, d;        // samples per axis
    int bx, by, bz;     // blocks per axis
    float ox, oy, oz;   // origin
    float cell;
};

__device__ __forceinline__ float3 grid_loc(const GridView& g, int x, int y, int z) {
    return f3(FMA((float)x, g.cell, g.ox), FMA((float)y, g.cell, g.oy), FMA((float)z, g.cell, g.oz));
}
__device__ __forceinline__ float edge_t(float v1, float v2) {
    const float denom = SUB(v2, v1);
    float t = 0.5f;
    if (fabsf(denom) > 1e-12f) t = DIV(SUB(0.f, v1), denom);
    t = CLAMP(t, 0.f, 1.f);
    if (t <= 0.f) t = 1e-7f;
    if (t >= 1.f) t = 1.f - 1e-7f;
    return t;
}
// lerp3 (:48-54) as inlined in interpEdgePoint and the DC solve: a*(1-t) fused
__device__ __forceinline__ float3 lerp3(float3 a, float3 b, float t) {
    const float u = SUB(1.f, t);
    return f3(FMA(a.x, u, MUL(b.x, t)), FMA(a.y, u, MUL(b.y, t)), FMA(a.z, u, MUL(b.z, t)));
}
__device__ __forceinline__ float len2_3(float3 v) { return FMA(v.z, v.z, FMA(v.x, v.x, MUL(v.y, v.y))); }
__device__ __forceinline__ bool degenerate(float3 a, float3 b, float3 c, float cell) {
    if (!finite3(a) || !finite3(b) || !finite3(c)) return true;
    const float me = DIV(cell, 1024.f), me2 = MUL(me, me);
    return len2_3(sub3(b, a)) < me2 || len2_3(sub3(c, b)) < me2 || len2_3(sub3(a, c)) < me2;
}

// corner offsets and edge endpoints (MarchingCubesTables.cuh:8-17), as bit-packed constants:
// corner c has offset (x, y, z) = bits (c*3, c*3+1, c*3+2) of kCornerBits
constexpr uint32_t kCornerBits = (0u << 0) | (1u << 3) | (3u << 6) | (2u << 9) | (4u << 12) | (5u << 15) |
                                 (7u << 18) | (6u << 21);
__device__ __forceinline__ int corner_dx(int c) { return (kCornerBits >> (3 * c)) & 1; }
__device__ __forceinline__ int corner_dy(int c) { return (kCornerBits >> (3 * c + 1)) & 1; }
__device__ __forceinline__ int corner_dz(int c) { return (kCornerBits >> (3 * c + 2)) & 1; }
// edge e joins corners (c0, c1): nibble e of kEdgeC0 / kEdgeC1
constexpr uint64_t kEdgeC0 = 0x321076543210ull;
constexpr uint64_t kEdgeC1 = 0x765447650321ull;
__device__ __forceinline__ int edge_c0(int e) { return (int)((kEdgeC0 >> (4 * e)) & 0xF); }
__device__ __forceinline__ int edge_c1(int e) { return (int)((kEdgeC1 >> (4 * e)) & 0xF); }

}  // namespace sdfb
