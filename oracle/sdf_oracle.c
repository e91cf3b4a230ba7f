/* CPU oracle for the SDF -> mesh hot path: TEST INFRASTRUCTURE, not part of the product.
 * See sdf_oracle.h. All citations are to the reference's src/SDFMesh/ files.
 *
 * Arithmetic convention: plain C operators are single IEEE roundings (built with
 * -ffp-contract=off); every place where the reference's compiled code fuses a multiply into an add
 * is written as fmaf(). Which product of a*b + c*d the reference's build fuses depends on the
 * expression; each choice below was pinned against the reference's own outputs on the GPU
 * (tests/golden/probes.npz, map_probes.npz): "len2a" = fma(x,x,y*y) fuses the first square,
 * "len2b" = fma(y,y,x*x) the second, and so on.
 */
#define _GNU_SOURCE
#include "sdf_oracle.h"

#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "mc_table_oracle.inc"

_Static_assert(sizeof(OrPrim) == 160, "OrPrim must match SDFPrimitive");
_Static_assert(sizeof(OrNode) == 32, "OrNode must match BVHNode");

/* corner and edge conventions (MarchingCubesTables.cuh:8-17) */
static const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                  {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
static const int kEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                 {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

enum { T_SPHERE = 0, T_BOX, T_TORUS, T_CYLINDER, T_CAPSULE, T_CONE, T_RBOX, T_RCYL, T_RCONE, T_ELLIPSOID,
       T_TRIPRISM, T_OCTA, T_HEXPRISM };
enum { OP_UNION = 0, OP_SUB, OP_INT, OP_UNION_BLEND, OP_SUB_BLEND, OP_INT_BLEND };
enum { D_NONE = 0, D_SINE, D_TWIST, D_BEND };

#define BLOCK 8
#define BLOCK3 512

typedef struct { float x, y, z; } v3;

static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 add3(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 scl3(v3 a, float s) { return mk(s * a.x, s * a.y, s * a.z); }
/* a.x*b.x + a.y*b.y + a.z*b.z  (Commons.cuh:261) */
static inline float dot3(v3 a, v3 b) { return fmaf(a.z, b.z, fmaf(a.x, b.x, a.y * b.y)); }
static inline float len3(v3 a) { return sqrtf(dot3(a, a)); }
/* length(float2) = sqrtf(x*x + y*y)  (MarchingCubesKernels.cu:112): len2a fuses x*x, len2b y*y */
static inline float len2(float x, float y) { return sqrtf(fmaf(x, x, y * y)); }
static inline float len2b(float x, float y) { return sqrtf(fmaf(y, y, x * x)); }
static inline float clampf(float v, float lo, float hi) { return fmaxf(lo, fminf(v, hi)); }
/* the cross product inlined in rotateVector: the subtracted product is fused,
 * fma(-a.z, b.y, a.y*b.z) */
static inline v3 cross3(v3 a, v3 b) {
    return mk(fmaf(-a.z, b.y, a.y * b.z), fmaf(-a.x, b.z, a.z * b.x), fmaf(-a.y, b.x, a.x * b.y));
}
static inline int finite3(v3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

/* rotateVector (Commons.cuh:264-273) with u = q.xyz, s = q.w:
 * 2*dot(u,v)*u + (s*s - dot(u,u))*v + 2*s*cross(u,v) */
static inline v3 rotate(v3 v, float ux, float uy, float uz, float s) {
    v3 u = mk(ux, uy, uz);
    float a = 2.0f * fmaf(u.z, v.z, fmaf(u.y, v.y, u.x * v.x));
    float b = fmaf(s, s, -dot3(u, u));
    float c = 2.0f * s;
    v3 cr = cross3(u, v);
    return mk(fmaf(c, cr.x, fmaf(b, v.x, a * u.x)), fmaf(c, cr.y, fmaf(b, v.y, a * u.y)),
              fmaf(c, cr.z, fmaf(b, v.z, a * u.z)));
}
/* invRotateVector (Commons.cuh:275-278): conjugate quaternion */
static inline v3 inv_rotate(v3 v, const float* q) { return rotate(v, -q[0], -q[1], -q[2], q[3]); }

/* world -> primitive local (MarchingCubesKernels.cu:597-599) */
static inline v3 to_local(v3 pw, const OrPrim* pr) {
    v3 p = sub3(pw, mk(pr->position[0], pr->position[1], pr->position[2]));
    p = inv_rotate(p, pr->rotation);
    return mk(p.x / pr->scale[0], p.y / pr->scale[1], p.z / pr->scale[2]);
}

/* ------------------------------------------------------------------------------------------------
 * primitive SDFs (MarchingCubesKernels.cu:129-219)
 * ---------------------------------------------------------------------------------------------- */
static float sd_sphere(v3 p, float r) { return len3(p) - r; }
static float sd_box(v3 p, float bx, float by, float bz) {
    v3 q = mk(fabsf(p.x) - bx, fabsf(p.y) - by, fabsf(p.z) - bz);
    return len3(mk(fmaxf(q.x, 0.0f), fmaxf(q.y, 0.0f), fmaxf(q.z, 0.0f))) +
           fminf(fmaxf(q.x, fmaxf(q.y, q.z)), 0.0f);
}
static float sd_torus(v3 p, float r1, float r2) { return len2b(len2(p.x, p.z) - r1, p.y) - r2; }
static float sd_cylinder(v3 p, float h, float r) {
    float dx = fabsf(len2(p.x, p.z)) - r, dy = fabsf(p.y) - h;
    return fminf(fmaxf(dx, dy), 0.0f) + len2b(fmaxf(dx, 0.0f), fmaxf(dy, 0.0f));
}
static float sd_capsule(v3 p, float h, float r) {
    p.y = p.y - clampf(p.y, 0.0f, h);
    return len3(p) - r;
}
static float sd_cone(v3 p, float h, float angle) {
    float cx = sinf(angle * 0.0174533f), cy = cosf(angle * 0.0174533f);
    float qx = h * (cx / cy), qy = -h;
    float wx = len2(p.x, p.z), wy = p.y;
    float dwq = fmaf(wx, qx, wy * qy);
    float dqq = fmaf(qx, qx, qy * qy);
    float t = clampf(dwq / dqq, 0.0f, 1.0f);
    float ax = fmaf(-qx, t, wx), ay = fmaf(-qy, t, wy);
    float tb = clampf(wx / qx, 0.0f, 1.0f);
    float bx = fmaf(-qx, tb, wx), by = wy - qy;
    float k = (qy > 0) ? 1.0f : -1.0f;
    float d = fminf(fmaf(ax, ax, ay * ay), fmaf(bx, bx, by * by));
    float s = fmaxf(k * fmaf(wx, qy, -(wy * qx)), k * (wy - qy));
    return sqrtf(d) * (s > 0.0f ? 1.0f : -1.0f);
}
static float sd_ellipsoid(v3 p, float rx, float ry, float rz) {
    float k0 = len3(mk(p.x / rx, p.y / ry, p.z / rz));
    float k1 = len3(mk(p.x / (rx * rx), p.y / (ry * ry), p.z / (rz * rz)));
    return k0 * (k0 - 1.0f) / k1;
}
static float sd_octahedron(v3 p, float s) {
    p = mk(fabsf(p.x), fabsf(p.y), fabsf(p.z));
    return (p.x + p.y + p.z - s) * 0.57735027f;
}
static float sd_triprism(v3 p, float hx, float hy) {
    v3 q = mk(fabsf(p.x), fabsf(p.y), fabsf(p.z));
    return fmaxf(q.z - hy, fmaf(-hx, 0.5f, fmaxf(fmaf(q.x, 0.866025f, p.y * 0.5f), -p.y)));
}
static float sd_rounded_cone(v3 p, float h, float r1, float r2) {
    float qx = len2(p.x, p.z), qy = p.y;
    float b = (r1 - r2) / h;
    float a = sqrtf(fmaf(-b, b, 1.0f));
    float k = fmaf(qx, -b, qy * a);
    if (k < 0.0f) return len2b(qx, qy) - r1;
    if (k > a * h) return len2b(qx, qy - h) - r2;
    /* inside map() the reference's build fuses q.y*b here (a standalone call fuses q.x*a) */
    return fmaf(qy, b, qx * a) - r1;
}
static float sd_rounded_cylinder(v3 p, float h, float r1, float r2) {
    float dx = fmaf(-2.0f, r1, len2(p.x, p.z)) + r2, dy = fabsf(p.y) - h;
    return fminf(fmaxf(dx, dy), 0.0f) + len2b(fmaxf(dx, 0.0f), fmaxf(dy, 0.0f)) - r2;
}
static float sd_hexprism(v3 p, float hx, float hy) {
    const float kx = -0.8660254f, ky = 0.5f, kz = 0.57735027f;
    p = mk(fabsf(p.x), fabsf(p.y), fabsf(p.z));
    float m = fminf(fmaf(ky, p.z, kx * p.x), 0.0f);
    float px = fmaf(-(kx * 2.0f), m, p.x), pz = fmaf(-(ky * 2.0f), m, p.z);
    float ex = px - clampf(px, -kz * hx, kz * hx), ez = pz - hx;
    float dx = len2b(ex, ez) * copysignf(1.0f, pz - hx), dy = p.y - hy;
    return fminf(fmaxf(dx, dy), 0.0f) + len2b(fmaxf(dx, 0.0f), fmaxf(dy, 0.0f));
}

/* the type switch of map() (MarchingCubesKernels.cu:608-624) */
static float sd_eval(int type, v3 p, const float* pm) {
    switch (type) {
        case T_SPHERE: return sd_sphere(p, pm[0]);
        case T_BOX: return sd_box(p, pm[0], pm[1], pm[2]);
        case T_TORUS: return sd_torus(p, pm[0], pm[1]);
        case T_CYLINDER: return sd_cylinder(p, pm[0], pm[1]);
        case T_CAPSULE: return sd_capsule(p, pm[0], pm[1]);
        case T_CONE: return sd_cone(p, pm[0], pm[1]);
        case T_RBOX: return sd_box(p, pm[0], pm[1], pm[2]) - pm[3];
        case T_ELLIPSOID: return sd_ellipsoid(p, pm[0], pm[1], pm[2]);
        case T_OCTA: return sd_octahedron(p, pm[0]);
        case T_TRIPRISM: return sd_triprism(p, pm[0], pm[1]);
        case T_RCYL: return sd_rounded_cylinder(p, pm[0], pm[1], pm[2]);
        case T_RCONE: return sd_rounded_cone(p, pm[0], pm[1], pm[2]);
        case T_HEXPRISM: return sd_hexprism(p, pm[0], pm[1]);
        default: return len3(p) - 1.0f;
    }
}

/* displacements (MarchingCubesKernels.cu:229-243, 604-606) */
static v3 disp_twist(v3 p, float k) {
    float c = cosf(k * p.y), s = sinf(k * p.y);
    return mk(fmaf(c, p.x, -(s * p.z)), p.y, fmaf(c, p.z, s * p.x));
}
static v3 disp_bend(v3 p, float k) {
    float c = cosf(k * p.x), s = sinf(k * p.x);
    return mk(fmaf(c, p.x, -(s * p.y)), fmaf(c, p.y, s * p.x), p.z);
}
static float disp_sine_y(v3 p, float k, float amp, float time) {
    return fmaf(sinf(fmaf(p.x, k, time)), amp, p.y);
}

/* leaf evaluation: world->local, displacement, SDF, scale, annular, rounding (:594-629) */
static float leaf_eval(const OrPrim* pr, v3 pw, float time, v3* pre) {
    v3 p = to_local(pw, pr);
    *pre = p;
    if (pr->displacement == D_TWIST) p = disp_twist(p, pr->dispParams[0]);
    else if (pr->displacement == D_BEND) p = disp_bend(p, pr->dispParams[0]);
    else if (pr->displacement == D_SINE) p.y = disp_sine_y(p, pr->dispParams[0], pr->dispParams[1], time);
    float d = sd_eval(pr->type, p, pr->params);
    d = d * fminf(pr->scale[0], fminf(pr->scale[1], pr->scale[2]));
    if (pr->annular > 0.0f) d = fabsf(d) - pr->annular;
    if (pr->rounding > 0.0f) d = d - pr->rounding;
    return d;
}

/* mix(x, y, a) = x*(1-a) + y*a (Commons.cuh:247). Inside the blends of map() the reference's
 * build fuses y*a for the union / intersect blends and the colour mix, and x*(1-a) for the
 * subtract blend; the trailing -/+ k*h*(1-h) is fused as fma(-/+(k*h), 1-h, mix). */
static inline float mix_fuse_y(float x, float y, float a) { return fmaf(y, a, x * (1.0f - a)); }
static inline float mix_fuse_x(float x, float y, float a) { return fmaf(x, 1.0f - a, y * a); }

typedef struct { float d; v3 color; int id; v3 local; } MapState;

/* the CSG combine of map() (MarchingCubesKernels.cu:631-694) */
static void combine(MapState* st, const OrPrim* pr, int i, float dp, v3 pre) {
    v3 pc = mk(pr->color[0], pr->color[1], pr->color[2]);
    if (st->d == 1e10f) {
        st->d = dp; st->color = pc; st->id = i; st->local = pre;
        return;
    }
    float k = pr->blendFactor, h;
    switch (pr->operation) {
        case OP_UNION:
            if (dp < st->d) { st->d = dp; st->color = pc; st->id = i; st->local = pre; }
            break;
        case OP_SUB: {
            float old = st->d;
            st->d = fmaxf(st->d, -dp);
            if (st->d > old) { st->color = pc; st->id = i; st->local = pre; }
        } break;
        case OP_INT:
            if (dp > st->d) { st->d = dp; st->color = pc; st->id = i; st->local = pre; }
            break;
        case OP_UNION_BLEND:
            h = clampf(0.5f + (0.5f * (st->d - dp)) / k, 0.0f, 1.0f);
            st->d = fmaf(-(k * h), 1.0f - h, mix_fuse_y(st->d, dp, h));
            st->color = mk(mix_fuse_y(st->color.x, pc.x, h), mix_fuse_y(st->color.y, pc.y, h), mix_fuse_y(st->color.z, pc.z, h));
            if (dp < st->d || h > 0.5f) { st->id = i; st->local = pre; }
            break;
        case OP_SUB_BLEND:
            h = clampf(0.5f - (0.5f * (st->d + dp)) / k, 0.0f, 1.0f);
            st->d = fmaf(k * h, 1.0f - h, mix_fuse_x(st->d, -dp, h));
            st->color = mk(mix_fuse_y(st->color.x, pc.x, h), mix_fuse_y(st->color.y, pc.y, h), mix_fuse_y(st->color.z, pc.z, h));
            if (h > 0.5f) { st->id = i; st->local = pre; }
            break;
        case OP_INT_BLEND:
            h = clampf(0.5f - (0.5f * (st->d - dp)) / k, 0.0f, 1.0f);
            st->d = fmaf(k * h, 1.0f - h, mix_fuse_y(st->d, dp, h));
            st->color = mk(mix_fuse_y(st->color.x, pc.x, h), mix_fuse_y(st->color.y, pc.y, h), mix_fuse_y(st->color.z, pc.z, h));
            if (dp > st->d || h > 0.5f) { st->id = i; st->local = pre; }
            break;
        default: break;
    }
}

/* intersectAABB (MarchingCubesKernels.cu:564-568) */
static inline int aabb_hit(v3 p, const float* mn, const float* mx, float dmin) {
    v3 d = mk(fmaxf(fmaxf(mn[0] - p.x, p.x - mx[0]), 0.0f), fmaxf(fmaxf(mn[1] - p.y, p.y - mx[1]), 0.0f),
              fmaxf(fmaxf(mn[2] - p.z, p.z - mx[2]), 0.0f));
    return len3(d) < dmin;
}

/* map() (MarchingCubesKernels.cu:570-808): capped DFS over the BVH (stack of 64, at most 256 popped
 * nodes, right child pushed first, pruning against the running distance), then a linear pass over
 * the non-union primitives. */
static MapState map_eval(const OrScene* s, v3 pw, float time, int* iters_out) {
    MapState st;
    st.d = 1e10f; st.color = mk(0, 0, 0); st.id = -1; st.local = mk(0, 0, 0);
    int stack[64], sp = 0, iter = 0;
    if (s->nnodes > 0) stack[sp++] = 0;
    while (sp > 0 && iter < 256) {
        iter++;
        const OrNode* nd = &s->nodes[stack[--sp]];
        if (!aabb_hit(pw, nd->mn, nd->mx, st.d)) continue;
        if (nd->right == -1) {
            const OrPrim* pr = &s->prims[nd->left];
            v3 pre;
            float dp = leaf_eval(pr, pw, time, &pre);
            combine(&st, pr, nd->left, dp, pre);
        } else {
            if (sp + 2 > 64) break; /* the reference overflows its stack here (undefined) */
            stack[sp++] = nd->right;
            stack[sp++] = nd->left;
        }
    }
    for (int i = s->nbvh; i < s->nprims; ++i) {
        const OrPrim* pr = &s->prims[i];
        v3 pre;
        float dp = leaf_eval(pr, pw, time, &pre);
        combine(&st, pr, i, dp, pre);
    }
    if (iters_out) *iters_out = iter;
    return st;
}

static inline float map_d(const OrScene* s, v3 p, float time) { return map_eval(s, p, time, NULL).d; }

/* computeNormal (MarchingCubesKernels.cu:814-844) */
static v3 normal_at(const OrScene* s, v3 p, float time, float cell) {
    const float h = cell * 0.001f;
    float dc = map_d(s, p, time);
    float dx = map_d(s, mk(p.x + h, p.y, p.z), time);
    float dy = map_d(s, mk(p.x, p.y + h, p.z), time);
    float dz = map_d(s, mk(p.x, p.y, p.z + h), time);
    v3 g = mk(dx - dc, dy - dc, dz - dc);
    float len = sqrtf(dot3(g, g));
    if (len > 1e-6f) return mk(g.x / len, g.y / len, g.z / len);
    return mk(0.0f, 1.0f, 0.0f);
}

/* ------------------------------------------------------------------------------------------------
 * marching-cubes helpers (MarchingCubesKernels.cu:33-103, Commons.cuh:209-215)
 * ---------------------------------------------------------------------------------------------- */
static inline float edge_t(float v1, float v2) {
    const float denom = v2 - v1;
    float t = 0.5f;
    if (fabsf(denom) > 1e-12f) t = (0.0f - v1) / denom;
    t = clampf(t, 0.0f, 1.0f);
    if (t <= 0.0f) t = 1e-7f;
    if (t >= 1.0f) t = 1.0f - 1e-7f;
    return t;
}
/* lerp3 (:48-54): a*(1-t) + b*t, the second product fused */
static inline v3 lerp3(v3 a, v3 b, float t) {
    float u = 1.0f - t;
    return mk(fmaf(b.x, t, a.x * u), fmaf(b.y, t, a.y * u), fmaf(b.z, t, a.z * u));
}
/* lerp3 as inlined into interpEdgePoint (:60-81): there the first product is fused */
static inline v3 lerp3_edge(v3 a, v3 b, float t) {
    float u = 1.0f - t;
    return mk(fmaf(a.x, u, b.x * t), fmaf(a.y, u, b.y * t), fmaf(a.z, u, b.z * t));
}
static inline v3 grid_loc(const OrGridDesc* g, int x, int y, int z) {
    return mk(fmaf((float)x, g->cell, g->origin[0]), fmaf((float)y, g->cell, g->origin[1]),
              fmaf((float)z, g->cell, g->origin[2]));
}
static inline float len2_3(v3 v) { return fmaf(v.z, v.z, fmaf(v.x, v.x, v.y * v.y)); }
static int degenerate(const v3 p[3], float cell) {
    if (!finite3(p[0]) || !finite3(p[1]) || !finite3(p[2])) return 1;
    const float me = cell / 1024.0f, me2 = me * me;
    if (len2_3(sub3(p[1], p[0])) < me2 || len2_3(sub3(p[2], p[1])) < me2 || len2_3(sub3(p[0], p[2])) < me2)
        return 1;
    return 0;
}

/* ------------------------------------------------------------------------------------------------
 * UV mapping (MarchingCubesKernels.cu:249-500)
 * ---------------------------------------------------------------------------------------------- */
#define OR_PI 3.14159265358979323846
#define OR_PI_2 1.57079632679489661923
typedef struct { float u, v; } v2;
static inline v2 mk2(float u, float v) { v2 r = {u, v}; return r; }

static v2 uv_sphere(v3 p) {
    float len = len3(p);
    if (len < 1e-6f) return mk2(0.5f, 0.5f);
    p = scl3(p, 1.0f / len);
    float theta = atan2f(p.z, p.x);
    float phi = asinf(clampf(p.y, -1.0f, 1.0f));
    return mk2((float)((theta + OR_PI) / (2.0 * OR_PI)), (float)((phi + OR_PI_2) / OR_PI));
}
static v2 uv_box(v3 p, v3 n) {
    v3 a = mk(fabsf(n.x), fabsf(n.y), fabsf(n.z));
    if (a.x > a.y && a.x > a.z) return mk2(fmaf(p.z, 0.5f, 0.5f), fmaf(p.y, 0.5f, 0.5f));
    if (a.y > a.z) return mk2(fmaf(p.x, 0.5f, 0.5f), fmaf(p.z, 0.5f, 0.5f));
    return mk2(fmaf(p.x, 0.5f, 0.5f), fmaf(p.y, 0.5f, 0.5f));
}
static v2 uv_cylinder(v3 p, float height) {
    float theta = atan2f(p.z, p.x);
    return mk2((float)((theta + OR_PI) / (2.0 * OR_PI)), clampf(fmaf(p.y / height, 0.5f, 0.5f), 0.0f, 1.0f));
}
static v2 uv_torus(v3 p, float R) {
    float theta = atan2f(p.z, p.x);
    float qx = len2(p.x, p.z) - R;
    float phi = atan2f(p.y, qx);
    return mk2((float)((theta + OR_PI) / (2.0 * OR_PI)), (float)((phi + OR_PI) / (2.0 * OR_PI)));
}
static v2 uv_capsule(v3 p, float height) {
    if (p.y > height) return uv_sphere(mk(p.x, p.y - height, p.z));
    if (p.y < 0.0f) return uv_sphere(p);
    return uv_cylinder(p, height);
}
static v3 approx_local_normal(v3 lp, const OrPrim* pr) {
    if (pr->type == T_BOX || pr->type == T_RBOX) {
        v3 a = mk(fabsf(lp.x), fabsf(lp.y), fabsf(lp.z));
        if (a.x > a.y && a.x > a.z) return mk(copysignf(1.0f, lp.x), 0, 0);
        if (a.y > a.z) return mk(0, copysignf(1.0f, lp.y), 0);
        return mk(0, 0, copysignf(1.0f, lp.z));
    }
    float len = len3(lp);
    return (len > 1e-6f) ? scl3(lp, 1.0f / len) : mk(0.0f, 1.0f, 0.0f);
}
static v2 seam_adjust(v2 uv, v2 ref) {
    v2 r = uv;
    if (fabsf(uv.u - ref.u) > 0.5f) r.u += (uv.u < ref.u) ? 1.0f : -1.0f;
    if (fabsf(uv.v - ref.v) > 0.5f) r.v += (uv.v < ref.v) ? 1.0f : -1.0f;
    return r;
}
static v2 uv_transform(v2 uv, const OrPrim* pr) {
    uv = mk2(uv.u * pr->uvScale[0], uv.v * pr->uvScale[1]);
    if (fabsf(pr->uvRotation) > 1e-6f) {
        float c = cosf(pr->uvRotation), s = sinf(pr->uvRotation);
        uv = mk2(fmaf(uv.u, c, -(uv.v * s)), fmaf(uv.u, s, uv.v * c));
    }
    return mk2(uv.u + pr->uvOffset[0], uv.v + pr->uvOffset[1]);
}
/* computeTriangleUVs (MarchingCubesKernels.cu:392-479) */
static void triangle_uvs(const v3 lp[3], const OrPrim* pr, v2 out[3]) {
    v3 ln[3] = {mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0)};
    int needs = (pr->type == T_BOX || pr->type == T_RBOX || pr->type == T_OCTA);
    if (needs)
        for (int i = 0; i < 3; ++i) ln[i] = approx_local_normal(lp[i], pr);
    for (int i = 0; i < 3; ++i) {
        v2 uv;
        switch (pr->type) {
            case T_SPHERE: case T_ELLIPSOID: uv = uv_sphere(lp[i]); break;
            case T_BOX: case T_RBOX: case T_OCTA: uv = uv_box(lp[i], ln[i]); break;
            case T_CYLINDER: case T_RCYL: uv = uv_cylinder(lp[i], pr->params[0]); break;
            case T_TORUS: uv = uv_torus(lp[i], pr->params[0]); break;
            case T_CAPSULE: uv = uv_capsule(lp[i], pr->params[0]); break;
            case T_CONE: case T_RCONE: uv = uv_cylinder(lp[i], pr->params[0]); break;
            case T_HEXPRISM: case T_TRIPRISM: uv = uv_cylinder(lp[i], pr->params[1]); break;
            default: uv = mk2(fmaf(lp[i].x, 0.5f, 0.5f), fmaf(lp[i].y, 0.5f, 0.5f)); break;
        }
        out[i] = uv;
    }
    out[1] = seam_adjust(out[1], out[0]);
    out[2] = seam_adjust(out[2], out[0]);
    float d01 = fabsf(out[0].u - out[1].u) + fabsf(out[0].v - out[1].v);
    float d02 = fabsf(out[0].u - out[2].u) + fabsf(out[0].v - out[2].v);
    float d12 = fabsf(out[1].u - out[2].u) + fabsf(out[1].v - out[2].v);
    if (d01 > 0.5f && d02 > 0.5f && d12 < 0.5f) out[0] = seam_adjust(out[0], out[1]);
    for (int i = 0; i < 3; ++i) out[i] = uv_transform(out[i], pr);
}

/* ------------------------------------------------------------------------------------------------
 * DC codecs and solvers (MarchingCubesKernels.cu:1133-1301)
 * ---------------------------------------------------------------------------------------------- */
static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static v3 dc_decode_vertex(const uint16_t q[3], v3 cmin, float cell) {
    const float inv = 1.0f / 65535.0f;
    return mk(fmaf((float)q[0] * inv, cell, cmin.x), fmaf((float)q[1] * inv, cell, cmin.y),
              fmaf((float)q[2] * inv, cell, cmin.z));
}
static v3 normalize_or_up(v3 n) {
    float len = sqrtf(dot3(n, n));
    if (len > 1e-6f) return mk(n.x / len, n.y / len, n.z / len);
    return mk(0.0f, 1.0f, 0.0f);
}
static v3 dc_decode_normal(const int16_t q[3]) {
    const float inv = 1.0f / 32767.0f;
    return normalize_or_up(mk((float)q[0] * inv, (float)q[1] * inv, (float)q[2] * inv));
}
static void dc_encode_normal(v3 n, int16_t out[4]) {
    n = normalize_or_up(n);
    out[0] = (int16_t)clampi((int)lrintf(clampf(n.x, -1.0f, 1.0f) * 32767.0f), -32767, 32767);
    out[1] = (int16_t)clampi((int)lrintf(clampf(n.y, -1.0f, 1.0f) * 32767.0f), -32767, 32767);
    out[2] = (int16_t)clampi((int)lrintf(clampf(n.z, -1.0f, 1.0f) * 32767.0f), -32767, 32767);
    out[3] = 0;
}
static void dc_encode_vertex(v3 pw, v3 cmin, float cell, uint16_t out[4]) {
    v3 t = mk((pw.x - cmin.x) / cell, (pw.y - cmin.y) / cell, (pw.z - cmin.z) / cell);
    t = mk(clampf(t.x, 0, 1), clampf(t.y, 0, 1), clampf(t.z, 0, 1));
    out[0] = (uint16_t)clampi((int)lrintf(t.x * 65535.0f), 0, 65535);
    out[1] = (uint16_t)clampi((int)lrintf(t.y * 65535.0f), 0, 65535);
    out[2] = (uint16_t)clampi((int)lrintf(t.z * 65535.0f), 0, 65535);
    out[3] = 0;
}
static inline float det2(float a, float b, float c, float d) { return fmaf(a, b, -(c * d)); } /* a*b - c*d */
/* solve3x3, Cramer's rule (MarchingCubesKernels.cu:1185-1218) */
static int solve3x3(const float A[9], const float b[3], float x[3]) {
    const float a00 = A[0], a01 = A[1], a02 = A[2], a10 = A[3], a11 = A[4], a12 = A[5], a20 = A[6], a21 = A[7],
                a22 = A[8];
    const float det = fmaf(a02, det2(a10, a21, a11, a20),
                           fmaf(a00, det2(a11, a22, a12, a21), -(a01 * det2(a10, a22, a12, a20))));
    if (fabsf(det) < 1e-12f) return 0;
    const float inv = 1.0f / det;
    const float bx = b[0], by = b[1], bz = b[2];
    const float dX = fmaf(a02, det2(by, a21, a11, bz), fmaf(bx, det2(a11, a22, a12, a21), -(a01 * det2(by, a22, a12, bz))));
    const float dY = fmaf(a02, det2(a10, bz, by, a20), fmaf(a00, det2(by, a22, a12, bz), -(bx * det2(a10, a22, a12, a20))));
    const float dZ = fmaf(bx, det2(a10, a21, a11, a20), fmaf(a00, fmaf(-by, a21, a11 * bz), -(a01 * det2(a10, bz, by, a20))));
    x[0] = dX * inv;
    x[1] = dY * inv;
    x[2] = dZ * inv;
    return 1;
}
/* accumulation shared by solveQEF / solveQEFRegularized (:1227-1247, :1269-1285) */
static void qef_accumulate(const v3* pts, const v3* ns, int m, float M[9], float rhs[3]) {
    for (int k = 0; k < 9; ++k) M[k] = 0.0f;
    rhs[0] = rhs[1] = rhs[2] = 0.0f;
    for (int i = 0; i < m; ++i) {
        v3 n = ns[i];
        const float len = sqrtf(dot3(n, n));
        if (len < 1e-6f) continue;
        n = mk(n.x / len, n.y / len, n.z / len);
        const float d = dot3(n, pts[i]);
        M[0] = fmaf(n.x, n.x, M[0]); M[1] = fmaf(n.x, n.y, M[1]); M[2] = fmaf(n.x, n.z, M[2]);
        M[3] = fmaf(n.y, n.x, M[3]); M[4] = fmaf(n.y, n.y, M[4]); M[5] = fmaf(n.y, n.z, M[5]);
        M[6] = fmaf(n.z, n.x, M[6]); M[7] = fmaf(n.z, n.y, M[7]); M[8] = fmaf(n.z, n.z, M[8]);
        rhs[0] = fmaf(n.x, d, rhs[0]); rhs[1] = fmaf(n.y, d, rhs[1]); rhs[2] = fmaf(n.z, d, rhs[2]);
    }
}
static int solve_qef(const v3* pts, const v3* ns, int m, v3* out) {
    if (m <= 0) return 0;
    float M[9], rhs[3], x[3];
    qef_accumulate(pts, ns, m, M, rhs);
    const float lambda = 1e-5f;
    M[0] += lambda; M[4] += lambda; M[8] += lambda;
    if (!solve3x3(M, rhs, x)) return 0;
    *out = mk(x[0], x[1], x[2]);
    return 1;
}
static int solve_qef_reg(const v3* pts, const v3* ns, int m, float alpha, v3 c, v3* out) {
    if (m <= 0) return 0;
    float M[9], rhs[3], x[3];
    qef_accumulate(pts, ns, m, M, rhs);
    const float a = fmaxf(alpha, 0.0f);
    M[0] += a; M[4] += a; M[8] += a;
    rhs[0] = fmaf(a, c.x, rhs[0]); rhs[1] = fmaf(a, c.y, rhs[1]); rhs[2] = fmaf(a, c.z, rhs[2]);
    const float lambda = 1e-6f;
    M[0] += lambda; M[4] += lambda; M[8] += lambda;
    if (!solve3x3(M, rhs, x)) return 0;
    *out = mk(x[0], x[1], x[2]);
    return 1;
}

/* ------------------------------------------------------------------------------------------------
 * grid set-up and BVH build
 * ---------------------------------------------------------------------------------------------- */
void or_grid_init(OrGridDesc* g, float cell, const float bmin[3], const float bmax[3]) {
    g->cell = cell;
    for (int k = 0; k < 3; ++k) g->origin[k] = bmin[k];
    g->width = (uint32_t)ceilf((bmax[0] - bmin[0]) / cell);
    g->height = (uint32_t)ceilf((bmax[1] - bmin[1]) / cell);
    g->depth = (uint32_t)ceilf((bmax[2] - bmin[2]) / cell);
    g->bx = (int32_t)((g->width + BLOCK - 1) / BLOCK);
    g->by = (int32_t)((g->height + BLOCK - 1) / BLOCK);
    g->bz = (int32_t)((g->depth + BLOCK - 1) / BLOCK);
}

/* host-side rotateVector: the host compiler does not contract (CudaSDFUtil.h:501-505) */
static v3 host_rotate(v3 v, const float* q) {
    v3 u = mk(q[0], q[1], q[2]);
    float s = q[3];
    float duv = (u.x * v.x + u.y * v.y) + u.z * v.z;
    float duu = (u.x * u.x + u.y * u.y) + u.z * u.z;
    float a = 2.0f * duv, b = s * s - duu, c = 2.0f * s;
    v3 cr = mk(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
    return mk((a * u.x + b * v.x) + c * cr.x, (a * u.y + b * v.y) + c * cr.y, (a * u.z + b * v.z) + c * cr.z);
}
/* getPrimitiveAABB (CudaSDFUtil.h:507-542) */
static void prim_aabb(const OrPrim* pr, v3* mn, v3* mx) {
    float pad = 0.1f;
    if (pr->displacement != D_NONE) pad += 0.5f;
    v3 dims = mk(1, 1, 1);
    if (pr->type == T_SPHERE) dims = mk(pr->params[0], pr->params[0], pr->params[0]);
    else if (pr->type == T_BOX || pr->type == T_RBOX) dims = mk(pr->params[0], pr->params[1], pr->params[2]);
    else if (pr->type == T_TORUS)
        dims = mk(pr->params[0] + pr->params[1], pr->params[1], pr->params[0] + pr->params[1]);
    dims = add3(dims, mk(pad, pad, pad));
    *mn = mk(1e10f, 1e10f, 1e10f);
    *mx = mk(-1e10f, -1e10f, -1e10f);
    for (int i = 0; i < 8; ++i) {
        v3 c = mk((i & 1) ? dims.x : -dims.x, (i & 2) ? dims.y : -dims.y, (i & 4) ? dims.z : -dims.z);
        v3 p = mk(c.x * pr->scale[0], c.y * pr->scale[1], c.z * pr->scale[2]);
        p = host_rotate(p, pr->rotation);
        p = add3(p, mk(pr->position[0], pr->position[1], pr->position[2]));
        mn->x = fminf(mn->x, p.x); mn->y = fminf(mn->y, p.y); mn->z = fminf(mn->z, p.z);
        mx->x = fmaxf(mx->x, p.x); mx->y = fmaxf(mx->y, p.y); mx->z = fmaxf(mx->z, p.z);
    }
}
/* buildBVHRecursive (CudaSDFUtil.h:544-603): mean-centroid split on the longest axis, in-place
 * partition, median-count fallback; node order = preorder with the parent written first. */
static int bvh_build(int* idx, int count, const OrPrim* prims, OrNode* nodes, int* nn) {
    OrNode node;
    node.mn[0] = node.mn[1] = node.mn[2] = 1e10f;
    node.mx[0] = node.mx[1] = node.mx[2] = -1e10f;
    v3 cc = mk(0, 0, 0);
    for (int i = 0; i < count; ++i) {
        v3 a, b;
        prim_aabb(&prims[idx[i]], &a, &b);
        node.mn[0] = fminf(node.mn[0], a.x); node.mn[1] = fminf(node.mn[1], a.y); node.mn[2] = fminf(node.mn[2], a.z);
        node.mx[0] = fmaxf(node.mx[0], b.x); node.mx[1] = fmaxf(node.mx[1], b.y); node.mx[2] = fmaxf(node.mx[2], b.z);
        cc = add3(cc, mk((a.x + b.x) * 0.5f, (a.y + b.y) * 0.5f, (a.z + b.z) * 0.5f));
    }
    const float invc = 1.0f / (float)count;
    cc = mk(cc.x * invc, cc.y * invc, cc.z * invc);
    if (count <= 1) {
        node.left = idx[0];
        node.right = -1;
        nodes[*nn] = node;
        return (*nn)++;
    }
    int axis = 0;
    v3 ext = mk(node.mx[0] - node.mn[0], node.mx[1] - node.mn[1], node.mx[2] - node.mn[2]);
    if (ext.y > ext.x) axis = 1;
    if (ext.z > ext.y && ext.z > ext.x) axis = 2;
    const float split = axis == 0 ? cc.x : (axis == 1 ? cc.y : cc.z);
    int mid = 0;
    for (int i = 0; i < count; ++i) {
        v3 a, b;
        prim_aabb(&prims[idx[i]], &a, &b);
        float c = axis == 0 ? (a.x + b.x) * 0.5f : (axis == 1 ? (a.y + b.y) * 0.5f : (a.z + b.z) * 0.5f);
        if (c < split) {
            int t = idx[i]; idx[i] = idx[mid]; idx[mid] = t;
            mid++;
        }
    }
    if (mid == 0 || mid == count) mid = count / 2;
    const int cur = (*nn)++;
    nodes[cur] = node;
    const int l = bvh_build(idx, mid, prims, nodes, nn);
    const int r = bvh_build(idx + mid, count - mid, prims, nodes, nn);
    nodes[cur].left = l;
    nodes[cur].right = r;
    return cur;
}

int or_build_scene(const OrPrim* prims, int n, OrPrim* sorted, OrNode* nodes, int* nbvh) {
    int k = 0;
    for (int i = 0; i < n; ++i)
        if (prims[i].operation == OP_UNION || prims[i].operation == OP_UNION_BLEND) sorted[k++] = prims[i];
    const int nu = k;
    for (int i = 0; i < n; ++i)
        if (!(prims[i].operation == OP_UNION || prims[i].operation == OP_UNION_BLEND)) sorted[k++] = prims[i];
    *nbvh = nu;
    if (nu == 0) return 0;
    int* idx = (int*)malloc(sizeof(int) * nu);
    for (int i = 0; i < nu; ++i) idx[i] = i;
    int nn = 0;
    bvh_build(idx, nu, sorted, nodes, &nn);
    free(idx);
    return nn;
}

/* ------------------------------------------------------------------------------------------------
 * batched point queries and function probes
 * ---------------------------------------------------------------------------------------------- */
void or_map_batch(const OrScene* s, int n, const float* pts, float time, float* out8, int* iters) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        int it = 0;
        MapState st = map_eval(s, mk(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), time, &it);
        float* o = out8 + 8 * (size_t)i;
        o[0] = st.d; o[1] = st.color.x; o[2] = st.color.y; o[3] = st.color.z; o[4] = (float)st.id;
        o[5] = st.local.x; o[6] = st.local.y; o[7] = st.local.z;
        if (iters) iters[i] = it;
    }
}

void or_normal_batch(const OrScene* s, int n, const float* pts, float time, float cell, float* out3) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        v3 nrm = normal_at(s, mk(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), time, cell);
        out3[3 * i] = nrm.x; out3[3 * i + 1] = nrm.y; out3[3 * i + 2] = nrm.z;
    }
}

/* probe ids: the same records as the reference probe kernels (oracle/ref/ref_probe.cu) */
void or_probe(int which, int n, const float* in, int is, float* out, int os) {
    for (int i = 0; i < n; ++i) {
        const float* a = in + (size_t)i * is;
        float* o = out + (size_t)i * os;
        switch (which) {
            case 0: o[0] = sd_eval((int)a[0], mk(a[1], a[2], a[3]), a + 4); break;
            case 1: {
                OrPrim pr;
                memset(&pr, 0, sizeof pr);
                for (int k = 0; k < 3; ++k) { pr.position[k] = a[3 + k]; pr.scale[k] = a[10 + k]; }
                for (int k = 0; k < 4; ++k) pr.rotation[k] = a[6 + k];
                v3 p = to_local(mk(a[0], a[1], a[2]), &pr);
                o[0] = p.x; o[1] = p.y; o[2] = p.z;
            } break;
            case 2: { v3 p = disp_twist(mk(a[0], a[1], a[2]), a[3]); o[0] = p.x; o[1] = p.y; o[2] = p.z; } break;
            case 3: { v3 p = disp_bend(mk(a[0], a[1], a[2]), a[3]); o[0] = p.x; o[1] = p.y; o[2] = p.z; } break;
            case 4: o[0] = disp_sine_y(mk(a[0], a[1], a[2]), a[3], a[4], a[5]); break;
            case 7: o[0] = edge_t(a[0], a[1]); break;
            case 8: { v3 p = lerp3(mk(a[0], a[1], a[2]), mk(a[3], a[4], a[5]), a[6]); o[0] = p.x; o[1] = p.y; o[2] = p.z; } break;
            case 9: {
                OrGridDesc g; memset(&g, 0, sizeof g);
                g.origin[0] = a[0]; g.origin[1] = a[1]; g.origin[2] = a[2]; g.cell = a[3];
                v3 p = grid_loc(&g, (int)a[4], (int)a[5], (int)a[6]);
                o[0] = p.x; o[1] = p.y; o[2] = p.z;
            } break;
            case 10: {
                OrGridDesc g; memset(&g, 0, sizeof g);
                g.origin[0] = a[0]; g.origin[1] = a[1]; g.origin[2] = a[2]; g.cell = a[3];
                const int x = (int)a[4], y = (int)a[5], z = (int)a[6], e = (int)a[15];
                const int c1 = kEdge[e][0], c2 = kEdge[e][1];
                const float t = edge_t(a[7 + c1], a[7 + c2]);
                v3 p1 = grid_loc(&g, x + kCorner[c1][0], y + kCorner[c1][1], z + kCorner[c1][2]);
                v3 p2 = grid_loc(&g, x + kCorner[c2][0], y + kCorner[c2][1], z + kCorner[c2][2]);
                v3 p = lerp3_edge(p1, p2, t);
                o[0] = p.x; o[1] = p.y; o[2] = p.z;
            } break;
            case 11: {
                v3 t[3] = {mk(a[0], a[1], a[2]), mk(a[3], a[4], a[5]), mk(a[6], a[7], a[8])};
                o[0] = degenerate(t, a[9]) ? 1.0f : 0.0f;
            } break;
            case 12: {
                float x[3] = {0, 0, 0};
                int ok = solve3x3(a, a + 9, x);
                o[0] = ok ? 1.0f : 0.0f; o[1] = x[0]; o[2] = x[1]; o[3] = x[2];
            } break;
            case 13: case 14: {
                v3 pts[12], ns[12], x = mk(0, 0, 0);
                for (int k = 0; k < 12; ++k) {
                    pts[k] = mk(a[5 + 3 * k], a[6 + 3 * k], a[7 + 3 * k]);
                    ns[k] = mk(a[41 + 3 * k], a[42 + 3 * k], a[43 + 3 * k]);
                }
                int ok = which == 13 ? solve_qef_reg(pts, ns, (int)a[0], a[1], mk(a[2], a[3], a[4]), &x)
                                     : solve_qef(pts, ns, (int)a[0], &x);
                o[0] = ok ? 1.0f : 0.0f; o[1] = x.x; o[2] = x.y; o[3] = x.z;
            } break;
            case 15: {
                uint16_t q[4];
                dc_encode_vertex(mk(a[0], a[1], a[2]), mk(a[3], a[4], a[5]), a[6], q);
                o[0] = q[0]; o[1] = q[1]; o[2] = q[2];
            } break;
            case 16: {
                uint16_t q[3] = {(uint16_t)a[0], (uint16_t)a[1], (uint16_t)a[2]};
                v3 p = dc_decode_vertex(q, mk(a[3], a[4], a[5]), a[6]);
                o[0] = p.x; o[1] = p.y; o[2] = p.z;
            } break;
            case 17: {
                int16_t q[4];
                dc_encode_normal(mk(a[0], a[1], a[2]), q);
                o[0] = q[0]; o[1] = q[1]; o[2] = q[2];
            } break;
            case 18: {
                int16_t q[3] = {(int16_t)a[0], (int16_t)a[1], (int16_t)a[2]};
                v3 nrm = dc_decode_normal(q);
                o[0] = nrm.x; o[1] = nrm.y; o[2] = nrm.z;
            } break;
            case 19: o[0] = aabb_hit(mk(a[0], a[1], a[2]), a + 3, a + 6, a[9]) ? 1.0f : 0.0f; break;
            default: break;
        }
    }
}

void or_exclusive_scan(const uint32_t* in, uint32_t* out, int64_t n) {
    uint32_t acc = 0;
    for (int64_t i = 0; i < n; ++i) {
        uint32_t v = in[i];
        out[i] = acc;
        acc += v;
    }
}

/* ------------------------------------------------------------------------------------------------
 * pipelines
 * ---------------------------------------------------------------------------------------------- */
struct OrResult {
    int64_t nActive, totalVerts, nDcVerts, scoutCount;
    int32_t* active;
    uint32_t* counts;
    uint32_t* offsets;
    float* verts;
    float* colors;
    uint32_t* indices;
    float* uvs;
    float* primids;
    float* normals;
    uint8_t* dcmask;
    uint32_t* dcvoff;
    uint16_t* dcvert;
    int16_t* dcnorm;
};

/* scout (MarchingCubesKernels.cu:850-889) */
static inline int scout_block(const OrScene* s, const OrGridDesc* g, float time, int64_t idx) {
    const int bx = (int)(idx % g->bx);
    const int64_t t = idx / g->bx;
    const int by = (int)(t % g->by), bz = (int)(t / g->by);
    v3 c = mk(fmaf((float)(bx * BLOCK) + 4.0f, g->cell, g->origin[0]),
              fmaf((float)(by * BLOCK) + 4.0f, g->cell, g->origin[1]),
              fmaf((float)(bz * BLOCK) + 4.0f, g->cell, g->origin[2]));
    const float r = (8 * 0.5f * 1.73205f + 2.0f) * g->cell;
    const float d = map_d(s, c, time);
    return fabsf(d) <= r;
}

/* 9^3 samples of one block; field[(z*9+y)*9+x] = map at sample (8b+x, 8b+y, 8b+z). Each value equals
 * what the reference's per-cell corner loop computes at that sample (same point, same function). */
static void block_field(const OrScene* s, const OrGridDesc* g, float time, int block, float* field) {
    const int bx = block % g->bx, t = block / g->bx, by = t % g->by, bz = t / g->by;
    for (int z = 0; z < 9; ++z)
        for (int y = 0; y < 9; ++y)
            for (int x = 0; x < 9; ++x) {
                const int gx = bx * BLOCK + x, gy = by * BLOCK + y, gz = bz * BLOCK + z;
                float v = 0.0f;
                if (gx < (int)g->width && gy < (int)g->height && gz < (int)g->depth)
                    v = map_d(s, grid_loc(g, gx, gy, gz), time);
                field[(z * 9 + y) * 9 + x] = v;
            }
}

static inline void cell_xyz(const OrGridDesc* g, int block, int tid, int* x, int* y, int* z, int* lx, int* ly,
                            int* lz) {
    const int bx = block % g->bx, t = block / g->bx, by = t % g->by, bz = t / g->by;
    *lz = tid / 64;
    *ly = (tid % 64) / 8;
    *lx = tid % 8;
    *x = bx * BLOCK + *lx;
    *y = by * BLOCK + *ly;
    *z = bz * BLOCK + *lz;
}
static inline int oob(const OrGridDesc* g, int x, int y, int z) {
    return x >= (int)g->width - 1 || y >= (int)g->height - 1 || z >= (int)g->depth - 1;
}

/* per-cell MC triangles: returns the number of triangles in the case and fills pts/valid */
static int mc_cell(const OrGridDesc* g, const float* field, int x, int y, int z, int lx, int ly, int lz,
                   v3 tri[5][3], int valid[5], int* code_out) {
    float cv[8];
    int code = 0;
    for (int i = 0; i < 8; ++i) {
        cv[i] = field[((lz + kCorner[i][2]) * 9 + (ly + kCorner[i][1])) * 9 + (lx + kCorner[i][0])];
        if (cv[i] > 0.0f) code |= 1 << i;
    }
    *code_out = code;
    int nt = 0;
    for (int k = 0; k < 15 && mc_tri[code][k] >= 0; k += 3, ++nt) {
        for (int j = 0; j < 3; ++j) {
            const int e = mc_tri[code][k + j], c1 = kEdge[e][0], c2 = kEdge[e][1];
            const float t = edge_t(cv[c1], cv[c2]);
            v3 p1 = grid_loc(g, x + kCorner[c1][0], y + kCorner[c1][1], z + kCorner[c1][2]);
            v3 p2 = grid_loc(g, x + kCorner[c2][0], y + kCorner[c2][1], z + kCorner[c2][2]);
            tri[nt][j] = lerp3_edge(p1, p2, t);
        }
        valid[nt] = !degenerate(tri[nt], g->cell);
    }
    return nt;
}

/* lookupPackedCell (MarchingCubesKernels.cu:1633-1657) */
static int lookup_packed(const OrGridDesc* g, const int32_t* b2a, int cx, int cy, int cz, int64_t* out) {
    if (cx < 0 || cy < 0 || cz < 0) return 0;
    if (cx >= (int)g->width - 1 || cy >= (int)g->height - 1 || cz >= (int)g->depth - 1) return 0;
    const int bx = cx / BLOCK, by = cy / BLOCK, bz = cz / BLOCK;
    if (bx >= g->bx || by >= g->by || bz >= g->bz) return 0;
    const int64_t bi = bx + (int64_t)by * g->bx + (int64_t)bz * g->bx * g->by;
    const int a = b2a[bi];
    if (a < 0) return 0;
    const int tid = (cx - bx * BLOCK) + (cy - by * BLOCK) * BLOCK + (cz - bz * BLOCK) * 64;
    *out = (int64_t)a * BLOCK3 + tid;
    return 1;
}

static inline int surface(uint8_t m) { return m != 0x00 && m != 0xFF; }

static void write_vertex_streams(OrResult* r, uint32_t outMask, int64_t w, v3 p, v3 color, float pid, v2 uv,
                                 v3 nrm, int has_normal) {
    r->verts[4 * w] = p.x; r->verts[4 * w + 1] = p.y; r->verts[4 * w + 2] = p.z; r->verts[4 * w + 3] = 1.0f;
    if (outMask & OR_COLORS) {
        r->colors[4 * w] = color.x; r->colors[4 * w + 1] = color.y; r->colors[4 * w + 2] = color.z;
        r->colors[4 * w + 3] = 1.0f;
    }
    if ((outMask & OR_NORMALS) && has_normal) {
        r->normals[4 * w] = nrm.x; r->normals[4 * w + 1] = nrm.y; r->normals[4 * w + 2] = nrm.z;
        r->normals[4 * w + 3] = 0.0f;
    }
    if (outMask & OR_PRIMIDS) r->primids[w] = pid;
    if (outMask & OR_UVS) { r->uvs[2 * w] = uv.u; r->uvs[2 * w + 1] = uv.v; }
    if (outMask & OR_INDICES) r->indices[w] = (uint32_t)w;
}

static void alloc_streams(OrResult* r, uint32_t outMask, int64_t V) {
    const size_t n = (size_t)(V > 0 ? V : 1);
    r->verts = (float*)calloc(n * 4, sizeof(float));
    if (outMask & OR_COLORS) r->colors = (float*)calloc(n * 4, sizeof(float));
    if (outMask & OR_INDICES) r->indices = (uint32_t*)calloc(n, sizeof(uint32_t));
    if (outMask & OR_UVS) r->uvs = (float*)calloc(n * 2, sizeof(float));
    if (outMask & OR_PRIMIDS) r->primids = (float*)calloc(n, sizeof(float));
    if (outMask & OR_NORMALS) r->normals = (float*)calloc(n * 4, sizeof(float));
}

/* marching cubes: countActiveBlockTriangles + scan + generateActiveBlockTriangles (:914-1110) */
static void run_mc(OrResult* r, const OrScene* s, const OrGridDesc* g, float time, uint32_t outMask,
                   uint32_t maxV, float* fields) {
    const int64_t nA = r->nActive;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t a = 0; a < nA; ++a) {
        float* field = fields + (size_t)a * 729;
        block_field(s, g, time, r->active[a], field);
        for (int tid = 0; tid < BLOCK3; ++tid) {
            int x, y, z, lx, ly, lz, code;
            cell_xyz(g, r->active[a], tid, &x, &y, &z, &lx, &ly, &lz);
            uint32_t cnt = 0;
            if (!oob(g, x, y, z)) {
                v3 tri[5][3];
                int valid[5];
                const int nt = mc_cell(g, field, x, y, z, lx, ly, lz, tri, valid, &code);
                for (int k = 0; k < nt; ++k) cnt += valid[k] ? 3 : 0;
            }
            r->counts[a * BLOCK3 + tid] = cnt;
        }
    }
    or_exclusive_scan(r->counts, r->offsets, nA * BLOCK3);
    r->totalVerts = nA ? (int64_t)r->offsets[nA * BLOCK3 - 1] + r->counts[nA * BLOCK3 - 1] : 0;
    alloc_streams(r, outMask, r->totalVerts);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t a = 0; a < nA; ++a) {
        const float* field = fields + (size_t)a * 729;
        for (int tid = 0; tid < BLOCK3; ++tid) {
            int x, y, z, lx, ly, lz, code;
            cell_xyz(g, r->active[a], tid, &x, &y, &z, &lx, &ly, &lz);
            if (oob(g, x, y, z)) continue;
            v3 tri[5][3];
            int valid[5];
            const int nt = mc_cell(g, field, x, y, z, lx, ly, lz, tri, valid, &code);
            uint32_t w = r->offsets[a * BLOCK3 + tid];
            for (int k = 0; k < nt; ++k) {
                if (!valid[k]) continue;
                if ((uint64_t)w + 2 >= maxV) break;
                v3 c = mk((tri[k][0].x + tri[k][1].x + tri[k][2].x) / 3.0f,
                          (tri[k][0].y + tri[k][1].y + tri[k][2].y) / 3.0f,
                          (tri[k][0].z + tri[k][1].z + tri[k][2].z) / 3.0f);
                MapState ms = map_eval(s, c, time, NULL);
                v2 uvs[3] = {mk2(0, 0), mk2(0, 0), mk2(0, 0)};
                if ((outMask & OR_UVS) && ms.id >= 0 && ms.id < s->nprims) {
                    const OrPrim* pr = &s->prims[ms.id];
                    v3 lp[3];
                    for (int j = 0; j < 3; ++j) lp[j] = to_local(tri[k][j], pr);
                    triangle_uvs(lp, pr, uvs);
                }
                for (int j = 0; j < 3; ++j) {
                    v3 nrm = mk(0, 0, 0);
                    if (outMask & OR_NORMALS) nrm = normal_at(s, tri[k][j], time, g->cell);
                    write_vertex_streams(r, outMask, (int64_t)w + j, tri[k][j], ms.color, (float)ms.id, uvs[j], nrm, 1);
                }
                w += 3;
            }
        }
    }
}

/* cross3 (MarchingCubesKernels.cu:21-27) as inlined in the DC kernels: the first product fused */
static inline v3 cross3_ff(v3 a, v3 b) {
    return mk(fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x)));
}
/* dcSolveCellVertices body for one cell (:1348-1597) */
static void dc_solve_cell(const OrScene* s, const OrGridDesc* g, float time, const float* field, int x, int y,
                          int z, int lx, int ly, int lz, float qefBlend, uint16_t qv[4], int16_t qn[4]) {
    float cv[8];
    unsigned mask = 0;
    for (int i = 0; i < 8; ++i) {
        cv[i] = field[((lz + kCorner[i][2]) * 9 + (ly + kCorner[i][1])) * 9 + (lx + kCorner[i][0])];
        if (cv[i] > 0.0f) mask |= 1u << i;
    }
    v3 pts[12], ns[12];
    int m = 0;
    for (int e = 0; e < 12; ++e) {
        const int c1 = kEdge[e][0], c2 = kEdge[e][1];
        if (((mask >> c1) & 1) == ((mask >> c2) & 1)) continue;
        const float t = edge_t(cv[c1], cv[c2]);
        v3 p1 = grid_loc(g, x + kCorner[c1][0], y + kCorner[c1][1], z + kCorner[c1][2]);
        v3 p2 = grid_loc(g, x + kCorner[c2][0], y + kCorner[c2][1], z + kCorner[c2][2]);
        v3 p = lerp3_edge(p1, p2, t);
        pts[m] = p;
        ns[m] = normal_at(s, p, time, g->cell);
        m++;
    }
    const v3 cmin = grid_loc(g, x, y, z);
    const v3 cmax = mk(cmin.x + g->cell, cmin.y + g->cell, cmin.z + g->cell);
    v3 xs = mk(fmaf(0.5f, g->cell, cmin.x), fmaf(0.5f, g->cell, cmin.y), fmaf(0.5f, g->cell, cmin.z));
    v3 centroid = xs;
    if (m > 0) {
        v3 sum = mk(0, 0, 0);
        for (int i = 0; i < m; ++i) sum = add3(sum, pts[i]);
        centroid = scl3(sum, 1.0f / (float)m);
    }
    v3 cN[3] = {mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0)}, cP[3] = {mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0)};
    int cC[3] = {0, 0, 0}, k = 0;
    for (int i = 0; i < m; ++i) {
        v3 n = ns[i];
        const float len = sqrtf(dot3(n, n));
        if (len < 1e-6f) continue;
        n = mk(n.x / len, n.y / len, n.z / len);
        int best = -1;
        float bestDot = -1.0f;
        for (int ci = 0; ci < k; ++ci) {
            v3 cn = cN[ci];
            const float cl = sqrtf(dot3(cn, cn));
            if (cl > 1e-6f) cn = mk(cn.x / cl, cn.y / cl, cn.z / cl);
            const float d = fabsf(dot3(cn, n));
            if (d > bestDot) { bestDot = d; best = ci; }
        }
        if (best >= 0 && bestDot > 0.92f) {
            cN[best] = add3(cN[best], n); cP[best] = add3(cP[best], pts[i]); cC[best]++;
        } else if (k < 3) {
            cN[k] = n; cP[k] = pts[i]; cC[k] = 1; k++;
        } else {
            cN[best] = add3(cN[best], n); cP[best] = add3(cP[best], pts[i]); cC[best]++;
        }
    }
    int solved = 0;
    v3 xsol = xs;
    if (k >= 2) {
        v3 n1 = cN[0], n2 = cN[1], n3 = cN[2];
        const float l1 = sqrtf(dot3(n1, n1)), l2 = sqrtf(dot3(n2, n2)), l3 = sqrtf(dot3(n3, n3));
        if (l1 > 1e-6f && l2 > 1e-6f) {
            n1 = mk(n1.x / l1, n1.y / l1, n1.z / l1);
            n2 = mk(n2.x / l2, n2.y / l2, n2.z / l2);
            if (l3 > 1e-6f) n3 = mk(n3.x / l3, n3.y / l3, n3.z / l3);
            const float d12 = fabsf(dot3(n1, n2));
            const float d13 = (k >= 3 && l3 > 1e-6f) ? fabsf(dot3(n1, n3)) : 1.0f;
            const float d23 = (k >= 3 && l3 > 1e-6f) ? fabsf(dot3(n2, n3)) : 1.0f;
            const int c01 = cC[0] >= 2 && cC[1] >= 2;
            const int c012 = c01 && k >= 3 && cC[2] >= 2 && l3 > 1e-6f;
            const int doEdge = k == 2 && c01 && d12 < 0.75f;
            const int doCorner = k >= 3 && c012 && d12 < 0.80f && d13 < 0.80f && d23 < 0.80f;
            if (doEdge || doCorner) {
                const float i0 = 1.0f / (float)(cC[0] > 0 ? cC[0] : 1), i1 = 1.0f / (float)(cC[1] > 0 ? cC[1] : 1);
                v3 p1 = scl3(cP[0], i0), p2 = scl3(cP[1], i1);
                float A[9], b[3], sol[3];
                if (doEdge) {
                    v3 ne = cross3_ff(n1, n2);
                    const float le = sqrtf(dot3(ne, ne));
                    if (le > 1e-6f) {
                        ne = mk(ne.x / le, ne.y / le, ne.z / le);
                        v3 pa = mk(0, 0, 0);
                        for (int i = 0; i < m; ++i) pa = add3(pa, pts[i]);
                        pa = scl3(pa, 1.0f / (float)(m > 0 ? m : 1));
                        A[0] = n1.x; A[1] = n1.y; A[2] = n1.z; A[3] = n2.x; A[4] = n2.y; A[5] = n2.z;
                        A[6] = ne.x; A[7] = ne.y; A[8] = ne.z;
                        b[0] = dot3(n1, p1); b[1] = dot3(n2, p2); b[2] = dot3(ne, pa);
                        if (solve3x3(A, b, sol)) { xsol = mk(sol[0], sol[1], sol[2]); solved = 1; }
                    }
                } else {
                    const float i2 = 1.0f / (float)(cC[2] > 0 ? cC[2] : 1);
                    v3 p3 = scl3(cP[2], i2);
                    A[0] = n1.x; A[1] = n1.y; A[2] = n1.z; A[3] = n2.x; A[4] = n2.y; A[5] = n2.z;
                    A[6] = n3.x; A[7] = n3.y; A[8] = n3.z;
                    b[0] = dot3(n1, p1); b[1] = dot3(n2, p2); b[2] = dot3(n3, p3);
                    if (solve3x3(A, b, sol)) { xsol = mk(sol[0], sol[1], sol[2]); solved = 1; }
                }
            }
        }
    }
    if (!solved) {
        if (!solve_qef_reg(pts, ns, m, 0.05f, centroid, &xsol)) (void)solve_qef(pts, ns, m, &xsol);
    }
    const float margin = 0.10f * g->cell;
    xsol = mk(clampf(xsol.x, cmin.x - margin, cmax.x + margin), clampf(xsol.y, cmin.y - margin, cmax.y + margin),
              clampf(xsol.z, cmin.z - margin, cmax.z + margin));
    xsol = mk(clampf(xsol.x, cmin.x, cmax.x), clampf(xsol.y, cmin.y, cmax.y), clampf(xsol.z, cmin.z, cmax.z));
    const v3 center = mk(fmaf(0.5f, g->cell, cmin.x), fmaf(0.5f, g->cell, cmin.y), fmaf(0.5f, g->cell, cmin.z));
    xsol = lerp3_edge(center, xsol, qefBlend);
    dc_encode_vertex(xsol, cmin, g->cell, qv);
    v3 nsum = mk(0, 0, 0);
    for (int i = 0; i < m; ++i) nsum = add3(nsum, ns[i]);
    const float len = sqrtf(dot3(nsum, nsum));
    v3 nout = (len > 1e-6f) ? mk(nsum.x / len, nsum.y / len, nsum.z / len) : normal_at(s, xsol, time, g->cell);
    const v3 nref = normal_at(s, xsol, time, g->cell);
    if (dot3(nout, nref) < 0.0f) nout = mk(-nout.x, -nout.y, -nout.z);
    dc_encode_normal(nout, qn);
}

/* the three edges leaving corner 0 and the four cells around each (:1735-1781, :2004-2043) */
static int dc_edge_cells(const OrGridDesc* g, const int32_t* b2a, int axis, int x, int y, int z, int64_t p[4]) {
    if (axis == 0) {
        if (!(y > 0 && z > 0)) return 0;
        return lookup_packed(g, b2a, x, y, z, &p[0]) && lookup_packed(g, b2a, x, y - 1, z, &p[1]) &&
               lookup_packed(g, b2a, x, y, z - 1, &p[2]) && lookup_packed(g, b2a, x, y - 1, z - 1, &p[3]);
    } else if (axis == 1) {
        if (!(x > 0 && z > 0)) return 0;
        return lookup_packed(g, b2a, x, y, z, &p[0]) && lookup_packed(g, b2a, x - 1, y, z, &p[1]) &&
               lookup_packed(g, b2a, x, y, z - 1, &p[2]) && lookup_packed(g, b2a, x - 1, y, z - 1, &p[3]);
    }
    if (!(x > 0 && y > 0)) return 0;
    return lookup_packed(g, b2a, x, y, z, &p[0]) && lookup_packed(g, b2a, x - 1, y, z, &p[1]) &&
           lookup_packed(g, b2a, x, y - 1, z, &p[2]) && lookup_packed(g, b2a, x - 1, y - 1, z, &p[3]);
}

static const int kQuadEdgeCorner[3] = {1, 3, 4};

static void run_dc(OrResult* r, const OrScene* s, const OrGridDesc* g, float time, uint32_t outMask,
                   uint32_t maxV, float qefBlend, float* fields) {
    const int64_t nA = r->nActive, nblocks = (int64_t)g->bx * g->by * g->bz;
    int32_t* b2a = (int32_t*)malloc(sizeof(int32_t) * (size_t)nblocks);
    for (int64_t i = 0; i < nblocks; ++i) b2a[i] = -1;
    for (int64_t a = 0; a < nA; ++a) b2a[r->active[a]] = (int32_t)a;
    uint32_t* hasv = (uint32_t*)calloc((size_t)(nA * BLOCK3 + 1), sizeof(uint32_t));
    r->dcmask = (uint8_t*)calloc((size_t)(nA * BLOCK3 + 1), 1);
    r->dcvoff = (uint32_t*)calloc((size_t)(nA * BLOCK3 + 1), sizeof(uint32_t));
    /* dcMarkCells (:1312-1346) */
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t a = 0; a < nA; ++a) {
        float* field = fields + (size_t)a * 729;
        block_field(s, g, time, r->active[a], field);
        for (int tid = 0; tid < BLOCK3; ++tid) {
            int x, y, z, lx, ly, lz;
            cell_xyz(g, r->active[a], tid, &x, &y, &z, &lx, &ly, &lz);
            uint8_t mask = 0;
            if (!oob(g, x, y, z))
                for (int i = 0; i < 8; ++i)
                    if (field[((lz + kCorner[i][2]) * 9 + (ly + kCorner[i][1])) * 9 + (lx + kCorner[i][0])] > 0.0f)
                        mask |= (uint8_t)(1u << i);
            r->dcmask[a * BLOCK3 + tid] = mask;
            hasv[a * BLOCK3 + tid] = surface(mask) ? 1u : 0u;
        }
    }
    or_exclusive_scan(hasv, r->dcvoff, nA * BLOCK3);
    r->nDcVerts = nA ? (int64_t)r->dcvoff[nA * BLOCK3 - 1] + hasv[nA * BLOCK3 - 1] : 0;
    r->dcvert = (uint16_t*)calloc((size_t)(r->nDcVerts + 1) * 4, sizeof(uint16_t));
    r->dcnorm = (int16_t*)calloc((size_t)(r->nDcVerts + 1) * 4, sizeof(int16_t));
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t a = 0; a < nA; ++a) {
        const float* field = fields + (size_t)a * 729;
        for (int tid = 0; tid < BLOCK3; ++tid) {
            const int64_t pk = a * BLOCK3 + tid;
            if (!hasv[pk]) continue;
            int x, y, z, lx, ly, lz;
            cell_xyz(g, r->active[a], tid, &x, &y, &z, &lx, &ly, &lz);
            const uint32_t vi = r->dcvoff[pk];
            if (vi >= maxV) continue;
            dc_solve_cell(s, g, time, field, x, y, z, lx, ly, lz, qefBlend, &r->dcvert[4 * (size_t)vi],
                          &r->dcnorm[4 * (size_t)vi]);
        }
    }
    /* dcCountQuads (:1714-1784) */
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t a = 0; a < nA; ++a) {
        for (int tid = 0; tid < BLOCK3; ++tid) {
            int x, y, z, lx, ly, lz;
            cell_xyz(g, r->active[a], tid, &x, &y, &z, &lx, &ly, &lz);
            uint32_t cnt = 0;
            if (!oob(g, x, y, z)) {
                const uint8_t mask = r->dcmask[a * BLOCK3 + tid];
                const unsigned s0 = mask & 1u;
                for (int ax = 0; ax < 3; ++ax) {
                    if (((mask >> kQuadEdgeCorner[ax]) & 1u) == s0) continue;
                    int64_t p[4];
                    if (dc_edge_cells(g, b2a, ax, x, y, z, p) && surface(r->dcmask[p[0]]) &&
                        surface(r->dcmask[p[1]]) && surface(r->dcmask[p[2]]) && surface(r->dcmask[p[3]]))
                        cnt += 6;
                }
            }
            r->counts[a * BLOCK3 + tid] = cnt;
        }
    }
    or_exclusive_scan(r->counts, r->offsets, nA * BLOCK3);
    r->totalVerts = nA ? (int64_t)r->offsets[nA * BLOCK3 - 1] + r->counts[nA * BLOCK3 - 1] : 0;
    alloc_streams(r, outMask, r->totalVerts);
    /* dcGenerateQuads (:1806-2044) */
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t a = 0; a < nA; ++a) {
        for (int tid = 0; tid < BLOCK3; ++tid) {
            const int64_t pk = a * BLOCK3 + tid;
            if (r->counts[pk] == 0) continue;
            int x, y, z, lx, ly, lz;
            cell_xyz(g, r->active[a], tid, &x, &y, &z, &lx, &ly, &lz);
            if (oob(g, x, y, z)) continue;
            const uint8_t mask = r->dcmask[pk];
            const unsigned s0 = mask & 1u;
            uint32_t w = r->offsets[pk];
            for (int ax = 0; ax < 3; ++ax) {
                if (((mask >> kQuadEdgeCorner[ax]) & 1u) == s0) continue;
                int64_t p[4];
                if (!dc_edge_cells(g, b2a, ax, x, y, z, p)) continue;
                /* vertex order per edge: X (A,B,D,C), Y (A,C,D,B), Z (A,B,D,C) */
                int64_t q[4];
                if (ax == 1) { q[0] = p[0]; q[1] = p[2]; q[2] = p[3]; q[3] = p[1]; }
                else { q[0] = p[0]; q[1] = p[1]; q[2] = p[3]; q[3] = p[2]; }
                if (!surface(r->dcmask[q[0]]) || !surface(r->dcmask[q[1]]) || !surface(r->dcmask[q[2]]) ||
                    !surface(r->dcmask[q[3]]))
                    continue;
                v3 v[4];
                int bad = 0;
                for (int j = 0; j < 4; ++j) {
                    const int64_t ab = q[j] / BLOCK3;
                    const int t = (int)(q[j] - ab * BLOCK3);
                    int cx, cy, cz, clx, cly, clz;
                    cell_xyz(g, r->active[ab], t, &cx, &cy, &cz, &clx, &cly, &clz);
                    const uint32_t vi = r->dcvoff[q[j]];
                    if (vi >= maxV) bad = 1;
                    else v[j] = dc_decode_vertex(&r->dcvert[4 * (size_t)vi], grid_loc(g, cx, cy, cz), g->cell);
                }
                if (bad) continue;
                const v3 qc = mk(0.25f * (((v[0].x + v[1].x) + v[2].x) + v[3].x),
                                 0.25f * (((v[0].y + v[1].y) + v[2].y) + v[3].y),
                                 0.25f * (((v[0].z + v[1].z) + v[2].z) + v[3].z));
                for (int j = 0; j < 4; ++j)
                    if (!finite3(v[j])) v[j] = qc;
                {
                    const v3 nref = normal_at(s, qc, time, g->cell);
                    const v3 nt = cross3_ff(sub3(v[1], v[0]), sub3(v[2], v[0]));
                    if (dot3(nt, nref) < 0.0f) { v3 tmp = v[1]; v[1] = v[3]; v[3] = tmp; }
                }
                MapState ms = map_eval(s, qc, time, NULL);
                v2 quv[4] = {mk2(0, 0), mk2(0, 0), mk2(0, 0), mk2(0, 0)};
                if ((outMask & OR_UVS) && ms.id >= 0 && ms.id < s->nprims) {
                    const OrPrim* pr = &s->prims[ms.id];
                    v3 lp[4];
                    for (int j = 0; j < 4; ++j) lp[j] = to_local(v[j], pr);
                    v3 t0[3] = {lp[0], lp[1], lp[2]}, t1[3] = {lp[0], lp[2], lp[3]};
                    v2 u0[3], u1[3];
                    triangle_uvs(t0, pr, u0);
                    triangle_uvs(t1, pr, u1);
                    quv[0] = mk2((u0[0].u + u1[0].u) * 0.5f, (u0[0].v + u1[0].v) * 0.5f);
                    quv[1] = u0[1];
                    quv[2] = mk2((u0[2].u + u1[1].u) * 0.5f, (u0[2].v + u1[1].v) * 0.5f);
                    quv[3] = u1[2];
                }
                v3 tn[6] = {mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0), mk(0, 0, 0)};
                if (outMask & OR_NORMALS) {
                    const float off = g->cell * 0.25f;
                    const int tv[2][3] = {{0, 1, 2}, {0, 2, 3}};
                    for (int t = 0; t < 2; ++t) {
                        v3 fn = cross3_ff(sub3(v[tv[t][1]], v[tv[t][0]]), sub3(v[tv[t][2]], v[tv[t][0]]));
                        const float len = sqrtf(dot3(fn, fn));
                        if (len > 1e-6f) fn = mk(fn.x / len, fn.y / len, fn.z / len);
                        else fn = normal_at(s, qc, time, g->cell);
                        for (int j = 0; j < 3; ++j) {
                            const v3 vv = v[tv[t][j]];
                            tn[3 * t + j] = normal_at(s, mk(fmaf(fn.x, off, vv.x), fmaf(fn.y, off, vv.y), fmaf(fn.z, off, vv.z)),
                                                      time, g->cell);
                        }
                    }
                }
                if ((uint64_t)w + 5 >= maxV) continue;
                const int order[6] = {0, 1, 2, 0, 2, 3};
                const v2 tuv[6] = {quv[0], quv[1], quv[2], quv[0], quv[2], quv[3]};
                for (int j = 0; j < 6; ++j)
                    write_vertex_streams(r, outMask, (int64_t)w + j, v[order[j]], ms.color, (float)ms.id, tuv[j], tn[j], 1);
                w += 6;
            }
        }
    }
    free(hasv);
    free(b2a);
}

OrResult* or_run(const OrScene* s, const OrGridDesc* g, float time, int technique, float qefBlend, uint32_t outMask,
                 uint32_t maxV, int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    OrResult* r = (OrResult*)calloc(1, sizeof(OrResult));
    const int64_t nb = (int64_t)g->bx * g->by * g->bz;
    uint8_t* act = (uint8_t*)calloc((size_t)nb, 1);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t b = 0; b < nb; ++b) act[b] = (uint8_t)scout_block(s, g, time, b);
    int64_t nA = 0;
    for (int64_t b = 0; b < nb; ++b) nA += act[b];
    r->scoutCount = nA;
    r->nActive = nA;
    r->active = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nA + 1));
    int64_t k = 0;
    for (int64_t b = 0; b < nb; ++b)
        if (act[b]) r->active[k++] = (int32_t)b;
    free(act);
    r->counts = (uint32_t*)calloc((size_t)(nA * BLOCK3 + 1), sizeof(uint32_t));
    r->offsets = (uint32_t*)calloc((size_t)(nA * BLOCK3 + 1), sizeof(uint32_t));
    float* fields = (float*)malloc(sizeof(float) * 729 * (size_t)(nA + 1));
    if (technique == 0) run_mc(r, s, g, time, outMask, maxV, fields);
    else run_dc(r, s, g, time, outMask, maxV, qefBlend, fields);
    free(fields);
    return r;
}

void or_result_sizes(const OrResult* r, int64_t out[4]) {
    out[0] = r->nActive; out[1] = r->totalVerts; out[2] = r->nDcVerts; out[3] = r->scoutCount;
}

int or_result_copy(const OrResult* r, int buf, void* dst, size_t bytes) {
    const void* src = NULL;
    switch (buf) {
        case ORB_ACTIVE: src = r->active; break;
        case ORB_COUNTS: src = r->counts; break;
        case ORB_OFFSETS: src = r->offsets; break;
        case ORB_VERTS: src = r->verts; break;
        case ORB_COLORS: src = r->colors; break;
        case ORB_INDICES: src = r->indices; break;
        case ORB_UVS: src = r->uvs; break;
        case ORB_PRIMIDS: src = r->primids; break;
        case ORB_NORMALS: src = r->normals; break;
        case ORB_DCMASK: src = r->dcmask; break;
        case ORB_DCVOFF: src = r->dcvoff; break;
        case ORB_DCVERT: src = r->dcvert; break;
        case ORB_DCNORM: src = r->dcnorm; break;
        default: return -1;
    }
    if (!src) return -2;
    if (bytes) memcpy(dst, src, bytes);
    return 0;
}

void or_result_free(OrResult* r) {
    if (!r) return;
    free(r->active); free(r->counts); free(r->offsets); free(r->verts); free(r->colors); free(r->indices);
    free(r->uvs); free(r->primids); free(r->normals); free(r->dcmask); free(r->dcvoff); free(r->dcvert);
    free(r->dcnorm);
    free(r);
}

int64_t or_scout_range(const OrScene* s, const OrGridDesc* g, float time, int64_t b0, int64_t b1, int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    int64_t n = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : n)
    for (int64_t b = b0; b < b1; ++b) n += scout_block(s, g, time, b);
    return n;
}

void or_scout_flags(const OrScene* s, const OrGridDesc* g, float time, const int32_t* blocks, int n, uint8_t* flags,
                    int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) flags[i] = (uint8_t)scout_block(s, g, time, blocks[i]);
}

int64_t or_mc_blocks(const OrScene* s, const OrGridDesc* g, float time, const int32_t* blocks, int nblocks,
                     int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    int64_t tris = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : tris)
    for (int a = 0; a < nblocks; ++a) {
        float field[729];
        block_field(s, g, time, blocks[a], field);
        for (int tid = 0; tid < BLOCK3; ++tid) {
            int x, y, z, lx, ly, lz, code;
            cell_xyz(g, blocks[a], tid, &x, &y, &z, &lx, &ly, &lz);
            if (oob(g, x, y, z)) continue;
            v3 tri[5][3];
            int valid[5];
            const int nt = mc_cell(g, field, x, y, z, lx, ly, lz, tri, valid, &code);
            for (int k = 0; k < nt; ++k) tris += valid[k];
        }
    }
    return tris;
}
