// Per-vertex UV mapping (MarchingCubesKernels.cu:249-479): canonical per-primitive mappings,
// seam-aware adjustment across a triangle, and the primitive's uv transform.
#pragma once

#include "sdf_device.cuh"

namespace sdfb {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kPi2 = 1.57079632679489661923f;

__device__ __forceinline__ float2 uv_sphere(float3 p) {
    const float len = len3(p);
    if (len < 1e-6f) return make_float2(0.5f, 0.5f);
    p = scl3(p, DIV(1.f, len));
    const float theta = atan2f(p.z, p.x);
    const float phi = asinf(CLAMP(p.y, -1.f, 1.f));
    // the reference divides in double (M_PI is a double literal)
    return make_float2((float)(((double)theta + 3.14159265358979323846) / (2.0 * 3.14159265358979323846)),
                       (float)(((double)phi + 1.57079632679489661923) / 3.14159265358979323846));
}
__device__ __forceinline__ float2 uv_box(float3 p, float3 n) {
    const float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
    if (ax > ay && ax > az) return make_float2(FMA(p.z, 0.5f, 0.5f), FMA(p.y, 0.5f, 0.5f));
    if (ay > az) return make_float2(FMA(p.x, 0.5f, 0.5f), FMA(p.z, 0.5f, 0.5f));
    return make_float2(FMA(p.x, 0.5f, 0.5f), FMA(p.y, 0.5f, 0.5f));
}
__device__ __forceinline__ float2 uv_cylinder(float3 p, float height) {
    const float theta = atan2f(p.z, p.x);
    return make_float2((float)(((double)theta + 3.14159265358979323846) / (2.0 * 3.14159265358979323846)),
                       CLAMP(FMA(DIV(p.y, height), 0.5f, 0.5f), 0.f, 1.f));
}
__device__ __forceinline__ float2 uv_torus(float3 p, float R) {
    const float theta = atan2f(p.z, p.x);
    const float qx = SUB(len2(p.x, p.z), R);
    const float phi = atan2f(p.y, qx);
    return make_float2((float)(((double)theta + 3.14159265358979323846) / (2.0 * 3.14159265358979323846)),
                       (float)(((double)phi + 3.14159265358979323846) / (2.0 * 3.14159265358979323846)));
}
__device__ __forceinline__ float2 uv_capsule(float3 p, float height) {
    if (p.y > height) return uv_sphere(f3(p.x, SUB(p.y, height), p.z));
    if (p.y < 0.f) return uv_sphere(p);
    return uv_cylinder(p, height);
}
__device__ __forceinline__ float3 approx_local_normal(float3 lp, int type) {
    if (type == P_BOX || type == P_RBOX) {
        const float ax = fabsf(lp.x), ay = fabsf(lp.y), az = fabsf(lp.z);
        if (ax > ay && ax > az) return f3(copysignf(1.f, lp.x), 0.f, 0.f);
        if (ay > az) return f3(0.f, copysignf(1.f, lp.y), 0.f);
        return f3(0.f, 0.f, copysignf(1.f, lp.z));
    }
    const float len = len3(lp);
    return (len > 1e-6f) ? scl3(lp, DIV(1.f, len)) : f3(0.f, 1.f, 0.f);
}
__device__ __forceinline__ float2 seam_adjust(float2 uv, float2 ref) {
    float2 r = uv;
    if (fabsf(SUB(uv.x, ref.x)) > 0.5f) r.x = ADD(r.x, (uv.x < ref.x) ? 1.f : -1.f);
    if (fabsf(SUB(uv.y, ref.y)) > 0.5f) r.y = ADD(r.y, (uv.y < ref.y) ? 1.f : -1.f);
    return r;
}

struct UvParams {
    int type;
    float p0, p1;          // params[0], params[1]
    float sx, sy, ox, oy;  // uvScale, uvOffset
    float rot;             // uvRotation
};

__device__ __forceinline__ UvParams load_uv_params(const float4* __restrict__ pr) {
    UvParams u;
    const float4 r5 = __ldg(pr + 5), r6 = __ldg(pr + 6), r7 = __ldg(pr + 7), r8 = __ldg(pr + 8);
    u.type = __float_as_int(r6.z);
    u.p0 = r5.x;
    u.p1 = r5.y;
    u.sx = r7.z;
    u.sy = r7.w;
    u.ox = r8.x;
    u.oy = r8.y;
    u.rot = r8.z;
    return u;
}

__device__ __forceinline__ float2 uv_transform(float2 uv, const UvParams& P) {
    uv = make_float2(MUL(uv.x, P.sx), MUL(uv.y, P.sy));
    if (fabsf(P.rot) > 1e-6f) {
        const float c = cosf(P.rot), s = sinf(P.rot);
        uv = make_float2(det2(uv.x, c, uv.y, s), FMA(uv.x, s, MUL(uv.y, c)));
    }
    return make_float2(ADD(uv.x, P.ox), ADD(uv.y, P.oy));
}

// computeTriangleUVs (MarchingCubesKernels.cu:392-479)
__device__ __forceinline__ void triangle_uvs(const float3 lp[3], const UvParams& P, float2 out[3]) {
    const bool needs = (P.type == P_BOX || P.type == P_RBOX || P.type == P_OCTA);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float3 ln = needs ? approx_local_normal(lp[i], P.type) : f3(0.f, 0.f, 0.f);
        float2 uv;
        switch (P.type) {
            case P_SPHERE: case P_ELLIPSOID: uv = uv_sphere(lp[i]); break;
            case P_BOX: case P_RBOX: case P_OCTA: uv = uv_box(lp[i], ln); break;
            case P_CYLINDER: case P_RCYL: uv = uv_cylinder(lp[i], P.p0); break;
            case P_TORUS: uv = uv_torus(lp[i], P.p0); break;
            case P_CAPSULE: uv = uv_capsule(lp[i], P.p0); break;
            case P_CONE: case P_RCONE: uv = uv_cylinder(lp[i], P.p0); break;
            case P_HEXPRISM: case P_TRIPRISM: uv = uv_cylinder(lp[i], P.p1); break;
            default: uv = make_float2(FMA(lp[i].x, 0.5f, 0.5f), FMA(lp[i].y, 0.5f, 0.5f)); break;
        }
        out[i] = uv;
    }
    out[1] = seam_adjust(out[1], out[0]);
    out[2] = seam_adjust(out[2], out[0]);
    const float d01 = ADD(fabsf(SUB(out[0].x, out[1].x)), fabsf(SUB(out[0].y, out[1].y)));
    const float d02 = ADD(fabsf(SUB(out[0].x, out[2].x)), fabsf(SUB(out[0].y, out[2].y)));
    const float d12 = ADD(fabsf(SUB(out[1].x, out[2].x)), fabsf(SUB(out[1].y, out[2].y)));
    if (d01 > 0.5f && d02 > 0.5f && d12 < 0.5f) out[0] = seam_adjust(out[0], out[1]);
#pragma unroll
    for (int i = 0; i < 3; ++i) out[i] = uv_transform(out[i], P);
}

}  // namespace sdfb
