// Reference probe harness (test infrastructure, never shipped, never on the product path).
//
// This translation unit compiles the reference's kernel source file unchanged, straight from the
// reference tree (the include path is set by oracle/ref/Makefile), and adds probe kernels that call
// the reference's own __device__ functions on caller-supplied inputs. Their outputs are the golden
// vectors that pin the CPU oracle (oracle/sdf_oracle.c) function by function:
//   sd* primitives      MarchingCubesKernels.cu:129-219
//   world->local        MarchingCubesKernels.cu:597-599 (Commons.cuh:264-278 quaternions)
//   displacements       MarchingCubesKernels.cu:229-243, 604-606
//   map()               MarchingCubesKernels.cu:570-808
//   computeNormal       MarchingCubesKernels.cu:814-844
//   safeEdgeT/lerp3     MarchingCubesKernels.cu:33-54, interpEdgePoint :60-81, isDegenerateTri :83-103
//   getLocation         Commons.cuh:209-215
//   DC codecs / solvers MarchingCubesKernels.cu:1133-1301
// Nothing here changes the reference's code; the probes only call it.
#include "MarchingCubesKernels.cu"

#include <cstdio>

namespace refprobe {

enum ProbeId {
    PR_SD = 0,      // in: type, p[3], params[6]                       out: d
    PR_XFORM = 1,   // in: p[3], pos[3], rot[4], scale[3]               out: local p[3]
    PR_TWIST = 2,   // in: p[3], k                                      out: p[3]
    PR_BEND = 3,    // in: p[3], k                                      out: p[3]
    PR_SINE = 4,    // in: p[3], k, amp, time                           out: p.y displaced
    PR_MAP = 5,     // in: p[3]  (scene in grid)                        out: d, color[3], primID, local[3]
    PR_NORMAL = 6,  // in: p[3]  (scene in grid)                        out: n[3]
    PR_EDGET = 7,   // in: v1, v2                                       out: t
    PR_LERP = 8,    // in: a[3], b[3], t                                out: p[3]
    PR_GETLOC = 9,  // in: origin[3], cell, ix, iy, iz                  out: p[3]
    PR_INTERP = 10, // in: origin[3], cell, ix, iy, iz, val[8], edge    out: p[3]
    PR_DEGEN = 11,  // in: p0[3], p1[3], p2[3], cell                    out: degenerate (0/1)
    PR_SOLVE3 = 12, // in: A[9], b[3]                                   out: ok, x[3]
    PR_QEFREG = 13, // in: m, alpha, c[3], pts[12*3], ns[12*3]          out: ok, x[3]
    PR_QEF = 14,    // in: m, pts[12*3], ns[12*3] (at offset 5)         out: ok, x[3]
    PR_ENCV = 15,   // in: pw[3], cellMin[3], cell                      out: q[3]
    PR_DECV = 16,   // in: q[3], cellMin[3], cell                       out: p[3]
    PR_ENCN = 17,   // in: n[3]                                         out: q[3]
    PR_DECN = 18,   // in: q[3]                                         out: n[3]
    PR_AABBD = 19,  // in: p[3], mn[3], mx[3], dmin                     out: hit (0/1)
};

constexpr int IN_STRIDE = 96;
constexpr int OUT_STRIDE = 8;

__device__ float probe_sd(int type, float3 p, const float* prm) {
    switch (type) {
        case SDF_SPHERE: return sdSphere(p, prm[0]);
        case SDF_BOX: return sdBox(p, make_float3(prm[0], prm[1], prm[2]));
        case SDF_TORUS: return sdTorus(p, prm[0], prm[1]);
        case SDF_CYLINDER: return sdCylinder(p, prm[0], prm[1]);
        case SDF_CAPSULE: return sdCapsule(p, prm[0], prm[1]);
        case SDF_CONE: return sdCone(p, prm[0], prm[1]);
        case SDF_ROUNDED_BOX: return sdRoundedBox(p, make_float3(prm[0], prm[1], prm[2]), prm[3]);
        case SDF_ELLIPSOID: return sdEllipsoid(p, make_float3(prm[0], prm[1], prm[2]));
        case SDF_OCTOHEDRON: return sdOctahedron(p, prm[0]);
        case SDF_TRIANGULAR_PRISM: return sdTriPrism(p, make_float2(prm[0], prm[1]));
        case SDF_ROUNDED_CYLINDER: return sdRoundedCylinder(p, prm[0], prm[1], prm[2]);
        case SDF_ROUNDED_CONE: return sdRoundedCone(p, prm[0], prm[1], prm[2]);
        case SDF_HEX_PRISM: return sdHexPrism(p, make_float2(prm[0], prm[1]));
        default: return length(p) - 1.0f;
    }
}

__global__ void probe_kernel(int which, int n, const float* __restrict__ in, float* __restrict__ out,
                             SDFGrid grid, float time) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* a = in + (size_t)i * IN_STRIDE;
    float* o = out + (size_t)i * OUT_STRIDE;
    switch (which) {
        case PR_SD: {
            o[0] = probe_sd((int)a[0], make_float3(a[1], a[2], a[3]), a + 4);
        } break;
        case PR_XFORM: {
            float3 p = make_float3(a[0], a[1], a[2]) - make_float3(a[3], a[4], a[5]);
            p = invRotateVector(p, make_float4(a[6], a[7], a[8], a[9]));
            p = make_float3(p.x / a[10], p.y / a[11], p.z / a[12]);
            o[0] = p.x; o[1] = p.y; o[2] = p.z;
        } break;
        case PR_TWIST: {
            float3 p = dispTwist(make_float3(a[0], a[1], a[2]), a[3]);
            o[0] = p.x; o[1] = p.y; o[2] = p.z;
        } break;
        case PR_BEND: {
            float3 p = dispBend(make_float3(a[0], a[1], a[2]), a[3]);
            o[0] = p.x; o[1] = p.y; o[2] = p.z;
        } break;
        case PR_SINE: {
            float3 p = make_float3(a[0], a[1], a[2]);
            p.y += sinf(p.x * a[3] + a[5]) * a[4];
            o[0] = p.y;
        } break;
        case PR_MAP: {
            float d; float3 c; int id; float3 lp;
            map(make_float3(a[0], a[1], a[2]), grid, time, d, c, id, lp);
            o[0] = d; o[1] = c.x; o[2] = c.y; o[3] = c.z; o[4] = (float)id;
            o[5] = lp.x; o[6] = lp.y; o[7] = lp.z;
        } break;
        case PR_NORMAL: {
            float3 nrm = computeNormal(make_float3(a[0], a[1], a[2]), grid, time);
            o[0] = nrm.x; o[1] = nrm.y; o[2] = nrm.z;
        } break;
        case PR_EDGET: {
            o[0] = safeEdgeT(a[0], a[1]);
        } break;
        case PR_LERP: {
            float3 p = lerp3(make_float3(a[0], a[1], a[2]), make_float3(a[3], a[4], a[5]), a[6]);
            o[0] = p.x; o[1] = p.y; o[2] = p.z;
        } break;
        case PR_GETLOC: {
            SDFGrid g = grid;
            g.origin = make_float3(a[0], a[1], a[2]);
            g.cellSize = a[3];
            float3 p = getLocation(g, make_int4((int)a[4], (int)a[5], (int)a[6], 0));
            o[0] = p.x; o[1] = p.y; o[2] = p.z;
        } break;
        case PR_INTERP: {
            SDFGrid g = grid;
            g.origin = make_float3(a[0], a[1], a[2]);
            g.cellSize = a[3];
            float cv[8];
            for (int k = 0; k < 8; ++k) cv[k] = a[7 + k];
            float3 p = interpEdgePoint(g, make_int4((int)a[4], (int)a[5], (int)a[6], 0), cv, (int)a[15]);
            o[0] = p.x; o[1] = p.y; o[2] = p.z;
        } break;
        case PR_DEGEN: {
            float3 t[3] = {make_float3(a[0], a[1], a[2]), make_float3(a[3], a[4], a[5]),
                           make_float3(a[6], a[7], a[8])};
            o[0] = isDegenerateTri(t, a[9]) ? 1.0f : 0.0f;
        } break;
        case PR_SOLVE3: {
            float A[9], b[3], x[3] = {0, 0, 0};
            for (int k = 0; k < 9; ++k) A[k] = a[k];
            for (int k = 0; k < 3; ++k) b[k] = a[9 + k];
            bool ok = solve3x3(A, b, x);
            o[0] = ok ? 1.0f : 0.0f; o[1] = x[0]; o[2] = x[1]; o[3] = x[2];
        } break;
        case PR_QEFREG: {
            int m = (int)a[0];
            float3 pts[12], ns[12];
            for (int k = 0; k < 12; ++k) {
                pts[k] = make_float3(a[5 + 3 * k], a[6 + 3 * k], a[7 + 3 * k]);
                ns[k] = make_float3(a[41 + 3 * k], a[42 + 3 * k], a[43 + 3 * k]);
            }
            float3 x = make_float3(0, 0, 0);
            bool ok = solveQEFRegularized(pts, ns, m, a[1], make_float3(a[2], a[3], a[4]), x);
            o[0] = ok ? 1.0f : 0.0f; o[1] = x.x; o[2] = x.y; o[3] = x.z;
        } break;
        case PR_QEF: {
            int m = (int)a[0];
            float3 pts[12], ns[12];
            for (int k = 0; k < 12; ++k) {
                pts[k] = make_float3(a[5 + 3 * k], a[6 + 3 * k], a[7 + 3 * k]);
                ns[k] = make_float3(a[41 + 3 * k], a[42 + 3 * k], a[43 + 3 * k]);
            }
            float3 x = make_float3(0, 0, 0);
            bool ok = solveQEF(pts, ns, m, x);
            o[0] = ok ? 1.0f : 0.0f; o[1] = x.x; o[2] = x.y; o[3] = x.z;
        } break;
        case PR_ENCV: {
            ushort4 q = encodeCellVertexLocal(make_float3(a[0], a[1], a[2]), make_float3(a[3], a[4], a[5]), a[6]);
            o[0] = (float)q.x; o[1] = (float)q.y; o[2] = (float)q.z;
        } break;
        case PR_DECV: {
            ushort4 q; q.x = (unsigned short)a[0]; q.y = (unsigned short)a[1]; q.z = (unsigned short)a[2]; q.w = 0;
            float3 p = decodeCellVertexWorld(q, make_float3(a[3], a[4], a[5]), a[6]);
            o[0] = p.x; o[1] = p.y; o[2] = p.z;
        } break;
        case PR_ENCN: {
            short4 q = encodeCellNormal(make_float3(a[0], a[1], a[2]));
            o[0] = (float)q.x; o[1] = (float)q.y; o[2] = (float)q.z;
        } break;
        case PR_DECN: {
            short4 q; q.x = (short)a[0]; q.y = (short)a[1]; q.z = (short)a[2]; q.w = 0;
            float3 nrm = decodeCellNormal(q);
            o[0] = nrm.x; o[1] = nrm.y; o[2] = nrm.z;
        } break;
        case PR_AABBD: {
            o[0] = intersectAABB(make_float3(a[0], a[1], a[2]), make_float3(a[3], a[4], a[5]),
                                 make_float3(a[6], a[7], a[8]), a[9]) ? 1.0f : 0.0f;
        } break;
        default: break;
    }
}

}  // namespace refprobe

// Runs probe `which` over n input records (IN_STRIDE floats each, host memory) and writes n output
// records (OUT_STRIDE floats each, host memory). `grid` carries the uploaded scene for PR_MAP and
// PR_NORMAL (device pointers filled by the driver), else may be zeroed. Returns a cudaError_t value.
extern "C" int ref_probe_run(int which, int n, const float* h_in, float* h_out, const SDFGrid* grid, float time) {
    using namespace refprobe;
    if (n <= 0) return 0;
    float *d_in = nullptr, *d_out = nullptr;
    cudaError_t e = cudaMalloc(&d_in, (size_t)n * IN_STRIDE * sizeof(float));
    if (e != cudaSuccess) return (int)e;
    e = cudaMalloc(&d_out, (size_t)n * OUT_STRIDE * sizeof(float));
    if (e != cudaSuccess) { cudaFree(d_in); return (int)e; }
    cudaMemcpy(d_in, h_in, (size_t)n * IN_STRIDE * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(d_out, 0, (size_t)n * OUT_STRIDE * sizeof(float));
    SDFGrid g;
    memset(&g, 0, sizeof(g));
    if (grid) g = *grid;
    probe_kernel<<<(n + 127) / 128, 128>>>(which, n, d_in, d_out, g, time);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(h_out, d_out, (size_t)n * OUT_STRIDE * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    return (int)e;
}

extern "C" int ref_probe_strides(int* in_stride, int* out_stride) {
    *in_stride = refprobe::IN_STRIDE;
    *out_stride = refprobe::OUT_STRIDE;
    return 0;
}
