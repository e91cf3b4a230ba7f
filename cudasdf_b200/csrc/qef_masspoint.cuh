// Mass-point-centred QEF for dual contouring (no counterpart in the reference's solver).
//
// For the Hermite samples (p_i, n_i) of a cell, minimise sum_i (n_i . (x - p_i))^2 with x written
// as c + y, c the mass point (mean of the p_i). The normal equations A y = b, A = sum n n^T,
// b = sum n (n . (p_i - c)), are formed in FP32. A symmetric Jacobi eigensolve gives A = V L V^T;
// y = sum_k v_k (v_k . b) / l_k over the eigenvalues l_k >= l_max / cond_threshold (pseudo-inverse
// truncation: directions the normals do not constrain stay at the mass point). Cells whose condition
// number l_max / l_min is above cond_threshold / 16 are solved in FP64 (FP64 on the GPU only for
// those cells).
#pragma once

#include "mc_kernels.cuh"

namespace sdfb {

template <class T>
__device__ __forceinline__ void jacobi3(T A[3][3], T V[3][3], int sweeps) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? T(1) : T(0);
    for (int s = 0; s < sweeps; ++s) {
        const T off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        const T diag = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (off <= diag * T(1e-30) || off == T(0)) break;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            const T apq = A[p][q];
            if (apq == T(0)) continue;
            const T theta = (A[q][q] - A[p][p]) / (T(2) * apq);
            const T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
            const T c = T(1) / sqrt(t * t + T(1));
            const T sn = t * c;
            // A <- J^T A J for the rotation in the (p, q) plane
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const T akp = A[k][p], akq = A[k][q];
                A[k][p] = c * akp - sn * akq;
                A[k][q] = sn * akp + c * akq;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const T apk = A[p][k], aqk = A[q][k];
                A[p][k] = c * apk - sn * aqk;
                A[q][k] = sn * apk + c * aqk;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const T vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - sn * vkq;
                V[k][q] = sn * vkp + c * vkq;
            }
        }
    }
}

template <class T>
__device__ __forceinline__ void pinv_solve(T A[3][3], const T b[3], T cond_threshold, int sweeps, T y[3]) {
    T V[3][3];
    jacobi3<T>(A, V, sweeps);
    const T l0 = A[0][0], l1 = A[1][1], l2 = A[2][2];
    const T lmax = fmax(fmax(fabs(l0), fabs(l1)), fabs(l2));
    y[0] = y[1] = y[2] = T(0);
    if (!(lmax > T(0))) return;
    const T lcut = lmax / cond_threshold;
    const T lam[3] = {l0, l1, l2};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (!(lam[k] >= lcut)) continue;
        const T proj = (V[0][k] * b[0] + V[1][k] * b[1] + V[2][k] * b[2]) / lam[k];
        y[0] += V[0][k] * proj;
        y[1] += V[1][k] * proj;
        y[2] += V[2][k] * proj;
    }
}

// The mass-point solve for one cell; returns the unclamped vertex. *used_fp64 reports the branch.
// The Hermite points are taken relative to the cell's corner (an exact subtraction for points of the
// cell, Sterbenz's lemma), so the mass point and the offsets p_i - c keep the full precision of the
// cell-sized differences. A backward-stable FP32 solve has a forward error of about
// cond * 2^-24 relative, so the FP32 branch (with one step of iterative refinement) takes the cells
// with cond <= cond_threshold / 16 (error below 4e-5 of the vertex offset); every other cell forms
// the normal equations from the Hermite data again in FP64 and solves them with the FP64 Jacobi
// eigensolve and the pseudo-inverse truncated at lmax / cond_threshold.
__device__ float3 solve_masspoint(const GridView& g, const CellInfo& c, const float cv[8],
                                  const float3* __restrict__ hn, const unsigned short* __restrict__ hcell, int m,
                                  float cond_threshold, int* used_fp64 = nullptr) {
    const float3 cmin = grid_loc(g, c.x, c.y, c.z);
    if (m <= 0) return f3(FMA(0.5f, g.cell, cmin.x), FMA(0.5f, g.cell, cmin.y), FMA(0.5f, g.cell, cmin.z));
    float3 sum = f3(0.f, 0.f, 0.f);
    for (int i = 0; i < m; ++i) sum = add3(sum, sub3(edge_point(g, c.x, c.y, c.z, cv, hcell[i] & 15), cmin));
    const float3 mq = scl3(sum, 1.f / (float)m);  // mass point relative to the corner
    float A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, b[3] = {0, 0, 0};
    for (int i = 0; i < m; ++i) {
        float3 n = hn[i];
        const float len = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
        if (len < 1e-6f) continue;
        n = f3(n.x / len, n.y / len, n.z / len);
        const float3 q = sub3(edge_point(g, c.x, c.y, c.z, cv, hcell[i] & 15), cmin);
        const float d = n.x * (q.x - mq.x) + n.y * (q.y - mq.y) + n.z * (q.z - mq.z);
        const float nn[3] = {n.x, n.y, n.z};
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int k = 0; k < 3; ++k) A[r][k] += nn[r] * nn[k];
            b[r] += nn[r] * d;
        }
    }
    // FP32 eigensolve; condition number from its eigenvalues
    float Af[3][3], Vf[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) Af[r][k] = A[r][k];
    jacobi3<float>(Af, Vf, 8);
    const float l0 = fabsf(Af[0][0]), l1 = fabsf(Af[1][1]), l2 = fabsf(Af[2][2]);
    const float lmax = fmaxf(fmaxf(l0, l1), l2), lmin = fminf(fminf(l0, l1), l2);
    const bool fp64 = !(lmin * (cond_threshold * 0.0625f) >= lmax);
    if (used_fp64) *used_fp64 = fp64 ? 1 : 0;
    if (!fp64) {
        const float lam[3] = {Af[0][0], Af[1][1], Af[2][2]};
        float y[3] = {0.f, 0.f, 0.f};
        // y = A^-1 b, then y += A^-1 (b - A y)
        for (int pass = 0; pass < 2; ++pass) {
            float r[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) r[k] = b[k] - (A[k][0] * y[0] + A[k][1] * y[1] + A[k][2] * y[2]);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float proj = (Vf[0][k] * r[0] + Vf[1][k] * r[1] + Vf[2][k] * r[2]) / lam[k];
                y[0] += Vf[0][k] * proj;
                y[1] += Vf[1][k] * proj;
                y[2] += Vf[2][k] * proj;
            }
        }
        return f3(cmin.x + (mq.x + y[0]), cmin.y + (mq.y + y[1]), cmin.z + (mq.z + y[2]));
    }
    // FP64: the same equations from the FP32 Hermite data
    double qd[12][3], sd[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < m; ++i) {
        const float3 q = sub3(edge_point(g, c.x, c.y, c.z, cv, hcell[i] & 15), cmin);
        qd[i][0] = q.x; qd[i][1] = q.y; qd[i][2] = q.z;
        sd[0] += q.x; sd[1] += q.y; sd[2] += q.z;
    }
    const double md[3] = {sd[0] / m, sd[1] / m, sd[2] / m};
    double Ad[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, bd[3] = {0, 0, 0}, yd[3];
    for (int i = 0; i < m; ++i) {
        const double nx = hn[i].x, ny = hn[i].y, nz = hn[i].z;
        const double len = sqrt(nx * nx + ny * ny + nz * nz);
        if (len < 1e-6) continue;
        const double nn[3] = {nx / len, ny / len, nz / len};
        const double d = nn[0] * (qd[i][0] - md[0]) + nn[1] * (qd[i][1] - md[1]) + nn[2] * (qd[i][2] - md[2]);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int k = 0; k < 3; ++k) Ad[r][k] += nn[r] * nn[k];
            bd[r] += nn[r] * d;
        }
    }
    pinv_solve<double>(Ad, bd, (double)cond_threshold, 24, yd);
    return f3((float)((double)cmin.x + (md[0] + yd[0])), (float)((double)cmin.y + (md[1] + yd[1])),
              (float)((double)cmin.z + (md[2] + yd[2])));
}

}  // namespace sdfb
