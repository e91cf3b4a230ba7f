// Mass-point-centred QEF for dual contouring (no counterpart in the reference's solver).
//
// For the Hermite samples (p_i, n_i) of a cell, minimise sum_i (n_i . (x - p_i))^2 with x written
// as c + y, c the mass point (mean of the p_i). The normal equations A y = b, A = sum n n^T,
// b = sum n (n . (p_i - c)), are formed in FP32. A symmetric Jacobi eigensolve gives A = V L V^T;
// y = sum_k v_k (v_k . b) / l_k over the eigenvalues l_k >= l_max / cond_threshold (pseudo-inverse
// truncation: directions the normals do not constrain stay at the mass point). When the condition
// number l_max / l_min exceeds cond_threshold, the eigensolve is repeated in FP64 (FP64 on the GPU
// only for those cells) before the truncated solve.
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
__device__ float3 solve_masspoint(const GridView& g, const CellInfo& c, const float cv[8],
                                  const float3* __restrict__ hn, const unsigned short* __restrict__ hcell, int m,
                                  float cond_threshold, int* used_fp64 = nullptr) {
    const float3 cmin = grid_loc(g, c.x, c.y, c.z);
    float3 mp = f3(FMA(0.5f, g.cell, cmin.x), FMA(0.5f, g.cell, cmin.y), FMA(0.5f, g.cell, cmin.z));
    if (m <= 0) return mp;
    float3 sum = f3(0.f, 0.f, 0.f);
    for (int i = 0; i < m; ++i) sum = add3(sum, edge_point(g, c.x, c.y, c.z, cv, hcell[i] & 15));
    mp = scl3(sum, 1.f / (float)m);
    float A[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, b[3] = {0, 0, 0};
    for (int i = 0; i < m; ++i) {
        float3 n = hn[i];
        const float len = sqrtf(n.x * n.x + n.y * n.y + n.z * n.z);
        if (len < 1e-6f) continue;
        n = f3(n.x / len, n.y / len, n.z / len);
        const float3 p = edge_point(g, c.x, c.y, c.z, cv, hcell[i] & 15);
        const float d = n.x * (p.x - mp.x) + n.y * (p.y - mp.y) + n.z * (p.z - mp.z);
        const float nn[3] = {n.x, n.y, n.z};
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int q = 0; q < 3; ++q) A[r][q] += nn[r] * nn[q];
            b[r] += nn[r] * d;
        }
    }
    // FP32 eigensolve; condition number from its eigenvalues
    float Af[3][3], y[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int q = 0; q < 3; ++q) Af[r][q] = A[r][q];
    float Vf[3][3];
    jacobi3<float>(Af, Vf, 8);
    const float l0 = fabsf(Af[0][0]), l1 = fabsf(Af[1][1]), l2 = fabsf(Af[2][2]);
    const float lmax = fmaxf(fmaxf(l0, l1), l2), lmin = fminf(fminf(l0, l1), l2);
    const bool ill = !(lmin * cond_threshold >= lmax);
    if (!ill) {
        y[0] = y[1] = y[2] = 0.f;
        const float lam[3] = {Af[0][0], Af[1][1], Af[2][2]};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float proj = (Vf[0][k] * b[0] + Vf[1][k] * b[1] + Vf[2][k] * b[2]) / lam[k];
            y[0] += Vf[0][k] * proj;
            y[1] += Vf[1][k] * proj;
            y[2] += Vf[2][k] * proj;
        }
    } else {
        double Ad[3][3], bd[3] = {(double)b[0], (double)b[1], (double)b[2]}, yd[3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int q = 0; q < 3; ++q) Ad[r][q] = (double)A[r][q];
        pinv_solve<double>(Ad, bd, (double)cond_threshold, 24, yd);
        y[0] = (float)yd[0];
        y[1] = (float)yd[1];
        y[2] = (float)yd[2];
    }
    if (used_fp64) *used_fp64 = ill ? 1 : 0;
    return f3(mp.x + y[0], mp.y + y[1], mp.z + y[2]);
}

}  // namespace sdfb
