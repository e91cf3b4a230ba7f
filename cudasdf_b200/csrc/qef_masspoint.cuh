// Mass-point-centred QEF for dual contouring (no counterpart in the reference's solver).
//
// For the Hermite samples (p_i, n_i) of a cell, minimise sum_i (n_i . (x - p_i))^2 with x written as
// c + y, c the mass point (mean of the p_i). The normal equations A y = b, A = sum n n^T,
// b = sum n (n . (p_i - c)), have the eigen-decomposition A = V L V^T.
//
// Condition number and the FP32 / FP64 split. The eigenvectors come from a Jacobi sweep of the FP32 A;
// each eigenvalue is then taken as the Rayleigh quotient sum_i (v_k . n_i)^2 of the unit normals
// themselves, which is accurate to the rounding of the normals (the diagonal of a Jacobi sweep of the
// rounded A errs by about cond x 2^-24 relative). cond = l_max / l_min. Cells with cond above
// cond_threshold form and solve the equations in FP64 (a Jacobi eigensolve and the pseudo-inverse
// truncated at l_max / cond_threshold: directions the normals do not constrain stay at the mass
// point); FP64 runs on the GPU only for those cells. Every other cell is solved in FP32:
// y = sum_k v_k (v_k . r) / l_k, refined twice, where the residual r = sum_i n_i (n_i . (p_i - c - y))
// is formed from the Hermite samples and not as b - A y from the rounded A (the rounding of A would
// limit the FP32 solution to about cond x 2^-24 of its size), and summed with its rounding errors
// carried.
//
// Every FP32 operation of the decision and of the FP32 solve is rounded on its own (no contraction),
// so a float32 restatement on the host reproduces the condition number, hence the FP32 / FP64 split,
// bit for bit.
#pragma once

#include "mc_kernels.cuh"

namespace sdfb {

// a.x*b.x + a.y*b.y + a.z*b.z, each product and sum rounded on its own
__device__ __forceinline__ float dot3_rn(float3 a, float3 b) {
    return ADD(ADD(MUL(a.x, b.x), MUL(a.y, b.y)), MUL(a.z, b.z));
}

// hi + lo += a * b, the sum kept unevaluated: the product's rounding error (exact by FMA) and the
// addition's rounding error (exact by Knuth's two-sum) are both carried in lo
__device__ __forceinline__ void acc2_rn(float& hi, float& lo, float a, float b) {
    const float p = MUL(a, b);
    const float pe = FMA(a, b, -p);
    const float s = ADD(hi, p);
    const float bb = SUB(s, hi);
    const float err = ADD(SUB(hi, SUB(s, bb)), SUB(p, bb));
    hi = s;
    lo = ADD(lo, ADD(err, pe));
}

// unit normal of a Hermite sample; false (and no normal) when its length is below 1e-6
__device__ __forceinline__ bool unit_normal_rn(float3 h, float3& n) {
    const float len = SQRT(dot3_rn(h, h));
    if (len < 1e-6f) return false;
    n = f3(DIV(h.x, len), DIV(h.y, len), DIV(h.z, len));
    return true;
}

// Cyclic Jacobi eigensolve of a symmetric 3x3 in FP32, every operation rounded on its own: A ends
// (nearly) diagonal, the columns of V are the eigenvectors.
__device__ __forceinline__ void jacobi3_rn(float A[3][3], float V[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? 1.f : 0.f;
    for (int s = 0; s < 8; ++s) {
        const float off = ADD(ADD(MUL(A[0][1], A[0][1]), MUL(A[0][2], A[0][2])), MUL(A[1][2], A[1][2]));
        const float dg = ADD(ADD(MUL(A[0][0], A[0][0]), MUL(A[1][1], A[1][1])), MUL(A[2][2], A[2][2]));
        if (off <= MUL(dg, 1e-30f) || off == 0.f) break;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            const float apq = A[p][q];
            if (apq == 0.f) continue;
            const float theta = DIV(SUB(A[q][q], A[p][p]), MUL(2.f, apq));
            const float t = DIV(theta >= 0.f ? 1.f : -1.f, ADD(fabsf(theta), SQRT(ADD(MUL(theta, theta), 1.f))));
            const float c = DIV(1.f, SQRT(ADD(MUL(t, t), 1.f)));
            const float sn = MUL(t, c);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float akp = A[k][p], akq = A[k][q];
                A[k][p] = SUB(MUL(c, akp), MUL(sn, akq));
                A[k][q] = ADD(MUL(sn, akp), MUL(c, akq));
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float apk = A[p][k], aqk = A[q][k];
                A[p][k] = SUB(MUL(c, apk), MUL(sn, aqk));
                A[q][k] = ADD(MUL(sn, apk), MUL(c, aqk));
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float vkp = V[k][p], vkq = V[k][q];
                V[k][p] = SUB(MUL(c, vkp), MUL(sn, vkq));
                V[k][q] = ADD(MUL(sn, vkp), MUL(c, vkq));
            }
        }
    }
}

// FP64 Jacobi eigensolve for the ill-conditioned cells
__device__ __forceinline__ void jacobi3_f64(double A[3][3], double V[3][3], int sweeps) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
    for (int s = 0; s < sweeps; ++s) {
        const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        const double diag = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (off <= diag * 1e-30 || off == 0.0) break;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            const double apq = A[p][q];
            if (apq == 0.0) continue;
            const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
            const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            const double c = 1.0 / sqrt(t * t + 1.0);
            const double sn = t * c;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double akp = A[k][p], akq = A[k][q];
                A[k][p] = c * akp - sn * akq;
                A[k][q] = sn * akp + c * akq;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double apk = A[p][k], aqk = A[q][k];
                A[p][k] = c * apk - sn * aqk;
                A[q][k] = sn * apk + c * aqk;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - sn * vkq;
                V[k][q] = sn * vkp + c * vkq;
            }
        }
    }
}

// The mass-point solve for one cell; returns the unclamped vertex. *used_fp64 reports the branch.
// The Hermite points are taken relative to the cell's corner, so the mass point and the offsets
// p_i - c keep the precision of cell-sized differences.
__device__ float3 solve_masspoint(const GridView& g, const CellInfo& c, const float cv[8],
                                  const float3* __restrict__ hn, const unsigned short* __restrict__ hcell, int m,
                                  float cond_threshold, int* used_fp64 = nullptr) {
    const float3 cmin = grid_loc(g, c.x, c.y, c.z);
    if (used_fp64) *used_fp64 = 0;
    if (m <= 0) return f3(FMA(0.5f, g.cell, cmin.x), FMA(0.5f, g.cell, cmin.y), FMA(0.5f, g.cell, cmin.z));
    float3 sum = f3(0.f, 0.f, 0.f);
    for (int i = 0; i < m; ++i) sum = add3(sum, sub3(edge_point(g, c.x, c.y, c.z, cv, hcell[i] & 15), cmin));
    const float3 mq = scl3(sum, DIV(1.f, (float)m));  // mass point relative to the corner
    // normal equations in FP32, for the eigenvectors
    float A[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
    for (int i = 0; i < m; ++i) {
        float3 n;
        if (!unit_normal_rn(hn[i], n)) continue;
        const float nn[3] = {n.x, n.y, n.z};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) A[r][k] = ADD(A[r][k], MUL(nn[r], nn[k]));
    }
    float V[3][3];
    jacobi3_rn(A, V);
    // eigenvalues: Rayleigh quotients of the unit normals
    float lam[3];
    float3 vk[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        vk[k] = f3(V[0][k], V[1][k], V[2][k]);
        float l = 0.f;
        for (int i = 0; i < m; ++i) {
            float3 n;
            if (!unit_normal_rn(hn[i], n)) continue;
            const float d = dot3_rn(vk[k], n);
            l = ADD(l, MUL(d, d));
        }
        lam[k] = l;
    }
    const float lmax = fmaxf(fmaxf(lam[0], lam[1]), lam[2]), lmin = fminf(fminf(lam[0], lam[1]), lam[2]);
    const bool fp64 = !(MUL(lmin, cond_threshold) >= lmax);  // cond = lmax / lmin > cond_threshold
    if (!fp64) {
        // FP32: y = sum_k v_k (v_k . r) / l_k, r from the Hermite samples, three passes; r is summed with
        // its rounding errors carried (acc2_rn): near the solution its terms cancel, and an error left
        // in r along the weakest direction grows by cond in y
        float3 y = f3(0.f, 0.f, 0.f);
        for (int pass = 0; pass < 3; ++pass) {
            float3 rh = f3(0.f, 0.f, 0.f), rl = f3(0.f, 0.f, 0.f);
            for (int i = 0; i < m; ++i) {
                float3 n;
                if (!unit_normal_rn(hn[i], n)) continue;
                const float3 q = sub3(edge_point(g, c.x, c.y, c.z, cv, hcell[i] & 15), cmin);
                const float e = dot3_rn(n, sub3(sub3(q, mq), y));
                acc2_rn(rh.x, rl.x, n.x, e);
                acc2_rn(rh.y, rl.y, n.y, e);
                acc2_rn(rh.z, rl.z, n.z, e);
            }
            const float3 r = add3(rh, rl);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (!(lam[k] > 0.f)) continue;
                y = add3(y, scl3(vk[k], DIV(dot3_rn(vk[k], r), lam[k])));
            }
        }
        return f3(ADD(cmin.x, ADD(mq.x, y.x)), ADD(cmin.y, ADD(mq.y, y.y)), ADD(cmin.z, ADD(mq.z, y.z)));
    }
    if (used_fp64) *used_fp64 = 1;
    // FP64: the equations from the FP32 Hermite data again, eigensolve, truncated pseudo-inverse
    double qd[12][3], sd[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < m; ++i) {
        const float3 q = sub3(edge_point(g, c.x, c.y, c.z, cv, hcell[i] & 15), cmin);
        qd[i][0] = q.x; qd[i][1] = q.y; qd[i][2] = q.z;
        sd[0] += q.x; sd[1] += q.y; sd[2] += q.z;
    }
    const double md[3] = {sd[0] / m, sd[1] / m, sd[2] / m};
    double Ad[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, bd[3] = {0, 0, 0};
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
    double Vd[3][3];
    jacobi3_f64(Ad, Vd, 24);
    const double l0 = Ad[0][0], l1 = Ad[1][1], l2 = Ad[2][2];
    const double lmaxd = fmax(fmax(fabs(l0), fabs(l1)), fabs(l2));
    double yd[3] = {0.0, 0.0, 0.0};
    if (lmaxd > 0.0) {
        const double lcut = lmaxd / (double)cond_threshold;
        const double ld[3] = {l0, l1, l2};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (!(ld[k] >= lcut)) continue;
            const double proj = (Vd[0][k] * bd[0] + Vd[1][k] * bd[1] + Vd[2][k] * bd[2]) / ld[k];
            yd[0] += Vd[0][k] * proj;
            yd[1] += Vd[1][k] * proj;
            yd[2] += Vd[2][k] * proj;
        }
    }
    return f3((float)((double)cmin.x + (md[0] + yd[0])), (float)((double)cmin.y + (md[1] + yd[1])),
              (float)((double)cmin.z + (md[2] + yd[2])));
}

}  // namespace sdfb
