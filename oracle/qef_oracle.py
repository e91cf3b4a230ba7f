"""FP64 restatement of the mass-point QEF for dual contouring (test infrastructure only: the tests use it
as the checker of the library's mass-point solver; nothing in the library calls it).

The solver has no counterpart in the reference. For the Hermite samples (p_i, n_i) of a surface cell
(edge crossings and the gradient there, as the reference's dcSolveCellVertices gathers them,
MarchingCubesKernels.cu:1383-1411), the vertex minimises sum_i (n_i . (x - p_i))^2 with x = c + y,
c the mass point (mean of the p_i): the normal equations A y = b, A = sum n n^T,
b = sum n (n . (p_i - c)), solved by a symmetric eigendecomposition with the eigen-directions whose
eigenvalue is below lmax / cond_threshold dropped (pseudo-inverse truncation; those directions stay at
the mass point). Optional projection steps x <- x - f(x) n move the vertex onto the surface along the
cell's mean Hermite normal n, each kept in the cell's box widened by 0.1 cell; the result is clamped to
the cell and blended towards the cell centre with qef_blend (MarchingCubesKernels.cu:1556-1577).

Two kinds of checker live here: FP64 solutions (masspoint_solve, masspoint_solve_batch, project_batch,
finish_batch), the numerical reference, and float32 restatements of the library's own operation order
(fp32_split_and_solve, mean_normals_f32, project_f32, finish_encode_f32, diagonal_lengths_f32), which
reproduce its FP32 / FP64 split and its FP32 results bit for bit.
"""
from __future__ import annotations

import numpy as np

# corner offsets and edge endpoints of the marching-cubes conventions (MarchingCubesTables.cuh:8-17)
CORNERS = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)])
EDGES = np.array([(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)])


def crossing_edges(cv):
    """Edges of a cell whose corner values change sign (d > 0 against d <= 0), in edge order."""
    inside = np.asarray(cv) > 0
    return [e for e in range(12) if inside[EDGES[e, 0]] != inside[EDGES[e, 1]]]


def masspoint_solve(points, normals, cond_threshold=1e4):
    """The mass-point QEF in FP64: returns (vertex, condition number of A)."""
    p = np.asarray(points, np.float64)
    c = p.mean(axis=0)
    A = np.zeros((3, 3))
    b = np.zeros(3)
    for pi, ni in zip(p, np.asarray(normals, np.float64)):
        ln = np.sqrt(ni @ ni)
        if ln < 1e-6:
            continue
        n = ni / ln
        A += np.outer(n, n)
        b += n * (n @ (pi - c))
    w, V = np.linalg.eigh(A)
    lmax = np.abs(w).max()
    if not lmax > 0:
        return c, np.inf
    lmin = np.abs(w).min()
    y = np.zeros(3)
    for k in range(3):
        if w[k] >= lmax / cond_threshold:
            y += V[:, k] * (V[:, k] @ b) / w[k]
    return c + y, (lmax / lmin if lmin > 0 else np.inf)


def finish(x, cmin, cell, qef_blend=1.0):
    """Soft clamp (0.1 cell), hard clamp to the cell, blend towards the centre."""
    cmin = np.asarray(cmin, np.float64)
    x = np.clip(x, cmin - 0.1 * cell, cmin + cell + 0.1 * cell)
    x = np.clip(x, cmin, cmin + cell)
    ctr = cmin + 0.5 * cell
    return ctr * (1.0 - qef_blend) + x * qef_blend


# ------------------------------------------------------------------------------------------------
# Batched forms over many cells. A cell's Hermite samples are padded to 12 (a cell has at most 12
# crossing edges): points P (nc, 12, 3) relative to the cell corner, normals N (nc, 12, 3), counts m.
# ------------------------------------------------------------------------------------------------

F32 = np.float32


def pad_hermite(values: np.ndarray, starts: np.ndarray, width: int = 12) -> np.ndarray:
    """(nc, width, k) array of the per-cell rows values[starts[c]:starts[c+1]], zero padded."""
    nc = len(starts) - 1
    cnt = np.diff(starts)
    out = np.zeros((nc, width) + values.shape[1:], values.dtype)
    slot = np.arange(len(values)) - np.repeat(starts[:-1], cnt)
    out[np.repeat(np.arange(nc), cnt), slot] = values
    return out


def _dot_rn(a, b):
    """(a.x*b.x + a.y*b.y) + a.z*b.z in float32, each operation rounded on its own."""
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def _unit_normals_rn(N, m):
    """float32 unit normals and the mask of samples that enter the equations (|n| >= 1e-6, i < m)."""
    ln = np.sqrt(_dot_rn(N, N))
    ok = (np.arange(N.shape[1])[None, :] < m[:, None]) & ~(ln < F32(1e-6))
    safe = np.where(ok, ln, F32(1))
    n = np.where(ok[..., None], N / safe[..., None], F32(0)).astype(F32)
    return n, ok


def _jacobi3_rn(A):
    """Cyclic Jacobi of symmetric 3x3 matrices in float32, every operation rounded on its own, with the
    per-matrix early exit and skipped zero pivots of the library's FP32 sweep (qef_masspoint.cuh)."""
    A = A.astype(F32).copy()
    nc = A.shape[0]
    V = np.tile(np.eye(3, dtype=F32), (nc, 1, 1))
    active = np.ones(nc, bool)
    one, two = F32(1), F32(2)
    with np.errstate(all="ignore"):
        for _ in range(8):
            off = (A[:, 0, 1] * A[:, 0, 1] + A[:, 0, 2] * A[:, 0, 2]) + A[:, 1, 2] * A[:, 1, 2]
            dg = (A[:, 0, 0] * A[:, 0, 0] + A[:, 1, 1] * A[:, 1, 1]) + A[:, 2, 2] * A[:, 2, 2]
            active &= ~((off <= dg * F32(1e-30)) | (off == 0))
            if not active.any():
                break
            for p, q in ((0, 1), (0, 2), (1, 2)):
                apq = A[:, p, q]
                doit = active & (apq != 0)
                theta = (A[:, q, q] - A[:, p, p]) / (two * np.where(doit, apq, one))
                t = np.where(theta >= 0, one, -one) / (np.abs(theta) + np.sqrt(theta * theta + one))
                c = one / np.sqrt(t * t + one)
                sn = t * c
                c, sn, d = c[:, None], sn[:, None], doit[:, None]
                kp, kq = A[:, :, p].copy(), A[:, :, q].copy()
                A[:, :, p] = np.where(d, c * kp - sn * kq, kp)
                A[:, :, q] = np.where(d, sn * kp + c * kq, kq)
                pk, qk = A[:, p, :].copy(), A[:, q, :].copy()
                A[:, p, :] = np.where(d, c * pk - sn * qk, pk)
                A[:, q, :] = np.where(d, sn * pk + c * qk, qk)
                vp, vq = V[:, :, p].copy(), V[:, :, q].copy()
                V[:, :, p] = np.where(d, c * vp - sn * vq, vp)
                V[:, :, q] = np.where(d, sn * vp + c * vq, vq)
    return A, V


def fp32_split_and_solve(P, N, m, cmin, cond_threshold=1e4):
    """Float32 restatement, operation for operation, of the library's mass-point solve up to its FP32 /
    FP64 decision and of its FP32 branch (cudasdf_b200/csrc/qef_masspoint.cuh, solve_masspoint): mass
    point, unit normals, FP32 normal equations, Jacobi eigenvectors, eigenvalues as Rayleigh quotients
    of the unit normals, cond > cond_threshold -> FP64, and for the other cells three passes of
    y += sum_k v_k (v_k . r) / l_k with r = sum_i n_i (n_i . ((p_i - c) - y)), summed with its rounding
    errors carried (the kernel's acc2_rn).

    P: float32 Hermite points minus the cell corner (nc, 12, 3); N: float32 normals as the kernel holds
    them; m: sample counts; cmin: float32 cell corners (nc, 3). Returns (fp64 mask, float32 vertices of
    the FP32 cells (garbage elsewhere), float32 eigenvalue estimates (nc, 3))."""
    P = np.asarray(P, F32)
    N = np.asarray(N, F32)
    m = np.asarray(m)
    nc, width = P.shape[0], P.shape[1]
    live = np.arange(width)[None, :] < m[:, None]
    with np.errstate(all="ignore"):
        s = np.zeros((nc, 3), F32)
        for i in range(width):
            s = np.where(live[:, i, None], s + P[:, i], s)
        mq = s * (F32(1) / np.maximum(m, 1).astype(F32))[:, None]
        n, ok = _unit_normals_rn(N, m)
        A = np.zeros((nc, 3, 3), F32)
        for i in range(width):
            outer = n[:, i, :, None] * n[:, i, None, :]
            A = np.where(ok[:, i, None, None], A + outer, A)
        _, V = _jacobi3_rn(A)
        lam = np.zeros((nc, 3), F32)
        for k in range(3):
            v = V[:, :, k]
            for i in range(width):
                d = _dot_rn(v, n[:, i])
                lam[:, k] = np.where(ok[:, i], lam[:, k] + d * d, lam[:, k])
        lmax = np.fmax(np.fmax(lam[:, 0], lam[:, 1]), lam[:, 2])
        lmin = np.fmin(np.fmin(lam[:, 0], lam[:, 1]), lam[:, 2])
        fp64 = ~(lmin * F32(cond_threshold) >= lmax)
        y = np.zeros((nc, 3), F32)
        for _ in range(3):
            rh = np.zeros((nc, 3), F32)
            rl = np.zeros((nc, 3), F32)
            for i in range(width):
                e = _dot_rn(n[:, i], (P[:, i] - mq) - y)
                # acc2_rn: the product's rounding error (exact: the product of two floats is exact in
                # float64) and the two-sum error of the addition go to rl
                p = (n[:, i] * e[:, None]).astype(F32)
                pe = (n[:, i].astype(np.float64) * e[:, None].astype(np.float64) - p.astype(np.float64)).astype(F32)
                s = (rh + p).astype(F32)
                bb = (s - rh).astype(F32)
                err = ((rh - (s - bb)) + (p - bb)).astype(F32)
                upd = ok[:, i, None]
                rl = np.where(upd, (rl + (err + pe)).astype(F32), rl)
                rh = np.where(upd, s, rh)
            r = (rh + rl).astype(F32)
            for k in range(3):
                v = V[:, :, k]
                pos = lam[:, k] > 0
                proj = _dot_rn(v, r) / np.where(pos, lam[:, k], F32(1))
                y = np.where(pos[:, None], y + v * proj[:, None], y)
        x = np.asarray(cmin, F32) + (mq + y)
    return fp64, x.astype(F32), lam


def masspoint_solve_batch(P, N, m, cmin, cond_threshold=1e4):
    """The mass-point QEF of every cell in FP64 (vectorised masspoint_solve): P and N as for
    fp32_split_and_solve; returns (vertices (nc, 3) in FP64, absolute coordinates; condition numbers)."""
    P = np.asarray(P, np.float64)
    N = np.asarray(N, np.float64)
    m = np.asarray(m)
    width = P.shape[1]
    live = np.arange(width)[None, :] < m[:, None]
    c = (P * live[..., None]).sum(1) / np.maximum(m, 1)[:, None]
    ln = np.sqrt((N * N).sum(-1))
    ok = live & ~(ln < 1e-6)
    n = np.where(ok[..., None], N / np.where(ok, ln, 1.0)[..., None], 0.0)
    A = np.einsum("nij,nik->njk", n, n)
    b = np.einsum("nij,ni->nj", n, (n * (P - c[:, None, :])).sum(-1) * ok)
    w, V = np.linalg.eigh(A)
    aw = np.abs(w)
    lmax = aw.max(1)
    lmin = aw.min(1)
    with np.errstate(divide="ignore", invalid="ignore"):
        cond = np.where(lmin > 0, lmax / np.where(lmin > 0, lmin, 1.0), np.inf)
        keep = (w >= (lmax / cond_threshold)[:, None]) & (lmax > 0)[:, None]
        proj = np.where(keep, np.einsum("nik,ni->nk", V, b) / np.where(keep, w, 1.0), 0.0)
    y = np.einsum("nik,nk->ni", V, proj)
    return np.asarray(cmin, np.float64) + c + y, cond


def mean_normals_f32(N, m):
    """Float32 restatement of the projection direction of each cell (dc_kernels.cuh, k_dc_solve): the
    normalised sum, in sample order, of the unit Hermite normals (unit_normal_rn of each, then of the
    sum). Returns (directions (nc, 3) float32, has_direction mask: the sum is at least 1e-6 long)."""
    n, ok = _unit_normals_rn(np.asarray(N, F32), np.asarray(m))
    s = np.zeros((n.shape[0], 3), F32)
    for i in range(n.shape[1]):
        s = np.where(ok[:, i, None], s + n[:, i], s)
    ln = np.sqrt(_dot_rn(s, s))
    has = ~(ln < F32(1e-6))
    with np.errstate(all="ignore"):
        nb = np.where(has[:, None], s / np.where(has, ln, F32(1))[:, None], F32(0)).astype(F32)
    return nb, has


def project_f32(x0, cmin, cell, nbar, has_dir, distance, iters, trace=None):
    """Float32 restatement, operation for operation, of the mass-point projection steps of k_dc_solve:
    y = clamp(x0 - cmin, -margin, cell + margin) with margin = float32(0.1 * cell), then `iters` times
    y = clamp(y - f(cmin + y) * nbar) where f is map() at the float32 point cmin + y (skipped where f is
    not finite or the cell has no direction). Returns float32 vertices cmin + y; `trace`, a list,
    receives (points, values) of every step."""
    x0 = np.asarray(x0, F32)
    cmin = np.asarray(cmin, F32)
    c32 = F32(cell)
    margin = F32(0.1) * c32
    hi = c32 + margin
    y = np.fmax(-margin, np.fmin((x0 - cmin).astype(F32), hi))
    for _ in range(iters):
        p = (cmin + y).astype(F32)
        d = np.asarray(distance(p), F32)
        if trace is not None:
            trace.append((p, d))
        upd = has_dir & np.isfinite(d)
        yn = np.fmax(-margin, np.fmin((y - nbar * d[:, None]).astype(F32), hi))
        y = np.where(upd[:, None], yn, y)
    return (cmin + y).astype(F32)


def project_batch(x, cmin, cell, N, m, distance, iters, trace=None):
    """The mass-point projection steps in FP64 (the library's definition, k_dc_solve): the direction is
    the normalised sum of the cell's unit Hermite normals (none where the sum is shorter than 1e-6); in
    cell-local coordinates y = x - cmin, starting from x clamped to the cell widened by 0.1 cell, each
    step y <- y - f n kept in that box, f being map() at the float32 point float32(cmin + y), skipped
    where f is not finite. `distance(points float32 (k, 3)) -> float32 (k,)` evaluates the field.
    Returns the absolute FP64 vertices; `trace`, a list, receives (points, values) of every step."""
    N = np.asarray(N, np.float64)
    m = np.asarray(m)
    live = np.arange(N.shape[1])[None, :] < m[:, None]
    ln = np.sqrt((N * N).sum(-1))
    ok = live & ~(ln < 1e-6)
    s = np.where(ok[..., None], N / np.where(ok, ln, 1.0)[..., None], 0.0).sum(1)
    sl = np.sqrt((s * s).sum(1))
    has = ~(sl < 1e-6)
    nb = np.where(has[:, None], s / np.where(has, sl, 1.0)[:, None], 0.0)
    cmin64 = np.asarray(cmin, F32).astype(np.float64)
    c32 = F32(cell)
    margin = F32(0.1) * c32
    lo, hi = -float(margin), float(c32 + margin)
    y = np.clip(np.asarray(x, np.float64) - cmin64, lo, hi)
    for _ in range(iters):
        p = (cmin64 + y).astype(F32)
        d = np.asarray(distance(p), F32).astype(np.float64)
        if trace is not None:
            trace.append((p, d))
        step = np.clip(y - d[:, None] * nb, lo, hi)
        y = np.where((has & np.isfinite(d))[:, None], step, y)
    return cmin64 + y


def finish_batch(x, cmin, cell, qef_blend=1.0):
    """finish() of many cells (soft clamp, clamp to the cell, blend towards the centre)."""
    cmin = np.asarray(cmin, np.float64)
    x = np.clip(x, cmin - 0.1 * cell, cmin + 1.1 * cell)
    x = np.clip(x, cmin, cmin + cell)
    return (cmin + 0.5 * cell) * (1.0 - qef_blend) + x * qef_blend


def finish_encode_f32(x, cmin, cell):
    """Float32 restatement of the end of k_dc_solve for qef_blend = 1 (the blend is then exact): clamp to
    the cell widened by 0.1 cell, clamp to the cell, and encode_vertex's quantisation to 16 bits per axis
    (t = clamp((x - cmin) / cell, 0, 1), round-half-even of t * 65535). Returns uint16 (nc, 3)."""
    x = np.asarray(x, F32)
    cmin = np.asarray(cmin, F32)
    c32 = F32(cell)
    cmax = cmin + c32
    margin = F32(0.1) * c32
    x = np.fmax(cmin - margin, np.fmin(x, cmax + margin))
    x = np.fmax(cmin, np.fmin(x, cmax))
    t = np.fmax(F32(0), np.fmin((x - cmin) / c32, F32(1))).astype(F32)
    return np.clip(np.rint(t * F32(65535)), 0, 65535).astype(np.uint16)


def diagonal_lengths_f32(a, b):
    """Squared length of b - a as the quads kernel computes it for the adaptive diagonal: float32,
    (dx*dx + dy*dy) + dz*dz with every operation rounded on its own."""
    e = np.asarray(b, F32) - np.asarray(a, F32)
    return _dot_rn(e, e)
