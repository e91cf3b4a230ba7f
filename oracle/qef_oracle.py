"""FP64 restatement of the mass-point QEF for dual contouring (test infrastructure only: the tests use it
as the checker of the library's mass-point solver; nothing in the library calls it).

The solver has no counterpart in the reference. For the Hermite samples (p_i, n_i) of a surface cell
(edge crossings and the gradient there, as the reference's dcSolveCellVertices gathers them,
MarchingCubesKernels.cu:1383-1411), the vertex minimises sum_i (n_i . (x - p_i))^2 with x = c + y,
c the mass point (mean of the p_i): the normal equations A y = b, A = sum n n^T,
b = sum n (n . (p_i - c)), solved by a symmetric eigendecomposition with the eigen-directions whose
eigenvalue is below lmax / cond_threshold dropped (pseudo-inverse truncation; those directions stay at
the mass point). Optional projection steps x <- x - f(x) grad f(x) move the vertex onto the surface,
each kept in the cell's box widened by 0.1 cell; the result is clamped to the cell and blended towards
the cell centre with qef_blend (MarchingCubesKernels.cu:1556-1577).
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


def project(x, cmin, cell, value_gradient, iters):
    """iters steps x <- x - f(x) grad f(x), each clamped to the cell widened by 0.1 cell;
    value_gradient(x) returns (f, unit gradient) at one point."""
    cmin = np.asarray(cmin, np.float64)
    for _ in range(iters):
        f, g = value_gradient(x)
        if not np.isfinite(f):
            continue
        x = np.clip(x - f * np.asarray(g, np.float64), cmin - 0.1 * cell, cmin + cell + 0.1 * cell)
    return x
