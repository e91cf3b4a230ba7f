"""The FP64 mass-point QEF restatement on Hermite data with known answers."""
import numpy as np

from oracle import qef_oracle as Q


def test_three_planes_meet_at_their_corner():
    corner = np.array([0.3, 0.6, 0.45])
    pts, nrm = [], []
    rng = np.random.default_rng(0)
    for axis in range(3):
        for _ in range(2):
            p = corner + rng.uniform(-0.2, 0.2, 3)
            p[axis] = corner[axis]
            n = np.zeros(3)
            n[axis] = 1.0
            pts.append(p)
            nrm.append(n * 2.5)  # normals need not be unit length
    x, cond = Q.masspoint_solve(pts, nrm)
    assert np.abs(x - corner).max() < 1e-12 and cond < 10


def test_single_plane_projects_the_mass_point():
    pts = np.array([[0.1, 0.2, 0.5], [0.9, 0.3, 0.5], [0.4, 0.8, 0.5], [0.6, 0.6, 0.5]])
    nrm = np.tile([0.0, 0.0, 1.0], (4, 1))
    x, cond = Q.masspoint_solve(pts, nrm)
    # the unconstrained directions stay at the mass point; the plane fixes z
    assert np.allclose(x, [0.5, 0.475, 0.5]) and cond == np.inf


def test_truncation_drops_weak_directions():
    # two nearly parallel planes: the weak direction is below lmax / 1e4 and is dropped
    eps = 1e-3
    pts = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    nrm = np.array([[1.0, 0.0, 0.0], [1.0, eps, 0.0]])
    x_trunc, cond = Q.masspoint_solve(pts, nrm, cond_threshold=1e4)
    assert cond == np.inf
    assert abs(x_trunc[1]) < 1e-9  # y stays at the mass point


def test_crossing_edges_and_finish():
    cv = np.array([-1, 1, 1, -1, -1, 1, 1, -1], np.float32)  # the plane x = 0.5
    assert Q.crossing_edges(cv) == [0, 2, 4, 6]
    x = Q.finish(np.array([1.5, 0.5, -0.2]), [1.0, 0.0, 0.0], 0.25)
    assert np.allclose(x, [1.25, 0.25, 0.0])
    assert np.allclose(Q.finish(np.array([1.1, 0.1, 0.1]), [1.0, 0.0, 0.0], 0.25, qef_blend=0.0), [1.125, 0.125, 0.125])


def _random_cells(rng, nc=4000, cell=0.05):
    """Hermite data of cells crossed by one to three random planes: points on the planes inside the
    cell, normals of the planes with a little noise; some cells nearly degenerate (planes almost
    parallel), so condition numbers spread over many decades."""
    P = np.zeros((nc, 12, 3), np.float32)
    N = np.zeros((nc, 12, 3), np.float32)
    m = rng.integers(3, 13, nc)
    cmin = (rng.uniform(-1, 1, (nc, 3)) // cell * cell).astype(np.float32)
    for c in range(nc):
        k = 3 if rng.random() < 0.8 else rng.integers(1, 3)
        base = rng.standard_normal(3)
        normals = [base / np.linalg.norm(base)]
        spread = 10.0 ** rng.uniform(-2.5, 0.3)
        for _ in range(k - 1):
            t = normals[0] + rng.standard_normal(3) * spread
            normals.append(t / np.linalg.norm(t))
        corner = rng.uniform(0.2, 0.8, 3) * cell
        for i in range(m[c]):
            n = normals[i % k]
            q = rng.uniform(0, cell, 3)
            q -= n * (n @ (q - corner))  # onto the plane through the feature point
            P[c, i] = np.clip(q, 0, cell)
            N[c, i] = n + rng.standard_normal(3) * 1e-3
    return P, N, m, cmin, cell


def test_batched_solve_matches_the_single_cell_solve():
    rng = np.random.default_rng(3)
    P, N, m, cmin, cell = _random_cells(rng, 300)
    xb, cb = Q.masspoint_solve_batch(P, N, m, cmin)
    for c in range(len(m)):
        x, cond = Q.masspoint_solve(P[c, :m[c]].astype(np.float64), N[c, :m[c]])
        assert np.abs(x + cmin[c] - xb[c]).max() < 1e-9 * cell or not np.isfinite(cond)
        assert np.isclose(cond, cb[c], rtol=1e-6) or (np.isinf(cond) and cb[c] > 1e12)


def test_fp32_restatement_splits_by_condition_and_solves_within_tolerance():
    """The float32 restatement of the library's solve: cells it keeps in FP32 are within 1e-4 cell of
    the FP64 solution, and its FP32/FP64 split agrees with the FP64 condition number except within a
    hair of the threshold."""
    rng = np.random.default_rng(5)
    P, N, m, cmin, cell = _random_cells(rng)
    fp64, x32, lam = Q.fp32_split_and_solve(P, N, m, cmin, 1e4)
    x64, cond = Q.masspoint_solve_batch(P, N, m, cmin, 1e4)
    assert 0.1 < fp64.mean() < 0.9  # both branches are exercised
    err = np.abs(x32.astype(np.float64) - x64).max(1) / cell
    assert err[~fp64].max() < 1e-4, err[~fp64].max()
    disagree = fp64 != (cond > 1e4)
    assert np.all(np.abs(cond[disagree] / 1e4 - 1) < 1e-4), cond[disagree]


def test_fp32_jacobi_restatement_diagonalises():
    rng = np.random.default_rng(9)
    B = rng.standard_normal((500, 3, 3)).astype(np.float32)
    A = (B @ np.transpose(B, (0, 2, 1))).astype(np.float32)
    D, V = Q._jacobi3_rn(A)
    off = np.abs(D[:, [0, 0, 1], [1, 2, 2]]).max(1)
    assert (off <= 1e-5 * np.abs(D).max((1, 2))).all()
    R = np.einsum("nij,njk,nlk->nil", V.astype(np.float64), D.astype(np.float64), V.astype(np.float64))
    assert np.abs(R - A).max() < 1e-4 * np.abs(A).max()


def test_projection_restatements_agree_on_a_smooth_field():
    """FP64 and float32 forms of the projection steps move vertices near a sphere onto it alike."""
    rng = np.random.default_rng(11)
    nc, cell, r = 2000, np.float32(0.02), 0.6
    d = rng.standard_normal((nc, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    surf = d * r
    cmin = (np.floor(surf / cell) * cell).astype(np.float32)
    x0 = (surf + rng.uniform(-0.3, 0.3, (nc, 3)) * cell).astype(np.float32)
    N = np.zeros((nc, 12, 3), np.float32)
    N[:, :4] = (d[:, None, :] + rng.standard_normal((nc, 4, 3)) * 0.01).astype(np.float32)
    m = np.full(nc, 4)

    def sphere(p):
        return (np.sqrt((np.asarray(p, np.float64) ** 2).sum(1)) - r).astype(np.float32)

    nb, has = Q.mean_normals_f32(N, m)
    assert has.all()
    x32 = Q.project_f32(x0, cmin, cell, nb, has, sphere, 3)
    x64 = Q.project_batch(x0, cmin, cell, N, m, sphere, 3)
    assert np.abs(x32 - x64).max() < 1e-5 * cell
    inside = (x64 > cmin - 0.1 * cell + 1e-9).all(1) & (x64 < cmin + 1.1 * cell - 1e-9).all(1)
    assert np.median(np.abs(sphere(x64[inside]))) < 0.05 * np.median(np.abs(sphere(x0[inside])))


def test_finish_encode_and_padding():
    cmin = np.array([[0.0, 0.5, -1.0]], np.float32)
    q = Q.finish_encode_f32(np.array([[0.025, 0.49, -0.99]], np.float32), cmin, 0.05)
    assert q.tolist() == [[32768, 0, 13107]]  # 0.5 -> 32767.5 rounds to even
    starts = np.array([0, 2, 2, 5])
    rows = np.arange(15, dtype=np.float32).reshape(5, 3)
    p = Q.pad_hermite(rows, starts)
    assert p.shape == (3, 12, 3) and (p[0, :2] == rows[:2]).all() and (p[1] == 0).all() and (p[2, :3] == rows[2:]).all()
