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
