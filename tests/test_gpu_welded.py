"""Indexed marching-cubes output (SDF_OUT_WELDED) against the triangle soup.

The reference writes a soup whose index buffer is the identity (CudaSDFMesh.cpp:466-469); the welded
mesh must carry the same triangles in the same order with one vertex per crossed grid edge. Checked:
the index count equals the soup's vertex count; every welded vertex is the soup vertex of each
corner that uses it, bit for bit where the cell walks the edge from its lower sample (8 of a cell's
12 edges) and within 1e-6 otherwise (the same interpolation from the other end); vertices are used
(except where the soup dropped every triangle on an edge as degenerate); and the sphere's mesh is
closed with Euler characteristic 2, which fails if two blocks create a vertex for one edge or an
edge has none.
"""
import numpy as np
import pytest

import gpu_helpers as H

pytestmark = pytest.mark.gpu


def welded_run(prims, res, bmin=(-1.0, -1.0, -1.0), bmax=(1.0, 1.0, 1.0), cell=None, debug=False, max_vertices=None,
               allow_capacity=False):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    cell = S.cell_size_for(res) if cell is None else cell
    eng = Engine()
    eng.configure(make_config(cell, bmin, bmax, out_mask=L.OUT_INDICES | L.OUT_WELDED))
    eng.set_debug(1 if debug else 0)
    eng.set_scene(prims)
    buf = MeshBuffers(max_vertices or 4_000_000, L.OUT_INDICES)
    st = eng.extract(buf, 0.0, allow_capacity=allow_capacity)
    V, U = int(st["total_vertices"]), int(st["welded_vertices"])
    r = {"stats": st, "verts": buf.vertices[:min(U, buf.max_vertices)].cpu().numpy(),
         "indices": buf.indices[:min(V, buf.max_vertices)].cpu().numpy().view(np.uint32)}
    eng.close()
    return r


def _check_against_soup(prims, res, **kw):
    from cudasdf_b200 import _lib as L
    soup = H.engine_run(prims, res, 0, L.OUT_INDICES, debug=False, **kw)
    w = welded_run(prims, res, **kw)
    V, U = int(soup["stats"]["total_vertices"]), int(w["stats"]["welded_vertices"])
    assert int(w["stats"]["total_vertices"]) == V and V > 0 and 0 < U < V
    idx = w["indices"]
    assert idx.max() < U
    used = np.unique(idx)
    # every crossed edge gets a vertex; one is left unused only where all triangles on its edge were
    # dropped by the soup's degenerate-triangle test (edges of a few ten-thousandths of a cell)
    assert U - len(used) <= max(2, U // 10000), (U - len(used))
    got = w["verts"][idx]
    assert (got[:, 3] == 1.0).all()
    d = np.abs(got[:, :3].astype(np.float64) - soup["verts"][:, :3]).max(1)
    exact = np.mean(d == 0)
    assert exact > 0.5 and d.max() <= 1e-6, (exact, d.max())
    return soup, w


def test_welded_sphere_closed_with_euler_characteristic_2():
    from cudasdf_b200 import scenes as S
    soup, w = _check_against_soup(S.sphere_scene(0.6), 128)
    tri = w["indices"].reshape(-1, 3).astype(np.int64)
    U = int(w["stats"]["welded_vertices"])
    e = np.sort(np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]]), axis=1)
    key = e[:, 0] * U + e[:, 1]
    uniq, cnt = np.unique(key, return_counts=True)
    assert (cnt == 2).all(), np.bincount(cnt)          # closed: every edge has two triangles
    assert U - len(uniq) + len(tri) == 2                 # V - E + F of a sphere
    # consistent orientation: each directed edge appears once
    d = tri[:, [0, 1, 1, 2, 2, 0]].reshape(-1, 2)
    dk = d[:, 0] * U + d[:, 1]
    assert len(np.unique(dk)) == len(dk)


@pytest.mark.parametrize("res", [64, 256])
def test_welded_matches_soup_benchmark_scene(res):
    from cudasdf_b200 import scenes as S
    _check_against_soup(S.config_scene(2), res)


def test_welded_matches_soup_odd_grid_and_bounds():
    """A grid whose size is not a multiple of the 8^3 block, bounds other than [-1, 1]^3, every
    primitive type and CSG operation but intersections."""
    from cudasdf_b200 import scenes as S
    rng = np.random.default_rng(3)
    p = S.random_scene(120, 3, size_range=(0.05, 0.3), center_range=0.7)
    p["type"] = rng.integers(0, 13, len(p))
    p["operation"] = rng.choice([0, 3, 3, 1, 4], len(p))
    p["operation"][0] = 0
    p["params"] = rng.uniform(0.2, 0.9, (len(p), 6))
    bmin, bmax = (-1.1, -1.05, -1.0), (1.1, 1.0, 1.05)
    cell = float(np.float32(2.2) / np.float32(77))
    _check_against_soup(p, 77, bmin=bmin, bmax=bmax, cell=cell)


def test_welded_with_debug_layout_and_capacity():
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    prims = S.config_scene(2)
    a = welded_run(prims, 96)
    b = welded_run(prims, 96, debug=True)
    assert a["verts"].tobytes() == b["verts"].tobytes() and a["indices"].tobytes() == b["indices"].tobytes()
    V = int(a["stats"]["total_vertices"])
    with pytest.raises(RuntimeError, match="SDF_ERR_CAPACITY"):
        welded_run(prims, 96, max_vertices=V - 3)
    c = welded_run(prims, 96, max_vertices=V - 3, allow_capacity=True)
    assert c["stats"]["status"] == L.SDF_ERR_CAPACITY
    W = 3 * ((V - 3 - 3) // 3) + 3  # a triangle starting at corner v is written iff v + 2 < capacity
    assert c["indices"][:W].tobytes() == a["indices"][:W].tobytes()


def test_welded_refuses_attributes_and_missing_indices():
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    eng = Engine()
    eng.configure(make_config(S.cell_size_for(64), out_mask=L.OUT_INDICES | L.OUT_WELDED | L.OUT_COLORS))
    eng.set_scene(S.sphere_scene(0.6))
    with pytest.raises(RuntimeError, match="SDF_ERR_INVALID"):
        eng.extract(MeshBuffers(100_000, L.OUT_INDICES | L.OUT_COLORS))
    eng.configure(make_config(S.cell_size_for(64), out_mask=L.OUT_WELDED))
    with pytest.raises(RuntimeError, match="SDF_ERR_INVALID"):
        eng.extract(MeshBuffers(100_000, 0))
    eng.close()


@pytest.mark.parametrize("solver", [0, 1])
def test_welded_dual_contouring_matches_soup(solver):
    """Dual contouring is indexed by nature: the welded output is the surface cells' vertices and six
    indices per quad (after the winding flip and the diagonal choice); every corner is its soup
    vertex bit for bit."""
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    prims = S.config_scene(2)
    kw = dict(technique=L.TECH_DC, dc_solver=solver, projection_iters=3 if solver else 0,
              adaptive_diagonal=1 if solver else 0)
    soup = H.engine_run(prims, 96, L.TECH_DC, L.OUT_INDICES, debug=False, **{k: v for k, v in kw.items()
                                                                               if k != "technique"})
    eng = Engine()
    eng.configure(make_config(S.cell_size_for(96), out_mask=L.OUT_INDICES | L.OUT_WELDED, **kw))
    eng.set_scene(prims)
    buf = MeshBuffers(2_000_000, L.OUT_INDICES)
    st = eng.extract(buf)
    V, U = int(st["total_vertices"]), int(st["welded_vertices"])
    assert V == int(soup["stats"]["total_vertices"]) and U == int(st["dc_cell_vertices"]) and 0 < U < V
    idx = buf.indices[:V].cpu().numpy().view(np.uint32)
    assert idx.max() < U
    verts = buf.vertices[:U].cpu().numpy()
    assert verts[idx].tobytes() == soup["verts"].tobytes()
    eng.close()
