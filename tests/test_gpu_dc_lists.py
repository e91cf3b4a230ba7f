"""Dual contouring's cross-block lists (Hermite normals, projection steps, quad winding normals) against
the in-block paths that take whatever does not fit them: with the lists limited to a few hundred
entries (engine debug bit 2) most blocks, passes and vertices go the in-block way beside listed ones,
and every output is the same as with full lists. Without per-quad attributes and with full lists the
quads are emitted from the quad list by k_dc_quad_normals, with small lists per block by k_dc_quads:
the meshes must be the same too."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def extract(prims, res, debug, out_mask, **kw):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    eng = Engine()
    eng.configure(make_config(S.cell_size_for(res), technique=L.TECH_DC, out_mask=out_mask, **kw))
    eng.set_debug(debug)
    eng.set_scene(prims)
    buf = MeshBuffers(8_000_000, out_mask)
    st = eng.extract(buf)
    st = eng.extract(buf)  # the lists sized by the first run's counts
    welded = bool(out_mask & L.OUT_WELDED)
    n = int(st["total_vertices"])
    out = {"dc": int(st["dc_cell_vertices"])}
    if welded:
        out["indices"] = buf.indices[:n].cpu().numpy()
        out["verts"] = buf.vertices[:int(st["welded_vertices"])].cpu().numpy()
    else:
        out["verts"] = buf.vertices[:n].cpu().numpy()
        if buf.indices is not None:
            out["indices"] = buf.indices[:n].cpu().numpy()
    if buf.normals is not None and not welded:
        out["normals"] = buf.normals[:n].cpu().numpy()
    if debug & 1:
        out["cell_normals"] = eng.buffer(6, np.int16, out["dc"] * 4)
    eng.close()
    return out


@pytest.mark.parametrize("outputs", ["indices_normals", "indices", "welded"])
@pytest.mark.parametrize("solver", ["reference", "masspoint"])
def test_small_lists_give_the_same_mesh(solver, outputs):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    kw = {} if solver == "reference" else dict(dc_solver=L.DC_SOLVER_MASSPOINT, projection_iters=3,
                                                 adaptive_diagonal=1)
    mask = {"indices_normals": L.OUT_INDICES | L.OUT_NORMALS, "indices": L.OUT_INDICES,
            "welded": L.OUT_INDICES | L.OUT_WELDED}[outputs]
    prims = S.config_scene(2)
    full = extract(prims, 160, 1, mask, **kw)
    small = extract(prims, 160, 1 | 4, mask, **kw)
    assert full["dc"] > 4096  # far more than the limited lists hold
    assert full.keys() == small.keys()
    for k in full:
        if k == "dc":
            assert full[k] == small[k]
            continue
        a, b = full[k], small[k]
        assert a.shape == b.shape, k
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), k
