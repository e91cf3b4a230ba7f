"""Dual contouring's cross-block lists (Hermite normals, projection steps, quad winding normals) against
the in-block paths that take whatever does not fit them: with the lists limited to a few hundred
entries (engine debug bit 2) most blocks, passes and vertices go the in-block way beside listed ones,
and every output is the same as with full lists."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def extract(prims, res, debug, **kw):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    eng = Engine()
    eng.configure(make_config(S.cell_size_for(res), technique=L.TECH_DC, out_mask=L.OUT_INDICES | L.OUT_NORMALS, **kw))
    eng.set_debug(debug)
    eng.set_scene(prims)
    buf = MeshBuffers(8_000_000, L.OUT_INDICES | L.OUT_NORMALS)
    st = eng.extract(buf)
    st = eng.extract(buf)  # the lists sized by the first run's counts
    V = int(st["total_vertices"])
    out = {"verts": buf.vertices[:V].cpu().numpy(), "normals": buf.normals[:V].cpu().numpy(),
           "dc": int(st["dc_cell_vertices"])}
    if debug & 1:
        out["cell_normals"] = eng.buffer(6, np.int16, out["dc"] * 4)
    eng.close()
    return out


@pytest.mark.parametrize("solver", ["reference", "masspoint"])
def test_small_lists_give_the_same_mesh(solver):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    kw = {} if solver == "reference" else dict(dc_solver=L.DC_SOLVER_MASSPOINT, projection_iters=3,
                                                 adaptive_diagonal=1)
    prims = S.config_scene(2)
    full = extract(prims, 160, 1, **kw)
    small = extract(prims, 160, 1 | 4, **kw)
    assert full["dc"] > 4096  # far more than the limited lists hold
    for k in ("verts", "normals", "cell_normals"):
        assert np.array_equal(full[k].view(np.uint32) if k != "cell_normals" else full[k],
                              small[k].view(np.uint32) if k != "cell_normals" else small[k]), k
