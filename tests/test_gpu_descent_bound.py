"""The replayed first descent of the warp walks (first_descent in sdf_device.cuh) against the oracle where
it must not apply: a scene whose boxes reach beyond 1e8 (the root's box then fails the bound and every
walk tests its boxes from the root), and points beyond 1e8 or NaN among ordinary ones (their warps walk
without the replay). Distances, attributes and an extracted mesh must equal the oracle bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _far_scene():
    from cudasdf_b200 import scenes as S
    near = S.random_scene(300, seed=11)
    far = S.primitive(S.SDF_SPHERE, (3.0e8, 0.0, 0.0), params=(0.5,), operation=S.SDF_UNION_BLEND, blend=0.05)
    return np.concatenate([near, far])


def _same(a, b):
    """Bit-equal floats, NaN matching NaN (the GPU's and the host's NaN payloads differ)."""
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    return a.shape == b.shape and np.array_equal(na, nb) and np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32))


def _points(n, seed, odd=True):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    if odd:
        p[5::97] = (2.0e8, 0.0, 0.0)            # beyond the bound
        p[7::101] = (0.1, np.nan, 0.2)          # NaN (the box distance drops the NaN axis)
        p[11::89] = (-1.0e8, 1.0e8, -1.0e8)     # exactly at the bound (not below it)
    return p


@pytest.mark.parametrize("scene", ["far_primitive", "ordinary"])
def test_eval_matches_oracle(scene):
    import torch
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, make_config
    from oracle import oracle as O
    prims = _far_scene() if scene == "far_primitive" else S.random_scene(300, seed=11)
    pts = _points(20000, 3)
    eng = Engine()
    eng.configure(make_config(S.cell_size_for(64)))
    eng.set_scene(prims)
    dev = torch.from_numpy(pts).cuda()
    d = eng.eval_distance(dev).cpu().numpy()
    full = eng.eval(dev).cpu().numpy()
    eng.close()
    ref, _ = O.Scene(prims).map(pts)
    assert _same(d, ref[:, 0])
    assert _same(full, ref)


def test_far_scene_mesh_matches_oracle():
    import gpu_helpers as H
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from oracle import oracle as O
    prims = _far_scene()
    res = 64
    r = H.engine_run(prims, res, L.TECH_MC, L.OUT_INDICES | L.OUT_COLORS)
    ref = O.run(O.Scene(prims), O.make_grid(S.cell_size_for(res)), out_mask=O.OR_INDICES | O.OR_COLORS)
    assert r["stats"]["total_vertices"] == ref["totalVertices"] > 0
    assert np.array_equal(r["active"], ref["active"])
    assert _same(r["verts"], ref["verts"])
    assert _same(r["colors"], ref["colors"])
