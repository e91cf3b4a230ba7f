"""Scene preparation on the GPU (sdf_engine_set_scene_device) against the host build.

The host build restates CudaSDFMesh::UpdateBVH and buildBVHRecursive (CudaSDFMesh.cpp:216-249,
CudaSDFUtil.h:507-603) and is pinned to the reference's node order by the golden fixtures; the GPU
build must give the same sorted primitives and the same nodes byte for byte, and hence the same
meshes. Scenes cover every primitive type, non-union operations (which stay out of the BVH),
displacements (which widen the boxes), coincident centroids (the split's fallback to count / 2),
trees of one and two primitives and scenes without unions.
"""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mixed(n, seed, dup=False, ops=(0, 3, 3, 1, 2, 4, 5)):
    from cudasdf_b200 import scenes as S
    rng = np.random.default_rng(seed)
    p = S.random_scene(n, seed, size_range=(0.02, 0.3), center_range=0.8)
    p["type"] = rng.integers(0, 15, n)
    p["operation"] = rng.choice(ops, n)
    p["params"] = rng.uniform(0.1, 0.9, (n, 6))
    p["displacement"] = rng.choice([0, 0, 0, 1, 2, 3], n)
    if dup:  # many primitives on a few centres: centroid ties and empty split sides
        p["position"] = rng.integers(0, 3, (n, 3)) * 0.25
        p["rotation"] = (0, 0, 0, 1)
        p["type"] = 0
    return p


def _both(prims):
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine
    host, dev = Engine(), Engine()
    host.set_scene(prims)
    dev.set_scene_device(prims)
    n = len(prims)
    hn, hb = host.bvh()
    dn, db = dev.bvh()
    hp = host.buffer(9, S.PRIM_DTYPE, n)
    dp = dev.buffer(9, S.PRIM_DTYPE, n)
    host.close()
    dev.close()
    return (hn, hb, hp), (dn, db, dp)


CASES = [("one", 1, 0, False), ("two", 2, 1, False), ("three", 3, 2, False), ("small", 37, 3, False),
         ("mixed_1k", 1000, 4, False), ("mixed_5k", 5000, 5, False), ("ties_300", 300, 6, True),
         ("ties_4k", 4096, 7, True), ("mixed_100k", 100_000, 8, False)]


@pytest.mark.parametrize("name,n,seed,dup", CASES)
def test_device_bvh_matches_host_build(name, n, seed, dup):
    (hn, hb, hp), (dn, db, dp) = _both(_mixed(n, seed, dup))
    assert hb == db and len(hn) == len(dn)
    assert hn.tobytes() == dn.tobytes(), int(np.sum(hn != dn))
    assert hp.tobytes() == dp.tobytes()


def test_device_bvh_benchmark_scenes():
    """The 256^3, 512^3 and 1024^3 benchmark scenes (256, 4,096 and 16,384 primitives)."""
    from cudasdf_b200 import scenes as S
    for cfg in (2, 3, 4):
        (hn, hb, hp), (dn, db, dp) = _both(S.config_scene(cfg))
        assert hb == db and hn.tobytes() == dn.tobytes() and hp.tobytes() == dp.tobytes(), cfg


def test_device_bvh_without_unions_and_empty():
    from cudasdf_b200 import scenes as S
    p = _mixed(50, 9)
    p["operation"] = 1  # subtract only: no BVH, a linear pass over all primitives
    (hn, hb, hp), (dn, db, dp) = _both(p)
    assert hb == db == 0 and len(hn) == len(dn) == 0 and hp.tobytes() == dp.tobytes()
    from cudasdf_b200.engine import Engine
    e = Engine()
    e.set_scene_device(np.zeros(0, S.PRIM_DTYPE))
    nodes, nb = e.bvh()
    assert len(nodes) == 0 and nb == 0
    e.close()


@pytest.mark.parametrize("technique", [0, 1])
def test_meshes_identical_after_device_build(technique):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    prims = _mixed(600, 11, ops=(0, 3, 3, 1, 4))
    res = 96
    digests = []
    for setter in ("set_scene", "set_scene_device"):
        e = Engine()
        e.configure(make_config(S.cell_size_for(res), technique=technique, out_mask=L.OUT_INDICES))
        getattr(e, setter)(prims)
        buf = MeshBuffers(4_000_000, L.OUT_INDICES)
        st = e.extract(buf, 0.25)
        V = int(st["total_vertices"])
        assert V > 1000
        digests.append(hashlib.sha256(buf.vertices[:V].cpu().numpy().tobytes()).hexdigest())
        e.close()
    assert digests[0] == digests[1]


def test_device_scene_then_host_scene_and_surrogate_scene_copy():
    """Switching between the two setters keeps each extraction's own scene; the surrogate's training
    run reads the device-built scene back (it has no host copy)."""
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    a, b = _mixed(300, 12, ops=(0, 3, 3, 1, 4)), _mixed(300, 13, ops=(0, 3, 3, 1, 4))
    e = Engine()
    e.configure(make_config(S.cell_size_for(64), out_mask=L.OUT_INDICES))
    buf = MeshBuffers(2_000_000, L.OUT_INDICES)
    counts = []
    for setter, p in (("set_scene_device", a), ("set_scene", b), ("set_scene_device", b), ("set_scene", a)):
        getattr(e, setter)(p)
        counts.append(int(e.extract(buf)["total_vertices"]))
    assert counts[0] == counts[3] and counts[1] == counts[2] and counts[0] != counts[1]
    e.set_scene_device(S.config_scene(2))
    st = e.surrogate_train(Engine.surrogate_config(samples=1 << 16, validation=1 << 14, steps=50))
    assert st["surface_points"] > 0
    e.close()
