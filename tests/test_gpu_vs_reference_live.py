"""Live parity against the reference's own CUDA path (oracle/_ref, built from the reference sources).

Randomised scenes beyond the golden fixtures: every primitive type, every CSG operation, the three
displacements, annular/rounding, non-zero time, grids whose size is not a multiple of the 8^3
block and bounds other than [-1, 1]^3. Skipped when oracle/_ref was not built.
"""
import numpy as np
import pytest

import gpu_helpers as H
from oracle import reflib as R

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")]


def mixed_scene(seed, n, ops="union", displaced=True, cones=True):
    """Random scene: every primitive type (optionally without cones); ops "union" (union / smooth
    union only) or "mixed" (also subtract and the smooth subtract); optional displacements and uv
    transforms."""
    from cudasdf_b200 import scenes as S
    rng = np.random.default_rng(seed)
    p = S.random_scene(n, seed, size_range=(0.08, 0.35), center_range=0.6)
    types = [t for t in range(15) if cones or t != S.SDF_CONE]
    p["type"] = rng.choice(types, n)
    p["operation"] = rng.choice([0, 3] if ops == "union" else [0, 0, 3, 3, 1, 4], n)
    p["operation"][0] = S.SDF_UNION  # at least one BVH primitive
    p["blendFactor"] = rng.uniform(0.02, 0.2, n)
    p["params"] = rng.uniform(0.2, 0.9, (n, 6))
    p["params"][:, 1] = np.where(p["type"] == S.SDF_CONE, rng.uniform(10, 50, n), p["params"][:, 1])
    p["params"][:, 2] = np.where(p["type"] == S.SDF_ROUNDED_CONE, rng.uniform(0.05, 0.15, n), p["params"][:, 2])
    p["annular"] = np.where(rng.random(n) < 0.2, rng.uniform(0, 0.03, n), 0)
    p["rounding"] = np.where(rng.random(n) < 0.2, rng.uniform(0, 0.03, n), 0)
    p["uvScale"] = rng.uniform(0.5, 3, (n, 2))
    if displaced:
        p["displacement"] = rng.choice([0, 0, 0, 1, 2, 3], n)
        p["dispParams"][:, 0] = rng.uniform(0.5, 3, n)
        p["dispParams"][:, 1] = rng.uniform(-0.1, 0.1, n)
        p["uvOffset"] = rng.uniform(-0.5, 0.5, (n, 2))
        p["uvRotation"] = np.where(rng.random(n) < 0.3, rng.uniform(-1, 1, n), 0)
    return p


def ref_run(prims, cell, bmin, bmax, technique, mask, time):
    m = R.RefMesh(cell, bmin, bmax, max_vertices=4_000_000)
    m.set_primitives(prims)
    st = m.run(time, technique, 1.0, mask, sort_active=True)
    nA, V = st["activeUsed"], st["totalVertices"]
    out = {"active": m.copy(R.RB_ACTIVE, np.int32, nA), "counts": m.copy(R.RB_COUNTS, np.uint32, nA * 512),
           "offsets": m.copy(R.RB_OFFSETS, np.uint32, nA * 512),
           "verts": m.copy(R.RB_VERTS, np.float32, V * 4).reshape(V, 4)}
    if mask & R.OUT_COLORS:
        out["colors"] = m.copy(R.RB_COLORS, np.float32, V * 4).reshape(V, 4)
    if mask & R.OUT_UVS:
        out["uvs"] = m.copy(R.RB_UVS, np.float32, V * 2).reshape(V, 2)
    if mask & R.OUT_PRIMIDS:
        out["primids"] = m.copy(R.RB_PRIMIDS, np.float32, V)
    if mask & R.OUT_NORMALS:
        out["normals"] = m.copy(R.RB_NORMALS, np.float32, V * 4).reshape(V, 4)
    if mask & R.OUT_INDICES:
        out["indices"] = m.copy(R.RB_INDICES, np.uint32, V)
    m.close()
    return out, st


class _Fixture(dict):
    @property
    def files(self):
        return list(self.keys())


# (A) undisplaced union scenes, every primitive type but the cone, smooth blends, annular/rounding
#     shells, uv scales: bit-exact on every stream. (The cone's distance, which goes through sinf and
#     cosf of its angle, differs from the reference in the last bits at a few per cent of points in
#     the reference's 8-corner context; it is in the tolerance tiers below.)
EXACT_CASES = [(31, 24, 45, 0), (32, 40, 64, 0), (33, 16, 37, 1), (34, 32, 50, 1), (35, 64, 72, 0)]
# (B) with displacements (twist/bend/sine) and uv offsets/rotations, and (C) with subtracted
#     primitives: the reference's build contracts some of these expressions differently inside its
#     8-corner and finite-difference stencils than in a lone map() call, so floats differ in the last
#     bits there; topology stays bit-exact and floats are compared within the stated tolerances.
DISPLACED_CASES = [(21, 24, 45, 0), (22, 40, 64, 0), (23, 16, 37, 1), (24, 32, 50, 1)]
SUBTRACT_CASES = [(11, 24, 45, 0), (12, 40, 64, 0), (13, 16, 37, 1), (14, 32, 50, 1)]
CONE_CASES = [(41, 24, 45, 0), (42, 32, 50, 1)]


@pytest.mark.parametrize("seed,n,res,technique", EXACT_CASES)
def test_undisplaced_union_scene_bit_exact(seed, n, res, technique):
    _run_case(mixed_scene(seed, n, "union", displaced=False, cones=False), seed, res, technique, exact=True)


@pytest.mark.parametrize("seed,n,res,technique", DISPLACED_CASES)
def test_displaced_scene_within_tolerance(seed, n, res, technique):
    _run_case(mixed_scene(seed, n, "union", displaced=True), seed, res, technique, exact=False)


@pytest.mark.parametrize("seed,n,res,technique", CONE_CASES)
def test_scene_with_cones_within_tolerance(seed, n, res, technique):
    _run_case(mixed_scene(seed, n, "union", displaced=False, cones=True), seed, res, technique, exact=False)


@pytest.mark.parametrize("seed,n,res,technique", SUBTRACT_CASES)
def test_subtract_scene_within_tolerance(seed, n, res, technique):
    _run_case(mixed_scene(seed, n, "mixed", displaced=False), seed, res, technique, exact=False)


def _run_case(prims, seed, res, technique, exact):
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    bmin, bmax = (-1.1, -1.05, -1.0), (1.1, 1.0, 1.05)
    cell = float(np.float32(2.2) / np.float32(res))
    mask = R.OUT_ALL
    time = 0.37 * seed
    ref, st = ref_run(prims, cell, bmin, bmax, technique, mask, time)
    assert st["totalVertices"] > 0
    eng = Engine()
    eng.configure(make_config(cell, bmin, bmax, technique=technique, out_mask=mask))
    eng.set_debug(1)
    eng.set_scene(prims)
    buf = MeshBuffers(st["totalVertices"] + 1024, mask)
    es = eng.extract(buf, time)
    assert es["active_blocks"] == st["activeUsed"] and es["total_vertices"] == st["totalVertices"]
    V = st["totalVertices"]
    A = st["activeUsed"]
    mine = {"active": eng.buffer(0, np.int32, A), "counts": eng.buffer(1, np.uint32, A * 512),
            "verts": buf.vertices[:V].cpu().numpy(), "colors": buf.colors[:V].cpu().numpy(),
            "uvs": buf.uvs[:V].cpu().numpy(), "primids": buf.primitive_ids[:V].cpu().numpy().view(np.float32),
            "normals": buf.normals[:V].cpu().numpy(), "indices": buf.indices[:V].cpu().numpy().view(np.uint32)}
    eng.close()
    mine["offsets"] = H.exclusive_scan(mine["counts"])
    topo = H.compare(mine, _Fixture(ref), ["active", "counts", "offsets", "indices"])
    assert not topo, topo
    if exact:
        bad = H.compare(mine, _Fixture(ref), ["primids", "verts", "colors", "uvs", "normals"])
        assert not bad, bad
        return
    d = np.abs(mine["verts"][:, :3].astype(np.float64) - ref["verts"][:, :3]).max(1) / cell
    if technique == 0:
        # marching-cubes positions: 1e-6 cell for 99 % of the vertices; a stencil distance that moves by
        # an ulp next to a zero crossing moves an edge point by up to a few 1e-4 cell, so 1e-2 cell for all
        assert np.mean(d <= 1e-6) > 0.99 and d.max() <= 1e-2, (np.mean(d <= 1e-6), d.max())
    else:
        # dual contouring: vertices within 1e-4 cell for almost all
        assert np.mean(d <= 1e-4) > 0.97 and d.max() < 0.05, (np.mean(d <= 1e-4), d.max())
    # normals are forward differences with step h = cell / 1000: one ulp of an O(1) intermediate
    # (1.2e-7) moves a component by about 1.2e-7 / h, i.e. 2.4e-3 at cell 0.05; most are unaffected
    dn = np.abs(mine["normals"][:, :3] - ref["normals"][:, :3]).max(1)
    assert np.mean(dn < 1e-4) > 0.8 and np.mean(dn < 1e-2) > 0.99, (np.mean(dn < 1e-4), np.mean(dn < 1e-2))


@pytest.mark.parametrize("seed,n,res", [(51, 24, 45), (52, 40, 64)])
def test_dc_normal_passes_match_reference(seed, n, res):
    """launchDCRecomputeNormalsAtVertices and launchDCSmoothCellNormals after a DC update, on the
    reference and on the library: the cell normals and the smoothed copies agree."""
    import torch

    from cudasdf_b200 import _lib as L
    from cudasdf_b200.dropin import CudaSDFMesh
    prims = mixed_scene(seed, n, "union", displaced=False, cones=False)
    bmin, bmax = (-1.1, -1.05, -1.0), (1.1, 1.0, 1.05)
    cell = float(np.float32(2.2) / np.float32(res))
    cos_t = float(np.cos(np.radians(30.0)))
    m = R.RefMesh(cell, bmin, bmax, max_vertices=4_000_000)
    m.set_primitives(prims)
    st = m.run(0.0, 1, 1.0, R.OUT_INDICES, sort_active=True)
    m.dc_normal_passes(0.0, cos_t)
    nA = st["activeUsed"]
    mask = m.copy(R.RB_DCMASK, np.uint8, nA * 512)
    voff = m.copy(R.RB_DCVOFF, np.uint32, nA * 512)
    nd = int(voff[-1]) + int(mask[-1] not in (0, 255))
    ref_n = m.copy(R.RB_DCNORM, np.int16, nd * 4).reshape(nd, 4)
    ref_t = m.copy(R.RB_DCNORMTMP, np.int16, nd * 4).reshape(nd, 4)
    m.close()
    mesh = CudaSDFMesh(max_active_blocks=1 << 30, max_vertices=4_000_000)
    mesh.Initialize(cell, bmin, bmax)
    for p in prims:
        mesh.AddPrimitive(p)
    verts = torch.empty((4_000_000, 4), dtype=torch.float32, device="cuda")
    idx = torch.empty(4_000_000, dtype=torch.int32, device="cuda")
    mesh.Update(0.0, verts, None, idx, technique=L.TECH_DC)
    mesh.DCNormalPasses(0.0, cos_t)
    assert mesh.num_active == nA
    got_n = mesh.dc_buffer("dcNormals", nd)[:, :3]
    got_t = mesh.dc_buffer("dcNormalsTmp", nd)[:, :3]
    assert (got_n == ref_n[:, :3]).all(), int((got_n != ref_n[:, :3]).any(1).sum())
    # the smoothing sums up to seven unit normals and renormalises; where the reference's build rounds
    # one of those sums differently the encoded result moves by a unit or two (one vertex in thousands)
    diff = np.abs(got_t.astype(np.int32) - ref_t[:, :3].astype(np.int32)).max(1)
    assert np.mean(diff == 0) > 0.998 and diff.max() <= 2, (int((diff > 0).sum()), int(diff.max()))
