"""UV atlas packing on the GPU against the oracle and the reference's own packer.

The reference's GridUVPacker (src/SDFMesh/GridUVPacker.cu) is compiled from its sources into
oracle/_ref/libuvpackref.so and run on the same inputs; the oracle (oracle/uvpack_oracle.cpp) is fed
the same curand draws the GPU attempts consume. Charts, island masks (all four grids and the row
bounds), every attempt's placements, the chosen atlas and the remapped UVs must be identical.
The reference is only run where every candidate loop of its packing kernel can end (its loop never
ends when an island has fewer aligned columns than the candidate budget).
"""
import os

import numpy as np
import pytest

import gpu_helpers as H
from oracle import uvpack_oracle as O

pytestmark = pytest.mark.gpu

HAVE_REF = os.path.exists(O.REF_LIB_PATH)


def mesh(prims, res):
    from cudasdf_b200 import _lib as L
    r = H.engine_run(prims, res, L.TECH_MC, L.OUT_UVS | L.OUT_PRIMIDS)
    return r["uvs"].astype(np.float32), r["primids"].astype(np.float32)


def scene(kind):
    from cudasdf_b200 import scenes as S
    if kind == "random24":
        return mesh(S.random_scene(24, 0x5DF0101, size_range=(0.15, 0.35), center_range=0.6), 96)
    if kind == "showcase":
        return mesh(S.showcase_scene(0.0, animate=False), 128)
    if kind == "random300":
        return mesh(S.random_scene(300, 0x5DF0102, size_range=(0.06, 0.12), center_range=0.8), 160)
    raise ValueError(kind)


def ours(uvs, prim, cfg, steps=4):
    import torch
    from cudasdf_b200.uvpack import PackingConfig, UVAtlas
    pc = PackingConfig(*[cfg[n] for n in O.CFG_FIELDS])
    a = UVAtlas()
    du = torch.from_numpy(uvs).cuda()
    dp = torch.from_numpy(prim).cuda()
    out = {}
    out["num_charts"] = a.extract_charts(du, dp)
    out["charts"] = a.read(0)
    out["tri_chart"] = a.read(1)
    if steps >= 2:
        a.create_islands(du, cfg["grid_resolution"], cfg["margin_cells"])
        out["islands"] = a.read(2)
        words, rb = a.read(3), a.read(4)
        out["grids"] = [a.grids(i, words, rb) for i in range(len(out["islands"]))]
    if steps >= 3:
        out["info"] = a.pack_islands(pc)
        out["seeds"] = a.read(6)
        out["solutions"] = a.read(7)
        out["all_placements"] = a.read(8)
        out["best"] = a.read(9)
    if steps >= 4:
        a.remap_uvs_to_atlas(du, dp, cfg["grid_resolution"])
        torch.cuda.synchronize()
        out["uvs"] = du.cpu().numpy()
    a.close()
    return out


def draws_for(seeds):
    from cudasdf_b200.uvpack import random_draws
    return random_draws(seeds, 1 << 14)


def check_charts(g, o):
    assert g["num_charts"] == len(o["prim"])
    assert np.array_equal(g["charts"]["primitive_id"], o["prim"])
    assert np.array_equal(g["charts"]["num_triangles"], o["ntris"])
    assert np.array_equal(g["charts"]["uv_min"], o["bounds"][:, :2]) and np.array_equal(g["charts"]["uv_max"], o["bounds"][:, 2:])
    assert np.array_equal(g["tri_chart"], o["tri_chart"])


def check_islands(g, oi):
    isl = g["islands"]
    assert np.array_equal(isl["island_index"], oi["order"]), "packing order (std::sort by area)"
    for slot, k in enumerate(oi["order"]):
        d = oi["islands"][k]
        assert (isl[slot]["width"], isl[slot]["height"], isl[slot]["min_cell_x"], isl[slot]["min_cell_y"]) == \
            (d["w"], d["h"], d["min_x"], d["min_y"])
        og = O.grids(oi, k)
        for name in ("mask", "collision", "mask90", "collision90", "row_bounds", "row_bounds90"):
            assert np.array_equal(g["grids"][slot][name], og[name]), (slot, name)


CONFIGS = {
    "app32": dict(O.APP_CONFIG, max_iterations=32),
    "plain": dict(O.APP_CONFIG, max_iterations=16, enable_rotation=0, shuffle_order_per_attempt=0, max_drop_steps=0,
                  margin_cells=0, x_alignment=1, max_candidates_per_island=4),
    "wide": dict(O.APP_CONFIG, max_iterations=12, max_candidates_per_island=64, x_alignment=4, margin_cells=2,
                 random_seed=77),
    "tight": dict(O.APP_CONFIG, max_iterations=24, grid_size=360),
}


@pytest.mark.parametrize("kind", ["random24", "showcase"])
def test_charts_and_islands(kind):
    uvs, prim = scene(kind)
    cfg = CONFIGS["app32"]
    g = ours(uvs, prim, cfg, steps=2)
    oc = O.extract_charts(uvs, prim)
    check_charts(g, oc)
    oi = O.create_islands(uvs, oc, cfg["grid_resolution"], cfg["margin_cells"])
    check_islands(g, oi)


@pytest.mark.parametrize("kind,cfg", [("random24", "app32"), ("random24", "plain"), ("random24", "wide"),
                                      ("random24", "tight"), ("showcase", "app32"), ("random300", "app32")])
def test_pack_matches_oracle(kind, cfg):
    uvs, prim = scene(kind)
    cfg = CONFIGS[cfg]
    if kind == "random300":
        cfg = dict(cfg, max_iterations=8)
    g = ours(uvs, prim, cfg)
    o = O.run(uvs, prim, cfg, draws_for)
    assert np.array_equal(g["seeds"], o["seeds"])
    assert not (o["packed"]["info"][:, 3] & O.DRAWS_EXHAUSTED).any()
    sol = g["solutions"]
    info = o["packed"]["info"]
    assert np.array_equal(sol["num_placed"], info[:, 0])
    assert np.array_equal(sol["utilized_width"], info[:, 1]) and np.array_equal(sol["utilized_height"], info[:, 2])
    assert np.array_equal(sol["fitness"], o["packed"]["fitness"])
    assert np.array_equal((sol["flags"] & 1) != 0, (info[:, 3] & O.CANDIDATE_LOOP_OPEN) != 0)
    n = o["packed"]["placements"].shape[1]
    allp = g["all_placements"].view(np.int32).reshape(len(sol), n, 4)
    for s in range(len(sol)):
        k = int(sol["num_placed"][s])
        assert np.array_equal(allp[s, :k], o["packed"]["placements"][s, :k]), s
    at = o["atlas"]
    gi = g["info"]
    assert (gi["success"], gi["atlas_width"], gi["atlas_height"], gi["num_placed"], gi["best_solution"]) == \
        (at["success"], at["width"], at["height"], at["placed"], at["best"])
    assert np.float32(gi["fitness"]) == at["fitness"] and np.float32(gi["scaling_factor"]) == at["scaling"]
    assert gi["shelf_width"] == o["packed"]["shelf"]
    assert np.array_equal(g["best"].view(np.int32).reshape(-1, 4), at["placements"])
    assert np.array_equal(g["uvs"].view(np.uint32), o["uvs"].view(np.uint32))
    if kind == "random300":
        assert gi["num_islands"] > 256 and not gi["success"]


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("kind,cfg", [("random24", "app32"), ("random24", "plain"), ("random24", "tight"),
                                      ("showcase", "app32")])
def test_matches_reference_packer(kind, cfg):
    uvs, prim = scene(kind)
    cfg = CONFIGS[cfg]
    ref = O.reference_run(uvs, prim, cfg)
    assert ref["loops_end"]
    g = ours(uvs, prim, cfg)
    assert np.array_equal(g["charts"]["primitive_id"], ref["charts"]["prim"])
    assert np.array_equal(g["charts"]["num_triangles"], ref["charts"]["ntris"])
    assert np.array_equal(g["charts"]["uv_min"], ref["charts"]["bounds"][:, :2])
    assert np.array_equal(g["charts"]["uv_max"], ref["charts"]["bounds"][:, 2:])
    isl = g["islands"]
    assert np.array_equal(isl["island_index"], ref["islands"][:, 0])
    assert np.array_equal(np.stack([isl["width"], isl["height"], isl["min_cell_x"], isl["min_cell_y"]], 1),
                          ref["islands"][:, 1:])
    for slot, rg in enumerate(O.reference_grids(ref)):
        for name, v in rg.items():
            assert np.array_equal(g["grids"][slot][name], v), (slot, name)
    at, gi = ref["atlas"], g["info"]
    assert (gi["success"], gi["atlas_width"], gi["atlas_height"], gi["num_placed"]) == \
        (at["success"], at["width"], at["height"], at["placed"])
    assert np.float32(gi["fitness"]) == at["fitness"] and np.float32(gi["scaling_factor"]) == at["scaling"]
    assert np.array_equal(g["best"].view(np.int32).reshape(-1, 4), at["placements"])
    assert np.array_equal(g["uvs"].view(np.uint32), ref["uvs"].view(np.uint32))


def test_empty_and_single_island():
    """No triangles: no charts, no atlas, UVs unchanged. One island under the app configuration: the
    reference's candidate loop cannot end there; this packer stops once every column is listed, as
    the oracle does, and reports it."""
    from cudasdf_b200 import scenes as S
    cfg = CONFIGS["app32"]
    e = ours(np.zeros((0, 2), np.float32), np.zeros(0, np.float32), cfg)
    assert e["num_charts"] == 0 and not e["info"]["success"] and e["uvs"].shape == (0, 2)
    uvs, prim = mesh(S.sphere_scene(0.6), 64)
    g = ours(uvs, prim, cfg)
    o = O.run(uvs, prim, cfg, draws_for)
    assert not o["loops_end"] and g["info"]["candidate_loop_open"] == 1
    assert g["info"]["success"] == o["atlas"]["success"] == 1
    assert np.array_equal(g["best"].view(np.int32).reshape(-1, 4), o["atlas"]["placements"])
    assert np.array_equal(g["uvs"].view(np.uint32), o["uvs"].view(np.uint32))
    assert g["uvs"].min() >= 0.0 and g["uvs"].max() <= 1.0


def test_atlas_has_no_overlap():
    """Every placed island's collision mask, written at its placement, touches no other (the
    reference's own overlap check, GridUVPacker.cu:1316-1395), and lies inside the atlas."""
    uvs, prim = scene("showcase")
    cfg = CONFIGS["app32"]
    g = ours(uvs, prim, cfg)
    assert g["info"]["success"]
    G = cfg["grid_size"]
    board = np.zeros((G, G), bool)
    by_index = {int(d["island_index"]): i for i, d in enumerate(g["islands"])}
    for p in g["best"]:
        slot = by_index[int(p["island_index"])]
        m = g["grids"][slot]["collision90" if p["rotation"] else "collision"]
        bits = np.unpackbits(m.view(np.uint8), bitorder="little").reshape(m.shape[0], -1).astype(bool)
        w = int(g["islands"][slot]["height" if p["rotation"] else "width"])
        bits = bits[:, :w]
        sub = board[p["grid_y"]:p["grid_y"] + bits.shape[0], p["grid_x"]:p["grid_x"] + w]
        assert sub.shape == bits.shape and not (sub & bits).any()
        sub |= bits
    assert g["info"]["atlas_width"] >= max(int(p["grid_x"]) for p in g["best"])


UVPACK_HOST = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cudasdf_b200", "dropin_host",
                           "_build", "uvpack_host")


@pytest.mark.skipif(not os.path.exists(UVPACK_HOST), reason="uvpack_host not built")
def test_cpp_api_host_matches(tmp_path):
    """The reference's call sequence (main.cpp:1417-1442) written against include/grid_uv_packer_b200.hpp
    (cudasdf_b200/dropin_host/uvpack_host.cpp) gives the atlas and UVs of the C entry points and of the
    oracle, with the app's full configuration (256 attempts)."""
    import json
    import subprocess
    uvs, prim = scene("showcase")
    cfg = dict(O.APP_CONFIG)
    fu, fp, fo = tmp_path / "uvs.bin", tmp_path / "prim.bin", tmp_path / "out.bin"
    uvs.tofile(fu)
    prim.tofile(fp)
    r = subprocess.run([UVPACK_HOST, str(fu), str(fp), str(len(prim)), str(fo), "2"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    host = json.loads(r.stdout.strip().splitlines()[-1])
    g = ours(uvs, prim, cfg)
    assert host["success"] == g["info"]["success"] == 1
    assert (host["atlas_width"], host["atlas_height"]) == (g["info"]["atlas_width"], g["info"]["atlas_height"])
    assert np.array_equal(np.array(host["placements"], np.int32).reshape(-1, 4), g["best"].view(np.int32).reshape(-1, 4))
    out = np.fromfile(fo, np.float32).reshape(-1, 2)
    assert np.array_equal(out.view(np.uint32), g["uvs"].view(np.uint32))
    o = O.run(uvs, prim, cfg, draws_for)
    assert np.array_equal(out.view(np.uint32), o["uvs"].view(np.uint32))


def synthetic_soup(seed, nchart=24, tris=150, nan_frac=0.01):
    """UV triangles in random patches, one primitive id per patch, with the inputs a mesh can hold and
    the reference reads in its own way: fractional ids (rounded by + 0.5 and truncation), -1 (which
    rounds to chart 0), -2 (no chart), NaN UVs in a few vertices (fminf skips them), triangles with a
    vertex on a cell boundary, degenerate (zero-area) triangles and triangles spanning tens of cells."""
    rng = np.random.default_rng(seed)
    uvs, ids = [], []
    for c in range(nchart):
        su, sv = rng.uniform(0.3, 1.2, 2)
        o = rng.uniform(-0.2, 0.6, 2)
        base = rng.uniform(0, 1, (tris, 1, 2)) * [su, sv] + o
        t = base + rng.normal(0, 0.04, (tris, 3, 2))
        t[: tris // 10] = base[: tris // 10] + rng.uniform(-0.4, 0.4, (tris // 10, 3, 2))  # large triangles
        t[tris // 10: tris // 10 + 5, 1] = t[tris // 10: tris // 10 + 5, 0]                 # degenerate
        k = slice(tris // 10 + 5, tris // 10 + 15)
        t[k] = np.round(t[k] * 64) / 64                                                    # on cell corners
        uvs.append(t.reshape(-1, 2))
        pid = float(c) + rng.choice([0.0, 0.3, -0.4])
        ids.append(np.full(tris * 3, pid, np.float32))
    uv = np.concatenate(uvs).astype(np.float32)
    pid = np.concatenate(ids)
    T = len(pid) // 3
    tri_ids = pid.reshape(T, 3)
    pick = rng.choice(T, T // 50, replace=False)
    tri_ids[pick[: len(pick) // 2], 0] = -1.0
    tri_ids[pick[len(pick) // 2:], 0] = -2.0
    nanv = rng.choice(len(uv), int(len(uv) * nan_frac), replace=False)
    uv[nanv, rng.integers(0, 2, len(nanv))] = np.nan
    order = rng.permutation(T)
    return uv.reshape(T, 3, 2)[order].reshape(-1, 2).copy(), tri_ids[order].reshape(-1).copy()


@pytest.mark.parametrize("seed", [1, 2])
def test_adversarial_soup_matches_oracle_and_reference(seed):
    uvs, prim = synthetic_soup(seed)
    cfg = dict(O.APP_CONFIG, max_iterations=16)
    g = ours(uvs, prim, cfg)
    o = O.run(uvs, prim, cfg, draws_for)
    check_charts(g, o["charts"])
    check_islands(g, o["islands"])
    assert np.array_equal(g["best"].view(np.int32).reshape(-1, 4), o["atlas"]["placements"])
    # NaN UVs stay NaN (the GPU writes its canonical NaN, the host keeps the input's bits); every other
    # value bit for bit
    nan = np.isnan(g["uvs"])
    assert np.array_equal(nan, np.isnan(o["uvs"])) and nan.any()
    assert np.array_equal(g["uvs"][~nan].view(np.uint32), o["uvs"][~nan].view(np.uint32))
    if HAVE_REF and o["loops_end"]:
        ref = O.reference_run(uvs, prim, cfg)
        assert np.array_equal(g["charts"]["primitive_id"], ref["charts"]["prim"])
        for slot, rg in enumerate(O.reference_grids(ref)):
            for name, v in rg.items():
                assert np.array_equal(g["grids"][slot][name], v), (slot, name)
        assert np.array_equal(g["best"].view(np.int32).reshape(-1, 4), ref["atlas"]["placements"])
        assert np.array_equal(g["uvs"].view(np.uint32), ref["uvs"].view(np.uint32))


def test_partial_triangle_and_limits():
    """A partial last triangle is not read; ids of 2^24 and more are refused (SDF_ERR_INVALID)."""
    import torch
    from cudasdf_b200 import _lib as L
    from cudasdf_b200.uvpack import UVAtlas
    uvs, prim = synthetic_soup(3, nchart=6, tris=40)
    a = UVAtlas()
    du, dp = torch.from_numpy(uvs[:-1].copy()).cuda(), torch.from_numpy(prim[:-1].copy()).cuda()
    assert a.extract_charts(du, dp) == len(O.extract_charts(uvs[:-3], prim[:-3])["prim"])
    big = prim.copy()
    big[0] = float(1 << 24)
    with pytest.raises(RuntimeError, match="SDF_ERR_INVALID"):
        a.extract_charts(torch.from_numpy(uvs).cuda(), torch.from_numpy(big).cuda())
    a.close()
    assert L.SDF_ERR_INVALID == 1
