"""The UV atlas packer oracle against the reference's own packer (golden fixtures, no GPU).

tests/golden/uvpack_ref.npz and uvpack_probes.npz are outputs of the reference's GridUVPacker and of
its raster helpers, compiled from the reference's sources (tests/golden/make_uvpack_golden.py).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import uvpack_oracle as O

REF = os.path.join(GOLDEN, "uvpack_ref.npz")
PROBES = os.path.join(GOLDEN, "uvpack_probes.npz")
need = pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(PROBES)), reason="fixtures not generated")


def config_of(arr):
    return dict(zip(O.CFG_FIELDS, (int(v) for v in arr)))


@need
def test_raster_helpers_match_reference_probes():
    """triangleArea2D bit for bit, pointInTriangle, orientSign, segmentsIntersect and
    triangleOverlapsCell exactly, including cells wholly inside a triangle where the corner test is
    decided by the rounding of the reference's compiled code."""
    Q = np.load(PROBES)
    r = O.probe(Q["rec"], Q["cells"])
    assert np.array_equal(r["area"].view(np.uint32), Q["area"].view(np.uint32))
    for k in ("pit", "ori", "seg", "ov"):
        assert np.array_equal(r[k], Q[k]), k
    # the corner test inside triangleOverlapsCell is not pointInTriangle alone: cells exist where a
    # corner passes pointInTriangle but the cell is not marked
    pit4, ov4 = Q["pit"].reshape(-1, 4), Q["ov"].reshape(-1, 4)[:, 0]
    assert (pit4.any(1) & (ov4 == 0)).any()


@need
def test_charts_match_reference():
    F = np.load(REF)
    c = O.extract_charts(F["uvs"], F["prim"])
    assert np.array_equal(c["prim"], F["chart_prim"]) and np.array_equal(c["ntris"], F["chart_ntris"])
    assert np.array_equal(c["bounds"], F["chart_bounds"])
    start = np.concatenate([[0], np.cumsum(F["chart_ntris"])])
    for k in range(len(c["prim"])):
        assert np.array_equal(np.nonzero(c["tri_chart"] == k)[0], F["chart_tris"][start[k]:start[k + 1]])


@need
def test_islands_match_reference():
    F = np.load(REF)
    cfg = config_of(F["config"])
    c = O.extract_charts(F["uvs"], F["prim"])
    isl = O.create_islands(F["uvs"], c, cfg["grid_resolution"], cfg["margin_cells"])
    assert np.array_equal(isl["order"], F["islands"][:, 0]), "packing order (std::sort by mask area)"
    ref = dict(islands=F["islands"], words=F["words"], rb=F["rb"])
    for slot, (k, rg) in enumerate(zip(isl["order"], O.reference_grids(ref))):
        d = isl["islands"][k]
        assert (d["w"], d["h"], d["min_x"], d["min_y"]) == tuple(F["islands"][slot, 1:])
        og = O.grids(isl, k)
        for name, v in rg.items():
            assert np.array_equal(og[name], v), (slot, name)


@need
def test_pack_and_remap_match_reference():
    F = np.load(REF)
    cfg = config_of(F["config"])
    assert np.array_equal(O.seeds(cfg["random_seed"], cfg["max_iterations"]), F["seeds"])
    r = O.run(F["uvs"], F["prim"], cfg, lambda s: F["draws"])
    assert r["loops_end"]
    assert not (r["packed"]["info"][:, 3] & O.DRAWS_EXHAUSTED).any()
    a = r["atlas"]
    assert [a["success"], a["width"], a["height"], a["placed"]] == F["atlas_i"].tolist()
    assert a["fitness"] == F["atlas_f"][0] and a["scaling"] == F["atlas_f"][1]
    assert np.array_equal(a["placements"], F["placements"])
    assert np.array_equal(r["uvs"].view(np.uint32), F["uvs_out"].view(np.uint32))


@need
def test_candidate_loop_check():
    """The reference's candidate loop can end for the fixture's islands; with one island it cannot
    (fewer aligned columns than the budget), and the oracle then lists every column and flags it."""
    F = np.load(REF)
    cfg = config_of(F["config"])
    c = O.extract_charts(F["uvs"], F["prim"])
    isl = O.create_islands(F["uvs"], c, cfg["grid_resolution"], cfg["margin_cells"])
    assert O.candidate_loops_end(isl, cfg)
    dims = [(int(d["w"]), int(d["h"])) for d in isl["islands"][isl["order"]]]
    assert O.loops_end_from_dims(dims, cfg)
    assert not O.loops_end_from_dims([(74, 74)], cfg)   # shelf 184, 14 aligned columns for a budget of 16
    small = int(np.argmin(isl["islands"]["w"]))
    assert not O.loops_end_from_dims([(int(isl["islands"][small]["w"]), int(isl["islands"][small]["h"]))], cfg)
    one = c["tri_chart"] == small
    keep = np.repeat(one, 3)
    uvs1, prim1 = F["uvs"][keep], F["prim"][keep]
    r = O.run(uvs1, prim1, cfg, lambda s: F["draws"])
    assert not r["loops_end"] and (r["packed"]["info"][:, 3] & O.CANDIDATE_LOOP_OPEN).all()
    assert r["atlas"]["success"] == 1


@need
def test_atlas_has_no_overlap():
    """The chosen placements' collision masks, written into the board, never overlap (the reference's
    own overlap check, GridUVPacker.cu:1316-1395, which reads its masks without their row stride)."""
    F = np.load(REF)
    cfg = config_of(F["config"])
    r = O.run(F["uvs"], F["prim"], cfg, lambda s: F["draws"])
    isl = r["islands"]
    board = np.zeros((cfg["grid_size"], cfg["grid_size"]), bool)
    for ii, x, y, rot in r["atlas"]["placements"]:
        g = O.grids(isl, ii)["collision90" if rot else "collision"]
        d = isl["islands"][ii]
        w = int(d["h"] if rot else d["w"])
        bits = np.unpackbits(g.view(np.uint8), bitorder="little").reshape(g.shape[0], -1)[:, :w].astype(bool)
        sub = board[y:y + bits.shape[0], x:x + w]
        assert not (sub & bits).any()
        sub |= bits


def test_config_defaults_match_reference():
    """PackingConfig() defaults (GridUVPacker.cuh:135-140) in the Python front end; no GPU."""
    from cudasdf_b200.uvpack import PackingConfig
    assert PackingConfig().as_dict() == dict(grid_size=128, grid_resolution=64, max_iterations=500, margin_cells=2,
                                             enable_rotation=1, x_alignment=8, max_candidates_per_island=32,
                                             max_drop_steps=0, shuffle_order_per_attempt=1, random_seed=0)
    assert PackingConfig.app().as_dict() == O.APP_CONFIG
