"""Batched extraction on the GPU: every scene's part of the batch's output equals the same scene
extracted alone by the engine (positions, colours and primitive ids bit for bit; identity indices
offset by the scene's first vertex), with direct launches and with the captured, autotuned graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _configs(n, seed=11):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import make_config
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        prims = S.random_scene(int(rng.integers(16, 300)), S.SEED_BASE + 900 + i)
        res = int(rng.choice([64, 72, 96, 128]))
        tech = int(i % 2)
        cfg = make_config(S.cell_size_for(res), technique=tech, out_mask=L.OUT_INDICES | L.OUT_COLORS | L.OUT_PRIMIDS,
                          dc_solver=L.DC_SOLVER_MASSPOINT if tech else L.DC_SOLVER_REFERENCE,
                          projection_iters=2 if tech else 0, adaptive_diagonal=1 if tech else 0)
        out.append((prims, cfg))
    return out


def _solo(prims, cfg):
    from cudasdf_b200.engine import Engine, MeshBuffers
    eng = Engine()
    eng.configure(cfg)
    eng.set_scene(prims)
    buf = MeshBuffers(2_000_000, cfg.out_mask)
    st = eng.extract(buf)
    V = int(st["total_vertices"])
    r = {"verts": buf.vertices[:V].cpu().numpy(), "colors": buf.colors[:V].cpu().numpy(),
         "primids": buf.primitive_ids[:V].cpu().numpy(), "indices": buf.indices[:V].cpu().numpy()}
    eng.close()
    return r


def _check(scenes, first, count, mc, dc, solos):
    for k, (prims, cfg) in enumerate(scenes):
        buf = dc if cfg.technique else mc
        f, c = int(first[k]), int(count[k])
        ref = solos[k]
        assert c == len(ref["verts"]), (k, c, len(ref["verts"]))
        got = buf.vertices[f:f + c].cpu().numpy()
        assert got.tobytes() == ref["verts"].tobytes(), f"scene {k}: positions"
        assert buf.colors[f:f + c].cpu().numpy().tobytes() == ref["colors"].tobytes(), f"scene {k}: colours"
        assert buf.primitive_ids[f:f + c].cpu().numpy().tobytes() == ref["primids"].tobytes(), f"scene {k}: ids"
        assert (buf.indices[f:f + c].cpu().numpy() - f == ref["indices"]).all(), f"scene {k}: indices"


def test_batch_matches_solo_extractions():
    from cudasdf_b200 import _lib as L
    from cudasdf_b200.engine import Batch, MeshBuffers
    scenes = _configs(12)
    solos = [_solo(p, c) for p, c in scenes]
    mask = L.OUT_INDICES | L.OUT_COLORS | L.OUT_PRIMIDS
    mc = MeshBuffers(8_000_000, mask)
    dc = MeshBuffers(8_000_000, mask)
    b = Batch()
    b.set_scenes(scenes, mask)
    first, count, st = b.extract(mc, dc)
    assert st["graph"] == 0 and st["scenes"] == 12
    _check(scenes, first, count, mc, dc, solos)
    # captured and autotuned: two replays in a row give the same meshes
    b.capture(mc, dc, tune=True)
    for _ in range(2):
        mc.vertices.zero_()
        dc.vertices.zero_()
        first2, count2, st2 = b.extract(mc, dc)
        assert st2["graph"] == 1
        assert (first2 == first).all() and (count2 == count).all()
        _check(scenes, first2, count2, mc, dc, solos)
    assert all(v in (0, 1, 2, 4) for v in st2["tuned_ctas"])
    b.close()


def test_batch_rejects_mixed_dc_options():
    from cudasdf_b200 import _lib as L
    from cudasdf_b200.engine import Batch
    scenes = _configs(4)
    scenes[3][1].projection_iters = 5  # the DC scenes of one batch share their options
    b = Batch()
    with pytest.raises(RuntimeError):
        b.set_scenes(scenes, L.OUT_INDICES)
    b.close()


def _sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _exclusive(x):
    out = np.zeros(len(x), np.uint64)
    out[1:] = np.cumsum(x.astype(np.uint64))[:-1]
    return out.astype(np.uint32)


def test_batch_benchmark_workload_matches_reference_digests():
    """The batched benchmark workload (256 scenes, primitive counts log-uniform in [16, 2048], grids from
    {64, 96, 128, 192, 256}^3, half marching cubes, half dual contouring with the reference's solver),
    extracted by the captured, autotuned graph, against digests of each scene run alone through the
    reference's own CUDA path (tests/golden/batch_c5.npz): per scene the active blocks, per-block vertex
    totals, VBO and EBO (as the scene's own identity indices), and for dual contouring the per-cell corner
    masks, cell-vertex offsets, cell vertices and quad-vertex counts with their scan."""
    import os

    from conftest import GOLDEN
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Batch, MeshBuffers, make_config
    path = os.path.join(GOLDEN, "batch_c5.npz")
    if not os.path.exists(path):
        pytest.skip("batch_c5.npz not generated")
    G = np.load(path)
    scn = S.batch_scenes(256)
    scenes = [(sc["primitives"], make_config(S.cell_size_for(sc["resolution"]), technique=sc["technique"],
                                             out_mask=L.OUT_INDICES)) for sc in scn]
    for k, sc in enumerate(scn):  # the generator still draws the scenes the digests were made of
        assert _sha(sc["primitives"]) == str(G["prims_sha"][k]) and sc["resolution"] == int(G["res"][k])
    tot = G["total_vertices"].astype(np.int64)
    tech = G["technique"]
    mc = MeshBuffers(int(tot[tech == 0].sum()) + 1024, L.OUT_INDICES)
    dc = MeshBuffers(int(tot[tech == 1].sum()) + 1024, L.OUT_INDICES)
    b = Batch()
    b.set_scenes(scenes, L.OUT_INDICES)
    b.capture(mc, dc, tune=True)
    first, count, st = b.extract(mc, dc)
    assert st["graph"] == 1
    lists = {t: b.read_buffer(t, 0, np.int32) for t in (0, 1)}
    totals = {t: b.read_buffer(t, 1, np.uint32) for t in (0, 1)}
    dcc = {"counts": b.read_buffer(1, 2, np.uint32), "mask": b.read_buffer(1, 3, np.uint8),
           "voff": b.read_buffer(1, 4, np.uint32), "vert": b.read_buffer(1, 5, np.uint16).reshape(-1, 4)}
    base = {0: 0, 1: 0}
    cell_vertex_base = 0
    bad = []
    for k, sc in enumerate(scn):
        t, res = int(tech[k]), sc["resolution"]
        nblocks = ((res + 7) // 8) ** 3
        lo, hi = base[t], base[t] + nblocks
        base[t] = hi
        lst = lists[t]
        sel = np.nonzero((lst >= lo) & (lst < hi))[0]
        a0, a1 = int(G["active_starts"][k]), int(G["active_starts"][k + 1])
        ok = len(sel) == a1 - a0 == int(G["active_count"][k])
        ok = ok and (sel.size == 0 or (np.diff(sel) == 1).all())  # one run of the sorted list
        ok = ok and (lst[sel] - lo == G["active"][a0:a1]).all() and (totals[t][sel] == G["block_totals"][a0:a1]).all()
        f, c = int(first[k]), int(count[k])
        ok = ok and c == int(tot[k])
        buf = dc if t else mc
        ok = ok and _sha(buf.vertices[f:f + c].cpu().numpy()) == str(G["verts_sha"][k])
        idx = buf.indices[f:f + c].cpu().numpy().astype(np.int64) - f
        ok = ok and _sha(idx.astype(np.uint32)) == str(G["indices_sha"][k])
        if t == 1 and sel.size:
            c0, c1 = int(sel[0]) * 512, (int(sel[-1]) + 1) * 512
            counts = dcc["counts"][c0:c1]
            ok = ok and _sha(counts) == str(G["counts_sha"][k]) and _sha(_exclusive(counts)) == str(G["offsets_sha"][k])
            ok = ok and _sha(dcc["mask"][c0:c1]) == str(G["dc_mask_sha"][k])
            voff = dcc["voff"][c0:c1].astype(np.int64) - cell_vertex_base
            ok = ok and _sha(voff.astype(np.uint32)) == str(G["dc_voff_sha"][k])
            nv = int(G["dc_vertices"][k])
            ok = ok and _sha(dcc["vert"][cell_vertex_base:cell_vertex_base + nv]) == str(G["dc_vert_sha"][k])
            cell_vertex_base += nv
        if not ok:
            bad.append(k)
    b.close()
    assert not bad, f"{len(bad)} scenes differ from the reference: {bad[:20]}"
