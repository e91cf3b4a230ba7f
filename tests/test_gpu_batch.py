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
