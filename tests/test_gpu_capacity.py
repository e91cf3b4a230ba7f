"""The engine's per-active-block buffers are sized by the active blocks, not by every block of the grid:
they start at a sixteenth of the blocks, and an extraction that finds more active blocks grows them and
runs again, with the same mesh as the reference's recorded run."""
import ctypes

import numpy as np
import pytest

import gpu_helpers as H

pytestmark = pytest.mark.gpu


def _rows_bytes(eng):
    n = ctypes.c_size_t(0)
    eng._lib.sdf_engine_buffer(eng.h, 8, ctypes.byref(n))
    return n.value


@pytest.mark.parametrize("technique,name", [(0, "full_mc_c2"), (1, "full_dc_c2")])
def test_buffers_grow_with_the_active_blocks(technique, name):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    G = H.load(name)
    st = H.stats_of(G)
    eng = Engine()
    eng.configure(make_config(S.cell_size_for(256), technique=technique, out_mask=int(G["out_mask"])))
    eng.set_scene(S.config_scene(2))
    row = 736 * 4
    nblocks = 32 ** 3
    assert _rows_bytes(eng) == max(4096, nblocks // 16) * row  # a 4,096-block start, fewer than the 12,524 active
    buf = MeshBuffers(st["totalVertices"] + 1024, int(G["out_mask"]))
    out = eng.extract(buf)
    assert out["active_blocks"] == st["activeUsed"] and out["total_vertices"] == st["totalVertices"]
    assert _rows_bytes(eng) >= st["activeUsed"] * row
    V = st["totalVertices"]
    assert H.sha(buf.vertices[:V].cpu().numpy()) == str(G["verts_sha"])
    # the next extraction runs once, in the grown buffers, to the same mesh
    grown = _rows_bytes(eng)
    buf.vertices.zero_()
    again = eng.extract(buf)
    assert again["total_vertices"] == V and _rows_bytes(eng) == grown
    assert H.sha(buf.vertices[:V].cpu().numpy()) == str(G["verts_sha"])
    eng.close()
