"""The allocation-free scout, sdf_scout_active_blocks_static, against launchScoutActiveBlocks.

Some callers cannot let a library allocate device memory while they run (a per-frame render loop or a
plugin host that forbids cudaMalloc/cudaFree, which synchronise the device and can fail under the
host's fixed budget, or an application that owns every allocation through its own allocator). The
static entry point keeps its working memory in one fixed device array instead. This file is named to
be collected last, so a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _prepared_mesh(prims, res):
    """A drop-in mesh whose grid has its scene on the device (one full Update)."""
    import torch

    from cudasdf_b200 import scenes as S
    from cudasdf_b200.dropin import CudaSDFMesh
    mesh = CudaSDFMesh(max_active_blocks=1 << 30, max_vertices=1 << 21)
    mesh.Initialize(S.cell_size_for(res), S.BOUNDS_MIN, S.BOUNDS_MAX)
    for p in prims:
        mesh.AddPrimitive(p)
    verts = torch.empty((1 << 21, 4), dtype=torch.float32, device="cuda")
    mesh.Update(0.0, verts)
    return mesh


def _outputs(mesh):
    import torch
    torch.cuda.synchronize()
    n = int(mesh._bufs["activeBlockCount"].item())
    return n, mesh._bufs["activeBlocks"][:n].cpu().numpy().copy()


@pytest.mark.parametrize("config,res", [(2, 128), (3, 512)])
def test_static_scout_matches_allocating_scout_twice(config, res):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    lib = L.lib()
    mesh = _prepared_mesh(S.config_scene(config), res)
    g = ctypes.byref(mesh.grid)
    lib.sdf_last_error()
    lib.launchScoutActiveBlocks(g, 0.0)
    n_ref, ref = _outputs(mesh)
    assert n_ref > 0
    for _ in range(2):  # two calls in a row: the shared array must not carry state between them
        mesh._bufs["activeBlocks"].fill_(-7)
        mesh._bufs["activeBlockCount"].fill_(-7)
        rc = lib.sdf_scout_active_blocks_static(g, 0.0)
        assert rc == L.SDF_OK, L.STATUS_NAMES.get(rc, rc)
        n, got = _outputs(mesh)
        assert n == n_ref
        assert (got == ref).all()
    assert lib.sdf_last_error() == 0


def test_static_scout_rejects_grids_beyond_its_limit():
    from cudasdf_b200 import _lib as L
    lib = L.lib()
    limit = L.SCOUT_STATIC_MAX_BLOCKS
    grid = L.SdfGrid()
    grid.blocksDim[0], grid.blocksDim[1], grid.blocksDim[2] = 128, 128, 128  # 2,097,152 blocks
    assert 128 ** 3 > limit
    grid.d_activeBlocks = 1
    grid.d_activeBlockCount = 1
    assert lib.sdf_scout_active_blocks_static(ctypes.byref(grid), 0.0) == L.SDF_ERR_CAPACITY
