"""The C ABI library loads without a GPU and exports every symbol include/sdfmesh_b200.h declares."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "sdfmesh_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:unsigned\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s+\**([A-Za-z_][A-Za-z0-9_]*)\s*\(", text, re.M)
    return sorted(set(n for n in names if n not in ("if", "return")))


def test_header_declares_the_reference_launchers():
    names = declared_functions()
    for n in ["launchScoutActiveBlocks", "launchCountActiveBlockTriangles", "launchGenerateActiveBlockTriangles",
              "launchBuildBlockToActiveMap", "launchDCMarkCells", "launchDCSolveCellVertices",
              "launchDCRecomputeNormalsAtVertices", "launchDCSmoothCellNormals", "launchDCCountQuads",
              "launchDCGenerateQuads", "getScanStorageSize", "launchScan"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    from cudasdf_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libsdfmesh_b200.so not built")
    L = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert set(_lib.DROPIN_SYMBOLS + _lib.ENGINE_SYMBOLS + _lib.SURROGATE_SYMBOLS + _lib.BATCH_SYMBOLS +
               _lib.STATIC_SCOUT_SYMBOLS + _lib.EXPORT_SYMBOLS + _lib.UVPACK_SYMBOLS) <= set(declared_functions())
    assert L.sdf_version().startswith(b"sdfmesh_b200")


def test_struct_layouts_match_reference():
    from cudasdf_b200 import _lib
    from cudasdf_b200.scenes import PRIM_DTYPE
    assert ctypes.sizeof(_lib.SdfGrid) == 232
    assert _lib.SdfGrid.cellSize.offset == 56 and _lib.SdfGrid.d_primitives.offset == 64
    assert _lib.SdfGrid.d_vertices.offset == 160 and _lib.SdfGrid.maxVertices.offset == 208
    assert PRIM_DTYPE.itemsize == 160 and PRIM_DTYPE.fields["type"][1] == 104


def test_header_compiles_as_c():
    """The header is plain C11, and its structs have the sizes the Python bindings assume."""
    import subprocess
    import tempfile

    from cudasdf_b200 import _lib
    structs = {"sdf_config": _lib.SdfConfig, "sdf_outputs": _lib.SdfOutputs, "sdf_stats": _lib.SdfStats,
               "sdf_surrogate_config": _lib.SurrogateConfig, "sdf_surrogate_stats": _lib.SurrogateStats,
               "sdf_grid": _lib.SdfGrid, "sdf_batch_scene": _lib.BatchScene, "sdf_batch_stats": _lib.BatchStats,
               "sdf_uv_pack_config": _lib.UvPackConfig, "sdf_uv_chart": _lib.UvChart, "sdf_uv_grid": _lib.UvGrid,
               "sdf_uv_island": _lib.UvIsland, "sdf_uv_placement": _lib.UvPlacement,
               "sdf_uv_solution": _lib.UvSolution, "sdf_uv_atlas_info": _lib.UvAtlasInfo}
    body = "".join(f'printf("%zu\\n", sizeof({n}));' for n in structs)
    src = ('#include <stdio.h>\n#include "sdfmesh_b200.h"\n'
           'int main(void){ if (sizeof(sdf_primitive) != 160) return 1; ' + body + ' return 0; }\n')
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        r = subprocess.run(["/usr/bin/gcc", "-std=c11", "-Wall", "-I", os.path.dirname(HEADER), c, "-o",
                            os.path.join(d, "t")], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        out = subprocess.run([os.path.join(d, "t")], capture_output=True, text=True)
        assert out.returncode == 0
        sizes = [int(x) for x in out.stdout.split()]
        assert sizes == [ctypes.sizeof(t) for t in structs.values()], dict(zip(structs, sizes))


def test_c_host_links_and_writes_obj():
    """A C program links the library and calls it through the header alone: the version string and
    the OBJ writer (host memory only, so no GPU is needed); the file matches the restatement of the
    reference's writer."""
    import subprocess
    import tempfile

    import numpy as np

    from cudasdf_b200 import _lib
    from oracle import obj_oracle
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libsdfmesh_b200.so not built")
    src = r'''
#include <stdio.h>
#include <string.h>
#include "sdfmesh_b200.h"
int main(int argc, char** argv) {
    sdf_float4 v[6];
    sdf_float2 uv[6];
    for (int i = 0; i < 6; ++i) {
        v[i].x = 0.125f * i; v[i].y = -1.5f + i; v[i].z = 1e-5f * (i + 1); v[i].w = 1.f;
        uv[i].x = 0.1f * i; uv[i].y = 1.f - 0.1f * i;
    }
    const uint32_t idx[6] = {0, 1, 2, 2, 1, 5};
    if (strncmp(sdf_version(), "sdfmesh_b200", 12) != 0) return 2;
    if (sdf_write_obj(argv[1], v, 6, NULL, 0, uv) != SDF_OK) return 3;
    if (sdf_write_obj(argv[2], v, 6, idx, 6, NULL) != SDF_OK) return 4;
    if (sdf_write_obj(argv[2], v, 5, idx, 6, NULL) != SDF_ERR_INVALID) return 5;  /* index 5 of 5 vertices */
    return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c, exe = os.path.join(d, "host.c"), os.path.join(d, "host")
        open(c, "w").write(src)
        libdir = os.path.dirname(_lib.LIB_PATH)
        r = subprocess.run(["/usr/bin/gcc", "-std=c11", "-Wall", "-I", os.path.dirname(HEADER), c, "-o", exe,
                            "-L", libdir, "-lsdfmesh_b200", "-Wl,-rpath," + libdir], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        soup, indexed = os.path.join(d, "soup.obj"), os.path.join(d, "indexed.obj")
        out = subprocess.run([exe, soup, indexed], capture_output=True, text=True)
        assert out.returncode == 0, (out.returncode, out.stderr)
        i = np.arange(6, dtype=np.float32)
        v = np.stack([np.float32(0.125) * i, np.float32(-1.5) + i, np.float32(1e-5) * (i + 1), np.ones(6, np.float32)], 1)
        uv = np.stack([np.float32(0.1) * i, np.float32(1.0) - np.float32(0.1) * i], 1)
        assert open(soup, "rb").read() == obj_oracle.obj_text("soup.obj", v, uv)
        assert open(indexed, "rb").read() == obj_oracle.obj_text("indexed.obj", v, None,
                                                                np.array([0, 1, 2, 2, 1, 5], np.uint32))


def test_static_scout_limit_and_error_status_without_a_device():
    """The header states the allocation-free scout's limit, and without a usable CUDA device the entry
    point reports SDF_ERR_CUDA (never SDF_OK with its outputs unwritten)."""
    from conftest import cuda_available
    from cudasdf_b200 import _lib
    text = open(HEADER).read()
    m = re.search(r"#define\s+SDF_SCOUT_STATIC_MAX_BLOCKS\s+(\d+)u", text)
    assert m and int(m.group(1)) == _lib.SCOUT_STATIC_MAX_BLOCKS
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libsdfmesh_b200.so not built")
    if cuda_available():
        pytest.skip("a CUDA device is present: the GPU tests cover the call")
    L = _lib.lib()
    grid = _lib.SdfGrid()
    grid.blocksDim[0], grid.blocksDim[1], grid.blocksDim[2] = 4, 4, 4
    grid.d_activeBlocks = 1  # never dereferenced on the host
    grid.d_activeBlockCount = 1
    assert L.sdf_scout_active_blocks_static(ctypes.byref(grid), 0.0) == _lib.SDF_ERR_CUDA
