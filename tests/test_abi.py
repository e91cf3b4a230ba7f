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
               _lib.STATIC_SCOUT_SYMBOLS + _lib.EXPORT_SYMBOLS) <= set(declared_functions())
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
               "sdf_grid": _lib.SdfGrid, "sdf_batch_scene": _lib.BatchScene, "sdf_batch_stats": _lib.BatchStats}
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
