"""OBJ export (sdf_write_obj) against the restatement of the reference's ExportMeshToOBJ
(src/main.cpp:1043-1115): byte-identical files for soups, UVs and indexed meshes."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import obj_oracle as OO


def _lib_or_skip():
    from cudasdf_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libsdfmesh_b200.so not built")
    return _lib


def _edge_floats(rng, n):
    """float32 values that exercise %g: exponents switching to scientific notation, trailing-zero
    removal, rounding to six digits, negative zero, denormals, extremes."""
    special = np.array([0.0, -0.0, 1.0, -1.0, 0.1, 1e-5, 1e-4, 9.999995e-5, 123456.0, 1234567.0, 999999.5,
                        3.4028235e38, -3.4028235e38, 1.17549435e-38, 1e-45, 0.5, 2.5e-7, -1.1, 1.1],
                       dtype=np.float32)
    r = np.concatenate([rng.standard_normal(n).astype(np.float32),
                        (rng.standard_normal(n) * 10.0 ** rng.integers(-12, 12, n)).astype(np.float32),
                        rng.integers(-1000, 1000, n).astype(np.float32)])
    return np.concatenate([special, r])


def test_ostream_default_float_format_is_printf_g():
    """Pins the oracle's formatting claim: std::ostream << float with default flags prints what
    printf("%g") prints (the reference writes every coordinate that way, main.cpp:1088)."""
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    import tempfile
    vals = _edge_floats(np.random.default_rng(7), 300)
    src = ("#include <iostream>\n#include <cstdio>\n#include <cstring>\n"
           "int main(){unsigned u; while (std::scanf(\"%x\", &u) == 1) { float f; std::memcpy(&f, &u, 4);"
           " std::cout << f << \"\\n\"; } return 0; }\n")
    with tempfile.TemporaryDirectory() as d:
        cpp, exe = os.path.join(d, "fmt.cpp"), os.path.join(d, "fmt")
        open(cpp, "w").write(src)
        subprocess.run([gxx, "-O1", cpp, "-o", exe], check=True)
        inp = "\n".join("%08x" % u for u in vals.view(np.uint32)) + "\n"
        got = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout.splitlines()
    assert got == ["%g" % float(v) for v in vals]


def _mesh(rng, n):
    v = np.zeros((n, 4), np.float32)
    vals = _edge_floats(rng, n)
    v[:, :3] = rng.choice(vals, (n, 3))
    v[:, 3] = 1.0
    uv = rng.choice(vals, (n, 2)).astype(np.float32)
    return v, uv


@pytest.mark.parametrize("n", [3, 30, 9000, 300_003])
def test_soup_matches_oracle(tmp_path, n):
    _lib_or_skip()
    from cudasdf_b200.export import write_obj
    v, uv = _mesh(np.random.default_rng(n), n)
    for with_uv in (False, True):
        p = tmp_path / f"mesh_{n}_{with_uv}.obj"
        write_obj(p, v, uvs=uv if with_uv else None)
        assert p.read_bytes() == OO.obj_text(p.name, v, uv if with_uv else None)


def test_indexed_matches_oracle(tmp_path):
    _lib_or_skip()
    from cudasdf_b200.export import write_obj
    rng = np.random.default_rng(3)
    v, uv = _mesh(rng, 5000)
    ix = rng.integers(0, 5000, 3 * 40_000).astype(np.uint32)
    for with_uv in (False, True):
        p = tmp_path / f"welded_{with_uv}.obj"
        write_obj(p, v, indices=ix, uvs=uv if with_uv else None)
        assert p.read_bytes() == OO.obj_text(p.name, v, uv if with_uv else None, ix)


def test_ragged_soup_drops_the_partial_triangle(tmp_path):
    _lib_or_skip()
    from cudasdf_b200.export import write_obj
    v, _ = _mesh(np.random.default_rng(1), 7)
    p = tmp_path / "ragged.obj"
    write_obj(p, v)
    text = p.read_bytes()
    assert text == OO.obj_text(p.name, v)
    assert text.count(b"\nf ") == 2 and text.count(b"\nv ") == 7


def test_errors(tmp_path):
    L = _lib_or_skip()
    from cudasdf_b200.export import write_obj
    v, _ = _mesh(np.random.default_rng(2), 6)
    with pytest.raises(RuntimeError):  # an index names a vertex that does not exist
        write_obj(tmp_path / "bad.obj", v, indices=np.array([0, 1, 6], np.uint32))
    with pytest.raises(RuntimeError):  # a directory that does not exist
        write_obj(tmp_path / "no" / "such" / "dir.obj", v)
    p = tmp_path / "empty.obj"
    with pytest.raises(RuntimeError):  # the reference reports the empty mesh and leaves the header
        write_obj(p, np.zeros((0, 4), np.float32))
    assert p.read_bytes() == OO.obj_text(p.name, np.zeros((0, 4), np.float32))
    assert L.lib().sdf_write_obj(None, None, 0, None, 0, None) == L.SDF_ERR_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("welded", [False, True])
def test_extracted_mesh_exports_like_the_reference(tmp_path, welded):
    """A mesh extracted on the GPU (a 64-primitive composite scene with UVs, or the welded output),
    read back and written through the library, gives the bytes of the reference's writer."""
    import gpu_helpers as H
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.export import write_obj
    prims = S.random_scene(64, seed=11)
    if welded:
        from test_gpu_welded import welded_run
        r = welded_run(prims, 128)
        v, ix, uv = r["verts"], r["indices"], None
    else:
        r = H.engine_run(prims, 128, L.TECH_MC, L.OUT_UVS, debug=False)
        v, ix, uv = r["verts"], None, r["uvs"]
    assert len(v) > 1000
    p = tmp_path / "mesh_export.obj"
    write_obj(p, v, indices=ix, uvs=uv)
    assert p.read_bytes() == OO.obj_text(p.name, v, uv, ix)


def test_torch_tensors_and_shapes(tmp_path):
    """write_obj takes torch tensors like numpy arrays, and refuses arrays of the wrong shape."""
    _lib_or_skip()
    import torch
    from cudasdf_b200.export import write_obj
    v, uv = _mesh(np.random.default_rng(5), 300)
    ix = np.random.default_rng(6).integers(0, 300, 600).astype(np.uint32)
    p = tmp_path / "torch.obj"
    write_obj(p, torch.from_numpy(v), indices=torch.from_numpy(ix.view(np.int32)), uvs=torch.from_numpy(uv))
    assert p.read_bytes() == OO.obj_text(p.name, v, uv, ix)
    with pytest.raises(ValueError):
        write_obj(tmp_path / "bad.obj", v[:, :3])
    with pytest.raises(ValueError):
        write_obj(tmp_path / "bad.obj", v, uvs=uv[:10])


def _comma_decimal_locale(d):
    """Builds a locale whose LC_NUMERIC decimal point is ',' under directory d (for LOCPATH), from a
    generated ASCII charmap; None when localedef is missing or fails."""
    localedef = shutil.which("localedef")
    if localedef is None:
        return None
    cm = os.path.join(d, "ascii.cm")
    with open(cm, "w") as f:
        f.write("<code_set_name> ASCII_TEST\n<mb_cur_max> 1\n<mb_cur_min> 1\nCHARMAP\n")
        f.writelines(f"<U{i:04X}> /x{i:02x} CHAR{i}\n" for i in range(128))
        f.write("END CHARMAP\n")
    src = os.path.join(d, "comma.def")
    with open(src, "w") as f:
        f.write('LC_NUMERIC\ndecimal_point ","\nthousands_sep ""\ngrouping -1\nEND LC_NUMERIC\n')
    subprocess.run([localedef, "-c", "-f", cm, "-i", src, os.path.join(d, "comma_decimal")],
                   capture_output=True)
    return "comma_decimal" if os.path.isdir(os.path.join(d, "comma_decimal")) else None


def test_comma_decimal_locale_does_not_change_the_file():
    """A host application that switched the process to a comma-decimal locale (setlocale(LC_ALL, ...))
    still gets the reference's bytes: the writer's number formatting ignores LC_NUMERIC."""
    import tempfile
    L = _lib_or_skip()
    gcc = shutil.which("gcc") or "/usr/bin/gcc"
    with tempfile.TemporaryDirectory() as d:
        name = _comma_decimal_locale(d)
        if name is None:
            pytest.skip("no way to build a comma-decimal locale here")
        src = r'''
#include <locale.h>
#include <stdio.h>
#include <string.h>
#include "sdfmesh_b200.h"
int main(int argc, char** argv) {
    if (!setlocale(LC_ALL, argv[2])) return 2;
    char probe[32];
    snprintf(probe, sizeof probe, "%g", 0.5);
    if (strcmp(probe, "0,5") != 0) return 3;  /* the locale is in force for printf */
    sdf_float4 v[6];
    sdf_float2 uv[6];
    for (int i = 0; i < 6; ++i) {
        v[i].x = 0.125f * i - 0.5f; v[i].y = 1.5f + i; v[i].z = 1e-5f * (i + 1); v[i].w = 1.f;
        uv[i].x = 0.1f * i; uv[i].y = 1.f - 0.25f * i;
    }
    return sdf_write_obj(argv[1], v, 6, NULL, 0, uv) == SDF_OK ? 0 : 4;
}
'''
        c, exe = os.path.join(d, "host.c"), os.path.join(d, "host")
        open(c, "w").write(src)
        libdir = os.path.dirname(L.LIB_PATH)
        inc = os.path.join(os.path.dirname(libdir), "include")
        r = subprocess.run([gcc, "-std=c11", "-Wall", "-I", inc, c, "-o", exe, "-L", libdir, "-lsdfmesh_b200",
                            "-Wl,-rpath," + libdir], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        path = os.path.join(d, "comma.obj")
        out = subprocess.run([exe, path, name], capture_output=True, text=True, env=dict(os.environ, LOCPATH=d))
        assert out.returncode == 0, (out.returncode, out.stderr)
        i = np.arange(6, dtype=np.float32)
        v = np.stack([np.float32(0.125) * i - np.float32(0.5), np.float32(1.5) + i, np.float32(1e-5) * (i + 1),
                      np.ones(6, np.float32)], 1)
        uv = np.stack([np.float32(0.1) * i, np.float32(1.0) - np.float32(0.25) * i], 1)
        got = open(path, "rb").read()
        assert b"," not in got
        assert got == OO.obj_text("comma.obj", v, uv)
