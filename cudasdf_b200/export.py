"""Wavefront OBJ export of an extracted mesh through the C ABI (``sdf_write_obj``).

The file format is the reference's ExportMeshToOBJ (src/main.cpp:1043-1115): the soup is written as
consecutive triangles; an indexed (SDF_OUT_WELDED) mesh is written with its index buffer.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib as L


def _host(a, dtype, cols):
    if a is None:
        return None
    if hasattr(a, "detach"):  # a torch tensor, possibly on the device
        a = a.detach().cpu().numpy()
    a = np.ascontiguousarray(np.asarray(a, dtype=dtype))
    if cols and (a.ndim != 2 or a.shape[1] != cols):
        raise ValueError(f"expected an (n, {cols}) array, got shape {a.shape}")
    return a


def write_obj(path: str | os.PathLike, vertices, indices=None, uvs=None) -> None:
    """Writes ``vertices`` ((n, 4) float32, the VBO layout), optional ``uvs`` ((n, 2) float32) and
    optional ``indices`` (uint32, 3 per triangle) to ``path`` as OBJ text. Raises RuntimeError when the
    library refuses (no vertices, an index out of range, a file that cannot be written)."""
    v = _host(vertices, np.float32, 4)
    uv = _host(uvs, np.float32, 2)
    ix = _host(indices, np.uint32, 0)
    if ix is not None:
        ix = ix.reshape(-1)
    if uv is not None and len(uv) < len(v):
        raise ValueError("uvs must have one entry per vertex")
    st = L.lib().sdf_write_obj(os.fsencode(os.fspath(path)), v.ctypes.data_as(ctypes.c_void_p), len(v),
                               None if ix is None else ix.ctypes.data_as(ctypes.c_void_p),
                               0 if ix is None else len(ix),
                               None if uv is None else uv.ctypes.data_as(ctypes.c_void_p))
    L.check(st, f"sdf_write_obj({os.fspath(path)})")
