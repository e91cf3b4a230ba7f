"""CPU restatement of the reference's OBJ export (src/main.cpp:1043-1115, ExportMeshToOBJ).

TEST INFRASTRUCTURE: only tests/ use it, as the checker of the library's sdf_write_obj.

The reference streams floats through std::ofstream with default flags, which formats as printf's
"%g" with six significant digits; Python's "%g" operator follows the same C rules for finite values.
"""
from __future__ import annotations

import os

import numpy as np


def obj_text(file_name: str, vertices: np.ndarray, uvs: np.ndarray | None = None,
             indices: np.ndarray | None = None) -> bytes:
    """The bytes the reference writes for this mesh (main.cpp:1059-1111). ``file_name`` is the name
    written on the "# Generated:" line (the reference writes its own timestamped file name there).
    ``indices`` None: the soup of the reference, face k = vertices 3k..3k+2 (main.cpp:1099-1111)."""
    out = ["# Exported from CudaSDF\n", f"# Generated: {file_name}\n", "\n"]  # main.cpp:1059-1061
    n = len(vertices)
    if n == 0:  # main.cpp:1066-1070: header only
        return "".join(out).encode()
    v = np.asarray(vertices, dtype=np.float32)
    for i in range(n):  # main.cpp:1087-1090
        out.append("v %g %g %g\n" % (float(v[i, 0]), float(v[i, 1]), float(v[i, 2])))
    out.append("\n")
    if uvs is not None:  # main.cpp:1093-1098
        t = np.asarray(uvs, dtype=np.float32)
        for i in range(n):
            out.append("vt %g %g\n" % (float(t[i, 0]), float(t[i, 1])))
        out.append("\n")
    if indices is None:
        faces = np.arange(n - n % 3, dtype=np.int64).reshape(-1, 3)
    else:
        ix = np.asarray(indices, dtype=np.int64).reshape(-1)
        faces = ix[: len(ix) - len(ix) % 3].reshape(-1, 3)
    for a, b, c in (faces + 1).tolist():  # main.cpp:1101-1111, 1-based
        out.append(f"f {a}/{a} {b}/{b} {c}/{c}\n" if uvs is not None else f"f {a} {b} {c}\n")
    return "".join(out).encode()


def write_obj(path: str, vertices, uvs=None, indices=None) -> None:
    with open(path, "wb") as f:
        f.write(obj_text(os.path.basename(path), vertices, uvs, indices))
