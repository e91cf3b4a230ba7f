"""ctypes binding of oracle/_ref/libsdfref.so: the reference's own CUDA path, built from its sources
by oracle/Makefile (target ``ref``), plus probe kernels over its __device__ functions.

Test infrastructure only: used by tests/ and by tests/golden/make_golden.py, never by the product.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libsdfref.so")

BVH_DTYPE = np.dtype([("min", "<f4", 3), ("max", "<f4", 3), ("left", "<i4"), ("right", "<i4")])
SDFGRID_BYTES = 232

# probe ids (oracle/ref/ref_probe.cu)
PR_SD, PR_XFORM, PR_TWIST, PR_BEND, PR_SINE, PR_MAP, PR_NORMAL, PR_EDGET, PR_LERP, PR_GETLOC = range(10)
PR_INTERP, PR_DEGEN, PR_SOLVE3, PR_QEFREG, PR_QEF, PR_ENCV, PR_DECV, PR_ENCN, PR_DECN, PR_AABBD = range(10, 20)

# ref_copy buffer ids
RB_ACTIVE, RB_COUNTS, RB_OFFSETS, RB_VERTS, RB_COLORS, RB_INDICES, RB_UVS, RB_PRIMIDS, RB_NORMALS = range(9)
RB_DCMASK, RB_DCVOFF, RB_DCVERT, RB_DCNORM, RB_B2A, RB_DCNORMTMP = range(9, 15)

OUT_COLORS, OUT_INDICES, OUT_UVS, OUT_PRIMIDS, OUT_NORMALS = 1, 2, 4, 8, 16
OUT_ALL = 31

_STATS_FIELDS = ["scoutCount", "activeUsed", "totalVertices", "error", "msScout", "msCount", "msScan1",
                 "msGenerate", "msBlockMap", "msMark", "msSolve", "msCountQuads", "msScan2", "msQuads",
                 "msTotalKernels", "msWall"]


class _Stats(ctypes.Structure):
    _fields_ = [("scoutCount", ctypes.c_int), ("activeUsed", ctypes.c_int), ("totalVertices", ctypes.c_uint),
                ("error", ctypes.c_int)] + [(f, ctypes.c_float) for f in _STATS_FIELDS[4:]]


def available() -> bool:
    return os.path.exists(LIB_PATH)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle ref)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, f, u, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_uint, ctypes.c_size_t
        L.ref_probe_run.argtypes = [i, i, vp, vp, vp, f]
        L.ref_probe_run.restype = i
        L.ref_create.argtypes = [f, vp, vp, i, u]
        L.ref_create.restype = vp
        L.ref_destroy.argtypes = [vp]
        L.ref_set_primitives.argtypes = [vp, vp, i]
        L.ref_set_primitives.restype = i
        L.ref_num_nodes.argtypes = [vp]
        L.ref_num_nodes.restype = i
        L.ref_get_nodes.argtypes = [vp, vp]
        L.ref_get_primitives.argtypes = [vp, vp]
        L.ref_get_grid.argtypes = [vp, vp]
        L.ref_run.argtypes = [vp, f, i, f, u, i, ctypes.POINTER(_Stats)]
        L.ref_run.restype = i
        L.ref_dc_normal_passes.argtypes = [vp, f, f]
        L.ref_dc_normal_passes.restype = i
        L.ref_copy.argtypes = [vp, i, vp, sz]
        L.ref_copy.restype = i
        L.ref_stats_size.restype = i
        L.ref_device_count.restype = i
        assert L.ref_stats_size() == ctypes.sizeof(_Stats)
        _lib = L
    return _lib


def probe_strides():
    return 96, 8


def probe(which: int, inputs: np.ndarray, grid: bytes | None = None, time: float = 0.0) -> np.ndarray:
    """Run a probe over float32 input records (n, 96); returns (n, 8) float32."""
    ins, outs = probe_strides()
    inp = np.ascontiguousarray(inputs, dtype=np.float32)
    assert inp.ndim == 2 and inp.shape[1] == ins
    n = inp.shape[0]
    out = np.zeros((n, outs), np.float32)
    gbuf = None
    if grid is not None:
        gbuf = ctypes.create_string_buffer(bytes(grid), SDFGRID_BYTES)
    rc = lib().ref_probe_run(which, n, inp.ctypes.data, out.ctypes.data,
                             ctypes.cast(gbuf, ctypes.c_void_p) if gbuf is not None else None, time)
    if rc != 0:
        raise RuntimeError(f"ref_probe_run({which}) failed with cudaError {rc}")
    return out


class RefMesh:
    """The reference pipeline (CudaSDFMesh::Update stage order) on the GPU, headless."""

    def __init__(self, cell_size: float, bmin=(-1.0, -1.0, -1.0), bmax=(1.0, 1.0, 1.0),
                 max_active_blocks: int = 0, max_vertices: int = 50_000_000):
        L = lib()
        bmin_a = np.asarray(bmin, np.float32)
        bmax_a = np.asarray(bmax, np.float32)
        self.h = L.ref_create(float(cell_size), bmin_a.ctypes.data, bmax_a.ctypes.data,
                              int(max_active_blocks), int(max_vertices))
        if not self.h:
            raise RuntimeError("ref_create failed")
        self.stats = None

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_primitives(self, prims: np.ndarray) -> int:
        p = np.ascontiguousarray(prims)
        return lib().ref_set_primitives(self.h, p.ctypes.data, len(p))

    def nodes(self) -> np.ndarray:
        n = lib().ref_num_nodes(self.h)
        out = np.zeros(n, BVH_DTYPE)
        if n:
            lib().ref_get_nodes(self.h, out.ctypes.data)
        return out

    def primitives(self, n: int, dtype) -> np.ndarray:
        out = np.zeros(n, dtype)
        lib().ref_get_primitives(self.h, out.ctypes.data)
        return out

    def grid_bytes(self) -> bytes:
        buf = ctypes.create_string_buffer(SDFGRID_BYTES)
        lib().ref_get_grid(self.h, buf)
        return buf.raw

    def grid_fields(self) -> dict:
        g = self.grid_bytes()
        i32 = np.frombuffer(g, np.int32)
        f32 = np.frombuffer(g, np.float32)
        return {"maxBlocks": int(i32[4]), "blocksDim": tuple(int(v) for v in i32[5:8]),
                "width": int(i32[8]), "height": int(i32[9]), "depth": int(i32[10]),
                "origin": tuple(float(v) for v in f32[11:14]), "cellSize": float(f32[14]),
                "maxVertices": int(np.frombuffer(g, np.uint32)[52])}

    def run(self, time: float = 0.0, technique: int = 0, qef_blend: float = 1.0, out_mask: int = OUT_ALL,
            sort_active: bool = True) -> dict:
        st = _Stats()
        rc = lib().ref_run(self.h, float(time), int(technique), float(qef_blend), int(out_mask),
                           1 if sort_active else 0, ctypes.byref(st))
        self.stats = {f: getattr(st, f) for f in _STATS_FIELDS}
        if rc != 0:
            raise RuntimeError(f"reference pipeline failed with cudaError {rc}")
        return self.stats

    def dc_normal_passes(self, time: float, cos_angle: float) -> None:
        rc = lib().ref_dc_normal_passes(self.h, float(time), float(cos_angle))
        if rc != 0:
            raise RuntimeError(f"reference DC normal passes failed with cudaError {rc}")

    def copy(self, buf: int, dtype, count: int) -> np.ndarray:
        dt = np.dtype(dtype)
        out = np.zeros(count, dt)
        if count == 0:
            return out
        rc = lib().ref_copy(self.h, int(buf), out.ctypes.data, out.nbytes)
        if rc != 0:
            raise RuntimeError(f"ref_copy({buf}) failed: {rc}")
        return out
