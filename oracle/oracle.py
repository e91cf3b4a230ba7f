"""ctypes binding of oracle/liboracle.so, the CPU restatement of the reference algorithm.

TEST INFRASTRUCTURE: only tests/, the smoke check and bench.py's CPU-baseline leg use it, and only
as the checker (or the timed CPU baseline), never as the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

NODE_DTYPE = np.dtype([("min", "<f4", 3), ("max", "<f4", 3), ("left", "<i4"), ("right", "<i4")])
OR_COLORS, OR_INDICES, OR_UVS, OR_PRIMIDS, OR_NORMALS = 1, 2, 4, 8, 16
ORB_ACTIVE, ORB_COUNTS, ORB_OFFSETS, ORB_VERTS, ORB_COLORS, ORB_INDICES, ORB_UVS, ORB_PRIMIDS = range(8)
ORB_NORMALS, ORB_DCMASK, ORB_DCVOFF, ORB_DCVERT, ORB_DCNORM = range(8, 13)


class _Scene(ctypes.Structure):
    _fields_ = [("prims", ctypes.c_void_p), ("nprims", ctypes.c_int32), ("nbvh", ctypes.c_int32),
                ("nodes", ctypes.c_void_p), ("nnodes", ctypes.c_int32)]


class _Grid(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("depth", ctypes.c_uint32),
                ("bx", ctypes.c_int32), ("by", ctypes.c_int32), ("bz", ctypes.c_int32),
                ("origin", ctypes.c_float * 3), ("cell", ctypes.c_float)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        L = ctypes.CDLL(LIB_PATH)
        vp, i, f, u, i64, sz = (ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_uint32, ctypes.c_int64,
                                ctypes.c_size_t)
        L.or_grid_init.argtypes = [ctypes.POINTER(_Grid), f, vp, vp]
        L.or_build_scene.argtypes = [vp, i, vp, vp, vp]
        L.or_build_scene.restype = i
        L.or_map_batch.argtypes = [ctypes.POINTER(_Scene), i, vp, f, vp, vp]
        L.or_normal_batch.argtypes = [ctypes.POINTER(_Scene), i, vp, f, f, vp]
        L.or_probe.argtypes = [i, i, vp, i, vp, i]
        L.or_run.argtypes = [ctypes.POINTER(_Scene), ctypes.POINTER(_Grid), f, i, f, u, u, i]
        L.or_run.restype = vp
        L.or_result_sizes.argtypes = [vp, vp]
        L.or_result_copy.argtypes = [vp, i, vp, sz]
        L.or_result_copy.restype = i
        L.or_result_free.argtypes = [vp]
        L.or_scout_range.argtypes = [ctypes.POINTER(_Scene), ctypes.POINTER(_Grid), f, i64, i64, i]
        L.or_scout_range.restype = i64
        L.or_scout_flags.argtypes = [ctypes.POINTER(_Scene), ctypes.POINTER(_Grid), f, vp, i, vp, i]
        L.or_mc_blocks.argtypes = [ctypes.POINTER(_Scene), ctypes.POINTER(_Grid), f, vp, i, i]
        L.or_mc_blocks.restype = i64
        L.or_exclusive_scan.argtypes = [vp, vp, i64]
        _lib = L
    return _lib


class Scene:
    """A scene prepared the reference's way: unions first, BVH over the unions."""

    def __init__(self, prims: np.ndarray):
        prims = np.ascontiguousarray(prims)
        n = len(prims)
        self.sorted = np.zeros(n, prims.dtype)
        self.nodes = np.zeros(max(2 * n, 1), NODE_DTYPE)
        nb = ctypes.c_int(0)
        nn = lib().or_build_scene(prims.ctypes.data, n, self.sorted.ctypes.data, self.nodes.ctypes.data,
                                  ctypes.byref(nb))
        self.nodes = self.nodes[:nn].copy()
        self.nbvh = nb.value
        self._c = _Scene(self.sorted.ctypes.data, n, self.nbvh, self.nodes.ctypes.data if nn else None, nn)

    def map(self, pts: np.ndarray, time: float = 0.0):
        p = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        out = np.zeros((len(p), 8), np.float32)
        iters = np.zeros(len(p), np.int32)
        lib().or_map_batch(ctypes.byref(self._c), len(p), p.ctypes.data, float(time), out.ctypes.data,
                           iters.ctypes.data)
        return out, iters

    def normals(self, pts: np.ndarray, cell: float, time: float = 0.0):
        p = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        out = np.zeros((len(p), 3), np.float32)
        lib().or_normal_batch(ctypes.byref(self._c), len(p), p.ctypes.data, float(time), float(cell),
                              out.ctypes.data)
        return out


def make_grid(cell: float, bmin=(-1.0, -1.0, -1.0), bmax=(1.0, 1.0, 1.0)) -> _Grid:
    g = _Grid()
    a = np.asarray(bmin, np.float32)
    b = np.asarray(bmax, np.float32)
    lib().or_grid_init(ctypes.byref(g), float(cell), a.ctypes.data, b.ctypes.data)
    return g


def probe(which: int, inputs: np.ndarray, in_stride: int = 96, out_stride: int = 8) -> np.ndarray:
    inp = np.zeros((len(inputs), in_stride), np.float32)
    inp[:, :inputs.shape[1]] = inputs
    out = np.zeros((len(inputs), out_stride), np.float32)
    lib().or_probe(which, len(inputs), inp.ctypes.data, in_stride, out.ctypes.data, out_stride)
    return out


def run(scene: Scene, grid: _Grid, time: float = 0.0, technique: int = 0, qef_blend: float = 1.0,
        out_mask: int = 31, max_vertices: int = 50_000_000, nthreads: int = 0) -> dict:
    L = lib()
    h = L.or_run(ctypes.byref(scene._c), ctypes.byref(grid), float(time), int(technique), float(qef_blend),
                 int(out_mask), int(max_vertices), int(nthreads))
    try:
        sz = np.zeros(4, np.int64)
        L.or_result_sizes(h, sz.ctypes.data)
        nA, V, nDC, scout = (int(v) for v in sz)

        def get(buf, dtype, shape):
            a = np.zeros(shape, dtype)
            if a.size:
                rc = L.or_result_copy(h, buf, a.ctypes.data, a.nbytes)
                if rc != 0:
                    return None
            return a

        out = {"nActive": nA, "totalVertices": V, "nDcVerts": nDC, "scoutCount": scout,
               "active": get(ORB_ACTIVE, np.int32, nA), "counts": get(ORB_COUNTS, np.uint32, nA * 512),
               "offsets": get(ORB_OFFSETS, np.uint32, nA * 512), "verts": get(ORB_VERTS, np.float32, (V, 4))}
        if out_mask & OR_COLORS:
            out["colors"] = get(ORB_COLORS, np.float32, (V, 4))
        if out_mask & OR_INDICES:
            out["indices"] = get(ORB_INDICES, np.uint32, V)
        if out_mask & OR_UVS:
            out["uvs"] = get(ORB_UVS, np.float32, (V, 2))
        if out_mask & OR_PRIMIDS:
            out["primids"] = get(ORB_PRIMIDS, np.float32, V)
        if out_mask & OR_NORMALS:
            out["normals"] = get(ORB_NORMALS, np.float32, (V, 4))
        if technique == 1:
            out["dc_mask"] = get(ORB_DCMASK, np.uint8, nA * 512)
            out["dc_voff"] = get(ORB_DCVOFF, np.uint32, nA * 512)
            out["dc_vert"] = get(ORB_DCVERT, np.uint16, (nDC, 4))
            out["dc_norm"] = get(ORB_DCNORM, np.int16, (nDC, 4))
        return out
    finally:
        L.or_result_free(h)


def scout_range(scene: Scene, grid: _Grid, b0: int, b1: int, time: float = 0.0, nthreads: int = 0) -> int:
    return int(lib().or_scout_range(ctypes.byref(scene._c), ctypes.byref(grid), float(time), int(b0), int(b1),
                                    int(nthreads)))


def scout_flags(scene: Scene, grid: _Grid, blocks: np.ndarray, time: float = 0.0, nthreads: int = 0) -> np.ndarray:
    b = np.ascontiguousarray(blocks, np.int32)
    out = np.zeros(len(b), np.uint8)
    lib().or_scout_flags(ctypes.byref(scene._c), ctypes.byref(grid), float(time), b.ctypes.data, len(b),
                         out.ctypes.data, int(nthreads))
    return out.astype(bool)


def mc_blocks(scene: Scene, grid: _Grid, blocks: np.ndarray, time: float = 0.0, nthreads: int = 0) -> int:
    b = np.ascontiguousarray(blocks, np.int32)
    return int(lib().or_mc_blocks(ctypes.byref(scene._c), ctypes.byref(grid), float(time), b.ctypes.data, len(b),
                                  int(nthreads)))


def exclusive_scan(x: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(x, np.uint32)
    out = np.zeros_like(a)
    lib().or_exclusive_scan(a.ctypes.data, out.ctypes.data, len(a))
    return out
