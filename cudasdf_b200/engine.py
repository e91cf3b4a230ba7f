"""Python front end of the fused engine (sdf_engine_* in include/sdfmesh_b200.h).

Device memory comes from torch (the caller's CUDA allocator); every kernel is the library's own.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from .scenes import PRIM_DTYPE


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class MeshBuffers:
    """Output streams in the reference's VBO/EBO layout (triangle soup)."""

    def __init__(self, max_vertices: int, out_mask: int, device="cuda"):
        import torch
        self.max_vertices = int(max_vertices)
        self.out_mask = int(out_mask)
        n = max(self.max_vertices, 1)
        self.vertices = torch.empty((n, 4), dtype=torch.float32, device=device)
        self.colors = torch.empty((n, 4), dtype=torch.float32, device=device) if out_mask & L.OUT_COLORS else None
        self.indices = torch.empty((n,), dtype=torch.int32, device=device) if out_mask & L.OUT_INDICES else None
        self.uvs = torch.empty((n, 2), dtype=torch.float32, device=device) if out_mask & L.OUT_UVS else None
        self.primitive_ids = torch.empty((n,), dtype=torch.int32, device=device) if out_mask & L.OUT_PRIMIDS else None
        self.normals = torch.empty((n, 4), dtype=torch.float32, device=device) if out_mask & L.OUT_NORMALS else None

    def c_struct(self) -> L.SdfOutputs:
        o = L.SdfOutputs()
        o.vertices = self.vertices.data_ptr()
        o.colors = self.colors.data_ptr() if self.colors is not None else None
        o.indices = self.indices.data_ptr() if self.indices is not None else None
        o.uvs = self.uvs.data_ptr() if self.uvs is not None else None
        o.primitive_ids = self.primitive_ids.data_ptr() if self.primitive_ids is not None else None
        o.normals = self.normals.data_ptr() if self.normals is not None else None
        o.max_vertices = self.max_vertices
        return o


def make_config(cell_size: float, bounds_min=(-1.0, -1.0, -1.0), bounds_max=(1.0, 1.0, 1.0), technique=L.TECH_MC,
                qef_blend=1.0, dc_solver=L.DC_SOLVER_REFERENCE, projection_iters=0, adaptive_diagonal=0,
                cond_threshold=1e4, out_mask=L.OUT_INDICES) -> L.SdfConfig:
    c = L.SdfConfig()
    c.cell_size = float(np.float32(cell_size))
    for k in range(3):
        c.bounds_min[k] = float(bounds_min[k])
        c.bounds_max[k] = float(bounds_max[k])
    c.technique = int(technique)
    c.qef_blend = float(qef_blend)
    c.dc_solver = int(dc_solver)
    c.projection_iters = int(projection_iters)
    c.adaptive_diagonal = int(adaptive_diagonal)
    c.cond_threshold = float(cond_threshold)
    c.out_mask = int(out_mask)
    return c


class Engine:
    """One engine instance: grid configuration, uploaded scene, reusable device buffers."""

    def __init__(self, device: int = -1):
        self._lib = L.lib()
        h = ctypes.c_void_p()
        L.check(self._lib.sdf_engine_create(ctypes.byref(h), int(device)), "sdf_engine_create")
        self.h = h
        self.config = None

    def close(self):
        if self.h:
            self._lib.sdf_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def configure(self, cfg: L.SdfConfig):
        L.check(self._lib.sdf_engine_configure(self.h, ctypes.byref(cfg)), "sdf_engine_configure")
        self.config = cfg

    def set_scene(self, prims: np.ndarray):
        p = np.ascontiguousarray(prims, dtype=PRIM_DTYPE)
        L.check(self._lib.sdf_engine_set_scene(self.h, p.ctypes.data, len(p)), "sdf_engine_set_scene")

    def set_scene_device(self, prims, stream=None):
        """The scene from primitives in device memory (a CUDA tensor of 160-byte records, or a host
        array, which is uploaded first); the BVH is built on the GPU (sdf_engine_set_scene_device)."""
        import torch
        if isinstance(prims, np.ndarray):
            p = np.ascontiguousarray(prims, dtype=PRIM_DTYPE)
            prims = torch.from_numpy(p.view(np.uint8).reshape(-1)).cuda()
        if not (prims.is_cuda and prims.is_contiguous()):
            raise ValueError("set_scene_device wants a contiguous CUDA tensor")
        n = prims.numel() * prims.element_size() // PRIM_DTYPE.itemsize
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        self._scene_keep = prims
        L.check(self._lib.sdf_engine_set_scene_device(self.h, prims.data_ptr(), n, sp), "sdf_engine_set_scene_device")

    def set_scene_async(self, prims: np.ndarray, stream=None):
        """set_scene with the upload enqueued on `stream` (sdf_engine_set_scene_async)."""
        p = np.ascontiguousarray(prims, dtype=PRIM_DTYPE)
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        L.check(self._lib.sdf_engine_set_scene_async(self.h, p.ctypes.data, len(p), sp), "sdf_engine_set_scene_async")

    def extract_async(self, out: MeshBuffers, time: float = 0.0, stream=None) -> int:
        """Enqueues an extraction; returns its ticket for extract_wait."""
        o = out.c_struct()
        t = ctypes.c_uint64(0)
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        L.check(self._lib.sdf_engine_extract_async(self.h, float(time), ctypes.byref(o), sp, ctypes.byref(t)),
                "sdf_engine_extract_async")
        return t.value

    def extract_wait(self, ticket: int, allow_capacity=False) -> dict:
        st = L.SdfStats()
        rc = self._lib.sdf_engine_extract_wait(self.h, ctypes.c_uint64(ticket), ctypes.byref(st))
        if not (allow_capacity and rc == L.SDF_ERR_CAPACITY):
            L.check(rc, "sdf_engine_extract_wait")
        d = st.as_dict()
        d["status"] = rc
        return d

    def set_timing(self, on: bool):
        self._lib.sdf_engine_set_timing(self.h, 1 if on else 0)

    def set_debug(self, flags: int):
        self._lib.sdf_engine_set_debug(self.h, int(flags))

    def extract(self, out: MeshBuffers, time: float = 0.0, stream=None, allow_capacity=False) -> dict:
        st = L.SdfStats()
        o = out.c_struct()
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        rc = self._lib.sdf_engine_extract(self.h, float(time), ctypes.byref(o), sp, ctypes.byref(st))
        if not (allow_capacity and rc == L.SDF_ERR_CAPACITY):
            L.check(rc, "sdf_engine_extract")
        d = st.as_dict()
        d["status"] = rc
        return d

    def eval(self, points, time: float = 0.0, stream=None):
        """map() at device points (torch float32 (n, 3)); returns a (n, 8) device tensor."""
        import torch
        pts = points.contiguous()
        out = torch.empty((pts.shape[0], 8), dtype=torch.float32, device=pts.device)
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        L.check(self._lib.sdf_engine_eval(self.h, ctypes.c_void_p(pts.data_ptr()), int(pts.shape[0]), float(time),
                                          ctypes.c_void_p(out.data_ptr()), sp), "sdf_engine_eval")
        return out

    def eval_distance(self, points, time: float = 0.0, stream=None):
        """Distance only at device points (torch float32 (n, 3)); returns a (n,) device tensor."""
        import torch
        pts = points.contiguous()
        out = torch.empty((pts.shape[0],), dtype=torch.float32, device=pts.device)
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        L.check(self._lib.sdf_engine_eval_distance(self.h, ctypes.c_void_p(pts.data_ptr()), int(pts.shape[0]),
                                                   float(time), ctypes.c_void_p(out.data_ptr()), sp),
                "sdf_engine_eval_distance")
        return out

    def eval_normals(self, points, cell: float, time: float = 0.0, stream=None):
        """computeNormal at device points (torch float32 (n, 3)); returns a (n, 3) device tensor."""
        import torch
        pts = points.contiguous()
        out = torch.empty((pts.shape[0], 3), dtype=torch.float32, device=pts.device)
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        L.check(self._lib.sdf_engine_eval_normals(self.h, ctypes.c_void_p(pts.data_ptr()), int(pts.shape[0]),
                                                  float(time), float(cell), ctypes.c_void_p(out.data_ptr()), sp),
                "sdf_engine_eval_normals")
        return out

    # ---- learned surrogate (sdf_surrogate_* in include/sdfmesh_b200.h) ----
    @staticmethod
    def surrogate_config(**overrides) -> L.SurrogateConfig:
        c = L.SurrogateConfig()
        L.lib().sdf_surrogate_default_config(ctypes.byref(c))
        for k, v in overrides.items():
            setattr(c, k, v)
        return c

    def surrogate_train(self, cfg: L.SurrogateConfig = None) -> dict:
        cfg = cfg or self.surrogate_config()
        st = L.SurrogateStats()
        L.check(self._lib.sdf_surrogate_train(self.h, ctypes.byref(cfg), ctypes.byref(st)), "sdf_surrogate_train")
        return st.as_dict()

    def surrogate_enable(self, on: bool):
        L.check(self._lib.sdf_surrogate_enable(self.h, 1 if on else 0), "sdf_surrogate_enable")

    def set_coarse_cull(self, mode: int, extra_margin: float = 0.0):
        """L.SDF_CULL_NONE, L.SDF_CULL_SURROGATE or L.SDF_CULL_EXACT (the exact map() at the coarse centres,
        culled beyond the reach plus extra_margin)."""
        L.check(self._lib.sdf_engine_set_coarse_cull(self.h, int(mode), float(extra_margin)),
                "sdf_engine_set_coarse_cull")

    def surrogate_audit(self, time: float = 0.0) -> dict:
        v, c, n = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        L.check(self._lib.sdf_surrogate_audit(self.h, float(time), ctypes.byref(v), ctypes.byref(c), ctypes.byref(n)),
                "sdf_surrogate_audit")
        return {"violations": v.value, "culled_coarse": c.value, "coarse_blocks": n.value}

    def surrogate_set_params(self, theta, freq, io):
        th = np.ascontiguousarray(theta, np.float32)
        fr = np.ascontiguousarray(freq, np.float32)
        iv = np.ascontiguousarray(io, np.float32)
        assert th.size == self._lib.sdf_surrogate_num_params() and fr.size == 96 and iv.size == 7
        L.check(self._lib.sdf_surrogate_set_params(self.h, th.ctypes.data, fr.ctypes.data, iv.ctypes.data),
                "sdf_surrogate_set_params")

    def surrogate_get_params(self):
        th = np.zeros(self._lib.sdf_surrogate_num_params(), np.float32)
        fr = np.zeros(96, np.float32)
        iv = np.zeros(7, np.float32)
        L.check(self._lib.sdf_surrogate_get_params(self.h, th.ctypes.data, fr.ctypes.data, iv.ctypes.data),
                "sdf_surrogate_get_params")
        return th, fr.reshape(32, 3), iv

    def surrogate_forward(self, points, stream=None):
        """f_net at device points (torch float32 (n, 3)); returns a (n,) device tensor."""
        import torch
        pts = points.contiguous()
        out = torch.empty((pts.shape[0],), dtype=torch.float32, device=pts.device)
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        L.check(self._lib.sdf_surrogate_forward(self.h, ctypes.c_void_p(pts.data_ptr()), int(pts.shape[0]),
                                                ctypes.c_void_p(out.data_ptr()), sp), "sdf_surrogate_forward")
        return out

    def surrogate_gradient(self, points, targets):
        """Gradient of the mean squared error over device samples (no update): (grad numpy, loss)."""
        pts = points.contiguous()
        tg = targets.contiguous()
        g = np.zeros(self._lib.sdf_surrogate_num_params(), np.float32)
        loss = ctypes.c_float()
        L.check(self._lib.sdf_surrogate_gradient(self.h, ctypes.c_void_p(pts.data_ptr()), ctypes.c_void_p(tg.data_ptr()),
                                                 int(pts.shape[0]), g.ctypes.data, ctypes.byref(loss)),
                "sdf_surrogate_gradient")
        return g, loss.value

    def bvh(self):
        nb = ctypes.c_int(0)
        n = self._lib.sdf_engine_get_bvh(self.h, None, 0, ctypes.byref(nb))
        nodes = np.zeros(max(n, 0), dtype=[("min", "<f4", 3), ("max", "<f4", 3), ("left", "<i4"), ("right", "<i4")])
        if n > 0:
            self._lib.sdf_engine_get_bvh(self.h, nodes.ctypes.data, n, ctypes.byref(nb))
        return nodes, nb.value

    def buffer(self, which: int, dtype, count: int) -> np.ndarray:
        """Copies `count` elements of an internal device array (see sdf_engine_buffer) to the host."""
        nbytes = ctypes.c_size_t(0)
        self._lib.sdf_engine_buffer(self.h, int(which), ctypes.byref(nbytes))
        dt = np.dtype(dtype)
        count = min(int(count), nbytes.value // dt.itemsize)
        out = np.zeros(count, dt)
        if count:
            L.check(self._lib.sdf_engine_read_buffer(self.h, int(which), out.ctypes.data, out.nbytes),
                    "sdf_engine_read_buffer")
        return out


class Batch:
    """Many scenes meshed together (sdf_batch_* in include/sdfmesh_b200.h).

    scenes: list of (primitives, SdfConfig). Marching-cubes scenes write one concatenated soup into
    the mc buffers, dual-contouring scenes into the dc buffers."""

    def __init__(self, device: int = -1):
        self._lib = L.lib()
        h = ctypes.c_void_p()
        L.check(self._lib.sdf_batch_create(ctypes.byref(h), int(device)), "sdf_batch_create")
        self.h = h
        self.n = 0

    def close(self):
        if self.h:
            self._lib.sdf_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_scenes(self, scenes, out_mask: int):
        self._keep = [np.ascontiguousarray(p, dtype=PRIM_DTYPE) for p, _ in scenes]
        arr = (L.BatchScene * len(scenes))()
        for k, ((_, cfg), p) in enumerate(zip(scenes, self._keep)):
            arr[k].prims = p.ctypes.data
            arr[k].count = len(p)
            arr[k].config = cfg
        L.check(self._lib.sdf_batch_set_scenes(self.h, arr, len(scenes), int(out_mask)), "sdf_batch_set_scenes")
        self.n = len(scenes)

    def _outs(self, mc: MeshBuffers, dc: MeshBuffers):
        return (ctypes.byref(mc.c_struct()) if mc is not None else None,
                ctypes.byref(dc.c_struct()) if dc is not None else None)

    def capture(self, mc: MeshBuffers, dc: MeshBuffers, time: float = 0.0, tune: bool = True, stream=None):
        om, od = self._outs(mc, dc)
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        L.check(self._lib.sdf_batch_capture(self.h, float(time), om, od, sp, 1 if tune else 0), "sdf_batch_capture")

    def read_buffer(self, technique: int, which: int, dtype) -> np.ndarray:
        """An internal array of one group's last extraction (see sdf_batch_read_buffer) on the host."""
        n = ctypes.c_size_t(0)
        L.check(self._lib.sdf_batch_read_buffer(self.h, int(technique), int(which), None, ctypes.byref(n)),
                "sdf_batch_read_buffer")
        out = np.zeros(n.value // np.dtype(dtype).itemsize, dtype)
        n = ctypes.c_size_t(out.nbytes)
        L.check(self._lib.sdf_batch_read_buffer(self.h, int(technique), int(which), out.ctypes.data,
                                                ctypes.byref(n)), "sdf_batch_read_buffer")
        return out

    def extract(self, mc: MeshBuffers, dc: MeshBuffers, time: float = 0.0, stream=None, allow_capacity=False):
        """Returns (first_vertex, vertex_count, stats); the counts are exact even when a buffer was too
        small (SDF_ERR_CAPACITY, raised unless allow_capacity)."""
        om, od = self._outs(mc, dc)
        first = np.zeros(self.n, np.int64)
        count = np.zeros(self.n, np.int64)
        st = L.BatchStats()
        sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        rc = self._lib.sdf_batch_extract(self.h, float(time), om, od, sp, first.ctypes.data, count.ctypes.data,
                                         ctypes.byref(st))
        if not (allow_capacity and rc == L.SDF_ERR_CAPACITY):
            L.check(rc, "sdf_batch_extract")
        return first, count, st.as_dict()
