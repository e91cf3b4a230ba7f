"""CudaSDFMesh over the drop-in launchers.

A mirror of the reference's host orchestrator (src/SDFMesh/CudaSDFMesh.{h,cpp}): the same methods,
argument meaning and stage order, calling the twelve extern "C" launchers that libsdfmesh_b200.so
exports under the reference's names (Wrappers.cu:19-136). It is what a user of the reference's
CudaSDFMesh gets when the reference's kernels are replaced by this library, and it is how the tests
exercise that boundary. Device memory is torch's.

Differences from the reference, all additive:
  * the 200000 active-block and 50M vertex caps (CudaSDFMesh.cpp:159, 187, 352) are constructor
    parameters (defaults: the reference's values);
  * every stage checks sdf_last_error() and raises instead of printing and continuing;
  * scenes without union primitives skip the BVH walk (the reference reads an unwritten node 0).
"""
from __future__ import annotations

import ctypes
import math
import time as _time

import numpy as np

from . import _lib as L
from .scenes import PRIM_DTYPE, SDF_UNION, SDF_UNION_BLEND

MARCHING_CUBES, DUAL_CONTOURING = 0, 1
BLOCK = 8
BLOCK3 = 512


def _f32(x):
    return np.float32(x)


class CudaSDFMesh:
    def __init__(self, max_active_blocks: int = 200000, max_vertices: int = 50_000_000, device: str = "cuda"):
        import torch
        self.torch = torch
        self.device = device
        self.max_active_cap = int(max_active_blocks)
        self.max_vertices = int(max_vertices)
        self.grid = L.SdfGrid()
        self.primitives = []
        self.bvh_nodes = None
        self.num_bvh_primitives = 0
        self.total_vertices = 0
        self.total_indices = 0
        self.timings = {}
        self._bufs = {}
        self.packed_size = 0

    # -- CudaSDFMesh::Initialize (CudaSDFMesh.cpp:90-206) ------------------------------------------
    def Initialize(self, cellSize: float, boundsMin, boundsMax):
        torch = self.torch
        cell = _f32(cellSize)
        if not cell > 0:
            raise ValueError("Invalid cell size (must be > 0)")
        size = [_f32(boundsMax[k]) - _f32(boundsMin[k]) for k in range(3)]
        if any(not s > 0 for s in size):
            raise ValueError("Invalid bounds size (must be > 0)")
        dims = [int(math.ceil(_f32(s / cell))) for s in size]
        if dims[0] * dims[1] * dims[2] > 8589934592:
            raise ValueError("Grid size too large")
        g = self.grid
        g.cellSize = float(cell)
        for k in range(3):
            g.origin[k] = float(_f32(boundsMin[k]))
        g.width, g.height, g.depth = dims
        bd = [(d + BLOCK - 1) // BLOCK for d in dims]
        for k in range(3):
            g.blocksDim[k] = bd[k]
        g.maxBlocks = bd[0] * bd[1] * bd[2]
        est = min(g.maxBlocks, self.max_active_cap)
        self.packed_size = est * BLOCK3
        dev = self.device
        b = self._bufs
        b["activeBlocks"] = torch.empty(g.maxBlocks, dtype=torch.int32, device=dev)
        b["activeBlockCount"] = torch.zeros(1, dtype=torch.int32, device=dev)
        b["counts"] = torch.empty(self.packed_size, dtype=torch.int32, device=dev)
        b["offsets"] = torch.empty(self.packed_size, dtype=torch.int32, device=dev)
        nbytes = ctypes.c_size_t(0)
        L.lib().getScanStorageSize(self.packed_size, ctypes.byref(nbytes))
        b["scanTemp"] = torch.empty(max(nbytes.value, 16), dtype=torch.uint8, device=dev)
        self.scan_bytes = nbytes.value
        for k in ("blockToActiveId", "dcMasks", "dcVertOffsets", "dcVerts", "dcNormals", "dcNormalsTmp"):
            b.pop(k, None)
        g.d_activeBlocks = b["activeBlocks"].data_ptr()
        g.d_activeBlockCount = b["activeBlockCount"].data_ptr()
        g.d_packetVertexCounts = b["counts"].data_ptr()
        g.d_packetVertexOffsets = b["offsets"].data_ptr()
        g.maxVertices = self.max_vertices
        g.maxIndices = self.max_vertices * 3 & 0xFFFFFFFF
        g.numPrimitives = 0

    def AddPrimitive(self, prim):
        self.primitives.append(np.asarray(prim, dtype=PRIM_DTYPE).reshape(()))

    def ClearPrimitives(self):
        self.primitives = []

    def GetPrimitives(self):
        return self.primitives

    def GetTotalVertexCount(self):
        return self.total_vertices

    def GetTotalIndexCount(self):
        return self.total_indices

    def GetNumBVHPrimitives(self):
        return self.num_bvh_primitives

    def GetBVHNodes(self):
        return self.bvh_nodes

    def GetKernelTimings(self):
        return dict(self.timings)

    def GetBounds(self):
        g = self.grid
        mn = tuple(g.origin)
        mx = (g.origin[0] + g.width * g.cellSize, g.origin[1] + g.height * g.cellSize, g.origin[2] + g.depth * g.cellSize)
        return mn, mx

    # -- CudaSDFMesh::UpdateBVH (CudaSDFMesh.cpp:216-249) ------------------------------------------
    def UpdateBVH(self):
        from .engine import Engine
        prims = np.array(self.primitives, dtype=PRIM_DTYPE) if self.primitives else np.zeros(0, PRIM_DTYPE)
        is_union = (prims["operation"] == SDF_UNION) | (prims["operation"] == SDF_UNION_BLEND)
        self.sorted = np.concatenate([prims[is_union], prims[~is_union]])
        self.primitives = list(self.sorted)
        eng = _bvh_engine()
        eng.set_scene(self.sorted)
        self.bvh_nodes, self.num_bvh_primitives = eng.bvh()

    def _ensure(self, name, n, dtype):
        torch = self.torch
        t = self._bufs.get(name)
        if t is None or t.numel() < n:
            t = torch.empty(max(n, 1), dtype=dtype, device=self.device)
            self._bufs[name] = t
        return t

    def _err(self, stage):
        e = L.lib().sdf_last_error()
        if e:
            raise RuntimeError(f"{stage}: CUDA error {e}")

    # -- CudaSDFMesh::Update (CudaSDFMesh.cpp:281-470) ---------------------------------------------
    def Update(self, time, d_outVertices, d_outColors=None, d_outIndices=None, d_outUVs=None, d_outPrimitiveIDs=None,
               d_outNormals=None, technique=MARCHING_CUBES, dcNormalSmoothAngleDeg=30.0, dcQefBlend=1.0,
               timing=False):
        torch = self.torch
        lib = L.lib()
        g = self.grid
        self.timings = {}
        self.UpdateBVH()
        n = len(self.sorted)
        prims_t = self._ensure("prims", n * 160, torch.uint8)
        if n:
            prims_t[: n * 160].copy_(torch.from_numpy(self.sorted.view(np.uint8).reshape(-1)))
        nodes = self.bvh_nodes
        nodes_t = self._ensure("nodes", len(nodes) * 32, torch.uint8)
        if len(nodes):
            nodes_t[: len(nodes) * 32].copy_(torch.from_numpy(np.ascontiguousarray(nodes).view(np.uint8).reshape(-1)))
        g.d_primitives = prims_t.data_ptr()
        g.numPrimitives = n
        g.numBVHPrimitives = self.num_bvh_primitives
        g.d_bvhNodes = nodes_t.data_ptr()
        g.numBVHNodes = len(nodes)
        ptr = lambda t: t.data_ptr() if t is not None else None  # noqa: E731
        g.d_vertices = ptr(d_outVertices)
        g.d_vertexColors = ptr(d_outColors)
        g.d_indices = ptr(d_outIndices)
        g.d_uvCoords = ptr(d_outUVs)
        g.d_primitiveIDs = ptr(d_outPrimitiveIDs)
        g.d_normals = ptr(d_outNormals)
        G = ctypes.byref(g)
        t_stage = [_time.perf_counter()]

        def stage(name):
            if timing:
                torch.cuda.synchronize()
                now = _time.perf_counter()
                self.timings[name] = (now - t_stage[0]) * 1e3
                t_stage[0] = now

        self._bufs["activeBlockCount"].zero_()
        lib.launchScoutActiveBlocks(G, float(time))
        self._err("scoutActiveBlocks")
        stage("scoutActiveBlocks")
        num_active = int(self._bufs["activeBlockCount"].item())
        if num_active <= 0:
            self.total_vertices = 0
            self.total_indices = 0
            return
        num_active = min(num_active, self.max_active_cap)
        total_items = num_active * BLOCK3
        if technique == MARCHING_CUBES:
            lib.launchCountActiveBlockTriangles(G, num_active, float(time))
            self._err("countActiveBlockTriangles")
            stage("mcCountTriangles")
            lib.launchScan(g.d_packetVertexCounts, g.d_packetVertexOffsets, total_items,
                           self._bufs["scanTemp"].data_ptr(), self.scan_bytes)
            self._err("scan")
            stage("scan1")
            lib.launchGenerateActiveBlockTriangles(G, num_active, float(time))
            self._err("generateActiveBlockTriangles")
            stage("mcGenerateTriangles")
        else:
            b2a = self._ensure("blockToActiveId", g.maxBlocks, torch.int32)
            masks = self._ensure("dcMasks", self.packed_size, torch.uint8)
            voff = self._ensure("dcVertOffsets", self.packed_size, torch.int32)
            verts = self._ensure("dcVerts", self.max_vertices * 4, torch.int16)
            norms = self._ensure("dcNormals", self.max_vertices * 4, torch.int16)
            norms_tmp = self._ensure("dcNormalsTmp", self.max_vertices * 4, torch.int16)
            g.d_blockToActiveId = b2a.data_ptr()
            g.d_dcCornerMasks = masks.data_ptr()
            g.d_dcCellVertexOffsets = voff.data_ptr()
            g.d_dcCellVertices = verts.data_ptr()
            g.d_dcCellNormals = norms.data_ptr()
            g.d_dcCellNormalsTmp = norms_tmp.data_ptr()
            b2a.fill_(-1)
            lib.launchBuildBlockToActiveMap(G, num_active)
            self._err("buildBlockToActiveMap")
            stage("dcBuildBlockMap")
            lib.launchDCMarkCells(G, num_active, float(time))
            self._err("dcMarkCells")
            stage("dcMarkCells")
            lib.launchScan(g.d_packetVertexCounts, g.d_dcCellVertexOffsets, total_items,
                           self._bufs["scanTemp"].data_ptr(), self.scan_bytes)
            self._err("scan1")
            stage("scan1")
            lib.launchDCSolveCellVertices(G, num_active, float(time), self.max_vertices, float(dcQefBlend))
            self._err("dcSolveCellVertices")
            stage("dcSolveCellVertices")
            lib.launchDCCountQuads(G, num_active)
            self._err("dcCountQuads")
            stage("dcCountQuads")
            lib.launchScan(g.d_packetVertexCounts, g.d_packetVertexOffsets, total_items,
                           self._bufs["scanTemp"].data_ptr(), self.scan_bytes)
            self._err("scan2")
            stage("scan2")
            lib.launchDCGenerateQuads(G, num_active, float(time))
            self._err("dcGenerateQuads")
            stage("dcGenerateQuads")
        last_off = int(self._bufs["offsets"][total_items - 1].item()) & 0xFFFFFFFF
        last_cnt = int(self._bufs["counts"][total_items - 1].item()) & 0xFFFFFFFF
        self.total_vertices = last_off + last_cnt
        self.total_indices = 0
        self.num_active = num_active

    def DCNormalPasses(self, time, cosAngleThreshold):
        """The two dual-contouring normal passes that CudaSDFMesh::Update never calls
        (Wrappers.cu:87-105): normals recomputed at the cell vertices, then the angle-gated smoothing
        into the tmp buffer. Run after Update with the dual-contouring technique."""
        lib = L.lib()
        G = ctypes.byref(self.grid)
        lib.launchDCRecomputeNormalsAtVertices(G, self.num_active, float(time))
        self._err("dcRecomputeNormalsAtVertices")
        lib.launchDCSmoothCellNormals(G, self.num_active, float(cosAngleThreshold))
        self._err("dcSmoothCellNormals")

    # inspection helpers for the tests
    def active_blocks(self):
        return self._bufs["activeBlocks"][: self.num_active].cpu().numpy()

    def packet(self, name):
        return self._bufs[name][: self.num_active * BLOCK3].cpu().numpy().view(np.uint32)

    def dc_buffer(self, name, count):
        t = self._bufs[name]
        if name in ("dcVerts", "dcNormals", "dcNormalsTmp"):
            return t[: count * 4].cpu().numpy().reshape(-1, 4)
        return t[:count].cpu().numpy()


_BVH_ENGINE = None


def _bvh_engine():
    """An engine used only for its host BVH builder (the reference's node order)."""
    global _BVH_ENGINE
    if _BVH_ENGINE is None:
        from .engine import Engine
        _BVH_ENGINE = Engine()
    return _BVH_ENGINE
