"""UV atlas packing on the GPU: the reference's GridUVPacker (src/SDFMesh/GridUVPacker.{cuh,cu}).

`UVAtlas` wraps the sdf_uv_atlas_* entry points of include/sdfmesh_b200.h. Its steps are the
reference's ExtractCharts, CreateIslands, PackIslands and RemapUVsToAtlas (GridUVPacker.cuh:186-219),
in the order of main.cpp:1429-1442; `run` does all four. Buffers are CUDA tensors: UVs (n, 2) float32
and primitive ids (n,) holding float bits (the SDF_OUT_UVS / SDF_OUT_PRIMIDS streams).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, fields

import numpy as np

from . import _lib as L


@dataclass
class PackingConfig:
    """PackingConfig (GridUVPacker.cuh:121-146): same fields and defaults."""
    gridSize: int = 128
    gridResolution: int = 64
    maxIterations: int = 500
    marginCells: int = 2
    enableRotation: bool = True
    xAlignment: int = 8
    maxCandidatesPerIsland: int = 32
    maxDropSteps: int = 0
    shuffleOrderPerAttempt: bool = True
    randomSeed: int = 0

    @staticmethod
    def app() -> "PackingConfig":
        """The configuration of the reference's only caller (main.cpp:1417-1427)."""
        return PackingConfig(gridSize=2048, gridResolution=64, maxIterations=256, marginCells=4, enableRotation=True,
                             xAlignment=8, maxCandidatesPerIsland=16, maxDropSteps=256, shuffleOrderPerAttempt=True,
                             randomSeed=1337)

    def c_struct(self) -> L.UvPackConfig:
        c = L.UvPackConfig()
        vals = [int(getattr(self, f.name)) for f in fields(self)]
        for (name, _), v in zip(L.UvPackConfig._fields_, vals):
            setattr(c, name, v)
        return c

    def as_dict(self) -> dict:
        return dict(zip([n for n, _ in L.UvPackConfig._fields_], self.c_struct().as_list()))


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


CHART_DTYPE = np.dtype([("primitive_id", "<i4"), ("num_triangles", "<i4"), ("uv_min", "<f4", 2), ("uv_max", "<f4", 2)])
GRID_DTYPE = np.dtype([("width", "<i4"), ("height", "<i4"), ("stride", "<i4"), ("pad", "<i4"), ("word_offset", "<i8")])
ISLAND_DTYPE = np.dtype([("island_index", "<i4"), ("primitive_id", "<i4"), ("num_triangles", "<i4"),
                         ("min_cell_x", "<i4"), ("min_cell_y", "<i4"), ("width", "<i4"), ("height", "<i4"),
                         ("pad", "<i4"), ("mask", GRID_DTYPE), ("collision", GRID_DTYPE), ("mask90", GRID_DTYPE),
                         ("collision90", GRID_DTYPE), ("row_bounds", "<i8"), ("row_bounds90", "<i8"),
                         ("profile", "<i8"), ("profile90", "<i8")])
PLACEMENT_DTYPE = np.dtype([("island_index", "<i4"), ("grid_x", "<i4"), ("grid_y", "<i4"), ("rotation", "<i4")])
SOLUTION_DTYPE = np.dtype([("num_placed", "<i4"), ("utilized_width", "<i4"), ("utilized_height", "<i4"),
                           ("flags", "<i4"), ("fitness", "<f4"), ("seed", "<i4")])
assert CHART_DTYPE.itemsize == ctypes.sizeof(L.UvChart) and ISLAND_DTYPE.itemsize == ctypes.sizeof(L.UvIsland)
READ_DTYPES = {0: CHART_DTYPE, 1: np.int32, 2: ISLAND_DTYPE, 3: np.uint32, 4: np.uint16, 5: np.int32, 6: np.int32,
               7: SOLUTION_DTYPE, 8: PLACEMENT_DTYPE, 9: PLACEMENT_DTYPE}


class UVAtlas:
    """One packer state (charts, islands, attempts). Not safe for concurrent use from several threads."""

    def __init__(self):
        h = ctypes.c_void_p()
        L.check(L.lib().sdf_uv_atlas_create(ctypes.byref(h)), "sdf_uv_atlas_create")
        self.h = h

    def close(self):
        if self.h:
            L.lib().sdf_uv_atlas_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def extract_charts(self, uvs, primitive_ids, stream=None) -> int:
        """ExtractCharts (GridUVPacker.cu:833-896); returns the chart count."""
        n = ctypes.c_int32()
        L.check(L.lib().sdf_uv_atlas_extract_charts(self.h, _ptr(uvs), _ptr(primitive_ids), int(uvs.shape[0]),
                                                     _stream(stream), ctypes.byref(n)), "sdf_uv_atlas_extract_charts")
        return n.value

    def create_islands(self, uvs, grid_resolution: int, margin_cells: int, stream=None):
        """CreateIslands (GridUVPacker.cu:898-1061)."""
        L.check(L.lib().sdf_uv_atlas_create_islands(self.h, _ptr(uvs), int(grid_resolution), int(margin_cells),
                                                     _stream(stream)), "sdf_uv_atlas_create_islands")

    def pack_islands(self, config: PackingConfig, stream=None) -> dict:
        """PackIslands (GridUVPacker.cu:1063-1439); the PackedAtlas fields and the run's counts."""
        info = L.UvAtlasInfo()
        c = config.c_struct()
        L.check(L.lib().sdf_uv_atlas_pack(self.h, ctypes.byref(c), _stream(stream), ctypes.byref(info)),
                "sdf_uv_atlas_pack")
        return info.as_dict()

    def remap_uvs_to_atlas(self, uvs, primitive_ids, grid_resolution: int, stream=None):
        """RemapUVsToAtlas (GridUVPacker.cu:1441-1547), in place."""
        L.check(L.lib().sdf_uv_atlas_remap(self.h, _ptr(uvs), _ptr(primitive_ids), int(uvs.shape[0]),
                                            int(grid_resolution), _stream(stream)), "sdf_uv_atlas_remap")

    def run(self, uvs, primitive_ids, config: PackingConfig, stream=None) -> dict:
        info = L.UvAtlasInfo()
        c = config.c_struct()
        L.check(L.lib().sdf_uv_atlas_run(self.h, _ptr(uvs), _ptr(primitive_ids), int(uvs.shape[0]), ctypes.byref(c),
                                          _stream(stream), ctypes.byref(info)), "sdf_uv_atlas_run")
        return info.as_dict()

    def read(self, which: int) -> np.ndarray:
        """One internal array (sdf_uv_atlas_read): 0 charts, 1 chart per triangle, 2 islands, 3 mask words,
        4 row bounds, 5 column profiles, 6 seeds, 7 attempts, 8 all placements, 9 chosen placements."""
        n = ctypes.c_size_t(0)
        L.check(L.lib().sdf_uv_atlas_read(self.h, int(which), None, ctypes.byref(n)), "sdf_uv_atlas_read")
        dt = np.dtype(READ_DTYPES[which])
        out = np.zeros(n.value // dt.itemsize, dt)
        if n.value:
            L.check(L.lib().sdf_uv_atlas_read(self.h, int(which), out.ctypes.data_as(ctypes.c_void_p),
                                               ctypes.byref(n)), "sdf_uv_atlas_read")
        return out

    def grids(self, slot: int, words=None, rb=None) -> dict:
        """The four grids and the two row-bound arrays of the island in packing position `slot`."""
        isl = self.read(2)[slot]
        words = self.read(3) if words is None else words
        rb = self.read(4) if rb is None else rb
        out = {}
        for k in ("mask", "collision", "mask90", "collision90"):
            g = isl[k]
            o, s, h = int(g["word_offset"]), int(g["stride"]), int(g["height"])
            out[k] = words[o:o + s * h].reshape(h, s)
        h, w = int(isl["height"]), int(isl["width"])
        out["row_bounds"] = rb[int(isl["row_bounds"]):int(isl["row_bounds"]) + 2 * h].reshape(2, h)
        out["row_bounds90"] = rb[int(isl["row_bounds90"]):int(isl["row_bounds90"]) + 2 * w].reshape(2, w)
        return out


def random_draws(seeds, per_seed: int) -> np.ndarray:
    """curand(curand_init(seed, 0, 0)) draws per seed, (len(seeds), per_seed) uint32 (the GPU's stream)."""
    s = np.ascontiguousarray(seeds, dtype=np.int32)
    out = np.zeros((len(s), int(per_seed)), np.uint32)
    L.check(L.lib().sdf_uv_pack_random_draws(s.ctypes.data_as(ctypes.c_void_p), len(s), int(per_seed),
                                             out.ctypes.data_as(ctypes.c_void_p)), "sdf_uv_pack_random_draws")
    return out
