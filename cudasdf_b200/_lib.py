"""ctypes binding of libsdfmesh_b200.so (include/sdfmesh_b200.h).

The library is built in-tree by ``build.py`` (or ``__graft_entry__.build()``). Importing this module
does not load it; ``lib()`` does, and raises if it is missing: there is no fallback path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsdfmesh_b200.so")

SDF_OK, SDF_ERR_INVALID, SDF_ERR_CUDA, SDF_ERR_CAPACITY, SDF_ERR_STACK, SDF_ERR_NOMEM, SDF_ERR_TIMEOUT = range(7)
STATUS_NAMES = {0: "SDF_OK", 1: "SDF_ERR_INVALID", 2: "SDF_ERR_CUDA", 3: "SDF_ERR_CAPACITY", 4: "SDF_ERR_STACK",
                5: "SDF_ERR_NOMEM", 6: "SDF_ERR_TIMEOUT"}
OUT_COLORS, OUT_INDICES, OUT_UVS, OUT_PRIMIDS, OUT_NORMALS, OUT_WELDED = 1, 2, 4, 8, 16, 32
TECH_MC, TECH_DC = 0, 1
DC_SOLVER_REFERENCE, DC_SOLVER_MASSPOINT = 0, 1


class SdfConfig(ctypes.Structure):
    _fields_ = [("cell_size", ctypes.c_float), ("bounds_min", ctypes.c_float * 3), ("bounds_max", ctypes.c_float * 3),
                ("technique", ctypes.c_int32), ("qef_blend", ctypes.c_float), ("dc_solver", ctypes.c_int32),
                ("projection_iters", ctypes.c_int32), ("adaptive_diagonal", ctypes.c_int32),
                ("cond_threshold", ctypes.c_float), ("out_mask", ctypes.c_uint32)]


class SdfOutputs(ctypes.Structure):
    _fields_ = [("vertices", ctypes.c_void_p), ("colors", ctypes.c_void_p), ("indices", ctypes.c_void_p),
                ("uvs", ctypes.c_void_p), ("primitive_ids", ctypes.c_void_p), ("normals", ctypes.c_void_p),
                ("max_vertices", ctypes.c_uint32)]


class SdfStats(ctypes.Structure):
    _fields_ = [("total_blocks", ctypes.c_int64), ("active_blocks", ctypes.c_int64),
                ("total_vertices", ctypes.c_int64), ("written_vertices", ctypes.c_int64),
                ("dc_cell_vertices", ctypes.c_int64), ("bvh_cap_hits", ctypes.c_int64),
                ("ms_scout", ctypes.c_float), ("ms_field", ctypes.c_float), ("ms_scan", ctypes.c_float),
                ("ms_emit", ctypes.c_float), ("ms_total", ctypes.c_float), ("scouted_blocks", ctypes.c_int64),
                ("dc_fp64_cells", ctypes.c_int64), ("welded_vertices", ctypes.c_int64),
                ("ms_classify", ctypes.c_float), ("reserved", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class SurrogateConfig(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_int32), ("validation", ctypes.c_int32), ("steps", ctypes.c_int32),
                ("batch", ctypes.c_int32), ("lr", ctypes.c_float), ("freq_sigma", ctypes.c_float),
                ("surface_sigma", ctypes.c_float), ("clamp", ctypes.c_float), ("surface_res", ctypes.c_int32),
                ("slack_cells", ctypes.c_float), ("time", ctypes.c_float), ("seed", ctypes.c_uint32)]


class SurrogateStats(ctypes.Structure):
    _fields_ = [("final_loss", ctypes.c_float), ("eps_max", ctypes.c_float), ("eps_cert", ctypes.c_float),
                ("margin", ctypes.c_float),
                ("surface_points", ctypes.c_int32), ("ms_samples", ctypes.c_float), ("ms_train", ctypes.c_float),
                ("ms_certify", ctypes.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class BatchScene(ctypes.Structure):
    _fields_ = [("prims", ctypes.c_void_p), ("count", ctypes.c_int32), ("config", SdfConfig)]


class BatchStats(ctypes.Structure):
    _fields_ = [("scenes", ctypes.c_int64), ("total_blocks", ctypes.c_int64), ("active_blocks", ctypes.c_int64),
                ("mc_vertices", ctypes.c_int64), ("dc_vertices", ctypes.c_int64), ("ms_total", ctypes.c_float),
                ("graph", ctypes.c_int32), ("tuned_ctas", ctypes.c_int32 * 4)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["tuned_ctas"] = list(self.tuned_ctas)
        return d


class SdfGrid(ctypes.Structure):
    """The reference's SDFGrid (Commons.cuh:115-186), 232 bytes."""
    _fields_ = [("d_activeBlocks", ctypes.c_void_p), ("d_activeBlockCount", ctypes.c_void_p),
                ("maxBlocks", ctypes.c_int32), ("blocksDim", ctypes.c_int32 * 3),
                ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("depth", ctypes.c_uint32),
                ("origin", ctypes.c_float * 3), ("cellSize", ctypes.c_float),
                ("d_primitives", ctypes.c_void_p), ("numPrimitives", ctypes.c_uint32),
                ("numBVHPrimitives", ctypes.c_uint32), ("d_bvhNodes", ctypes.c_void_p),
                ("numBVHNodes", ctypes.c_uint32), ("d_packetVertexCounts", ctypes.c_void_p),
                ("d_packetVertexOffsets", ctypes.c_void_p), ("d_blockToActiveId", ctypes.c_void_p),
                ("d_dcCornerMasks", ctypes.c_void_p), ("d_dcCellVertexOffsets", ctypes.c_void_p),
                ("d_dcCellVertices", ctypes.c_void_p), ("d_dcCellNormals", ctypes.c_void_p),
                ("d_dcCellNormalsTmp", ctypes.c_void_p), ("d_vertices", ctypes.c_void_p),
                ("d_vertexColors", ctypes.c_void_p), ("d_indices", ctypes.c_void_p),
                ("d_uvCoords", ctypes.c_void_p), ("d_primitiveIDs", ctypes.c_void_p),
                ("d_normals", ctypes.c_void_p), ("maxVertices", ctypes.c_uint32), ("maxIndices", ctypes.c_uint32),
                ("d_totalVertices", ctypes.c_void_p), ("d_totalIndices", ctypes.c_void_p)]


assert ctypes.sizeof(SdfGrid) == 232

# every symbol include/sdfmesh_b200.h declares
DROPIN_SYMBOLS = ["launchScoutActiveBlocks", "launchCountActiveBlockTriangles", "launchGenerateActiveBlockTriangles",
                  "launchBuildBlockToActiveMap", "launchDCMarkCells", "launchDCSolveCellVertices",
                  "launchDCRecomputeNormalsAtVertices", "launchDCSmoothCellNormals", "launchDCCountQuads",
                  "launchDCGenerateQuads", "getScanStorageSize", "launchScan"]
SDF_CULL_NONE, SDF_CULL_SURROGATE, SDF_CULL_EXACT = 0, 1, 2
SURROGATE_SYMBOLS = ["sdf_engine_set_coarse_cull", "sdf_surrogate_default_config", "sdf_surrogate_train", "sdf_surrogate_enable",
                     "sdf_surrogate_audit", "sdf_surrogate_num_params", "sdf_surrogate_set_params",
                     "sdf_surrogate_get_params", "sdf_surrogate_forward", "sdf_surrogate_gradient"]
BATCH_SYMBOLS = ["sdf_batch_create", "sdf_batch_destroy", "sdf_batch_set_scenes", "sdf_batch_extract",
                 "sdf_batch_capture", "sdf_batch_read_buffer"]
STATIC_SCOUT_SYMBOLS = ["sdf_scout_active_blocks_static"]
SCOUT_STATIC_MAX_BLOCKS = 1 << 20  # SDF_SCOUT_STATIC_MAX_BLOCKS of the header
EXPORT_SYMBOLS = ["sdf_write_obj"]
UVPACK_SYMBOLS = ["sdf_uv_pack_default_config", "sdf_uv_atlas_create", "sdf_uv_atlas_destroy",
                  "sdf_uv_atlas_extract_charts", "sdf_uv_atlas_create_islands", "sdf_uv_atlas_pack",
                  "sdf_uv_atlas_remap", "sdf_uv_atlas_remap_placements", "sdf_uv_atlas_run", "sdf_uv_atlas_read",
                  "sdf_uv_pack_random_draws"]


class UvPackConfig(ctypes.Structure):
    """sdf_uv_pack_config (the reference's PackingConfig)."""
    _fields_ = [(n, ctypes.c_int32) for n in (
        "grid_size", "grid_resolution", "max_iterations", "margin_cells", "enable_rotation", "x_alignment",
        "max_candidates_per_island", "max_drop_steps", "shuffle_order_per_attempt", "random_seed")]

    def as_list(self):
        return [getattr(self, n) for n, _ in self._fields_]


class UvChart(ctypes.Structure):
    _fields_ = [("primitive_id", ctypes.c_int32), ("num_triangles", ctypes.c_int32),
                ("uv_min", ctypes.c_float * 2), ("uv_max", ctypes.c_float * 2)]


class UvGrid(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("stride", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("word_offset", ctypes.c_int64)]


class UvIsland(ctypes.Structure):
    _fields_ = [("island_index", ctypes.c_int32), ("primitive_id", ctypes.c_int32), ("num_triangles", ctypes.c_int32),
                ("min_cell_x", ctypes.c_int32), ("min_cell_y", ctypes.c_int32), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32), ("pad", ctypes.c_int32), ("mask", UvGrid), ("collision", UvGrid),
                ("mask90", UvGrid), ("collision90", UvGrid), ("row_bounds", ctypes.c_int64),
                ("row_bounds90", ctypes.c_int64), ("profile", ctypes.c_int64), ("profile90", ctypes.c_int64)]


class UvPlacement(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("island_index", "grid_x", "grid_y", "rotation")]


class UvSolution(ctypes.Structure):
    _fields_ = [("num_placed", ctypes.c_int32), ("utilized_width", ctypes.c_int32),
                ("utilized_height", ctypes.c_int32), ("flags", ctypes.c_int32), ("fitness", ctypes.c_float),
                ("seed", ctypes.c_int32)]


class UvAtlasInfo(ctypes.Structure):
    _fields_ = [("success", ctypes.c_int32), ("atlas_width", ctypes.c_int32), ("atlas_height", ctypes.c_int32),
                ("num_placed", ctypes.c_int32), ("fitness", ctypes.c_float), ("scaling_factor", ctypes.c_float),
                ("num_charts", ctypes.c_int32), ("num_islands", ctypes.c_int32), ("num_solutions", ctypes.c_int32),
                ("best_solution", ctypes.c_int32), ("shelf_width", ctypes.c_int32),
                ("candidate_loop_open", ctypes.c_int32), ("ms_pack", ctypes.c_float),
                ("reserved", ctypes.c_float * 3)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}
ENGINE_SYMBOLS = ["sdf_engine_create", "sdf_engine_destroy", "sdf_engine_configure", "sdf_engine_set_scene",
                  "sdf_engine_set_scene_device",
                  "sdf_engine_set_scene_async", "sdf_engine_extract_async", "sdf_engine_extract_wait",
                  "sdf_engine_extract", "sdf_engine_set_timing", "sdf_engine_set_debug", "sdf_engine_get_bvh",
                  "sdf_build_bvh_host",
                  "sdf_engine_buffer", "sdf_engine_read_buffer", "sdf_engine_eval", "sdf_engine_eval_distance", "sdf_engine_eval_normals", "sdf_engine_count_work", "sdf_measure_fp32_peak", "sdf_extract", "sdf_last_error", "sdf_version"]

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built; run `python -m cudasdf_b200.build` first")
    L = ctypes.CDLL(LIB_PATH)
    vp, i, f, u, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_uint, ctypes.c_size_t
    G = ctypes.POINTER(SdfGrid)
    L.launchScoutActiveBlocks.argtypes = [G, f]
    L.launchCountActiveBlockTriangles.argtypes = [G, i, f]
    L.launchGenerateActiveBlockTriangles.argtypes = [G, i, f]
    L.launchBuildBlockToActiveMap.argtypes = [G, i]
    L.launchDCMarkCells.argtypes = [G, i, f]
    L.launchDCSolveCellVertices.argtypes = [G, i, f, u, f]
    L.launchDCRecomputeNormalsAtVertices.argtypes = [G, i, f]
    L.launchDCSmoothCellNormals.argtypes = [G, i, f]
    L.launchDCCountQuads.argtypes = [G, i]
    L.launchDCGenerateQuads.argtypes = [G, i, f]
    L.getScanStorageSize.argtypes = [u, ctypes.POINTER(sz)]
    L.launchScan.argtypes = [vp, vp, u, vp, sz]
    for name in DROPIN_SYMBOLS:
        getattr(L, name).restype = None
    L.sdf_engine_create.argtypes = [ctypes.POINTER(vp), i]
    L.sdf_engine_create.restype = i
    L.sdf_engine_destroy.argtypes = [vp]
    L.sdf_engine_destroy.restype = None
    L.sdf_engine_configure.argtypes = [vp, ctypes.POINTER(SdfConfig)]
    L.sdf_engine_configure.restype = i
    L.sdf_engine_set_scene.argtypes = [vp, vp, i]
    L.sdf_engine_set_scene.restype = i
    L.sdf_engine_set_scene_device.argtypes = [vp, vp, i, vp]
    L.sdf_engine_set_scene_device.restype = i
    L.sdf_engine_set_scene_async.argtypes = [vp, vp, i, vp]
    L.sdf_engine_set_scene_async.restype = i
    L.sdf_engine_extract_async.argtypes = [vp, f, ctypes.POINTER(SdfOutputs), vp, ctypes.POINTER(ctypes.c_uint64)]
    L.sdf_engine_extract_async.restype = i
    L.sdf_engine_extract_wait.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(SdfStats)]
    L.sdf_engine_extract_wait.restype = i
    L.sdf_engine_extract.argtypes = [vp, f, ctypes.POINTER(SdfOutputs), vp, ctypes.POINTER(SdfStats)]
    L.sdf_engine_extract.restype = i
    L.sdf_engine_set_timing.argtypes = [vp, i]
    L.sdf_engine_set_timing.restype = None
    L.sdf_engine_set_debug.argtypes = [vp, i]
    L.sdf_engine_set_debug.restype = None
    L.sdf_engine_get_bvh.argtypes = [vp, vp, i, ctypes.POINTER(i)]
    L.sdf_engine_get_bvh.restype = i
    L.sdf_engine_buffer.argtypes = [vp, i, ctypes.POINTER(sz)]
    L.sdf_engine_buffer.restype = vp
    L.sdf_engine_count_work.argtypes = [vp, vp]
    L.sdf_engine_count_work.restype = i
    L.sdf_measure_fp32_peak.argtypes = [vp]
    L.sdf_measure_fp32_peak.restype = i
    L.sdf_engine_eval.argtypes = [vp, vp, i, f, vp, vp]
    L.sdf_engine_eval_distance.argtypes = [vp, vp, i, f, vp, vp]
    L.sdf_engine_eval_distance.restype = i
    L.sdf_engine_eval_normals.argtypes = [vp, vp, i, f, f, vp, vp]
    L.sdf_engine_eval_normals.restype = i
    L.sdf_engine_eval.restype = i
    L.sdf_engine_read_buffer.argtypes = [vp, i, vp, sz]
    L.sdf_engine_read_buffer.restype = i
    L.sdf_extract.argtypes = [vp, i, ctypes.POINTER(SdfConfig), f, ctypes.POINTER(SdfOutputs), vp,
                              ctypes.POINTER(SdfStats)]
    L.sdf_extract.restype = i
    L.sdf_surrogate_default_config.argtypes = [ctypes.POINTER(SurrogateConfig)]
    L.sdf_surrogate_default_config.restype = None
    L.sdf_surrogate_train.argtypes = [vp, ctypes.POINTER(SurrogateConfig), ctypes.POINTER(SurrogateStats)]
    L.sdf_surrogate_train.restype = i
    L.sdf_surrogate_enable.argtypes = [vp, i]
    L.sdf_surrogate_enable.restype = i
    L.sdf_engine_set_coarse_cull.argtypes = [vp, i, f]
    L.sdf_engine_set_coarse_cull.restype = i
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.sdf_surrogate_audit.argtypes = [vp, f, i64p, i64p, i64p]
    L.sdf_surrogate_audit.restype = i
    L.sdf_surrogate_num_params.restype = i
    L.sdf_surrogate_set_params.argtypes = [vp, vp, vp, vp]
    L.sdf_surrogate_set_params.restype = i
    L.sdf_surrogate_get_params.argtypes = [vp, vp, vp, vp]
    L.sdf_surrogate_get_params.restype = i
    L.sdf_surrogate_forward.argtypes = [vp, vp, i, vp, vp]
    L.sdf_surrogate_forward.restype = i
    L.sdf_surrogate_gradient.argtypes = [vp, vp, vp, i, vp, vp]
    L.sdf_surrogate_gradient.restype = i
    L.sdf_batch_create.argtypes = [ctypes.POINTER(vp), i]
    L.sdf_batch_create.restype = i
    L.sdf_batch_destroy.argtypes = [vp]
    L.sdf_batch_destroy.restype = None
    L.sdf_batch_set_scenes.argtypes = [vp, ctypes.POINTER(BatchScene), i, u]
    L.sdf_batch_set_scenes.restype = i
    L.sdf_batch_extract.argtypes = [vp, f, ctypes.POINTER(SdfOutputs), ctypes.POINTER(SdfOutputs), vp, vp, vp,
                                    ctypes.POINTER(BatchStats)]
    L.sdf_batch_extract.restype = i
    L.sdf_batch_capture.argtypes = [vp, f, ctypes.POINTER(SdfOutputs), ctypes.POINTER(SdfOutputs), vp, i]
    L.sdf_batch_capture.restype = i
    L.sdf_batch_read_buffer.argtypes = [vp, i, i, vp, ctypes.POINTER(ctypes.c_size_t)]
    L.sdf_batch_read_buffer.restype = i
    L.sdf_scout_active_blocks_static.argtypes = [G, f]
    L.sdf_scout_active_blocks_static.restype = i
    L.sdf_write_obj.argtypes = [ctypes.c_char_p, vp, ctypes.c_uint64, vp, ctypes.c_uint64, vp]
    L.sdf_write_obj.restype = i
    L.sdf_uv_pack_default_config.argtypes = [ctypes.POINTER(UvPackConfig)]
    L.sdf_uv_pack_default_config.restype = None
    L.sdf_uv_atlas_create.argtypes = [ctypes.POINTER(vp)]
    L.sdf_uv_atlas_create.restype = i
    L.sdf_uv_atlas_destroy.argtypes = [vp]
    L.sdf_uv_atlas_destroy.restype = None
    L.sdf_uv_atlas_extract_charts.argtypes = [vp, vp, vp, ctypes.c_int64, vp, ctypes.POINTER(ctypes.c_int32)]
    L.sdf_uv_atlas_extract_charts.restype = i
    L.sdf_uv_atlas_create_islands.argtypes = [vp, vp, i, i, vp]
    L.sdf_uv_atlas_create_islands.restype = i
    L.sdf_uv_atlas_pack.argtypes = [vp, ctypes.POINTER(UvPackConfig), vp, ctypes.POINTER(UvAtlasInfo)]
    L.sdf_uv_atlas_pack.restype = i
    L.sdf_uv_atlas_remap.argtypes = [vp, vp, vp, ctypes.c_int64, i, vp]
    L.sdf_uv_atlas_remap.restype = i
    L.sdf_uv_atlas_remap_placements.argtypes = [vp, vp, vp, ctypes.c_int64, i, vp, i, i, i, i, vp]
    L.sdf_uv_atlas_remap_placements.restype = i
    L.sdf_uv_atlas_run.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.POINTER(UvPackConfig), vp,
                                   ctypes.POINTER(UvAtlasInfo)]
    L.sdf_uv_atlas_run.restype = i
    L.sdf_uv_atlas_read.argtypes = [vp, i, vp, ctypes.POINTER(ctypes.c_size_t)]
    L.sdf_uv_atlas_read.restype = i
    L.sdf_uv_pack_random_draws.argtypes = [vp, i, i, vp]
    L.sdf_uv_pack_random_draws.restype = i
    L.sdf_last_error.restype = i
    L.sdf_version.restype = ctypes.c_char_p
    _lib = L
    return L


def check(status: int, what: str = "") -> None:
    if status != SDF_OK:
        raise RuntimeError(f"{what}: {STATUS_NAMES.get(status, status)} (cuda error {lib().sdf_last_error()})")
