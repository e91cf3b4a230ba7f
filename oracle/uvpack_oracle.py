"""Python front end of the UV atlas packer oracle (oracle/uvpack_oracle.cpp): TEST INFRASTRUCTURE.

Restates the reference's GridUVPacker (src/SDFMesh/GridUVPacker.cu) step by step; only tests/ and
bench.py's CPU-baseline leg use it. `run()` does the four steps of main.cpp:1429-1442 for one mesh.
The packing attempts need each attempt's random draws (curand of the attempt's seed); the caller
passes a function seeds -> draws array.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libuvpack_oracle.so")

ISLAND_DTYPE = np.dtype([
    ("island_index", "<i4"), ("primitive_id", "<i4"), ("num_triangles", "<i4"), ("min_x", "<i4"), ("min_y", "<i4"),
    ("w", "<i4"), ("h", "<i4"), ("stride", "<i4"), ("stride90", "<i4"), ("pad", "<i4"),
    ("off_mask", "<i8"), ("off_coll", "<i8"), ("off_mask90", "<i8"), ("off_coll90", "<i8"),
    ("off_rb", "<i8"), ("off_rb90", "<i8")])
assert ISLAND_DTYPE.itemsize == 88

CFG_FIELDS = ("grid_size", "grid_resolution", "max_iterations", "margin_cells", "enable_rotation", "x_alignment",
              "max_candidates_per_island", "max_drop_steps", "shuffle_order_per_attempt", "random_seed")
# PackingConfig of the reference's only caller (main.cpp:1417-1427)
APP_CONFIG = dict(grid_size=2048, grid_resolution=64, max_iterations=256, margin_cells=4, enable_rotation=1,
                  x_alignment=8, max_candidates_per_island=16, max_drop_steps=256, shuffle_order_per_attempt=1,
                  random_seed=1337)
DRAWS_EXHAUSTED, CANDIDATE_LOOP_OPEN = 1, 2

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle oracle`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
        L.uvo_extract_charts.argtypes = [vp, vp, i64, vp, vp, vp, vp, i64]
        L.uvo_extract_charts.restype = i64
        L.uvo_island_plan.argtypes = [i, vp, vp, vp, i, i, vp, ctypes.POINTER(i64), ctypes.POINTER(i64)]
        L.uvo_island_plan.restype = i
        L.uvo_island_build.argtypes = [vp, i64, vp, i, vp, i, i, vp, vp]
        L.uvo_island_build.restype = i
        L.uvo_island_sort.argtypes = [i, vp, vp]
        L.uvo_island_sort.restype = None
        L.uvo_seeds.argtypes = [i, i, vp]
        L.uvo_seeds.restype = None
        L.uvo_shelf_width.argtypes = [i, vp, i]
        L.uvo_shelf_width.restype = i
        L.uvo_candidate_loops_end.argtypes = [i, vp, vp, i]
        L.uvo_candidate_loops_end.restype = i
        L.uvo_pack.argtypes = [i, vp, vp, vp, vp, i, i, vp, i64, vp, vp, vp, i]
        L.uvo_pack.restype = i
        L.uvo_select.argtypes = [i, vp, vp, i, i, vp, vp]
        L.uvo_select.restype = i
        L.uvo_remap.argtypes = [vp, vp, i64, i, vp, vp, vp, i, i, i, i]
        L.uvo_remap.restype = None
        L.uvo_probe.argtypes = [vp, vp, i64, vp, vp, vp, vp, vp]
        L.uvo_probe.restype = None
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def config_list(cfg: dict) -> np.ndarray:
    return np.array([int(cfg[n]) for n in CFG_FIELDS], dtype=np.int32)


def extract_charts(uvs: np.ndarray, prim: np.ndarray) -> dict:
    """ExtractCharts (GridUVPacker.cu:833-896)."""
    uvs = np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 2)
    prim = np.ascontiguousarray(prim, dtype=np.float32).reshape(-1)
    n = len(prim)
    T = n // 3
    tri_chart = np.empty(max(T, 1), np.int32)
    cap = max(T, 1)
    cp, cn, cb = np.empty(cap, np.int32), np.empty(cap, np.int32), np.empty((cap, 4), np.float32)
    nc = lib().uvo_extract_charts(_p(uvs), _p(prim), n, _p(tri_chart), _p(cp), _p(cn), _p(cb), cap)
    assert nc >= 0
    return dict(tri_chart=tri_chart[:T], prim=cp[:nc].copy(), ntris=cn[:nc].copy(), bounds=cb[:nc].copy())


def create_islands(uvs: np.ndarray, charts: dict, res: int, margin: int) -> dict:
    """CreateIslands (GridUVPacker.cu:898-1061). islands: chart order; order: the packing order (chart
    index of each sorted position)."""
    uvs = np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 2)
    nc = len(charts["prim"])
    isl = np.zeros(max(nc, 1), ISLAND_DTYPE)
    tw, tr = ctypes.c_int64(), ctypes.c_int64()
    L = lib()
    assert L.uvo_island_plan(nc, _p(charts["prim"]), _p(charts["ntris"]), _p(charts["bounds"]), res, margin,
                             _p(isl), ctypes.byref(tw), ctypes.byref(tr)) == 0
    words = np.zeros(max(tw.value, 1), np.uint32)
    rb = np.zeros(max(tr.value, 1), np.uint16)
    tri = np.ascontiguousarray(charts["tri_chart"], dtype=np.int32)
    assert L.uvo_island_build(_p(uvs), len(uvs), _p(tri), nc, _p(isl), res, margin, _p(words), _p(rb)) == 0
    order = np.zeros(max(nc, 1), np.int32)
    L.uvo_island_sort(nc, _p(isl), _p(order))
    return dict(islands=isl[:nc], words=words, rb=rb, order=order[:nc])


def probe(rec: np.ndarray, cells: np.ndarray) -> dict:
    """The raster helpers on (a, b, c, p) records with a cell each (uvo_probe)."""
    rec = np.ascontiguousarray(rec, dtype=np.float32).reshape(-1, 8)
    cells = np.ascontiguousarray(cells, dtype=np.int32).reshape(-1, 2)
    n = len(rec)
    out = dict(area=np.zeros(n, np.float32), pit=np.zeros(n, np.int32), ori=np.zeros(n, np.int32),
               seg=np.zeros(n, np.int32), ov=np.zeros(n, np.int32))
    lib().uvo_probe(_p(rec), _p(cells), n, _p(out["area"]), _p(out["pit"]), _p(out["ori"]), _p(out["seg"]),
                    _p(out["ov"]))
    return out


def seeds(random_seed: int, n: int) -> np.ndarray:
    out = np.zeros(max(n, 1), np.int32)
    lib().uvo_seeds(int(random_seed), int(n), _p(out))
    return out[:n]


def sorted_islands(isl: dict) -> np.ndarray:
    return np.ascontiguousarray(isl["islands"][isl["order"]])


def shelf_width(isl: dict, grid_size: int) -> int:
    s = sorted_islands(isl)
    return lib().uvo_shelf_width(len(s), _p(s), int(grid_size))


def candidate_loops_end(isl: dict, cfg: dict) -> bool:
    """False when the reference's packing kernel would draw candidates forever (GridUVPacker.cu:660-665)."""
    s = sorted_islands(isl)
    c = config_list(cfg)
    return bool(lib().uvo_candidate_loops_end(len(s), _p(s), _p(c), shelf_width(isl, cfg["grid_size"])))


def pack(isl: dict, cfg: dict, draws: np.ndarray, nthreads: int = 0) -> dict:
    """packSolutionKernel (GridUVPacker.cu:585-777) for every attempt, each fed with draws[attempt]."""
    s = sorted_islands(isl)
    c = config_list(cfg)
    nsol = min(int(cfg["max_iterations"]), 256)
    n = min(len(s), 256)
    draws = np.ascontiguousarray(draws, dtype=np.uint32).reshape(nsol, -1)
    info = np.zeros((max(nsol, 1), 5), np.int32)
    fit = np.zeros(max(nsol, 1), np.float32)
    pl = np.zeros((max(nsol, 1), max(n, 1), 4), np.int32)
    shelf = shelf_width(isl, cfg["grid_size"])
    threads = nthreads or os.cpu_count() or 1
    lib().uvo_pack(len(s), _p(s), _p(isl["words"]), _p(isl["rb"]), _p(c), shelf, nsol, _p(draws), draws.shape[1],
                   _p(info), _p(fit), _p(pl), threads)
    return dict(info=info[:nsol], fitness=fit[:nsol], placements=pl[:nsol, :n], shelf=shelf)


def select(packed: dict, num_islands: int, grid_size: int) -> dict:
    """The choice of PackIslands (GridUVPacker.cu:1188-1214, 1403-1420)."""
    ai = np.zeros(5, np.int32)
    af = np.zeros(2, np.float32)
    info = np.ascontiguousarray(packed["info"], dtype=np.int32)
    fit = np.ascontiguousarray(packed["fitness"], dtype=np.float32)
    lib().uvo_select(len(info), _p(info), _p(fit), num_islands, grid_size, _p(ai), _p(af))
    best = int(ai[4])
    placements = packed["placements"][best, :ai[3]].copy() if best >= 0 else np.zeros((0, 4), np.int32)
    return dict(success=int(ai[0]), width=int(ai[1]), height=int(ai[2]), placed=int(ai[3]), best=best,
                fitness=np.float32(af[0]), scaling=np.float32(af[1]), placements=placements)


def remap(uvs: np.ndarray, prim: np.ndarray, charts: dict, isl: dict, atlas: dict, res: int) -> np.ndarray:
    """RemapUVsToAtlas (GridUVPacker.cu:1441-1547); returns the new UVs (a copy)."""
    out = np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 2).copy()
    if not atlas["success"] or len(atlas["placements"]) == 0:
        return out
    prim = np.ascontiguousarray(prim, dtype=np.float32).reshape(-1)
    pl = np.ascontiguousarray(atlas["placements"], dtype=np.int32)
    isl_c = np.ascontiguousarray(isl["islands"])
    lib().uvo_remap(_p(out), _p(prim), len(out), len(charts["prim"]), _p(charts["prim"]), _p(isl_c), _p(pl),
                    len(pl), atlas["width"], atlas["height"], res)
    return out


def grids(isl: dict, k: int) -> dict:
    """The four grids of chart k as 2-D uint32 arrays (rows x stride words)."""
    d = isl["islands"][k]
    w, h, s0, s9 = int(d["w"]), int(d["h"]), int(d["stride"]), int(d["stride90"])
    W = isl["words"]
    return dict(mask=W[d["off_mask"]:d["off_mask"] + s0 * h].reshape(h, s0),
                collision=W[d["off_coll"]:d["off_coll"] + s0 * h].reshape(h, s0),
                mask90=W[d["off_mask90"]:d["off_mask90"] + s9 * w].reshape(w, s9),
                collision90=W[d["off_coll90"]:d["off_coll90"] + s9 * w].reshape(w, s9),
                row_bounds=isl["rb"][d["off_rb"]:d["off_rb"] + 2 * h].reshape(2, h),
                row_bounds90=isl["rb"][d["off_rb90"]:d["off_rb90"] + 2 * w].reshape(2, w))


def run(uvs: np.ndarray, prim: np.ndarray, cfg: dict, draws_for, nthreads: int = 0) -> dict:
    """The four steps of main.cpp:1429-1442. draws_for(seeds) -> (attempts, k) uint32 draws."""
    charts = extract_charts(uvs, prim)
    isl = create_islands(uvs, charts, cfg["grid_resolution"], cfg["margin_cells"])
    res = dict(charts=charts, islands=isl, loops_end=True)
    nisl = len(charts["prim"])
    too_big = any(int(d["w"]) > cfg["grid_size"] or int(d["h"]) > cfg["grid_size"] for d in isl["islands"])
    nsol = min(int(cfg["max_iterations"]), 256)
    if nisl == 0 or too_big or nsol <= 0:
        res["atlas"] = dict(success=0, width=0, height=0, placed=0, best=-1, fitness=np.float32(0),
                            scaling=np.float32(1), placements=np.zeros((0, 4), np.int32))
        res["uvs"] = np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 2).copy()
        return res
    res["loops_end"] = candidate_loops_end(isl, cfg)
    sd = seeds(cfg["random_seed"], nsol)
    packed = pack(isl, cfg, draws_for(sd), nthreads)
    res["seeds"] = sd
    res["packed"] = packed
    res["atlas"] = select(packed, nisl, cfg["grid_size"])
    res["uvs"] = remap(uvs, prim, charts, isl, res["atlas"], cfg["grid_resolution"])
    return res


# ------------------------------------------------------------------------------------------------
# the reference's own packer, compiled from its sources into oracle/_ref (GPU; tests only)
# ------------------------------------------------------------------------------------------------
REF_LIB_PATH = os.path.join(HERE, "_ref", "libuvpackref.so")
_ref = None


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB_PATH):
            raise RuntimeError(f"{REF_LIB_PATH} missing: run `make -C oracle ref`")
        R = ctypes.CDLL(REF_LIB_PATH)
        vp, i, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
        R.ref_uvpack_islands.argtypes = [vp, vp, i, i, i, i, vp, vp, vp, vp, i64, vp, vp, i64, ctypes.POINTER(i64), vp,
                                         i64, ctypes.POINTER(i64), vp]
        R.ref_uvpack_islands.restype = i
        R.ref_uvpack_pack.argtypes = [vp, vp, vp, vp, i, vp, vp]
        R.ref_uvpack_pack.restype = i
        R.ref_uvpack_release.restype = None
        _ref = R
    return _ref


def loops_end_from_dims(dims_sorted, cfg: dict) -> bool:
    """uvo_candidate_loops_end from the islands' (width, height) in packing order: shelf width
    (GridUVPacker.cu:1126-1138) and the candidate budget of packSolutionKernel (GridUVPacker.cu:601-665)."""
    G, A = int(cfg["grid_size"]), max(1, int(cfg["x_alignment"]))
    maxW = max((w for w, _ in dims_sorted), default=0)
    total = sum(w * h for w, h in dims_sorted)
    target = int(np.sqrt(np.float32(total) * np.float32(1.3), dtype=np.float32))
    shelf = max(maxW * 2 + maxW // 2, min(target, G))
    s1 = max(1, shelf)
    shelf_max = min(G, s1 - s1 % A if A > 1 else s1)
    budget = max(4, min(64, int(cfg["max_candidates_per_island"])))
    for w, h in list(dims_sorted)[:256]:
        for rot in ((0, 1) if cfg["enable_rotation"] else (0,)):
            iw, ih = (h, w) if rot else (w, h)
            if iw > G or ih > G:
                continue
            maxX = min(shelf_max, G) - iw
            if maxX >= 0 and maxX // A + 1 < budget:
                return False
    return True


def reference_run(uvs: np.ndarray, prim: np.ndarray, cfg: dict) -> dict:
    """The reference's ExtractCharts + CreateIslands, then, when every candidate loop of its packing
    kernel can end, PackIslands + RemapUVsToAtlas (main.cpp:1429-1442). Runs the reference's CUDA code."""
    uvs = np.ascontiguousarray(uvs, dtype=np.float32).reshape(-1, 2)
    prim = np.ascontiguousarray(prim, dtype=np.float32).reshape(-1)
    n = len(prim)
    T = n // 3 + 1
    R = ref_lib()
    cp, cn, cb = np.zeros(T, np.int32), np.zeros(T, np.int32), np.zeros((T, 4), np.float32)
    tri = np.zeros(T, np.uint32)
    info = np.zeros((T, 5), np.int32)
    wcap = 1 << 26
    words = np.zeros(wcap, np.uint32)
    rb = np.zeros(1 << 24, np.uint16)
    wu, ru = ctypes.c_int64(), ctypes.c_int64()
    ms = np.zeros(2, np.float64)
    nc = R.ref_uvpack_islands(_p(uvs), _p(prim), n, int(cfg["grid_resolution"]), int(cfg["margin_cells"]), T, _p(cp),
                              _p(cn), _p(cb), _p(tri), T, _p(info), _p(words), wcap, ctypes.byref(wu), _p(rb),
                              len(rb), ctypes.byref(ru), _p(ms))
    assert nc >= 0, "reference ExtractCharts / CreateIslands failed"
    out = dict(charts=dict(prim=cp[:nc].copy(), ntris=cn[:nc].copy(), bounds=cb[:nc].copy(),
                           tri_lists=tri[:int(cn[:nc].sum())].copy()),
               islands=info[:nc].copy(), words=words[:wu.value].copy(), rb=rb[:ru.value].copy(),
               ms_charts=float(ms[0]), ms_islands=float(ms[1]))
    dims = [(int(w), int(h)) for _, w, h, _, _ in info[:nc]]
    out["loops_end"] = loops_end_from_dims(dims, cfg)
    if not out["loops_end"]:
        R.ref_uvpack_release()
        return out
    ai, af = np.zeros(4, np.int32), np.zeros(2, np.float32)
    pl = np.zeros((max(nc, 1), 4), np.int32)
    uv_out = np.zeros_like(uvs)
    c = config_list(cfg)
    assert R.ref_uvpack_pack(_p(c), _p(ai), _p(af), _p(pl), len(pl), _p(uv_out), _p(ms)) == 0
    R.ref_uvpack_release()
    out["atlas"] = dict(success=int(ai[0]), width=int(ai[1]), height=int(ai[2]), placed=int(ai[3]),
                        fitness=np.float32(af[0]), scaling=np.float32(af[1]), placements=pl[:ai[3]].copy())
    out["uvs"] = uv_out
    out["ms_pack"], out["ms_remap"] = float(ms[0]), float(ms[1])
    return out


def reference_grids(ref: dict):
    """Per island of a reference_run (packing order): its four grids and row bounds, as `grids` gives them."""
    o, r = 0, 0
    res = []
    for _, w, h, _, _ in ref["islands"]:
        w, h = int(w), int(h)
        s0, s9 = (w + 31) // 32, (h + 31) // 32
        g = {}
        for k, (rows, s) in zip(("mask", "collision", "mask90", "collision90"), ((h, s0), (h, s0), (w, s9), (w, s9))):
            g[k] = ref["words"][o:o + rows * s].reshape(rows, s)
            o += rows * s
        g["row_bounds"] = ref["rb"][r:r + 2 * h].reshape(2, h)
        g["row_bounds90"] = ref["rb"][r + 2 * h:r + 2 * h + 2 * w].reshape(2, w)
        r += 2 * (h + w)
        res.append(g)
    return res
