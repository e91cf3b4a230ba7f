"""Generate the UV atlas packer fixtures in tests/golden/ by running the reference's own CUDA code.

uvpack_ref.npz: a triangle soup with UVs and primitive ids made by the reference's own marching cubes
(oracle/_ref/libsdfref.so), and the reference's GridUVPacker (oracle/_ref/libuvpackref.so, compiled
from GridUVPacker.cu) run on it through its host API in main.cpp's order: the charts, the island masks,
the atlas and the remapped UVs. It also holds the curand draws each packing attempt consumes
(curand_init(seed, 0, 0) / curand(), recorded by the library's sdf_uv_pack_random_draws), so the CPU
oracle can replay the attempts.
uvpack_probes.npz: the reference's raster helpers (triangleArea2D, pointInTriangle, orientSign,
segmentsIntersect, triangleOverlapsCell, GridUVPacker.cu:41-165) through probe kernels, on cells of the
mesh's triangles in island cell space, half of them cells that lie wholly inside a triangle (where the
corner test decides by rounding alone).

Run on a GPU machine:

    python tests/golden/make_uvpack_golden.py --out <dir>

and copy the two .npz files into tests/golden/. Inputs are seeded, so a rerun reproduces them.
"""
from __future__ import annotations

import argparse
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cudasdf_b200 import scenes as S  # noqa: E402
from oracle import reflib as R  # noqa: E402
from oracle import uvpack_oracle as O  # noqa: E402

SCENE_SEED = 0x5DF0201
RES = 48
CONFIG = dict(O.APP_CONFIG, max_iterations=16)


def reference_mesh():
    prims = S.random_scene(20, SCENE_SEED, size_range=(0.15, 0.35), center_range=0.6)
    m = R.RefMesh(S.cell_size_for(RES))
    m.set_primitives(prims)
    st = m.run(technique=0)
    V = int(st["totalVertices"])
    uvs = m.copy(R.RB_UVS, np.float32, V * 2).reshape(V, 2)
    prim = m.copy(R.RB_PRIMIDS, np.float32, V)
    m.close()
    return uvs, prim


def probe_inputs(uvs, prim, rng, cells_per_kind=1500):
    """(a, b, c, corner) records with their cell, four per cell, from the mesh's triangles in the cell
    space of their island (uv * 64 - minCell)."""
    charts = O.extract_charts(uvs, prim)
    isl = O.create_islands(uvs, charts, 64, 4)
    tri = uvs.reshape(-1, 3, 2).astype(np.float32)
    mins = np.stack([isl["islands"]["min_x"], isl["islands"]["min_y"]], 1).astype(np.float32)
    inside, other = [], []
    for t in rng.permutation(len(charts["tri_chart"])):
        c = charts["tri_chart"][t]
        if c < 0:
            continue
        p = (tri[t] * np.float32(64) - mins[c]).astype(np.float32)
        x0, x1 = int(np.floor(p[:, 0].min())), int(np.ceil(p[:, 0].max()))
        y0, y1 = int(np.floor(p[:, 1].min())), int(np.ceil(p[:, 1].max()))
        o = lambda a, b, q: (b[0] - a[0]) * (q[1] - a[1]) - (b[1] - a[1]) * (q[0] - a[0])  # noqa: E731
        for y in range(y0, y1):
            for x in range(x0, x1):
                ks = [(x, y), (x + 1, y), (x + 1, y + 1), (x, y + 1)]
                s = [np.sign([o(p[0], p[1], k), o(p[1], p[2], k), o(p[2], p[0], k)]) for k in ks]
                full = all(abs(v.sum()) == 3 for v in s) and len({int(v[0]) for v in s}) == 1
                (inside if full else other).append((p, x, y))
        if len(inside) >= cells_per_kind and len(other) >= cells_per_kind:
            break
    rec, cells = [], []
    for p, x, y in inside[:cells_per_kind] + other[:cells_per_kind]:
        for k in ((x, y), (x + 1, y), (x + 1, y + 1), (x, y + 1)):
            rec.append([*p[0], *p[1], *p[2], *k])
            cells.append([x, y])
    return np.array(rec, np.float32), np.array(cells, np.int32)


def reference_probe(rec, cells):
    L = O.ref_lib()
    L.ref_uvpack_probe.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 5
    L.ref_uvpack_probe.restype = ctypes.c_int
    n = len(rec)
    out = dict(area=np.zeros(n, np.float32), pit=np.zeros(n, np.int32), ori=np.zeros(n, np.int32),
               seg=np.zeros(n, np.int32), ov=np.zeros(n, np.int32))
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    assert L.ref_uvpack_probe(p(rec), p(cells), n, p(out["area"]), p(out["pit"]), p(out["ori"]), p(out["seg"]),
                              p(out["ov"])) == 0
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    from cudasdf_b200.uvpack import random_draws
    uvs, prim = reference_mesh()
    ref = O.reference_run(uvs, prim, CONFIG)
    assert ref["loops_end"] and ref["atlas"]["success"]
    seeds = O.seeds(CONFIG["random_seed"], CONFIG["max_iterations"])
    draws = random_draws(seeds, 1 << 13)
    o = O.run(uvs, prim, CONFIG, lambda s: draws)
    used = int(o["packed"]["info"][:, 4].max())
    d = dict(uvs=uvs, prim=prim, config=O.config_list(CONFIG), seeds=seeds, draws=draws[:, :used + 64],
             chart_prim=ref["charts"]["prim"], chart_ntris=ref["charts"]["ntris"], chart_bounds=ref["charts"]["bounds"],
             chart_tris=ref["charts"]["tri_lists"], islands=ref["islands"], words=ref["words"], rb=ref["rb"],
             atlas_i=np.array([ref["atlas"][k] for k in ("success", "width", "height", "placed")], np.int32),
             atlas_f=np.array([ref["atlas"]["fitness"], ref["atlas"]["scaling"]], np.float32),
             placements=ref["atlas"]["placements"], uvs_out=ref["uvs"])
    np.savez_compressed(os.path.join(args.out, "uvpack_ref.npz"), **d)
    rec, cells = probe_inputs(uvs, prim, np.random.default_rng(SCENE_SEED))
    np.savez_compressed(os.path.join(args.out, "uvpack_probes.npz"), rec=rec, cells=cells, **reference_probe(rec, cells))
    print("vertices", len(uvs), "charts", len(d["chart_prim"]), "probes", len(rec), "draws used", used)


if __name__ == "__main__":
    main()
