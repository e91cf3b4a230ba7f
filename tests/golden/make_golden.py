"""Generate the golden fixtures in tests/golden/ by running the reference's own CUDA code.

The reference has no tests and no golden data of its own, so every fixture here is an output of
the reference itself: its __device__ functions through the probe kernels and its full
marching-cubes / dual-contouring pipelines through its own launchers (oracle/ref/, built by
``make -C oracle ref`` from the reference's sources). Run on a GPU machine:

    python tests/golden/make_golden.py --out <dir>

and copy the written .npz files into tests/golden/. Inputs are seeded, so a rerun reproduces them.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cudasdf_b200 import scenes as S  # noqa: E402
from oracle import reflib as R  # noqa: E402

IN_STRIDE = 96


def pad(cols: np.ndarray) -> np.ndarray:
    cols = np.asarray(cols, np.float32)
    out = np.zeros((cols.shape[0], IN_STRIDE), np.float32)
    out[:, :cols.shape[1]] = cols
    return out


def unit(v):
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def sd_params(rng, t, n):
    U = lambda a, b, k=1: rng.uniform(a, b, (n, k))  # noqa: E731
    z = lambda k: np.zeros((n, k))  # noqa: E731
    table = {
        S.SDF_SPHERE: lambda: np.hstack([U(0.2, 1.0), z(5)]),
        S.SDF_BOX: lambda: np.hstack([U(0.1, 0.8, 3), z(3)]),
        S.SDF_TORUS: lambda: np.hstack([U(0.3, 0.8), U(0.05, 0.3), z(4)]),
        S.SDF_CYLINDER: lambda: np.hstack([U(0.2, 1.0), U(0.1, 0.6), z(4)]),
        S.SDF_CAPSULE: lambda: np.hstack([U(0.2, 1.0), U(0.05, 0.4), z(4)]),
        S.SDF_CONE: lambda: np.hstack([U(0.2, 1.0), U(10.0, 60.0), z(4)]),
        S.SDF_ROUNDED_BOX: lambda: np.hstack([U(0.1, 0.8, 3), U(0.0, 0.2), z(2)]),
        S.SDF_ROUNDED_CYLINDER: lambda: np.hstack([U(0.2, 0.8), U(0.1, 0.4), U(0.02, 0.1), z(3)]),
        S.SDF_ROUNDED_CONE: lambda: np.hstack([U(0.3, 1.0), U(0.1, 0.4), U(0.02, 0.2), z(3)]),
        S.SDF_ELLIPSOID: lambda: np.hstack([U(0.2, 1.0, 3), z(3)]),
        S.SDF_TRIANGULAR_PRISM: lambda: np.hstack([U(0.2, 1.0, 2), z(4)]),
        S.SDF_OCTOHEDRON: lambda: np.hstack([U(0.2, 1.0), z(5)]),
        S.SDF_HEX_PRISM: lambda: np.hstack([U(0.1, 0.6, 2), z(4)]),
    }
    return table.get(t, lambda: U(0.1, 1.0, 6))()


def gen_probes(rng) -> dict:
    out = {}

    def run(name, which, cols, ncols_out, grid=None, t=0.0):
        res = R.probe(which, pad(cols), grid, t)
        out[name + "_in"] = np.asarray(cols, np.float32)
        out[name + "_out"] = res[:, :ncols_out].copy()

    # primitive SDFs, every type (15 = outside the enum: the default branch)
    for t in list(range(0, 13)) + [14, 15]:
        n = 1024
        p = rng.uniform(-1.2, 1.2, (n, 3))
        cols = np.hstack([np.full((n, 1), t), p, sd_params(rng, t, n)])
        run(f"sd{t}", R.PR_SD, cols, 1)

    n = 4096
    q = S.random_unit_quaternions(rng, n)
    sc = rng.uniform(0.02, 1.5, (n, 3))
    sc[: n // 2] = sc[: n // 2, :1]
    cols = np.hstack([rng.uniform(-1, 1, (n, 3)), rng.uniform(-0.8, 0.8, (n, 3)), q, sc])
    run("xform", R.PR_XFORM, cols, 3)

    n = 1024
    run("twist", R.PR_TWIST, np.hstack([rng.uniform(-1, 1, (n, 3)), rng.uniform(-4, 4, (n, 1))]), 3)
    run("bend", R.PR_BEND, np.hstack([rng.uniform(-1, 1, (n, 3)), rng.uniform(-4, 4, (n, 1))]), 3)
    run("sine", R.PR_SINE, np.hstack([rng.uniform(-1, 1, (n, 3)), rng.uniform(0, 10, (n, 1)),
                                      rng.uniform(-0.2, 0.2, (n, 1)), rng.uniform(0, 10, (n, 1))]), 1)

    # edge parameter: opposite signs, equal values, zeros, tiny gaps
    n = 4096
    v1 = rng.normal(0, 0.05, n)
    v2 = -np.sign(v1) * np.abs(rng.normal(0, 0.05, n))
    v2[:256] = v1[:256]
    v1[256:384] = 0.0
    v2[384:512] = 0.0
    v2[512:768] = v1[512:768] + rng.normal(0, 1e-12, 256)
    v1[768:1024] = rng.normal(0, 1e-8, 256)
    run("edget", R.PR_EDGET, np.stack([v1, v2], 1), 1)

    n = 4096
    run("lerp", R.PR_LERP, np.hstack([rng.uniform(-1, 1, (n, 6)), rng.uniform(0, 1, (n, 1))]), 3)

    n = 4096
    res = rng.choice([64, 96, 128, 192, 256, 512, 1024], n).astype(np.float32)
    cell = (np.float32(2.0) / res).astype(np.float32)
    ijk = np.floor(rng.uniform(0, 1, (n, 3)) * (res[:, None] + 1))
    org = np.full((n, 3), -1.0)
    org[n // 2:] = rng.uniform(-2, 2, (n // 2, 3))
    run("getloc", R.PR_GETLOC, np.hstack([org, cell[:, None], ijk]), 3)

    n = 4096
    res = rng.choice([64, 128, 256, 512, 1024], n).astype(np.float32)
    cell = (np.float32(2.0) / res).astype(np.float32)
    ijk = np.floor(rng.uniform(0, 1, (n, 3)) * (res[:, None] - 1))
    vals = rng.normal(0, 0.02, (n, 8))
    vals[: n // 8] = np.round(vals[: n // 8] * 100) / 100  # some exact ties
    edges = rng.integers(0, 12, (n, 1))
    run("interp", R.PR_INTERP, np.hstack([np.full((n, 3), -1.0), cell[:, None], ijk, vals, edges]), 3)

    n = 4096
    res = rng.choice([64, 128, 256, 512, 1024], n).astype(np.float32)
    cell = (np.float32(2.0) / res).astype(np.float32)
    p0 = rng.uniform(-1, 1, (n, 3))
    scale = cell[:, None] * rng.choice([1e-4, 5e-4, 9e-4, 1e-3, 1.1e-3, 0.5], (n, 1))
    p1 = p0 + rng.normal(0, 1, (n, 3)) * scale
    p2 = p0 + rng.normal(0, 1, (n, 3)) * cell[:, None]
    p2[:64, 0] = np.nan
    p1[64:128, 1] = np.inf
    run("degen", R.PR_DEGEN, np.hstack([p0, p1, p2, cell[:, None]]), 1)

    n = 4096
    A = rng.normal(0, 1, (n, 9))
    A[:256, 6:9] = A[:256, 3:6] * 2  # singular
    A[256:512, 6:9] = A[256:512, 3:6] + rng.normal(0, 1e-4, (256, 3))
    run("solve3", R.PR_SOLVE3, np.hstack([A, rng.normal(0, 1, (n, 3))]), 4)

    def qef_inputs(n, cellsz=0.01):
        m = rng.integers(0, 13, (n, 1))
        c = rng.uniform(-1, 1, (n, 3))
        pts = c[:, None, :] + rng.uniform(-0.5, 0.5, (n, 12, 3)) * cellsz
        base = unit(rng.normal(0, 1, (n, 3)))
        ns = base[:, None, :] + rng.normal(0, 1, (n, 12, 3)) * rng.choice([0.02, 0.3, 2.0], (n, 1, 1))
        ns[: n // 16, 3] = 0.0  # zero-length normals are skipped
        return m, c, pts.reshape(n, 36), ns.reshape(n, 36)

    n = 4096
    m, c, pts, ns = qef_inputs(n)
    run("qefreg", R.PR_QEFREG, np.hstack([m, np.full((n, 1), 0.05), c, pts, ns]), 4)
    m, c, pts, ns = qef_inputs(n)
    run("qef", R.PR_QEF, np.hstack([m, np.zeros((n, 4)), pts, ns]), 4)

    n = 4096
    res = rng.choice([64, 128, 256, 512, 1024], n).astype(np.float32)
    cell = (np.float32(2.0) / res).astype(np.float32)
    cmin = rng.uniform(-1, 1, (n, 3))
    pw = cmin + rng.uniform(-0.2, 1.2, (n, 3)) * cell[:, None]
    run("encv", R.PR_ENCV, np.hstack([pw, cmin, cell[:, None]]), 3)
    qv = rng.integers(0, 65536, (n, 3))
    run("decv", R.PR_DECV, np.hstack([qv, cmin, cell[:, None]]), 3)
    nn = rng.normal(0, 1, (n, 3)) * rng.choice([1e-7, 1.0, 3.0], (n, 1))
    run("encn", R.PR_ENCN, nn, 3)
    qn = rng.integers(-32767, 32768, (n, 3))
    qn[:64] = 0
    run("decn", R.PR_DECN, qn, 3)

    n = 8192
    p = rng.uniform(-1, 1, (n, 3))
    lo = rng.uniform(-1, 1, (n, 3))
    hi = lo + rng.uniform(0, 0.5, (n, 3))
    dv = np.maximum(np.maximum(lo - p, p - hi), 0)
    dist = np.sqrt((dv ** 2).sum(1)).astype(np.float32)
    dmin = dist * rng.choice([0.5, 1.0, 2.0], n).astype(np.float32)
    k = n // 4  # borderline: d_min one ulp either side of the float distance
    dmin[:k] = np.nextafter(dist[:k], np.float32(np.inf))
    dmin[k:2 * k] = np.nextafter(dist[k:2 * k], np.float32(-np.inf))
    run("aabb", R.PR_AABBD, np.hstack([p, lo, hi, dmin[:, None]]), 1)
    return out


def map_scene_probes(name: str, prims: np.ndarray, pts: np.ndarray, t: float, normals: int = 0) -> dict:
    mesh = R.RefMesh(2.0 / 64)
    nb = mesh.set_primitives(prims)
    grid = mesh.grid_bytes()
    res = R.probe(R.PR_MAP, pad(pts), grid, t)
    d = {f"{name}_prims": prims, f"{name}_nbvh": np.int32(nb), f"{name}_nodes": mesh.nodes(),
         f"{name}_sorted": mesh.primitives(len(prims), S.PRIM_DTYPE),
         f"{name}_pts": pts.astype(np.float32), f"{name}_map": res, f"{name}_time": np.float32(t)}
    if normals:
        npts = pts[:normals]
        d[f"{name}_npts"] = npts.astype(np.float32)
        d[f"{name}_normal"] = R.probe(R.PR_NORMAL, pad(npts), grid, t)[:, :3]
    mesh.close()
    return d


def gen_map_probes(rng) -> dict:
    out = {}
    for t in list(range(0, 13)) + [14]:
        prm = sd_params(rng, t, 1)[0]
        p = S.primitive(t, rng.uniform(-0.3, 0.3, 3), S.random_unit_quaternions(rng, 1)[0],
                        rng.uniform(0, 1, 3), S.SDF_UNION, 0.0, prm, rng.uniform(0.3, 1.2, 3))
        if t % 3 == 1:
            p["annular"] = rng.uniform(0.0, 0.05)
        if t % 4 == 2:
            p["rounding"] = rng.uniform(0.0, 0.05)
        out.update(map_scene_probes(f"single{t}", p, rng.uniform(-1, 1, (512, 3)), 0.0))
    for op in range(6):
        for k in (0.05, 0.3):
            a = S.primitive(S.SDF_SPHERE, (-0.15, 0.0, 0.0), color=(1, 0, 0), params=(0.35,))
            b = S.primitive(S.SDF_BOX, (0.15, 0.05, 0.0), S.random_unit_quaternions(rng, 1)[0], (0, 0, 1),
                            op, k, (0.25, 0.25, 0.25))
            c = S.primitive(S.SDF_TORUS, (0.0, -0.2, 0.1), color=(0, 1, 0), operation=S.SDF_UNION_BLEND,
                            blend=k, params=(0.3, 0.08))
            prims = np.concatenate([a, b, c])
            out.update(map_scene_probes(f"op{op}_k{int(k * 100)}", prims, rng.uniform(-0.7, 0.7, (1024, 3)), 0.0))
    out.update(map_scene_probes("c2", S.config_scene(2), rng.uniform(-1, 1, (32768, 3)), 0.0, normals=4096))
    out.update(map_scene_probes("c4", S.config_scene(4), rng.uniform(-1, 1, (16384, 3)), 0.0))
    out.update(map_scene_probes("showcase", S.showcase_scene(0.7), rng.uniform(-1.1, 1.1, (4096, 3)), 0.7,
                                normals=2048))
    return out


def run_pipeline(prims, res, technique, out_mask, t=0.0, qef_blend=1.0, max_vertices=50_000_000,
                 full=True, dc_normal_passes=False, cell=None, bmin=S.BOUNDS_MIN, bmax=S.BOUNDS_MAX) -> dict:
    mesh = R.RefMesh(cell if cell is not None else S.cell_size_for(res), bmin, bmax, max_vertices=max_vertices)
    mesh.set_primitives(prims)
    st = mesh.run(t, technique, qef_blend, out_mask, sort_active=True)
    nA = st["activeUsed"]
    V = st["totalVertices"]
    d = {"stats": json.dumps(st), "grid": json.dumps(mesh.grid_fields())}
    d["active"] = mesh.copy(R.RB_ACTIVE, np.int32, nA)
    counts = mesh.copy(R.RB_COUNTS, np.uint32, nA * 512)
    offsets = mesh.copy(R.RB_OFFSETS, np.uint32, nA * 512)
    verts = mesh.copy(R.RB_VERTS, np.float32, V * 4).reshape(V, 4)
    streams = {"verts": verts}
    if out_mask & R.OUT_COLORS:
        streams["colors"] = mesh.copy(R.RB_COLORS, np.float32, V * 4).reshape(V, 4)
    if out_mask & R.OUT_INDICES:
        streams["indices"] = mesh.copy(R.RB_INDICES, np.uint32, V)
    if out_mask & R.OUT_UVS:
        streams["uvs"] = mesh.copy(R.RB_UVS, np.float32, V * 2).reshape(V, 2)
    if out_mask & R.OUT_PRIMIDS:
        streams["primids"] = mesh.copy(R.RB_PRIMIDS, np.float32, V)
    if out_mask & R.OUT_NORMALS:
        streams["normals"] = mesh.copy(R.RB_NORMALS, np.float32, V * 4).reshape(V, 4)
    if technique == 1:
        d["dc_mask"] = mesh.copy(R.RB_DCMASK, np.uint8, nA * 512)
        dvoff = mesh.copy(R.RB_DCVOFF, np.uint32, nA * 512)
        nv = int(dvoff[-1] + (1 if d["dc_mask"][-1] not in (0, 255) else 0)) if nA else 0
        d["dc_voff"] = dvoff
        d["dc_vert"] = mesh.copy(R.RB_DCVERT, np.uint16, nv * 4).reshape(nv, 4)
        d["dc_norm"] = mesh.copy(R.RB_DCNORM, np.int16, nv * 4).reshape(nv, 4)
        if dc_normal_passes:
            mesh.dc_normal_passes(t, float(np.cos(np.deg2rad(30.0))))
            d["dc_norm_recomputed"] = mesh.copy(R.RB_DCNORM, np.int16, nv * 4).reshape(nv, 4)
            d["dc_norm_smoothed"] = mesh.copy(R.RB_DCNORMTMP, np.int16, nv * 4).reshape(nv, 4)
    if full:
        d["counts"] = counts
        d["offsets"] = offsets
        d.update(streams)
    else:
        d["counts_sha"] = hashlib.sha256(counts.tobytes()).hexdigest()
        d["offsets_sha"] = hashlib.sha256(offsets.tobytes()).hexdigest()
        d["counts_sum"] = np.uint64(counts.astype(np.uint64).sum())
        nz = counts.reshape(nA, 512).sum(1) if nA else np.zeros(0)
        d["block_totals"] = nz.astype(np.uint32)
        stride = max(1, V // 8192)
        for k, v in streams.items():
            d[k + "_sha"] = hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
            d[k + "_sum"] = v.astype(np.float64).reshape(V, -1).sum(0) if v.dtype != np.uint32 else np.uint64(v.astype(np.uint64).sum())
            d[k + "_sample"] = v[::stride].copy()
        d["sample_stride"] = np.int64(stride)
        for k in list(d.keys()):
            if k.startswith("dc_") and d[k].size > 200000:
                arr = d.pop(k)
                d[k + "_sha"] = hashlib.sha256(np.ascontiguousarray(arr).tobytes()).hexdigest()
                d[k + "_sample"] = arr[::max(1, len(arr) // 8192)].copy()
    mesh.close()
    return d


def batch_digests(out_dir, count=256):
    """Digests of the batched workload (scenes.batch_scenes: 256 scenes, primitive counts log-uniform in
    [16, 2048], grids from {64, 96, 128, 192, 256}^3, half marching cubes, half dual contouring with the
    reference's solver), each scene run alone through the reference's own CUDA path with a fresh mesh
    object (CudaSDFMesh.cpp keeps process-wide allocation sizes, :301, :314), VBO + EBO outputs, sorted
    active list. Per scene: primitive-record sha, active blocks, per-block vertex totals, per-cell count
    and offset sha, VBO and EBO sha, and for dual contouring the corner-mask, cell-vertex-offset and
    cell-vertex sha. Written to batch_c5.npz."""
    scenes = S.batch_scenes(count)
    cols = {k: [] for k in ("res", "technique", "nprims", "prims_sha", "active_count", "total_vertices",
                            "counts_sha", "offsets_sha", "verts_sha", "indices_sha", "dc_mask_sha", "dc_voff_sha",
                            "dc_vert_sha", "dc_vertices")}
    actives, totals = [], []
    for sc in scenes:
        prims, res, tech = sc["primitives"], sc["resolution"], sc["technique"]
        mesh = R.RefMesh(S.cell_size_for(res), max_vertices=24_000_000)
        mesh.set_primitives(prims)
        st = mesh.run(0.0, tech, 1.0, R.OUT_INDICES, sort_active=True)
        nA, V = st["activeUsed"], st["totalVertices"]
        counts = mesh.copy(R.RB_COUNTS, np.uint32, nA * 512)
        offsets = mesh.copy(R.RB_OFFSETS, np.uint32, nA * 512)
        verts = mesh.copy(R.RB_VERTS, np.float32, V * 4).reshape(V, 4)
        indices = mesh.copy(R.RB_INDICES, np.uint32, V)
        h = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()  # noqa: E731
        cols["res"].append(res)
        cols["technique"].append(tech)
        cols["nprims"].append(len(prims))
        cols["prims_sha"].append(h(prims))
        cols["active_count"].append(nA)
        cols["total_vertices"].append(V)
        cols["counts_sha"].append(h(counts))
        cols["offsets_sha"].append(h(offsets))
        cols["verts_sha"].append(h(verts))
        cols["indices_sha"].append(h(indices))
        actives.append(mesh.copy(R.RB_ACTIVE, np.int32, nA))
        totals.append(counts.reshape(nA, 512).sum(1).astype(np.uint32) if nA else np.zeros(0, np.uint32))
        if tech == 1:
            mask = mesh.copy(R.RB_DCMASK, np.uint8, nA * 512)
            dvoff = mesh.copy(R.RB_DCVOFF, np.uint32, nA * 512)
            nv = int(dvoff[-1] + (1 if mask[-1] not in (0, 255) else 0)) if nA else 0
            cols["dc_mask_sha"].append(h(mask))
            cols["dc_voff_sha"].append(h(dvoff))
            cols["dc_vert_sha"].append(h(mesh.copy(R.RB_DCVERT, np.uint16, nv * 4)))
            cols["dc_vertices"].append(nv)
        else:
            for k in ("dc_mask_sha", "dc_voff_sha", "dc_vert_sha"):
                cols[k].append("")
            cols["dc_vertices"].append(0)
        mesh.close()
    starts = np.concatenate([[0], np.cumsum([len(a) for a in actives])]).astype(np.int64)
    np.savez_compressed(os.path.join(out_dir, "batch_c5.npz"), active=np.concatenate(actives).astype(np.int32),
                        block_totals=np.concatenate(totals).astype(np.uint32), active_starts=starts,
                        **{k: np.asarray(v) for k, v in cols.items()})


def single_type_scene(t, n, seed):
    rng = np.random.default_rng(seed)
    p = S.random_scene(n, seed, size_range=(0.1, 0.35), center_range=0.6)
    p["type"] = t
    p["operation"] = rng.choice([S.SDF_UNION, S.SDF_UNION_BLEND], n)
    p["blendFactor"] = rng.uniform(0.02, 0.2, n)
    prm = sd_params(rng, t, n)
    p["params"] = prm
    p["annular"] = np.where(rng.random(n) < 0.25, rng.uniform(0, 0.03, n), 0)
    p["rounding"] = np.where(rng.random(n) < 0.25, rng.uniform(0, 0.03, n), 0)
    return p


def mixed_scene_notrig(seed, n):
    """Every primitive type without transcendentals (the cone calls sinf/cosf), every operation,
    annular/rounding shells; no displacement."""
    rng = np.random.default_rng(seed)
    p = S.random_scene(n, seed, size_range=(0.08, 0.35), center_range=0.6)
    types = [t for t in range(15) if t != S.SDF_CONE]
    p["type"] = rng.choice(types, n)
    p["operation"] = rng.choice([0, 0, 3, 3, 1, 2, 4, 5], n)
    p["operation"][0] = S.SDF_UNION
    p["blendFactor"] = rng.uniform(0.02, 0.2, n)
    p["params"] = rng.uniform(0.2, 0.9, (n, 6))
    p["params"][:, 2] = np.where(p["type"] == S.SDF_ROUNDED_CONE, rng.uniform(0.05, 0.15, n), p["params"][:, 2])
    p["annular"] = np.where(rng.random(n) < 0.2, rng.uniform(0, 0.03, n), 0)
    p["rounding"] = np.where(rng.random(n) < 0.2, rng.uniform(0, 0.03, n), 0)
    return p


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True, help="directory for the fixture files")
    ap.add_argument("--skip-full", action="store_true", help="skip the full-size digests")
    ap.add_argument("--only-odd", action="store_true", help="only the non-power-of-two grid fixtures")
    ap.add_argument("--only-types", action="store_true", help="only the per-primitive-type fixtures")
    ap.add_argument("--only-batch", action="store_true", help="only the batched-workload digests")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    t0 = time.time()
    if args.only_batch:
        batch_digests(args.out)
        print("done", time.time() - t0)
        return
    # one marching-cubes run per primitive type: union scenes of that type only, random transforms,
    # annular / rounding shells on some primitives (pins the per-type arithmetic inside the reference's
    # 8-corner evaluation, which can contract differently than a lone map() call)
    for t in list(range(0, 13)) + [14]:
        prims = single_type_scene(t, 24, S.SEED_BASE + 300 + t)
        d = run_pipeline(prims, 48, 0, R.OUT_ALL, 0.0)
        np.savez_compressed(os.path.join(args.out, f"mc_type{t}_48.npz"), prims=prims, res=np.int32(48),
                            technique=np.int32(0), out_mask=np.int32(R.OUT_ALL), time=np.float32(0.0), **d)
        print(f"mc_type{t}_48", json.loads(d["stats"])["totalVertices"], time.time() - t0, flush=True)
    if args.only_types:
        return
    # grids whose cell size is not a power of two and whose origin is not -1: here the products
    # i * cellSize round, so these pin how grid points are formed
    odd_bmin, odd_bmax = (-1.1, -1.05, -1.0), (1.1, 1.0, 1.05)
    odd_cell = float(np.float32(2.2) / np.float32(50))
    notrig = mixed_scene_notrig(21, 48)
    odd = [
        ("mc_c2_odd50", S.config_scene(2), 0, R.OUT_ALL, 0.0),
        ("dc_c2_odd50", S.config_scene(2), 1, R.OUT_ALL, 0.0),
        ("mc_mixed_odd50", notrig, 0, R.OUT_ALL, 0.0),
        ("dc_mixed_odd50", notrig, 1, R.OUT_ALL, 0.0),
    ]
    for name, prims, tech, mask, t in odd:
        d = run_pipeline(prims, 50, tech, mask, t, cell=odd_cell, bmin=odd_bmin, bmax=odd_bmax)
        np.savez_compressed(os.path.join(args.out, name + ".npz"), prims=prims, res=np.int32(50),
                            technique=np.int32(tech), out_mask=np.int32(mask), time=np.float32(t),
                            cell=np.float32(odd_cell), bmin=np.float32(odd_bmin), bmax=np.float32(odd_bmax), **d)
        print(name, json.loads(d["stats"]), time.time() - t0, flush=True)
    if args.only_odd:
        return
    rng = np.random.Generator(np.random.PCG64(S.SEED_BASE + 100))
    np.savez_compressed(os.path.join(args.out, "probes.npz"), **gen_probes(rng))
    print("probes", time.time() - t0, flush=True)
    rng = np.random.Generator(np.random.PCG64(S.SEED_BASE + 200))
    np.savez_compressed(os.path.join(args.out, "map_probes.npz"), **gen_map_probes(rng))
    print("map probes", time.time() - t0, flush=True)

    small = [
        ("mc_sphere64", S.sphere_scene(), 64, 0, R.OUT_ALL, 0.0),
        ("mc_sphere128", S.sphere_scene(), 128, 0, R.OUT_COLORS | R.OUT_INDICES | R.OUT_PRIMIDS, 0.0),
        ("mc_c2_64", S.config_scene(2), 64, 0, R.OUT_ALL, 0.0),
        ("mc_showcase64", S.showcase_scene(0.7), 64, 0, R.OUT_ALL, 0.7),
        ("dc_sphere64", S.sphere_scene(), 64, 1, R.OUT_ALL, 0.0),
        ("dc_c2_64", S.config_scene(2), 64, 1, R.OUT_ALL, 0.0),
        ("dc_showcase64", S.showcase_scene(0.7), 64, 1, R.OUT_ALL, 0.7),
        ("dc_c3_128", S.config_scene(3), 128, 1, R.OUT_COLORS | R.OUT_INDICES, 0.0),
    ]
    for name, prims, res, tech, mask, t in small:
        d = run_pipeline(prims, res, tech, mask, t, dc_normal_passes=(name == "dc_c2_64"))
        np.savez_compressed(os.path.join(args.out, name + ".npz"), prims=prims, res=np.int32(res),
                            technique=np.int32(tech), out_mask=np.int32(mask), time=np.float32(t), **d)
        print(name, json.loads(d["stats"]), time.time() - t0, flush=True)

    if not args.skip_full:
        full = [
            ("full_mc_c1", 1, 0, R.OUT_COLORS | R.OUT_INDICES, 50_000_000),
            ("full_mc_c2", 2, 0, R.OUT_COLORS | R.OUT_INDICES, 50_000_000),
            ("full_dc_c2", 2, 1, R.OUT_COLORS | R.OUT_INDICES, 50_000_000),
            ("full_dc_c3", 3, 1, R.OUT_INDICES, 100_000_000),
            ("full_mc_c4", 4, 0, R.OUT_INDICES, 150_000_000),
        ]
        for name, cfg, tech, mask, maxv in full:
            prims = S.config_scene(cfg)
            res = S.config_resolution(cfg)
            d = run_pipeline(prims, res, tech, mask, 0.0, max_vertices=maxv, full=False)
            np.savez_compressed(os.path.join(args.out, name + ".npz"), res=np.int32(res), config=np.int32(cfg),
                                technique=np.int32(tech), out_mask=np.int32(mask), **d)
            print(name, json.loads(d["stats"]), time.time() - t0, flush=True)
    print("done", time.time() - t0)


if __name__ == "__main__":
    main()
