"""Shared helpers of the GPU parity tests: run the engine or the drop-in path and collect outputs."""
import hashlib
import json
import os

import numpy as np

from conftest import GOLDEN

STREAMS = ("verts", "colors", "indices", "uvs", "primids", "normals")


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def exclusive_scan(x):
    x = np.asarray(x, np.uint64)
    out = np.zeros(len(x), np.uint64)
    if len(x):
        out[1:] = np.cumsum(x)[:-1]
    return out.astype(np.uint32)


def engine_run(prims, res, technique, out_mask, time=0.0, max_vertices=None, debug=True, cell=None,
               bmin=(-1.0, -1.0, -1.0), bmax=(1.0, 1.0, 1.0), allow_capacity=False, **cfg_kw):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    cell = S.cell_size_for(res) if cell is None else cell
    eng = Engine()
    eng.configure(make_config(cell, bmin, bmax, technique=technique, out_mask=out_mask, **cfg_kw))
    eng.set_debug(1 if debug else 0)
    eng.set_scene(prims)
    buf = MeshBuffers(max_vertices or 4_000_000, out_mask)
    st = eng.extract(buf, time, allow_capacity=allow_capacity)
    A, V = int(st["active_blocks"]), int(st["total_vertices"])
    r = {"stats": st, "active": eng.buffer(0, np.int32, A)}
    r["verts"] = buf.vertices[:V].cpu().numpy()
    if buf.colors is not None:
        r["colors"] = buf.colors[:V].cpu().numpy()
    if buf.indices is not None:
        r["indices"] = buf.indices[:V].cpu().numpy().view(np.uint32)
    if buf.uvs is not None:
        r["uvs"] = buf.uvs[:V].cpu().numpy()
    if buf.primitive_ids is not None:
        r["primids"] = buf.primitive_ids[:V].cpu().numpy().view(np.float32)
    if buf.normals is not None:
        r["normals"] = buf.normals[:V].cpu().numpy()
    if technique == L.TECH_MC:
        if debug:
            r["counts"] = eng.buffer(1, np.uint32, A * 512)
            r["offsets"] = eng.buffer(2, np.uint32, A * 512)
    else:
        r["counts"] = eng.buffer(1, np.uint32, A * 512)
        r["offsets"] = exclusive_scan(r["counts"])
        r["dc_mask"] = eng.buffer(3, np.uint8, A * 512)
        r["dc_voff"] = eng.buffer(4, np.uint32, A * 512)
        nd = int(st["dc_cell_vertices"])
        r["dc_vert"] = eng.buffer(5, np.uint16, nd * 4).reshape(nd, 4)
        r["dc_norm"] = eng.buffer(6, np.int16, nd * 4).reshape(nd, 4)
    eng.close()
    return r


def dropin_run(prims, res, technique, out_mask, time=0.0, max_vertices=4_000_000, max_active=1 << 30, cell=None,
               bmin=(-1.0, -1.0, -1.0), bmax=(1.0, 1.0, 1.0)):
    import torch

    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.dropin import CudaSDFMesh
    mesh = CudaSDFMesh(max_active_blocks=max_active, max_vertices=max_vertices)
    mesh.Initialize(S.cell_size_for(res) if cell is None else cell, bmin, bmax)
    for p in prims:
        mesh.AddPrimitive(p)
    n = max_vertices
    dev = "cuda"
    bufs = {"verts": torch.empty((n, 4), dtype=torch.float32, device=dev)}
    if out_mask & L.OUT_COLORS:
        bufs["colors"] = torch.empty((n, 4), dtype=torch.float32, device=dev)
    if out_mask & L.OUT_INDICES:
        bufs["indices"] = torch.empty(n, dtype=torch.int32, device=dev)
    if out_mask & L.OUT_UVS:
        bufs["uvs"] = torch.empty((n, 2), dtype=torch.float32, device=dev)
    if out_mask & L.OUT_PRIMIDS:
        bufs["primids"] = torch.empty(n, dtype=torch.int32, device=dev)
    if out_mask & L.OUT_NORMALS:
        bufs["normals"] = torch.empty((n, 4), dtype=torch.float32, device=dev)
    mesh.Update(time, bufs["verts"], bufs.get("colors"), bufs.get("indices"), bufs.get("uvs"), bufs.get("primids"),
                bufs.get("normals"), technique=technique)
    V = mesh.GetTotalVertexCount()
    r = {"active": mesh.active_blocks(), "counts": mesh.packet("counts"), "offsets": mesh.packet("offsets")}
    for k, t in bufs.items():
        a = t[:V].cpu().numpy()
        if k == "indices":
            a = a.view(np.uint32)
        if k == "primids":
            a = a.view(np.float32)
        r[k] = a
    if technique == L.TECH_DC:
        r["dc_mask"] = mesh.dc_buffer("dcMasks", len(r["counts"]))
        r["dc_voff"] = mesh.dc_buffer("dcVertOffsets", len(r["counts"])).view(np.uint32)
        m = r["dc_mask"]
        nd = int(r["dc_voff"][-1]) + int(m[-1] not in (0, 255)) if len(m) else 0
        r["dc_vert"] = mesh.dc_buffer("dcVerts", nd).view(np.uint16)
        r["dc_norm"] = mesh.dc_buffer("dcNormals", nd)
    r["total_vertices"] = V
    return r


def compare(r, G, keys, exact=True):
    """Returns a list of human-readable mismatches (empty when all equal)."""
    bad = []
    for k in keys:
        if k not in G.files or k not in r:
            continue
        a, b = np.asarray(r[k]), np.asarray(G[k])
        if a.shape != b.shape:
            bad.append(f"{k}: shape {a.shape} != {b.shape}")
            continue
        if a.dtype.kind == "f":
            eq = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
        else:
            eq = a == b
        if not eq.all():
            rows = ~eq.reshape(len(eq), -1).all(1) if eq.ndim > 1 else ~eq
            bad.append(f"{k}: {int(rows.sum())} of {len(rows)} differ")
    return bad


def stats_of(G):
    return json.loads(str(G["stats"]))
