"""Mass-point QEF dual contouring on the GPU against the oracles of oracle/qef_oracle.py, up to the
benchmark configuration: 512^3, 4,096 primitives, 3 projection steps, adaptive quad diagonal, FP64 for
cells with condition number above 1e4.

The Hermite samples are the kernel's own: edge points from the CPU oracle's interpEdgePoint (the
reference's arithmetic, bit-exact with the GPU's) and normals from the library's computeNormal entry
point (the same map() stencil and arithmetic the solve kernel runs). The engine's debug bit 1 keeps each
cell's QEF vertex before projection. Checks per cell:

* the FP32 / FP64 split equals, cell for cell, the float32 restatement of the kernel's decision, and the
  set of cells with FP64 condition number above the threshold (no allowance beyond cells within 1e-4
  relative of the threshold); the FP64-cell counter equals that count;
* the QEF vertex before projection, clamped to its cell as the mesh vertex is, is within 1e-4 cell of
  the FP64 oracle's, every cell; FP32-solved cells equal the float32 restatement bit for bit;
* the final quantised vertex equals the float32 restatement of projection, clamps and quantisation bit
  for bit (projection evaluates map() with the CPU oracle, bit-exact with the GPU's), and is within 1e-4
  cell of the FP64 oracle (QEF, projection, clamps) wherever the field is continuous along the two
  paths. The reference's map() jumps where its 256-step traversal cap or its BVH pruning cuts off a
  smooth-blended primitive; a cell whose FP64 and float32 paths sample the field on two sides of such a
  jump (|f difference| above the 1-Lipschitz bound plus 1e-5 cell) is counted, not compared;
* every quad is split along its shorter diagonal: the float32 restatement of the kernel's squared
  lengths from the decoded vertices, and the exact comparison in FP64 except where the two lengths agree
  to 1e-6 relative.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import qef_oracle as Q

pytestmark = pytest.mark.gpu

F32 = np.float32
T = 1e4  # cond_threshold of the benchmark configuration


def _extract(prims, res, projection_iters, adaptive=1, welded=False):
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    cell = S.cell_size_for(res)
    eng = Engine()
    eng.set_debug(2)
    mask = L.OUT_INDICES | (L.OUT_WELDED if welded else 0)
    eng.configure(make_config(cell, technique=L.TECH_DC, dc_solver=L.DC_SOLVER_MASSPOINT,
                              projection_iters=projection_iters, adaptive_diagonal=adaptive, cond_threshold=T,
                              out_mask=mask))
    eng.set_scene(prims)
    probe = MeshBuffers(1 << 16, mask)
    st = eng.extract(probe, allow_capacity=True)
    need = int(st["dc_cell_vertices"]) if welded else int(st["total_vertices"])
    del probe
    buf = MeshBuffers(max(need, int(st["total_vertices"])) + 1024, mask)
    st = eng.extract(buf)
    A, nd = int(st["active_blocks"]), int(st["dc_cell_vertices"])
    return {"eng": eng, "stats": st, "cell": cell, "res": res, "A": A, "nd": nd, "buf": buf,
            "list": eng.buffer(0, np.int32, A), "voff": eng.buffer(4, np.uint32, A * 512),
            "verts": eng.buffer(5, np.uint16, nd * 4).reshape(nd, 4),
            "qef": eng.buffer(11, np.float32, nd * 4).reshape(nd, 4)}


def _surface_cells(r):
    """(cell coords, corner values, vertex index) of every surface cell, in block / cell order."""
    res, eng = r["res"], r["eng"]
    nbx = (res + 7) // 8
    t = np.arange(512)
    lx, ly, lz = t % 8, (t // 8) % 8, t // 64
    corner_idx = np.stack([(lz + dz) * 81 + (ly + dy) * 9 + (lx + dx) for dx, dy, dz in Q.CORNERS], 1)
    out_xyz, out_cv, out_v = [], [], []
    all_rows = eng.buffer(8, np.float32, r["A"] * 736).reshape(r["A"], 736)  # 9^3 samples + pad per block
    chunk = 2048
    for a0 in range(0, r["A"], chunk):
        a1 = min(r["A"], a0 + chunk)
        rows = all_rows[a0:a1]
        lin = r["list"][a0:a1]
        bx, by, bz = lin % nbx, (lin // nbx) % nbx, lin // (nbx * nbx)
        x = 8 * bx[:, None] + lx[None, :]
        y = 8 * by[:, None] + ly[None, :]
        z = 8 * bz[:, None] + lz[None, :]
        inb = (x < res - 1) & (y < res - 1) & (z < res - 1)
        cv = rows[:, corner_idx]  # (blocks, 512, 8)
        code = ((cv > 0) * (1 << np.arange(8))).sum(-1)
        surf = inb & (code != 0) & (code != 255)
        out_xyz.append(np.stack([x[surf], y[surf], z[surf]], 1))
        out_cv.append(cv[surf])
        out_v.append(r["voff"][(np.arange(a0, a1)[:, None] * 512 + t[None, :])[surf]])
    return np.concatenate(out_xyz), np.concatenate(out_cv), np.concatenate(out_v).astype(np.int64)


def _hermite(r, xyz, cvs):
    """Padded Hermite samples of every cell: points relative to the cell corner (float32, as the kernel
    forms them), the library's normals there, counts; and the cell corners."""
    import torch
    cell = r["cell"]
    inside = cvs > 0
    cross = np.stack([inside[:, Q.EDGES[e, 0]] != inside[:, Q.EDGES[e, 1]] for e in range(12)], 1)
    owner, edge = np.nonzero(cross)  # cell-major, edges ascending: the kernel's sample order
    m = cross.sum(1)
    starts = np.concatenate([[0], np.cumsum(m)])
    pts = np.zeros((len(owner), 3), F32)
    step = 200_000
    for s0 in range(0, len(owner), step):
        o, e = owner[s0:s0 + step], edge[s0:s0 + step]
        rows = np.zeros((len(o), 16), F32)
        rows[:, :3] = -1.0
        rows[:, 3] = cell
        rows[:, 4:7] = xyz[o]
        rows[:, 7:15] = cvs[o]
        rows[:, 15] = e
        pts[s0:s0 + step] = O.probe(10, rows)[:, :3]
    nrm = r["eng"].eval_normals(torch.from_numpy(pts).cuda(), cell).cpu().numpy()
    cmin = (xyz.astype(np.float64) * np.float64(F32(cell)) - 1.0).astype(F32)  # fma(x, cell, -1)
    prel = (pts - cmin[owner]).astype(F32)
    return Q.pad_hermite(prel, starts), Q.pad_hermite(nrm.astype(F32), starts), m, cmin


def _check_cells(r, prims, iters):
    cell = r["cell"]
    xyz, cvs, vidx = _surface_cells(r)
    assert len(xyz) == r["nd"] and len(xyz) > 1000
    P, N, m, cmin = _hermite(r, xyz, cvs)
    x0 = r["qef"][vidx]
    gpu_fp64 = x0[:, 3] != 0
    x0 = x0[:, :3].copy()
    # split and FP32 branch: the float32 restatement of the kernel
    fp64_r, x32_r, _ = Q.fp32_split_and_solve(P, N, m, cmin, T)
    assert (gpu_fp64 == fp64_r).all(), int((gpu_fp64 != fp64_r).sum())
    assert int(r["stats"]["dc_fp64_cells"]) == int(fp64_r.sum())
    assert (x0[~fp64_r].view(np.uint32) == x32_r[~fp64_r].view(np.uint32)).all()
    # split and QEF vertices against FP64
    x64, cond = Q.masspoint_solve_batch(P, N, m, cmin, T)
    flips = gpu_fp64 != (cond > T)
    assert np.all(np.abs(cond[flips] / T - 1) < 1e-4), cond[flips][:10]
    # the QEF minimum can lie cells away from an ill-conditioned cell; what reaches the mesh is the
    # vertex clamped to the cell (widened by 0.1 cell, then the cell), compared in cell units there
    err0 = np.abs(Q.finish_batch(x0.astype(np.float64), cmin, cell) - Q.finish_batch(x64, cmin, cell)).max(1) / cell
    ok0 = ~flips
    assert err0[ok0].max() <= 1e-4, (err0[ok0].max(), cond[np.argmax(np.where(ok0, err0, 0))])
    # final vertices: float32 restatement bit for bit, FP64 within 1e-4 where the field is continuous
    scene = O.Scene(prims)

    def dist(p):
        return scene.map(p)[0][:, 0]

    q_gpu = r["verts"][vidx, :3]
    if iters > 0:
        nb, has = Q.mean_normals_f32(N, m)
        tr32, tr64 = [], []
        xp32 = Q.project_f32(x0, cmin, cell, nb, has, dist, iters, trace=tr32)
        q_r = Q.finish_encode_f32(xp32, cmin, cell)
        xp64 = Q.project_batch(x64, cmin, cell, N, m, dist, iters, trace=tr64)
        jump = np.zeros(len(xyz), bool)
        for (p32, d32), (p64, d64) in zip(tr32, tr64):
            gap = np.abs(p32.astype(np.float64) - p64.astype(np.float64)).max(1) * np.sqrt(3)
            jump |= np.abs(d32.astype(np.float64) - d64) > gap + 1e-5 * cell
    else:
        q_r = Q.finish_encode_f32(x0, cmin, cell)
        xp64 = x64
        jump = np.zeros(len(xyz), bool)
    assert (q_gpu == q_r).all(), int((q_gpu != q_r).any(1).sum())
    dec = cmin.astype(np.float64) + q_gpu.astype(np.float64) / 65535.0 * cell
    fin = Q.finish_batch(xp64, cmin, cell)
    err = np.abs(dec - fin).max(1) / cell
    keep = ~flips & ~jump
    assert jump.mean() < 0.005, jump.mean()
    worst = np.argsort(np.where(keep, err, 0))[-5:]
    assert err[keep].max() <= 1e-4, (err[worst], cond[worst])
    return {"cells": len(xyz), "fp64": int(fp64_r.sum()), "flips": int(flips.sum()), "jumps": int(jump.sum()),
            "max_err_qef": float(err0[ok0].max()), "max_err_final": float(err[keep].max())}


CASES = [(2, 64, 0), (3, 96, 3)]


@pytest.mark.parametrize("config,res,iters", CASES)
def test_masspoint_vertices_match_the_oracles(config, res, iters):
    from cudasdf_b200 import scenes as S
    prims = S.config_scene(config)
    r = _extract(prims, res, iters)
    _check_cells(r, prims, iters)
    r["eng"].close()


def _check_diagonals(r):
    """Every quad of the indexed output splits along a diagonal no longer than the other one."""
    V = int(r["stats"]["total_vertices"])
    idx = r["buf"].indices[:V].cpu().numpy().astype(np.int64).reshape(-1, 6)
    verts = r["buf"].vertices[:r["nd"]].cpu().numpy()[:, :3]  # the cell vertices, at their indices
    assert (idx >= 0).all() and (idx < r["nd"]).all()
    # a quad's two triangles (a, b, c), (a, c, d) share the diagonal a-c; the other runs b-d
    assert (idx[:, 0] == idx[:, 3]).all() and (idx[:, 2] == idx[:, 4]).all()
    a, b, c, d = verts[idx[:, 0]], verts[idx[:, 1]], verts[idx[:, 2]], verts[idx[:, 5]]
    shared = Q.diagonal_lengths_f32(a, c)
    other = Q.diagonal_lengths_f32(b, d)
    assert (shared <= other).all(), int((shared > other).sum())
    s64 = ((c.astype(np.float64) - a) ** 2).sum(1)
    o64 = ((d.astype(np.float64) - b) ** 2).sum(1)
    tie = np.abs(s64 - o64) <= 1e-6 * np.maximum(s64, o64)
    assert ((s64 <= o64) | tie).all()
    return len(idx)


@pytest.fixture(scope="module")
def c3_benchmark():
    """The benchmark configuration: 512^3, the 4,096-primitive scene, mass-point QEF with 3 projection
    steps and the adaptive diagonal, FP64 above cond 1e4; extracted once with the indexed output."""
    from cudasdf_b200 import scenes as S
    prims = S.config_scene(3)
    r = _extract(prims, 512, 3, welded=True)
    yield prims, r
    r["eng"].close()


def test_masspoint_benchmark_configuration_matches_the_oracles(c3_benchmark):
    prims, r = c3_benchmark
    info = _check_cells(r, prims, 3)
    assert info["cells"] > 100_000 and info["fp64"] > 1000
    print("c3 512^3:", info)


def test_adaptive_diagonal_benchmark_configuration(c3_benchmark):
    _, r = c3_benchmark
    assert _check_diagonals(r) > 100_000


def test_adaptive_diagonal_small():
    from cudasdf_b200 import scenes as S
    r = _extract(S.config_scene(2), 64, 3, welded=True)
    assert _check_diagonals(r) > 1000
    r["eng"].close()
