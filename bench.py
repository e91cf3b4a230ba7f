"""Benchmark: Gvoxels/s of SDF -> mesh extraction on one B200 (or N, one process per GPU).

Workload (default, c4): marching cubes over a 1024^3 grid on [-1, 1]^3 of a seeded composite scene of
16384 smooth-blended primitives (sphere/box/capsule/torus, sizes log-uniform in [0.02, 0.2]); VBO
(float4 positions) + EBO (uint32 indices). A step is one full extraction with the scene already on
the device: (surrogate coarse-block inference, once per scene ->) scout -> compaction -> block field
(own samples, then halos, then the gather's classification and counts) -> block scan -> emission.

  value  = grid samples (1024^3) per second of device time of the surrogate-culled extraction, summed
           over ranks; the network is trained, certified and audited once before the timed region
           (its cost is reported under "surrogate"), and the culled mesh is checked byte-identical
           to the plain one
  plain  = the same for the plain exact extraction (no surrogate)
  e2e    = the surrogate-culled extraction through the public engine API with host buffers: scene
           upload from pinned host memory + extraction + read-back of counts and the whole vertex buffer
  --impl reference: the reference's algorithm on the host cores (its own path exists only as CUDA,
           so the C restatement in oracle/ with OpenMP stands in), a bounded sample per step
  --impl reference-cuda: the reference's own CUDA sources (built into oracle/_ref) on the same GPU,
           driven in CudaSDFMesh::Update's stage order

Run: python bench.py [--gpus N --steps K --warmup W --config c4 --impl ours|reference --plain]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "c1": {"config": 1, "technique": 0, "workload": "mc_sphere_128"},
    "c2": {"config": 2, "technique": 0, "workload": "mc_256prims_256"},
    "c3": {"config": 3, "technique": 1, "workload": "dc_masspoint_4096prims_512",
           "dc": {"dc_solver": 1, "projection_iters": 3, "adaptive_diagonal": 1, "cond_threshold": 1e4}},
    "c4": {"config": 4, "technique": 0, "workload": "mc_16384prims_1024", "surrogate": True},
    # the 16,384-primitive scene of c4 on a 256^3 grid, surrogate on: a case small enough for captures of
    # the surrogate's tensor-core kernels and of the memory-bound stages
    "c4s": {"config": 4, "technique": 0, "workload": "mc_16384prims_256", "surrogate": True, "res": 256},
    # the 256^3 scene with the dual-contouring options of c3: a case small enough for kernel captures
    "c3s": {"config": 2, "technique": 1, "workload": "dc_masspoint_256prims_256",
            "dc": {"dc_solver": 1, "projection_iters": 3, "adaptive_diagonal": 1, "cond_threshold": 1e4}},
    "c5": {"config": 5, "technique": -1, "workload": "batch_256scenes_mixed_mc_dc", "batch": True},
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c4", choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-cuda"],
                    help="reference: the reference's algorithm on the host cores (its path exists only as CUDA, "
                         "so the CPU restatement in oracle/ stands in); reference-cuda: the reference's own "
                         "CUDA sources (oracle/_ref) on this GPU")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--plain", action="store_true", help="time the plain exact path only (no surrogate)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def max_over_ranks(x, world):
    """The maximum of x over all ranks (every rank's device time; the job takes the slowest)."""
    import torch
    if world == 1:
        return x
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, units_per_rank, ms_max):
    """Whole-job throughput of N replicas: every rank processes its own units; the job lasts as long
    as the slowest rank."""
    return world * units_per_rank / (ms_max * 1e-3) / 1e9


def fp32_peak_tflops():
    """FP32 FMA throughput of this GPU, measured by the library's own FMA loop (TFLOP/s)."""
    import ctypes

    from cudasdf_b200 import _lib as L
    v = ctypes.c_double(0)
    rc = L.lib().sdf_measure_fp32_peak(ctypes.byref(v))
    return v.value if rc == 0 else None


STAGES = ("ms_scout", "ms_field", "ms_scan", "ms_emit", "ms_classify")


def timed_extractions(eng, buf, steps, flush, world):
    """K extractions, each timed with CUDA events on the launching stream, L2 flushed before each; the
    engine's own per-stage events (recorded on the same stream) give the stage split of the same steps."""
    import torch
    stream = torch.cuda.current_stream()
    eng.set_timing(True)
    barrier(world)
    times, stages = [], {k: [] for k in STAGES}
    st = None
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = eng.extract(buf)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        for k in STAGES:
            stages[k].append(st[k])
    barrier(world)
    eng.set_timing(False)
    return times, st, {k: sum(v) / len(v) for k, v in stages.items()}


def run_ours(args, rank, world):
    import numpy as np
    import torch

    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config

    spec = CONFIGS[args.config]
    cfg_id, tech = spec["config"], spec["technique"]
    res = spec.get("res") or S.config_resolution(cfg_id)
    cell = S.cell_size_for(res)
    prims = S.config_scene(cfg_id)
    mask = L.OUT_INDICES
    surrogate = spec.get("surrogate", False) and not args.plain
    eng = Engine()
    eng.configure(make_config(cell, technique=tech, out_mask=mask, **spec.get("dc", {})))
    eng.set_scene(prims)
    # capacity: one extraction to size the buffers
    probe_buf = MeshBuffers(1 << 20, mask)
    st0 = eng.extract(probe_buf, allow_capacity=True)
    V = int(st0["total_vertices"])
    del probe_buf
    buf = MeshBuffers(V + 1024, mask)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    voxels = float(res) ** 3
    out = {"V": V, "res": res, "nprims": len(prims)}

    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    # ---- plain exact extraction
    for _ in range(args.warmup):
        eng.extract(buf)
    times, st, out["plain_stages"] = timed_extractions(eng, buf, args.steps, flush, world)
    plain_ms = max_over_ranks(sum(times) / len(times), world)
    out["plain"] = {"ms": plain_ms, "value": job_throughput(world, voxels, plain_ms), "stats": st}
    # marching cubes: scout, compaction, halo plan, own samples, halo misses, gather (classification and
    # counts), block scan, emission; dual contouring (mass-point, projection steps): scout, compaction,
    # block map, halo plan, own samples, halo misses, gather, mark, cell scan, Hermite representatives,
    # Hermite normals, solve, projection, quad counts, block scan, quad list, quad normals (and their
    # emission), quads
    launches_per_step = 8 if tech == 0 else 18
    if surrogate:
        plain_verts = buf.vertices[:V].clone()
        t0 = time.perf_counter()
        sst = eng.surrogate_train()
        torch.cuda.synchronize()
        train_wall = (time.perf_counter() - t0) * 1e3
        audit = eng.surrogate_audit(0.0)
        out["surrogate"] = {"train": sst, "train_wall_ms": train_wall, "audit": audit}
        if audit["violations"] == 0:
            eng.surrogate_enable(True)  # the coarse values are kept while the scene is unchanged
        else:  # the exact audit decides: a violated certificate falls back to the plain path
            out["surrogate"]["fallback"] = "audit found active blocks in culled coarse blocks"
        for _ in range(args.warmup):
            eng.extract(buf)
        buf.vertices.zero_()
        times, st, out["stages"] = timed_extractions(eng, buf, args.steps, flush, world)
        out["surrogate"]["identical_mesh"] = bool(int(st["total_vertices"]) == V and
                                                  torch.equal(buf.vertices[:V], plain_verts))
        # the method without the network: the exact map() at the coarse centres. With the reach alone
        # (no extra margin) its audit counts the active blocks it would lose; with the surrogate's
        # certified eps as extra margin it is timed like the surrogate
        eng.set_coarse_cull(L.SDF_CULL_EXACT, 0.0)
        audit_reach_only = eng.surrogate_audit(0.0)
        eng.set_coarse_cull(L.SDF_CULL_EXACT, float(sst["eps_cert"]))
        audit_x = eng.surrogate_audit(0.0)
        for _ in range(args.warmup):
            eng.extract(buf)
        buf.vertices.zero_()
        tx, stx, stages_x = timed_extractions(eng, buf, args.steps, flush, world)
        ms_x = max_over_ranks(sum(tx) / len(tx), world)
        out["exact_coarse"] = {"ms": ms_x, "value": job_throughput(world, voxels, ms_x), "stage_ms": stages_x,
                               "audit": audit_x, "audit_reach_only": audit_reach_only,
                               "scouted_blocks": int(stx["scouted_blocks"]),
                               "identical_mesh": bool(int(stx["total_vertices"]) == V and
                                                      torch.equal(buf.vertices[:V], plain_verts))}
        # back to the culling the timed value used
        eng.set_coarse_cull(L.SDF_CULL_SURROGATE if audit["violations"] == 0 else L.SDF_CULL_NONE)
        del plain_verts
    else:
        out["stages"] = out["plain_stages"]
    clk = clocks.stop()
    ms = max_over_ranks(sum(times) / len(times), world)
    out.update({"ms": ms, "value": job_throughput(world, voxels, ms), "stats": st, "clocks": clk, "times": times,
                "launches_per_step": launches_per_step})
    # end to end through the public API with host buffers, every step: the scene from host memory
    # (compared with the engine's copy; an unchanged scene keeps its BVH and surrogate) uploaded from
    # pinned memory, the extraction, and the whole vertex buffer read back into pinned host memory
    if not args.no_e2e:
        nodes, _ = eng.bvh()
        h2d = int(len(prims) * 160 + len(nodes) * 32)
        # (a) one step at a time: sdf_engine_set_scene, sdf_engine_extract, then the read-back
        host_verts = torch.empty((V + 1024, 4), dtype=torch.float32, pin_memory=True)
        pinned_prims = torch.from_numpy(prims.view(np.uint8).copy()).pin_memory()
        e2e_times = []
        for i in range(args.warmup + args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.set_scene(pinned_prims.numpy().view(S.PRIM_DTYPE))
            st = eng.extract(buf)
            n = int(st["total_vertices"])
            host_verts[:n].copy_(buf.vertices[:n], non_blocking=True)
            torch.cuda.synchronize()
            if i >= args.warmup:
                e2e_times.append((time.perf_counter() - t0) * 1e3)
        sync_ms = max_over_ranks(sum(e2e_times) / len(e2e_times), world)
        # (b) streamed: sdf_engine_set_scene_async + sdf_engine_extract_async on an extraction stream,
        # and step k's read-back on a copy stream while step k + 1 computes (two output buffers)
        e2e_ms = streamed_e2e(args, eng, prims, buf, V, mask, flush, world)
        out["e2e"] = {"value": world * voxels / (e2e_ms * 1e-3) / 1e9, "unit": "Gvoxels/s",
                      "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(V * 16 + 8), "ms_per_step": e2e_ms,
                      "mode": "streamed: step k+1 computes while step k's vertices are read back",
                      "one_step_at_a_time": {"value": world * voxels / (sync_ms * 1e-3) / 1e9,
                                             "ms_per_step": sync_ms}}
    if tech == L.TECH_MC:
        out["welded"] = welded_output(args, world, eng, buf, V, flush, voxels,
                                      make_config(cell, technique=tech, out_mask=mask | L.OUT_WELDED))
        eng.configure(make_config(cell, technique=tech, out_mask=mask))  # same grid: buffers and surrogate stay
    if tech == L.TECH_MC and rank == 0:
        out["dropin"] = dropin_host_timing(args, prims, res, voxels)
        out["uv_atlas"] = uv_atlas_timing(args)
    out["fp32_peak"] = fp32_peak_tflops()
    out["counters"] = count_work(eng, buf, res) if rank == 0 else None
    eng.close()
    if not args.no_e2e:
        del buf
        out["dynamic_scene"] = dynamic_scene(args, world, prims, res, cell, tech, mask, spec, V, flush)
    return out


DROPIN_HOST = os.path.join(ROOT, "cudasdf_b200", "dropin_host", "_build", "dropin_host")

# UV atlas packing (the reference's GridUVPacker): the mesh of the reference's own scene at 128^3 with
# UVs and primitive ids, packed with the configuration of its only caller (main.cpp:1417-1427)
UV_ATLAS_RES = 128
UV_ATLAS_WORKLOAD = ("uv atlas of the 128^3 showcase mesh, main.cpp:1417-1427 configuration "
                     "(2048^2 board, 256 attempts, margin 4, 16 candidates, drop cap 256, seed 1337)")


def uv_atlas_config():
    from cudasdf_b200.uvpack import PackingConfig
    return PackingConfig.app()


def uv_atlas_timing(args):
    """sdf_uv_atlas_run (charts, islands, the 256 packing attempts, remap) on this library's mesh of the
    scene, host wall time per atlas with the UVs restored between runs (outside the timed region)."""
    import torch

    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    from cudasdf_b200.uvpack import UVAtlas
    mask = L.OUT_UVS | L.OUT_PRIMIDS
    eng = Engine()
    eng.configure(make_config(S.cell_size_for(UV_ATLAS_RES), out_mask=mask))
    eng.set_scene(S.showcase_scene(0.0, animate=False))
    buf = MeshBuffers(4_000_000, mask)
    V = int(eng.extract(buf, 0.0)["total_vertices"])
    eng.close()
    uvs0 = buf.uvs[:V].clone()
    uvs = buf.uvs[:V].clone()
    prim = buf.primitive_ids[:V].view(torch.float32).clone()
    cfg = uv_atlas_config()
    a = UVAtlas()
    times, info = [], None
    for i in range(args.warmup + args.steps):
        uvs.copy_(uvs0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info = a.run(uvs, prim, cfg)
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append((time.perf_counter() - t0) * 1e3)
    a.close()
    ms = sorted(times)[len(times) // 2]
    return {"workload": UV_ATLAS_WORKLOAD, "ms_per_atlas": ms, "unit": "ms (host wall, median)",
            "ms_pack_kernel": info["ms_pack"], "vertices": V, "charts": info["num_charts"],
            "attempts": info["num_solutions"], "success": info["success"], "atlas": info["atlas_width"],
            "fitness": info["fitness"], "launches_per_atlas": 14}


def uv_atlas_reference(args):
    """The reference's GridUVPacker (oracle/_ref/libuvpackref.so, its own sources) on the reference's own
    mesh of the scene (its marching cubes, oracle/_ref/libsdfref.so), through its host API in main.cpp's
    order; the wall time of its four calls, which synchronise internally."""
    from cudasdf_b200 import scenes as S
    from oracle import reflib as R
    from oracle import uvpack_oracle as O
    import numpy as np
    m = R.RefMesh(S.cell_size_for(UV_ATLAS_RES))
    m.set_primitives(S.showcase_scene(0.0, animate=False))
    V = int(m.run(technique=0)["totalVertices"])
    uvs = m.copy(R.RB_UVS, np.float32, V * 2).reshape(V, 2)
    prim = m.copy(R.RB_PRIMIDS, np.float32, V)
    m.close()
    cfg = uv_atlas_config().as_dict()
    runs = []
    for _ in range(max(1, min(args.steps, 3))):
        r = O.reference_run(uvs, prim, cfg)
        if not r["loops_end"]:
            return {"workload": UV_ATLAS_WORKLOAD, "unavailable": "the reference's candidate loop would not end"}
        runs.append(r["ms_charts"] + r["ms_islands"] + r["ms_pack"] + r["ms_remap"])
    return {"workload": UV_ATLAS_WORKLOAD, "ms_per_atlas": sorted(runs)[len(runs) // 2],
            "unit": "ms (host wall, median)", "ms_pack": r["ms_pack"], "ms_islands": r["ms_islands"],
            "ms_charts": r["ms_charts"], "vertices": V, "success": r["atlas"]["success"],
            "atlas": r["atlas"]["width"], "runs": len(runs)}


def uv_atlas_cpu():
    """The CPU oracle of the packer (oracle/uvpack_oracle.cpp, the reference's loops, OpenMP over the
    attempts) on this library's mesh, fed with the attempts' curand draws."""
    import torch

    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    from cudasdf_b200.uvpack import random_draws
    from oracle import uvpack_oracle as O
    mask = L.OUT_UVS | L.OUT_PRIMIDS
    eng = Engine()
    eng.configure(make_config(S.cell_size_for(UV_ATLAS_RES), out_mask=mask))
    eng.set_scene(S.showcase_scene(0.0, animate=False))
    buf = MeshBuffers(4_000_000, mask)
    V = int(eng.extract(buf, 0.0)["total_vertices"])
    eng.close()
    uvs = buf.uvs[:V].cpu().numpy()
    prim = buf.primitive_ids[:V].view(torch.float32).cpu().numpy()
    cfg = uv_atlas_config().as_dict()
    draws = random_draws(O.seeds(cfg["random_seed"], cfg["max_iterations"]), 1 << 14)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    r = O.run(uvs, prim, cfg, lambda s: draws, nthreads=cores)
    secs = time.perf_counter() - t0
    return {"workload": UV_ATLAS_WORKLOAD, "ms_per_atlas": secs * 1e3, "cores": cores, "kind": "port",
            "success": r["atlas"]["success"], "atlas": r["atlas"]["width"]}


def dropin_host_timing(args, prims, res, voxels):
    """The drop-in as a user of the reference runs it: the reference's CudaSDFMesh.cpp, unchanged, linked
    against this library (cudasdf_b200/dropin_host), one Update per step with its host BVH build,
    primitive and node uploads, per-stage synchronisations and count read-back (VBO + EBO outputs).
    Host wall time per Update (after one warm-up Update) and the sum of Update's own kernel timers."""
    import tempfile

    import numpy as np
    if not os.path.exists(DROPIN_HOST):
        return {"unavailable": "dropin_host not built (it needs the reference tree at build time)"}
    with tempfile.TemporaryDirectory() as d:
        pf = os.path.join(d, "prims.bin")
        np.ascontiguousarray(prims).tofile(pf)
        r = subprocess.run([DROPIN_HOST, pf, str(res), "0", "2", str(max(args.steps, 1)), "-"], capture_output=True,
                           text=True, timeout=900)
    if r.returncode != 0:
        return {"unavailable": f"dropin_host exited {r.returncode}: {r.stderr.strip()[-200:]}"}
    info = json.loads(r.stdout.strip().splitlines()[-1])
    ms = float(info["ms_update_wall"])
    return {"value": voxels / (ms * 1e-3) / 1e9, "unit": "Gvoxels/s", "ms_per_step": ms,
            "ms_kernels": float(info["ms_update_kernels"]), "vertices": int(info["vertices"]),
            "steps": int(info["repeat"]),
            "path": "the reference's CudaSDFMesh::Update (CudaSDFMesh.cpp, unchanged) on this library's launch* "
                    "entry points: host BVH build, uploads and per-stage syncs every step, host wall time"}


def streamed_e2e(args, eng, prims, buf, V, mask, flush, world):
    """Milliseconds per step of the streamed end-to-end loop (see run_ours), over args.steps steps
    after args.warmup untimed ones."""
    import torch

    from cudasdf_b200.engine import MeshBuffers
    ext, cpy = torch.cuda.Stream(), torch.cuda.Stream()
    bufs = [buf, MeshBuffers(V + 1024, mask)]
    hosts = [torch.empty((V + 1024, 4), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    pending = []  # (ticket, buffer)

    def drain_one():
        tk, b = pending.pop(0)
        st = eng.extract_wait(tk)
        n = int(st["total_vertices"])
        with torch.cuda.stream(cpy):
            hosts[b][:n].copy_(bufs[b].vertices[:n], non_blocking=True)
            copied[b].record(cpy)

    def run(k, first):
        for i in range(k):
            b = (first + i) % 2
            ext.wait_event(copied[b])  # the buffer's previous read-back has left
            with torch.cuda.stream(ext):
                flush.zero_()
            eng.set_scene_async(prims, ext)
            tk = eng.extract_async(bufs[b], 0.0, ext)
            if pending:
                drain_one()
            pending.append((tk, b))
        while pending:
            drain_one()
        cpy.synchronize()
        ext.synchronize()

    run(max(args.warmup, 2), 0)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    run(args.steps, 0)
    ms = (time.perf_counter() - t0) * 1e3 / args.steps
    return max_over_ranks(ms, world)


def welded_output(args, world, eng, soup_buf, V, flush, voxels, cfg):
    """The same extraction (surrogate-culled when the engine has it enabled) with the indexed output:
    one vertex per crossed grid edge and three indices per triangle. Device time, a check of the mesh
    against the soup just extracted (every corner's welded vertex within 1e-6 of its soup vertex), and
    the end-to-end time with the smaller read-back (vertices + indices)."""
    import torch

    from cudasdf_b200 import _lib as L
    from cudasdf_b200.engine import MeshBuffers
    eng.configure(cfg)
    wbuf = MeshBuffers(V + 1024, L.OUT_INDICES)
    for _ in range(args.warmup):
        eng.extract(wbuf)
    times, st, stages = timed_extractions(eng, wbuf, args.steps, flush, world)
    ms = max_over_ranks(sum(times) / len(times), world)
    U = int(st["welded_vertices"])
    idx = wbuf.indices[:V].long()
    ok = int(st["total_vertices"]) == V and bool((idx >= 0).all() and (idx < U).all())
    if ok:
        err = (wbuf.vertices[idx, :3] - soup_buf.vertices[:V, :3]).abs().max().item()
        ok = err <= 1e-6
    res = {"value": job_throughput(world, voxels, ms), "ms_per_step": ms, "stage_ms": stages,
           "welded_vertices": U, "indices": V, "matches_soup": ok}
    if not args.no_e2e:
        host_v = torch.empty((U + 1, 4), dtype=torch.float32, pin_memory=True)
        host_i = torch.empty(V + 1, dtype=torch.int32, pin_memory=True)
        e2e = []
        for i in range(args.warmup + args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st = eng.extract(wbuf)
            u, n = int(st["welded_vertices"]), int(st["total_vertices"])
            host_v[:u].copy_(wbuf.vertices[:u], non_blocking=True)
            host_i[:n].copy_(wbuf.indices[:n], non_blocking=True)
            torch.cuda.synchronize()
            if i >= args.warmup:
                e2e.append((time.perf_counter() - t0) * 1e3)
        e_ms = max_over_ranks(sum(e2e) / len(e2e), world)
        res["e2e"] = {"value": world * voxels / (e_ms * 1e-3) / 1e9, "unit": "Gvoxels/s", "ms_per_step": e_ms,
                      "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(U * 16 + V * 4)}
    return res


def dynamic_scene(args, world, prims, grid, cell, tech, mask, spec, V, flush):
    """End to end with a scene that changes at every step (every primitive moved), as in an animated
    or edited scene: the reference rebuilds its BVH on the host at every Update (CudaSDFMesh.cpp:293).
    Two ways through the engine API: the host build (sdf_engine_set_scene) and the raw records copied
    from pinned host memory and the BVH built on the GPU (sdf_engine_set_scene_device). Each step:
    scene up, plain exact extraction, the vertex buffer down."""
    import numpy as np
    import torch

    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    eng = Engine()
    eng.configure(make_config(cell, technique=tech, out_mask=mask, **spec.get("dc", {})))
    moved = []
    for k in range(2):
        m = prims.copy()
        m["position"][:, 0] += np.float32(2e-3 * (k + 1))
        moved.append(m)
    pinned = [torch.from_numpy(m.view(np.uint8).reshape(-1).copy()).pin_memory() for m in moved]
    dev_prims = torch.empty(pinned[0].numel(), dtype=torch.uint8, device="cuda")
    cap = int(V * 1.05) + 4096
    dbuf = MeshBuffers(cap, mask)
    host_verts = torch.empty((cap, 4), dtype=torch.float32, pin_memory=True)
    voxels = float(grid) ** 3
    res = {}
    for path in ("host_bvh", "device_bvh"):
        times, build = [], []
        for i in range(args.warmup + args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if path == "host_bvh":
                eng.set_scene(moved[i % 2])
            else:
                dev_prims.copy_(pinned[i % 2], non_blocking=True)
                eng.set_scene_device(dev_prims)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            st = eng.extract(dbuf, allow_capacity=True)
            n = min(int(st["total_vertices"]), cap)
            host_verts[:n].copy_(dbuf.vertices[:n], non_blocking=True)
            torch.cuda.synchronize()
            if i >= args.warmup:
                times.append((time.perf_counter() - t0) * 1e3)
                build.append((t1 - t0) * 1e3)
        ms = max_over_ranks(sum(times) / len(times), world)
        res[path] = {"value": world * voxels / (ms * 1e-3) / 1e9, "unit": "Gvoxels/s", "ms_per_step": ms,
                     "scene_ms": sum(build) / len(build)}
    eng.close()
    res["primitives"] = len(prims)
    res["h2d_bytes_per_step"] = int(len(prims) * 160)
    res["d2h_bytes_per_step"] = int(V * 16)
    return res



def batch_configs():
    """The batched workload: 256 scenes, primitive counts log-uniform in [16, 2048], grids from
    {64, 96, 128, 192, 256}^3, half marching cubes and half dual contouring."""
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import make_config
    out = []
    for sc in S.batch_scenes(256):
        out.append((sc["primitives"], make_config(S.cell_size_for(sc["resolution"]), technique=sc["technique"],
                                                  out_mask=L.OUT_INDICES), sc["resolution"]))
    return out


def run_batch(args, rank, world):
    import numpy as np
    import torch

    from cudasdf_b200 import _lib as L
    from cudasdf_b200.engine import Batch, Engine, MeshBuffers
    cfgs = batch_configs()
    scenes = [(p, c) for p, c, _ in cfgs]
    voxels = float(sum(float(r) ** 3 for _, _, r in cfgs))
    b = Batch()
    t0 = time.perf_counter()
    b.set_scenes(scenes, L.OUT_INDICES)
    setup_ms = (time.perf_counter() - t0) * 1e3
    small_mc = MeshBuffers(1 << 20, L.OUT_INDICES)
    small_dc = MeshBuffers(1 << 20, L.OUT_INDICES)
    first, count, st0 = b.extract(small_mc, small_dc, allow_capacity=True)  # exact counts size the buffers
    del small_mc, small_dc
    mc = MeshBuffers(int(st0["mc_vertices"]) + 1024, L.OUT_INDICES)
    dc = MeshBuffers(int(st0["dc_vertices"]) + 1024, L.OUT_INDICES)
    t0 = time.perf_counter()
    b.capture(mc, dc, tune=True)
    tune_ms = (time.perf_counter() - t0) * 1e3
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        b.extract(mc, dc)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    barrier(world)
    times = []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        first, count, st = b.extract(mc, dc)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    barrier(world)
    clk = clocks.stop()
    ms = max_over_ranks(sum(times) / len(times), world)
    out = {"ms": ms, "value": world * voxels / (ms * 1e-3) / 1e9, "stats": st, "clocks": clk, "voxels": voxels,
           "setup_ms": setup_ms, "tune_ms": tune_ms, "scenes": len(cfgs)}
    # the same scenes one at a time through the engine (scene uploaded beforehand, extraction timed);
    # two untimed extractions first: the second sizes the dual-contouring lists by the first's counts
    solo = 0.0
    for p, c, _ in cfgs:
        eng = Engine()
        eng.configure(c)
        eng.set_scene(p)
        buf = MeshBuffers(int(np.max(count)) + 1024, L.OUT_INDICES)
        eng.extract(buf)
        eng.extract(buf)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.extract(buf)
        e1.record(stream)
        e1.synchronize()
        solo += e0.elapsed_time(e1)
        eng.close()
    out["solo_ms"] = solo
    # end to end: graph replay + read-back of both concatenated vertex buffers
    if not args.no_e2e:
        hm = torch.empty((int(st["mc_vertices"]), 4), dtype=torch.float32, pin_memory=True)
        hd = torch.empty((int(st["dc_vertices"]), 4), dtype=torch.float32, pin_memory=True)
        e2e = []
        for i in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, _, s2 = b.extract(mc, dc)
            hm.copy_(mc.vertices[:hm.shape[0]], non_blocking=True)
            hd.copy_(dc.vertices[:hd.shape[0]], non_blocking=True)
            torch.cuda.synchronize()
            if i >= args.warmup:
                e2e.append((time.perf_counter() - t0) * 1e3)
        e2e_ms = max_over_ranks(sum(e2e) / len(e2e), world)
        out["e2e"] = {"value": world * voxels / (e2e_ms * 1e-3) / 1e9, "unit": "Gvoxels/s", "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": int((hm.shape[0] + hd.shape[0]) * 16 + 8 * len(cfgs)),
                      "ms_per_step": e2e_ms,
                      "note": "the scenes stay resident between steps (uploaded once by sdf_batch_set_scenes)"}
    b.close()
    return out


def count_work(eng, buf, res):
    """One extraction with the library's work counters on: BVH node visits and leaf evaluations of
    the block-field kernel (algorithmic work for its FP32 roofline)."""
    import ctypes

    from cudasdf_b200 import _lib as L
    c = (ctypes.c_ulonglong * 8)()
    rc = L.lib().sdf_engine_count_work(eng.h, ctypes.byref(c))
    if rc != 0:
        return None
    return {"field_node_visits": int(c[0]), "field_leaf_evals": int(c[1]), "field_points": int(c[2]),
            "warp_pops": int(c[4]), "warp_box_tests": int(c[5]), "warp_leaf_steps": int(c[6]),
            "lane_efficiency_pops": int(c[0]) / max(32 * int(c[4]), 1),
            "lane_efficiency_leaves": int(c[1]) / max(32 * int(c[6]), 1)}


def cpu_full_extraction(cfg_id, res, cores):
    """One whole extraction of the workload by the CPU restatement of the reference's algorithm
    (oracle/sdf_oracle.c: scout of every block, then the block field, cases, counts, scan and vertex
    and index emission of every active block), OpenMP over `cores` host threads. Returns
    (seconds, active blocks, vertices)."""
    from cudasdf_b200 import scenes as S
    from oracle import oracle as O
    sc = O.Scene(S.config_scene(cfg_id))
    g = O.make_grid(S.cell_size_for(res))
    t0 = time.perf_counter()
    out = O.run(sc, g, 0.0, 0, 1.0, O.OR_INDICES, max_vertices=200_000_000, nthreads=cores)
    return time.perf_counter() - t0, out["nActive"], out["totalVertices"]


def cpu_baseline(args):
    """The CPU oracle (the reference's algorithm restated in C, OpenMP over all host threads): one whole
    extraction of the same workload, timed; the one-thread figure is a sample (a slice of the scout and
    a sample of the active blocks' marching cubes) scaled to the grid."""
    import numpy as np

    from cudasdf_b200 import scenes as S
    from oracle import oracle as O
    spec = CONFIGS[args.config]
    cfg_id = spec["config"]
    res = spec.get("res") or S.config_resolution(cfg_id)
    cores = os.cpu_count() or 1
    secs, nact, nverts = cpu_full_extraction(cfg_id, res, cores)
    # one thread, on a sample
    sc = O.Scene(S.config_scene(cfg_id))
    g = O.make_grid(S.cell_size_for(res))
    nblocks = g.bx * g.by * g.bz
    scout_n = min(nblocks, 16384)
    t0 = time.perf_counter()
    O.scout_range(sc, g, 0, scout_n, 0.0, 1)
    t1_scout = (time.perf_counter() - t0) / scout_n * nblocks
    rng = np.random.default_rng(0)
    cand = rng.choice(nblocks, size=min(nblocks, 262144), replace=False).astype(np.int32)
    flags = O.scout_flags(sc, g, cand, 0.0, cores)
    sample = cand[flags][:128]
    t0 = time.perf_counter()
    O.mc_blocks(sc, g, sample, 0.0, 1)
    t1_mc = (time.perf_counter() - t0) / max(len(sample), 1) * nact
    try:
        uv = uv_atlas_cpu()
    except Exception as ex:  # reported, never required
        uv = {"error": str(ex)}
    return {"value": float(res) ** 3 / secs / 1e9, "unit": "Gvoxels/s", "cores": cores, "kind": "port",
            "seconds": secs, "vertices": nverts, "uv_atlas": uv,
            "value_1thread": float(res) ** 3 / (t1_scout + t1_mc) / 1e9,
            "sample": f"one whole {res}^3 extraction ({nblocks} blocks scouted, {nact} active blocks meshed, "
                      f"{nverts} vertices) in {secs:.1f} s on {cores} threads; value_1thread: a scout slice of "
                      f"{scout_n} blocks + marching cubes of {len(sample)} active blocks on one thread, scaled"}


def run_reference_cpu(args):
    """The reference arm on the host cores: the reference's algorithm (restated in oracle/sdf_oracle.c,
    OpenMP over all host threads); every step, warm-up and timed, is one whole extraction of the
    workload (the scout of every block and the marching cubes of every active block)."""
    from cudasdf_b200 import scenes as S
    spec = CONFIGS[args.config]
    cfg_id = spec["config"]
    res = spec.get("res") or S.config_resolution(cfg_id)
    cores = os.cpu_count() or 1
    times = []
    nact = nverts = 0
    for step in range(args.warmup + args.steps):
        secs, nact, nverts = cpu_full_extraction(cfg_id, res, cores)
        if step >= args.warmup:
            times.append(secs)
    ms = sum(times) / len(times) * 1e3
    return {"value": float(res) ** 3 / (ms * 1e-3) / 1e9, "ms": ms, "cores": cores, "res": res,
            "sample": f"every step one whole {res}^3 extraction: {nact} active blocks, {nverts} vertices"}


def run_reference_batch(args):
    """The batched workload through the reference's path: one fresh mesh object per scene (its size
    caches are process-wide), the scenes one after another; time of the runs alone."""
    from cudasdf_b200 import scenes as S
    from oracle import reflib as R
    total = 0.0
    voxels = 0.0
    for sc in S.batch_scenes(256):
        res = sc["resolution"]
        voxels += float(res) ** 3
        m = R.RefMesh(S.cell_size_for(res), max_vertices=16_000_000)
        m.set_primitives(sc["primitives"])
        m.run(0.0, sc["technique"], 1.0, R.OUT_INDICES, sort_active=False)
        st = m.run(0.0, sc["technique"], 1.0, R.OUT_INDICES, sort_active=False)
        total += st["msWall"]
        m.close()
    return {"ms": total, "value": voxels / (total * 1e-3) / 1e9, "ms_kernels": None, "stats": {},
            "clocks": {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}, "res": "mixed"}


def run_reference(args, rank, world):
    """The reference's own CUDA path (oracle/_ref, built from the reference sources)."""
    import numpy as np

    from cudasdf_b200 import scenes as S
    from oracle import reflib as R
    spec = CONFIGS[args.config]
    if spec.get("batch"):
        return run_reference_batch(args)
    cfg_id, tech = spec["config"], spec["technique"]
    res = S.config_resolution(cfg_id)
    prims = S.config_scene(cfg_id)
    m = R.RefMesh(S.cell_size_for(res), max_vertices=150_000_000 if cfg_id >= 3 else 50_000_000)
    m.set_primitives(prims)
    for _ in range(args.warmup):
        m.run(0.0, tech, 1.0, R.OUT_INDICES, sort_active=False)
    clocks = ClockSampler(0)
    clocks.start()
    walls, kern = [], []
    for _ in range(args.steps):
        st = m.run(0.0, tech, 1.0, R.OUT_INDICES, sort_active=False)
        walls.append(st["msWall"])
        kern.append(st["msTotalKernels"])
    clk = clocks.stop()
    m.close()
    ms = sum(walls) / len(walls)
    out = {"ms": ms, "ms_kernels": sum(kern) / len(kern), "value": float(res) ** 3 / (ms * 1e-3) / 1e9,
           "stats": st, "clocks": clk, "res": res}
    if tech == 0:
        out["uv_atlas"] = uv_atlas_reference(args)
    return out


METRIC = "Gvoxels/s SDF\u2192mesh at 1024\u00b3, surrogate-culled vs plain, identical topology"


def main():
    args = parse()
    if args.impl != "ours":
        # the reference arms run on rank 0 alone; no process group, no CUDA context of ours
        rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    else:
        rank, world, local = dist_setup(args.gpus)
    spec = CONFIGS[args.config]
    headline = spec.get("surrogate", False)
    base = {"metric": METRIC if headline else f"Gvoxels/s SDF\u2192mesh extraction ({spec['workload']})",
            "unit": "Gvoxels/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene with the benchmark configuration's primitive law, sizes and counts)"}
    nprims = (len(__import__("cudasdf_b200.scenes", fromlist=["x"]).config_scene(spec["config"]))
              if spec["config"] <= 4 else "256 scenes")
    if args.impl == "reference" and spec["technique"] == 0:
        if rank != 0:
            return
        r = run_reference_cpu(args)
        line = dict(base)
        line.update({"impl": "reference", "value": r["value"], "ms_per_step": r["ms"],
                     "config": {"workload": spec["workload"], "grid": r["res"], "primitives": nprims,
                                "outputs": "VBO float4 + EBO uint32", "parallelism": f"{r['cores']} host threads",
                                "path": "plain exact marching cubes: the reference's algorithm restated in C, "
                                        "OpenMP; the reference's own path is CUDA only (see --impl reference-cuda)"},
                     "cpu_baseline": {"value": r["value"], "unit": "Gvoxels/s", "cores": r["cores"], "kind": "port",
                                      "sample": r["sample"]},
                     "e2e": {"value": r["value"], "unit": "Gvoxels/s", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0}})
        print(json.dumps(line))
        return
    if args.impl in ("reference", "reference-cuda"):
        if rank != 0:
            return
        r = run_reference(args, rank, world)
        line = dict(base)
        line.update({"impl": "reference", "value": r["value"], "ms_per_step": r["ms"],
                     "config": {"workload": spec["workload"], "grid": r["res"], "primitives": nprims,
                                "outputs": "VBO float4 + EBO uint32", "parallelism": "single GPU",
                                "path": "the reference's plain exact path (it has no surrogate)",
                                "l2": "per-stage host syncs of the reference (CudaSDFMesh.cpp:83-88)"},
                     "reference_kernel_ms": r["ms_kernels"], "reference_stats": r["stats"], "clocks": r["clocks"],
                     "uv_atlas": r.get("uv_atlas"),
                     "reference_cuda_path": {"value": r["value"], "unit": "Gvoxels/s",
                                             "sample": "the reference's own CUDA sources (oracle/_ref) on this GPU: "
                                                       "its per-stage launches, host syncs and count read-backs"},
                     "e2e": {"value": r["value"], "unit": "Gvoxels/s", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0}})
        print(json.dumps(line))
        return
    if spec.get("batch"):
        r = run_batch(args, rank, world)
        if rank != 0:
            return
        st = r["stats"]
        line = dict(base)
        line.update({"value": r["value"], "ms_per_step": r["ms"],
                     "config": {"workload": spec["workload"], "scenes": r["scenes"], "grids": "{64,96,128,192,256}^3",
                                "primitives": "log-uniform [16, 2048]", "techniques": "50 % MC / 50 % DC",
                                "total_blocks": st["total_blocks"], "active_blocks": st["active_blocks"],
                                "vertices": st["mc_vertices"] + st["dc_vertices"], "parallelism": f"replicas x{world}",
                                "execution": "one CUDA graph (one launch per stage for all scenes)",
                                "l2": "flushed between timed steps (256 MiB write)"},
                     "solo_sequential": {"ms_per_step": r["solo_ms"],
                                         "value": r["voxels"] / (r["solo_ms"] * 1e-3) / 1e9},
                     "setup_ms": r["setup_ms"], "autotune_and_capture_ms": r["tune_ms"],
                     "tuned_ctas_per_sm": st["tuned_ctas"], "clocks": r["clocks"],
                     "gpu_launches": 27 * args.steps})
        if "e2e" in r:
            line["e2e"] = r["e2e"]
        line["roofline"] = None
        print(json.dumps(line))
        return
    r = run_ours(args, rank, world)
    if rank != 0:
        return
    st = r["stats"]
    line = dict(base)
    line.update({"value": r["value"], "ms_per_step": r["ms"],
                 "config": {"workload": spec["workload"],
                            "path": "surrogate-culled exact marching cubes" if "surrogate" in r else "plain exact",
                            "grid": r["res"], "primitives": r["nprims"], "outputs": "VBO float4 + EBO uint32",
                            "active_blocks": st["active_blocks"], "vertices": st["total_vertices"],
                            "scouted_blocks": st["scouted_blocks"], "parallelism": f"replicas x{world}",
                            "l2": "flushed between timed steps (256 MiB write)"},
                 "stage_ms": r["stages"],
                 "plain": {"value": r["plain"]["value"], "ms_per_step": r["plain"]["ms"],
                           "stage_ms": r["plain_stages"]},
                 "triangles_per_s": (st["total_vertices"] // 3) / (r["ms"] * 1e-3),
                 "bvh_cap_hits": st["bvh_cap_hits"], "clocks": r["clocks"],
                 "dynamic_scene": r.get("dynamic_scene"), "welded": r.get("welded"), "dropin": r.get("dropin"),
                 "uv_atlas": r.get("uv_atlas"),
                 "gpu_launches": r["launches_per_step"] * args.steps})
    if "surrogate" in r:
        sg = r["surrogate"]
        line["surrogate"] = {"ratio_vs_plain": r["value"] / r["plain"]["value"],
                             "identical_mesh": sg.get("identical_mesh"), "audit": sg["audit"],
                             "eps_max": sg["train"]["eps_max"], "eps_cert": sg["train"]["eps_cert"],
                             "margin": sg["train"]["margin"], "final_loss": sg["train"]["final_loss"],
                             "train_ms": {"samples": sg["train"]["ms_samples"], "train": sg["train"]["ms_train"],
                                          "certify": sg["train"]["ms_certify"], "wall": sg["train_wall_ms"]},
                             "fallback": sg.get("fallback")}
        if "exact_coarse" in r:
            x = r["exact_coarse"]
            line["surrogate"]["without_network"] = {
                "method": "exact map() at every 32^3 coarse centre, culled beyond the surrogate's margin "
                          "(reach + eps_cert; SDF_CULL_EXACT)",
                "value": x["value"], "ms_per_step": x["ms"], "stage_ms": x["stage_ms"], "audit": x["audit"],
                "audit_reach_only": x["audit_reach_only"],
                "scouted_blocks": x["scouted_blocks"], "identical_mesh": x["identical_mesh"],
                "network_gain": r["value"] / x["value"]}
    if "e2e" in r:
        line["e2e"] = r["e2e"]
    line["roofline"] = roofline(r)
    line["stage_roofline"] = stage_roofline(r) if spec["technique"] == 0 else None  # marching cubes stages
    if not args.no_cpu_baseline and world == 1:
        try:
            line["cpu_baseline"] = cpu_baseline(args)
        except Exception as ex:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(ex)}
    print(json.dumps(line))


# FP32 operations per unit of algorithmic work in the block-field kernel (see the design notes):
# a BVH box test is 6 subtractions, 2 FMAs + 1 multiply (squared distance) and a square root;
# a leaf evaluation is the world->local transform (3 subtractions, the quaternion rotation: 2 dots,
# 3 products, 3 cross terms, 3 x (2 FMA + 1 mul), 3 divisions), the primitive's distance (about 12)
# and the smooth-union blend (about 12).
FLOP_PER_NODE = 12
# DRAM bytes per active block of the block-field stage (k_field_own + k_field_miss), from a one-pass ncu
# capture of the 1024^3 workload: 85.60 + 85.64 MB and 23.63 + 15.04 MB for its 44,270 active blocks
TRAFFIC_PER_ACTIVE_BLOCK = (85.60e6 + 85.64e6 + 23.63e6 + 15.04e6) / 44270
# the same capture's DRAM bytes per active block of the gather (classification and counts) and the emission
DRAM_PER_ACTIVE_BLOCK = {"gather": (133.37e6 + 134.72e6) / 44270, "emission": (133.75e6 + 86.49e6) / 44270}
FLOP_PER_LEAF = 44 + 12 + 12 + 1


def roofline(r):
    c = r.get("counters")
    peak = r.get("fp32_peak")
    ms_field = r["stages"]["ms_field"]
    if not c or not peak or not ms_field:
        return None
    # the walks' time: the block-field stage without its gather (timed by its own events), which
    # classifies and counts
    ms_walks = ms_field - (r["stages"].get("ms_classify") or 0.0)
    flops = c["field_node_visits"] * FLOP_PER_NODE + c["field_leaf_evals"] * FLOP_PER_LEAF
    achieved = flops / (ms_walks * 1e-3) / 1e12
    active = r["stats"]["active_blocks"]
    return {"kernel": "block field stage (k_field_plan + k_field_own + k_field_miss: warp-coherent BVH map())",
            "bound": "fp32", "ms": ms_walks,
            "achieved": achieved,
            "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "measured by the library's FMA loop on this GPU (no FP32 figure in MEASURED_PEAKS.json)",
            "traffic": TRAFFIC_PER_ACTIVE_BLOCK * active,
            "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of k_field_own + k_field_miss in one "
                              "ncu capture of the 1024^3, 16,384-primitive workload, 4.74 KB per active block, "
                              "scaled by this run's active blocks",
            "work": c}


# HBM copy bandwidth used as the denominator of the memory-bound stages
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth of MEASURED_PEAKS.json when present, else the
    fallback figure measured earlier on the same kind of GPU."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        v = float(d.get("hbm_gbs") or d["hbm"]["gbs"])
        return v, "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback (6.65 TB/s; MEASURED_PEAKS.json absent)"


def stage_roofline(r):
    """Achieved HBM fraction of the memory-bound stages by their algorithmic bytes, A active blocks and
    V vertices (one index per vertex): classification and counting (the gather kernel, timed by its own
    events inside the block-field stage) read the 4-byte samples of the 512 A cells and write 4 B per
    block; scan 8 B x A; emission reads the 4-byte cell word of each of the 512 A cells and writes 16 B
    (float4 position) + 4 B (index) per vertex. Beside each, the DRAM bytes ncu measured."""
    st, stages = r["stats"], r["stages"]
    a, v = st["active_blocks"], st["total_vertices"]
    peak, source = hbm_peak()
    out = {"peak": peak, "unit": "GB/s", "peak_source": source,
           "dram_source": "dram__bytes_read.sum + dram__bytes_write.sum per active block from a one-pass ncu "
                          "capture of the 1024^3 workload, scaled by this run's active blocks"}
    for name, ms, nbytes, dram in (("classify_count", stages.get("ms_classify"), 4 * 512 * a + 4 * a,
                                    DRAM_PER_ACTIVE_BLOCK["gather"] * a),
                                   ("scan", stages.get("ms_scan"), 8 * a, None),
                                   ("emission", stages.get("ms_emit"), 4 * 512 * a + 20 * v,
                                    DRAM_PER_ACTIVE_BLOCK["emission"] * a)):
        if ms:
            gbs = nbytes / (ms * 1e-3) / 1e9
            out[name] = {"bytes": nbytes, "ms": ms, "achieved": gbs, "frac": gbs / peak}
            if dram:
                out[name]["dram_bytes"] = dram
                out[name]["dram_gbs"] = dram / (ms * 1e-3) / 1e9
    return out


if __name__ == "__main__":
    main()
