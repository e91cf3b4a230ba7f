"""bench.py's multi-process path on CPU: two gloo ranks (one process per rank, as torchrun starts
them) meet at the barrier, agree on the slowest rank's time and report the whole-job throughput of
two independent replicas. The extraction itself does not shard (replicas only), so no data moves
between ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    bench.barrier(world)
    ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
    ms_max = bench.max_over_ranks(ms, world)
    value = bench.job_throughput(world, 1024.0 ** 3, ms_max)
    out[rank] = (ms_max, value)
    bench.barrier(world)
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert out[0] == out[1]
    ms_max, value = out[0]
    assert ms_max == 15.0
    assert abs(value - 2 * 1024.0 ** 3 / 15e-3 / 1e9) < 1e-9


def test_stage_roofline_arithmetic():
    """The memory-bound stages' fractions in the bench line: algorithmic bytes / stage time / peak."""
    import bench
    r = {"stats": {"active_blocks": 1000, "total_vertices": 30000},
         "stages": {"ms_scan": 0.01, "ms_emit": 0.1, "ms_field": 1.0, "ms_scout": 0.1}}
    out = bench.stage_roofline(r)
    peak = out["peak"]
    assert out["scan"]["bytes"] == 8000
    assert abs(out["scan"]["achieved"] - 8000 / 1e-5 / 1e9) < 1e-9
    assert out["emission"]["bytes"] == 4 * 512 * 1000 + 20 * 30000
    assert abs(out["emission"]["frac"] - out["emission"]["achieved"] / peak) < 1e-12
    untimed = bench.stage_roofline({"stats": r["stats"], "stages": {}})  # timing off: no stage entries
    assert "scan" not in untimed and "emission" not in untimed and untimed["peak"] == peak


def test_field_roofline_arithmetic():
    """The dominant kernel's FP32 fraction: counted FLOPs over the field stage's time without its gather."""
    import bench
    c = {"field_node_visits": 1_000_000, "field_leaf_evals": 100_000}
    r = {"counters": c, "fp32_peak": 70.0, "stats": {"active_blocks": 1000},
         "stages": {"ms_field": 1.2, "ms_classify": 0.2}}
    out = bench.roofline(r)
    flops = 1_000_000 * bench.FLOP_PER_NODE + 100_000 * bench.FLOP_PER_LEAF
    assert abs(out["ms"] - 1.0) < 1e-12
    assert abs(out["achieved"] - flops / 1e-3 / 1e12) < 1e-9
    assert abs(out["frac"] - out["achieved"] / 70.0) < 1e-12
    assert abs(out["traffic"] - bench.TRAFFIC_PER_ACTIVE_BLOCK * 1000) < 1e-6
    # without the gather's own timing the whole stage counts
    r["stages"] = {"ms_field": 1.2}
    assert abs(bench.roofline(r)["ms"] - 1.2) < 1e-12
    assert bench.roofline({"counters": None, "fp32_peak": 70.0, "stats": {}, "stages": {"ms_field": 1.0}}) is None
