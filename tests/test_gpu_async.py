"""The asynchronous extraction API (sdf_engine_set_scene_async, sdf_engine_extract_async / _wait)
against the synchronous one: the same meshes, in flight several at a time on one stream, with scene
changes between them, and the ticket bookkeeping (a collected or evicted ticket is refused)."""
import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scenes():
    from cudasdf_b200 import scenes as S
    a = S.config_scene(2)
    b = a.copy()
    b["position"][:, 1] += np.float32(0.01)
    return a, b


def _digest(buf, n):
    return hashlib.sha256(buf.vertices[:n].cpu().numpy().tobytes()).hexdigest()


def test_async_matches_sync_with_scene_changes():
    import torch

    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    a, b = _scenes()
    order = [a, b, b, a, b, a]
    cfg = make_config(S.cell_size_for(128), out_mask=L.OUT_INDICES)
    ref = []
    e = Engine()
    e.configure(cfg)
    buf = MeshBuffers(2_000_000, L.OUT_INDICES)
    for p in order:
        e.set_scene(p)
        st = e.extract(buf, 0.5)
        ref.append((int(st["total_vertices"]), _digest(buf, int(st["total_vertices"]))))
    e.close()
    e = Engine()
    e.configure(cfg)
    stream = torch.cuda.Stream()
    bufs = [MeshBuffers(2_000_000, L.OUT_INDICES) for _ in range(len(order))]
    tickets = []
    for p, bb in zip(order, bufs):
        e.set_scene_async(p, stream)
        tickets.append(e.extract_async(bb, 0.5, stream))  # the fifth and sixth evict the oldest two
    got = []
    for k, (t, bb) in enumerate(zip(tickets, bufs)):
        if k < len(tickets) - 4:
            # the fifth and sixth extraction evicted the first two: their tickets are refused
            with pytest.raises(RuntimeError, match="SDF_ERR_INVALID"):
                e.extract_wait(t)
            continue
        st = e.extract_wait(t)
        got.append((int(st["total_vertices"]), _digest(bb, int(st["total_vertices"]))))
    stream.synchronize()
    # every buffer holds its own scene's mesh, the evicted ones included
    for k, bb in enumerate(bufs):
        assert _digest(bb, ref[k][0]) == ref[k][1], k
    assert got == ref[len(order) - len(got):]
    with pytest.raises(RuntimeError, match="SDF_ERR_INVALID"):
        e.extract_wait(tickets[-1])  # already collected
    e.close()


def test_async_streamed_loop_two_buffers():
    """The streamed pattern of the benchmark: step k + 1 enqueued before step k is collected."""
    import torch

    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    a, _ = _scenes()
    e = Engine()
    e.configure(make_config(S.cell_size_for(128), out_mask=L.OUT_INDICES))
    e.set_scene(a)
    one = MeshBuffers(2_000_000, L.OUT_INDICES)
    st = e.extract(one)
    V = int(st["total_vertices"])
    want = _digest(one, V)
    ext, cpy = torch.cuda.Stream(), torch.cuda.Stream()
    bufs = [MeshBuffers(V + 16, L.OUT_INDICES) for _ in range(2)]
    hosts = [torch.empty((V + 16, 4), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    pending, seen = [], []
    for i in range(6):
        bi = i % 2
        ext.wait_event(copied[bi])
        e.set_scene_async(a, ext)
        t = e.extract_async(bufs[bi], 0.0, ext)
        if pending:
            tk, bp = pending.pop(0)
            n = int(e.extract_wait(tk)["total_vertices"])
            with torch.cuda.stream(cpy):
                hosts[bp][:n].copy_(bufs[bp].vertices[:n], non_blocking=True)
                copied[bp].record(cpy)
            cpy.synchronize()
            seen.append(hashlib.sha256(hosts[bp][:n].numpy().tobytes()).hexdigest())
        pending.append((t, bi))
    tk, bp = pending.pop(0)
    n = int(e.extract_wait(tk)["total_vertices"])
    hosts[bp][:n].copy_(bufs[bp].vertices[:n])
    seen.append(hashlib.sha256(hosts[bp][:n].numpy().tobytes()).hexdigest())
    assert seen == [want] * 6
    e.close()
