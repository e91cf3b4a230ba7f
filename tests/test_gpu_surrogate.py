"""The learned surrogate on the GPU: the tensor-core forward and backward kernels against the CPU
restatement (oracle/surrogate_oracle.py), and what the trained network gains: surrogate-culled
extraction of the 1024^3, 16,384-primitive scene skips most of the exact scout and gives the plain
extraction's mesh byte for byte, with the exact audit finding no active block in a culled coarse block.
"""
import hashlib

import numpy as np
import pytest

from oracle import surrogate_oracle as O

pytestmark = pytest.mark.gpu

IO = np.array([0, 0, 0, 1, 1, 1, 0.25], np.float32)


def _engine():
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, make_config
    eng = Engine()
    eng.configure(make_config(2 / 128))
    eng.set_scene(S.config_scene(2))
    return eng


@pytest.mark.parametrize("n", [1, 127, 1000, 128 * 37 + 5])
def test_forward_matches_oracle(n):
    import torch
    eng = _engine()
    theta, freq = O.random_params(5)
    eng.surrogate_set_params(theta, freq, IO)
    pts = np.random.default_rng(n).uniform(-1, 1, (n, 3)).astype(np.float32)
    f = eng.surrogate_forward(torch.from_numpy(pts).cuda()).cpu().numpy()
    ref = O.forward(pts, theta, freq, IO)
    d = np.abs(f - ref)
    # BF16 operands agree exactly except where a hardware tanh / sincospi ulp flips a BF16 rounding:
    # observed max 3e-5 at |f| ~ 0.12
    assert d.max() <= 3e-4 and d.mean() <= 3e-6, (d.max(), d.mean())
    eng.close()


@pytest.mark.parametrize("n", [1000, 128 * 37 + 5, 65536])
def test_gradient_matches_oracle(n):
    import torch
    eng = _engine()
    theta, freq = O.random_params(7)
    eng.surrogate_set_params(theta, freq, IO)
    rng = np.random.default_rng(n + 1)
    pts = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    tgt = rng.uniform(-0.3, 0.3, n).astype(np.float32)
    g, loss = eng.surrogate_gradient(torch.from_numpy(pts).cuda(), torch.from_numpy(tgt).cuda())
    gr, lr = O.gradient(pts, tgt, theta, freq, IO)
    assert abs(loss - lr) <= 1e-4 * lr
    rel = np.linalg.norm(g - gr) / np.linalg.norm(gr)
    assert rel <= 1e-4, rel
    blocks = [slice(l * 4096, (l + 1) * 4096) for l in range(4)] + [slice(16384, 16640), slice(16640, 16704)]
    for b in blocks:  # each parameter block on its own (observed <= 2.3e-4 for the first layer's weights)
        rb = np.linalg.norm(g[b] - gr[b]) / np.linalg.norm(gr[b])
        assert rb <= 5e-3, (b, rb)
    assert abs(g[-1] - gr[-1]) <= 1e-4 * abs(gr[-1]) + 1e-7
    # the parameters are untouched by a gradient evaluation
    th, fr, io = eng.surrogate_get_params()
    assert (th == theta).all() and (fr.reshape(-1) == freq.reshape(-1)).all()
    eng.close()


def test_training_culls_and_keeps_the_mesh():
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    eng = Engine()
    eng.configure(make_config(S.cell_size_for(1024), out_mask=L.OUT_INDICES))
    eng.set_scene(S.config_scene(4))
    buf = MeshBuffers(8_000_000, L.OUT_INDICES)
    plain = eng.extract(buf, 0.0)
    V = plain["total_vertices"]
    h_plain = hashlib.sha256(buf.vertices[:V].cpu().numpy().tobytes()).hexdigest()
    st = eng.surrogate_train()
    assert 0 < st["eps_cert"] <= st["eps_max"] and st["margin"] > st["eps_cert"]
    assert st["final_loss"] < 1e-3  # the clamped targets have a variance of about 1e-2
    audit = eng.surrogate_audit(0.0)
    assert audit["violations"] == 0
    assert audit["culled_coarse"] > 0.5 * audit["coarse_blocks"], audit
    eng.surrogate_enable(True)
    buf.vertices.zero_()
    culled = eng.extract(buf, 0.0)
    assert culled["total_vertices"] == V and culled["active_blocks"] == plain["active_blocks"]
    assert culled["scouted_blocks"] < 0.5 * plain["scouted_blocks"], (culled["scouted_blocks"], plain["scouted_blocks"])
    assert hashlib.sha256(buf.vertices[:V].cpu().numpy().tobytes()).hexdigest() == h_plain
    # an unchanged scene keeps the surrogate; a changed one drops it
    eng.set_scene(S.config_scene(4))
    assert eng.extract(buf, 0.0)["scouted_blocks"] == culled["scouted_blocks"]
    eng.set_scene(S.config_scene(2))
    assert eng.extract(buf, 0.0, allow_capacity=True)["scouted_blocks"] == plain["scouted_blocks"]
    with pytest.raises(RuntimeError):
        eng.surrogate_enable(True)
    eng.close()


def test_network_against_the_method_without_it():
    """What the trained network gains over culling without it. The method without the network evaluates
    the exact map() at every 32^3 coarse centre and culls beyond a margin (SDF_CULL_EXACT); the
    surrogate evaluates f_net on tensor cores and culls beyond its certified margin eps_cert + reach.
    With the reach alone (no extra margin) the exact field culls coarse blocks that hold active blocks:
    the capped, pruned field of blended primitives is not 1-Lipschitz, and a coarse centre whose search
    hits the 256-step cap reads too large a distance. Given the surrogate's certified eps as its extra
    margin it keeps the plain mesh; the test reports the coarse blocks each mode culls and the blocks
    each leaves to the exact scout (the time of each is in the bench line)."""
    from cudasdf_b200 import _lib as L
    from cudasdf_b200 import scenes as S
    from cudasdf_b200.engine import Engine, MeshBuffers, make_config
    eng = Engine()
    eng.configure(make_config(S.cell_size_for(1024), out_mask=L.OUT_INDICES))
    eng.set_scene(S.config_scene(4))
    buf = MeshBuffers(8_000_000, L.OUT_INDICES)
    plain = eng.extract(buf, 0.0)
    V = plain["total_vertices"]
    h_plain = hashlib.sha256(buf.vertices[:V].cpu().numpy().tobytes()).hexdigest()
    res = {}
    eng.set_coarse_cull(L.SDF_CULL_EXACT, 0.0)  # no training needed
    res["exact_reach_only"] = eng.surrogate_audit(0.0)
    st = eng.surrogate_train()
    res["eps_cert"] = st["eps_cert"]
    for name, mode, extra in (("surrogate", L.SDF_CULL_SURROGATE, 0.0),
                              ("exact_same_margin", L.SDF_CULL_EXACT, st["eps_cert"])):
        eng.set_coarse_cull(mode, extra)
        res[name] = eng.surrogate_audit(0.0)
        buf.vertices.zero_()
        out = eng.extract(buf, 0.0)
        res[name]["scouted_blocks"] = out["scouted_blocks"]
        assert res[name]["violations"] == 0, (name, res)
        assert out["total_vertices"] == V
        assert hashlib.sha256(buf.vertices[:V].cpu().numpy().tobytes()).hexdigest() == h_plain
    eng.set_coarse_cull(L.SDF_CULL_NONE)
    assert eng.extract(buf, 0.0)["scouted_blocks"] == plain["scouted_blocks"]
    print("coarse culling at 1024^3:", res, "plain scouted", plain["scouted_blocks"])
    eng.close()
