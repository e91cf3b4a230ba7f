"""The library's host scene build (sdf_build_bvh_host: unions first, the BVH over the unions; boxes on
several threads, the two subtrees of large nodes built at once) against the oracle's sequential
restatement of CudaSDFMesh::UpdateBVH (CudaSDFMesh.cpp:216-249, CudaSDFUtil.h:507-603): sorted
primitives and nodes byte for byte. No GPU is needed."""
import ctypes
import os

import numpy as np
import pytest

from cudasdf_b200 import _lib
from cudasdf_b200 import scenes as S
from oracle import oracle as O


def _build(prims):
    L = _lib.lib()
    f = L.sdf_build_bvh_host
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_int)]
    prims = np.ascontiguousarray(prims)
    n = len(prims)
    sorted_out = np.zeros(n, prims.dtype)
    cap = max(2 * n - 1, 1)
    nodes = np.zeros(cap, O.NODE_DTYPE)
    nb = ctypes.c_int(-7)
    nn = f(prims.ctypes.data, n, sorted_out.ctypes.data, nodes.ctypes.data, cap, ctypes.byref(nb))
    return nn, nb.value, sorted_out, nodes[:max(nn, 0)]


def _scenes():
    rng = np.random.default_rng(5)
    out = {f"config{c}": S.config_scene(c) for c in (1, 2, 3, 4)}
    for n in (1, 2, 7, 100, 4095, 4096, 6000, 20000):
        out[f"random{n}"] = S.random_scene(n, seed=n)
    same = S.random_scene(5000, seed=3)
    same["position"] = (0.25, 0.25, 0.25)  # every centroid equal: the split falls back to the middle
    out["same_centroids"] = same
    flat = S.random_scene(5000, seed=4)
    flat["position"][:, 2] = 0.0
    out["flat"] = flat
    mixed = S.random_scene(6000, seed=6)
    mixed["operation"] = rng.integers(0, 6, len(mixed))  # subtractions and intersections stay out of the BVH
    out["mixed_operations"] = mixed
    zeros = S.random_scene(5000, seed=8)
    zeros["position"][::3] = (-0.0, 0.0, -0.0)
    out["signed_zeros"] = zeros
    return out


@pytest.mark.parametrize("name", sorted(_scenes()))
def test_host_build_matches_the_oracle(name):
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libsdfmesh_b200.so not built")
    prims = _scenes()[name]
    nn, nb, sorted_out, nodes = _build(prims)
    ref = O.Scene(prims)
    assert nb == ref.nbvh
    assert nn == len(ref.nodes)
    assert sorted_out.tobytes() == ref.sorted.tobytes()
    assert nodes.tobytes() == ref.nodes.tobytes()


def test_host_build_arguments():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libsdfmesh_b200.so not built")
    L = _lib.lib()
    f = L.sdf_build_bvh_host
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_int)]
    prims = S.random_scene(10, seed=1)
    out = np.zeros(10, prims.dtype)
    nodes = np.zeros(19, O.NODE_DTYPE)
    assert f(prims.ctypes.data, 10, out.ctypes.data, nodes.ctypes.data, 18, None) == -1  # capacity too small
    assert f(prims.ctypes.data, -1, out.ctypes.data, nodes.ctypes.data, 19, None) == -1
    assert f(None, 10, out.ctypes.data, nodes.ctypes.data, 19, None) == -1
    assert f(None, 0, None, None, 0, None) == 0  # an empty scene has no nodes
    assert f(prims.ctypes.data, 10, out.ctypes.data, nodes.ctypes.data, 19, None) == 19
