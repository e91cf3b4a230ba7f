"""Seeded synthetic scenes in the reference's primitive layout.

The reference ships no dataset: its only scene is the interactive showcase
(main.cpp:1130-1207). The benchmark workloads are seeded synthetic scenes with
the shapes, sizes and value ranges of the five benchmark configurations:

* ``sphere_scene``     - one sphere of radius 0.6 at the origin (128^3 case).
* ``random_scene(n)``  - n primitives, types uniform over sphere/box/capsule/torus,
  centres U[-0.8, 0.8]^3, size s log-uniform in [0.02, 0.2] encoded through
  ``scale = (s, s, s)`` with canonical parameters (the reference's BVH box is
  only tight for sphere/box/torus and is a fixed +-1.1 local box for every other
  type, CudaSDFUtil.h:507-542, so size must live in ``scale``), uniform random
  rotations (Shoemake), smooth union with k = 0.05.
* ``showcase_scene(t)`` - the reference's five-primitive showcase with its
  animation at time t (main.cpp:1136-1207, 1308-1315).
* ``batch_scenes``     - the many-scene batch workload.

Primitive records are numpy structured arrays whose dtype is byte-identical to
the reference's ``SDFPrimitive`` (Commons.cuh:68-102, 160 bytes).
"""
from __future__ import annotations

import math

import numpy as np

# PrimitiveType (Commons.cuh:17-34)
SDF_SPHERE, SDF_BOX, SDF_TORUS, SDF_CYLINDER, SDF_CAPSULE, SDF_CONE = 0, 1, 2, 3, 4, 5
SDF_ROUNDED_BOX, SDF_ROUNDED_CYLINDER, SDF_ROUNDED_CONE, SDF_ELLIPSOID = 6, 7, 8, 9
SDF_TRIANGULAR_PRISM, SDF_OCTOHEDRON, SDF_HEX_PRISM, SDF_SOLID_ANGLE = 10, 11, 12, 13
SDF_CUSTOM_FLOAT, SDF_CUSTOM_VECTOR = 14, 15
# OperationType (Commons.cuh:37-44)
SDF_UNION, SDF_SUBTRACT, SDF_INTERSECT = 0, 1, 2
SDF_UNION_BLEND, SDF_SUBTRACT_BLEND, SDF_INTERSECT_BLEND = 3, 4, 5
# DisplacementType (Commons.cuh:47-57)
DISP_NONE, DISP_SINE, DISP_TWIST, DISP_BEND = 0, 1, 2, 3

PRIM_DTYPE = np.dtype({
    "names": ["rotation", "dispParams", "position", "blendFactor", "scale", "rounding",
              "color", "annular", "params", "type", "operation", "displacement", "_pad1",
              "uvScale", "uvOffset", "uvRotation", "uvMode", "textureID", "atlasIslandID", "_pad2"],
    "formats": [("<f4", 4), ("<f4", 4), ("<f4", 3), "<f4", ("<f4", 3), "<f4",
                ("<f4", 3), "<f4", ("<f4", 6), "<i4", "<i4", "<i4", "<i4",
                ("<f4", 2), ("<f4", 2), "<f4", "<i4", "<i4", "<i4", ("<f4", 2)],
    "offsets": [0, 16, 32, 44, 48, 60, 64, 76, 80, 104, 108, 112, 116,
                120, 128, 136, 140, 144, 148, 152],
    "itemsize": 160,
})
assert PRIM_DTYPE.itemsize == 160

SEED_BASE = 0x5DF0000


def make_primitives(n: int) -> np.ndarray:
    """n default-initialised primitives (the defaults of CreatePrimitive, CudaSDFUtil.h:8-38)."""
    p = np.zeros(n, dtype=PRIM_DTYPE)
    p["rotation"] = (0.0, 0.0, 0.0, 1.0)
    p["scale"] = (1.0, 1.0, 1.0)
    p["uvScale"] = (1.0, 1.0)
    p["atlasIslandID"] = -1
    return p


def primitive(ptype, position, rotation=(0.0, 0.0, 0.0, 1.0), color=(1.0, 1.0, 1.0),
              operation=SDF_UNION, blend=0.0, params=(), scale=(1.0, 1.0, 1.0)) -> np.ndarray:
    p = make_primitives(1)
    p["type"] = ptype
    p["position"] = position
    p["rotation"] = rotation
    p["color"] = color
    p["operation"] = operation
    p["blendFactor"] = blend
    p["scale"] = scale
    prm = np.zeros(6, np.float32)
    prm[:len(params)] = params
    p["params"] = prm
    return p


def random_unit_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotations (Shoemake's subgroup algorithm), as (x, y, z, w) float32."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    q = np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2),
                  b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)], axis=1)
    return q.astype(np.float32)


def sphere_scene(radius: float = 0.6) -> np.ndarray:
    return primitive(SDF_SPHERE, (0.0, 0.0, 0.0), color=(0.8, 0.8, 0.8), params=(radius,))


_CANONICAL_PARAMS = {
    SDF_SPHERE: (1.0,),
    SDF_BOX: (1.0, 1.0, 1.0),
    SDF_CAPSULE: (0.8, 0.2),      # local y in [-0.2, 1.0]: inside the fixed +-1.1 BVH box
    SDF_TORUS: (0.75, 0.25),
}
_RANDOM_TYPES = np.array([SDF_SPHERE, SDF_BOX, SDF_CAPSULE, SDF_TORUS], np.int32)


def random_scene(n: int, seed: int, blend: float = 0.05, size_range=(0.02, 0.2),
                 center_range=0.8) -> np.ndarray:
    """n seeded primitives following the composite-scene law of the benchmark configurations."""
    rng = np.random.Generator(np.random.PCG64(seed))
    types = _RANDOM_TYPES[rng.integers(0, 4, n)]
    centres = rng.uniform(-center_range, center_range, (n, 3)).astype(np.float32)
    lo, hi = math.log(size_range[0]), math.log(size_range[1])
    sizes = np.exp(rng.uniform(lo, hi, n)).astype(np.float32)
    quats = random_unit_quaternions(rng, n)
    colors = rng.uniform(0.1, 1.0, (n, 3)).astype(np.float32)
    p = make_primitives(n)
    p["type"] = types
    p["position"] = centres
    p["rotation"] = quats
    p["scale"] = np.repeat(sizes[:, None], 3, axis=1)
    p["color"] = colors
    p["operation"] = SDF_UNION_BLEND
    p["blendFactor"] = blend
    for t, prm in _CANONICAL_PARAMS.items():
        sel = types == t
        row = np.zeros(6, np.float32)
        row[:len(prm)] = prm
        p["params"][sel] = row
    return p


def config_seed(config: int) -> int:
    return SEED_BASE + config


def showcase_scene(time: float = 0.0, animate: bool = True) -> np.ndarray:
    """The reference's showcase (main.cpp:1136-1207) with its animation (main.cpp:1308-1315)."""
    q0 = (0.0, 0.0, 0.0, 1.0)
    torus = primitive(SDF_TORUS, (-0.5, 0.5, 0.0), q0, (0.2, 0.8, 0.2), SDF_UNION, 0.0, (0.4, 0.15))
    torus["uvScale"] = (4.0, 2.0)
    torus["textureID"] = 0
    hexp = primitive(SDF_HEX_PRISM, (0.5, 0.5, 0.0), q0, (1.0, 0.2, 0.2), SDF_UNION, 0.0, (0.3, 0.4))
    hexp["displacement"] = DISP_TWIST
    hexp["dispParams"] = (2.0, 0.0, 0.0, 0.0)
    hexp["uvScale"] = (2.0, 1.0)
    hexp["textureID"] = 1
    cone = primitive(SDF_ROUNDED_CONE, (-0.5, -0.5, 0.0), q0, (0.2, 0.2, 1.0), SDF_UNION, 0.0, (0.5, 0.3, 0.1))
    cone["textureID"] = 2
    cyl = primitive(SDF_ROUNDED_CYLINDER, (0.5, -0.5, 0.0), q0, (1.0, 1.0, 0.2), SDF_UNION, 0.0, (0.4, 0.2, 0.1))
    cyl["uvScale"] = (3.0, 1.5)
    cyl["textureID"] = 3
    sph = primitive(SDF_SPHERE, (0.0, 0.0, 0.0), q0, (0.5, 0.0, 0.5), SDF_SUBTRACT, 0.0, (0.6,))
    sph["uvScale"] = (2.0, 2.0)
    sph["textureID"] = 4
    prims = np.concatenate([torus, hexp, cone, cyl, sph])
    if animate:
        t = np.float32(time)
        prims[0]["dispParams"][1] = np.float32(5.0) * np.float32(math.sin(np.float32(t * np.float32(0.1))))
        c, s = np.float32(math.cos(t)), np.float32(math.sin(t))
        prims[1]["rotation"] = (0.0, s, 0.0, c)
        prims[2]["position"][1] = np.float32(-0.5) + np.float32(0.2) * np.float32(math.sin(np.float32(t * np.float32(2.0))))
        prims[3]["params"][2] = np.float32(0.1) + np.float32(0.05) * np.float32(math.sin(np.float32(t * np.float32(3.0))))
    return prims


# ---------------------------------------------------------------------------------------------
# Benchmark configurations (grid = samples per axis over [-1, 1]^3)
# ---------------------------------------------------------------------------------------------

BOUNDS_MIN = (-1.0, -1.0, -1.0)
BOUNDS_MAX = (1.0, 1.0, 1.0)


def config_scene(config: int) -> np.ndarray:
    """Primitives of benchmark configuration 1..4 (1-based, as in the benchmark list)."""
    if config == 1:
        return sphere_scene()
    n = {2: 256, 3: 4096, 4: 16384}[config]
    return random_scene(n, config_seed(config))


def config_resolution(config: int) -> int:
    return {1: 128, 2: 256, 3: 512, 4: 1024}[config]


def cell_size_for(resolution: int) -> float:
    return float(np.float32(2.0) / np.float32(resolution))


def batch_scenes(count: int = 256, seed: int = SEED_BASE + 5):
    """The batched workload: primitive counts log-uniform in [16, 2048], grids drawn from
    {64, 96, 128, 192, 256}^3, technique 50 % marching cubes / 50 % dual contouring."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(16), math.log(2048)))))
        res = int(rng.choice([64, 96, 128, 192, 256]))
        tech = int(rng.integers(0, 2))
        out.append({"primitives": random_scene(n, seed * 1000 + i), "resolution": res, "technique": tech})
    return out
