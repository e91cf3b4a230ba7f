"""Builds libsdfmesh_b200.so in-tree for sm_100a (python -m cudasdf_b200.build)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libsdfmesh_b200.so")
SOURCES = ["sdfmesh.cu", "engine.inl", "mc_kernels.cuh", "dc_kernels.cuh", "sdf_device.cuh", "scan.cuh", "uv.cuh",
           "qef_masspoint.cuh", "bvh_host.h", "mc_cases.inc", "surrogate.cuh", "surrogate.inl", "noalloc.inl", "batch.inl",
           "bvh_device.cuh", "weld.cuh", "obj_export.inl", "uvpack.cuh", "uvpack.inl"]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    # host code (BVH construction) must round like the reference's host build: no contraction
    "-Xcompiler", "-fPIC,-ffp-contract=off",
    "-shared",
]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(HERE, "..", "include", "sdfmesh_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", OUT + ".tmp",
                                                                          os.path.join(CSRC, "sdfmesh.cu")]
    r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libsdfmesh_b200.so")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
