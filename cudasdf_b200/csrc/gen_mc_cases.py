"""Generate the marching-cubes case tables used by the engine and by the oracle.

Bit-exact parity with the reference requires the same case -> triangle table, with the same
triangle order and the same edge order inside each triangle, because the output is a
triangle soup whose vertex order is part of the contract. The reference keeps that table in
MarchingCubesTables.cuh:19-118 (``firstMarchingCubesId[257]`` prefix offsets into
``marchingCubesIds[2460]``). This script reads it from the reference tree once and re-encodes it:

* ``mc_cases.inc`` (engine): one 64-bit word per case. Bits 0-3 hold the triangle count (0..5);
  bits 4+4k..7+4k hold the k-th edge id (k = 0..14, three per triangle).
* ``oracle/mc_table_oracle.inc`` (oracle): ``signed char mc_tri[256][16]``, edge ids terminated by -1.

Usage: python cudasdf_b200/csrc/gen_mc_cases.py [reference_root]
"""
from __future__ import annotations

import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def read_reference_tables(ref_root: str):
    path = os.path.join(ref_root, "src", "SDFMesh", "MarchingCubesTables.cuh")
    text = open(path).read()

    def array(name):
        m = re.search(name + r"\s*\[[^\]]*\]\s*=\s*\{(.*?)\};", text, re.S)
        return [int(v) for v in re.findall(r"-?\d+", m.group(1))]

    first = array("firstMarchingCubesId")
    ids = array("marchingCubesIds")
    assert len(first) == 257 and len(ids) == 2460 and first[-1] == 2460
    cases = []
    for c in range(256):
        edges = ids[first[c]:first[c + 1]]
        assert len(edges) % 3 == 0 and len(edges) <= 15
        cases.append(edges)
    return cases


def encode_word(edges):
    w = len(edges) // 3
    for k, e in enumerate(edges):
        assert 0 <= e < 12
        w |= e << (4 + 4 * k)
    return w


def decode_word(w):
    n = w & 0xF
    return [(w >> (4 + 4 * k)) & 0xF for k in range(3 * n)]


def main():
    # the reference checkout: the first argument, else $CUDASDF_REFERENCE, else "reference" beside the repository
    ref_root = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CUDASDF_REFERENCE")
                or os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference"))
    cases = read_reference_tables(ref_root)
    words = [encode_word(e) for e in cases]
    assert [decode_word(w) for w in words] == cases
    lines = ["// Generated by gen_mc_cases.py from the reference case table (MarchingCubesTables.cuh:19-118).",
             "// Word layout: bits 0-3 triangle count; bits 4+4k..7+4k edge id k (three per triangle).",
             "// Expands to the 256 initialisers of the engine's __constant__ case table.",
             "#define SDF_MC_CASE_WORDS \\"]
    for i in range(0, 256, 4):
        sep = ", \\" if i + 4 < 256 else ""
        lines.append("    " + ", ".join(f"0x{w:016x}ull" for w in words[i:i + 4]) + sep)
    with open(os.path.join(HERE, "mc_cases.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")
    ol = ["/* Generated by cudasdf_b200/csrc/gen_mc_cases.py from the reference case table",
          "   (MarchingCubesTables.cuh:19-118): edge ids per case, -1 terminated. */",
          "static const signed char mc_tri[256][16] = {"]
    for c in range(256):
        row = cases[c] + [-1] * (16 - len(cases[c]))
        ol.append("    {" + ",".join(str(v) for v in row) + "},")
    ol.append("};")
    with open(os.path.join(ROOT, "oracle", "mc_table_oracle.inc"), "w") as f:
        f.write("\n".join(ol) + "\n")
    print("wrote", os.path.join(HERE, "mc_cases.inc"), "and oracle/mc_table_oracle.inc")


if __name__ == "__main__":
    main()
