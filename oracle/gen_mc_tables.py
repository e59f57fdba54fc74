"""Generate the marching-cubes lookup tables used by the oracle and the CUDA path.

The reference triangulates each active cube with the classic Lorensen-Cline
tables in the form Paul Bourke published them ("Polygonising a scalar field",
1994): ``edgeTable[256]`` and ``triTable[256][16]`` (marchingCubes.cpp:49-362).
Parity needs the very same triangulation -- the triangle order feeds the FP64
volume sum -- so the table *data* must be identical.  This script reads the two
tables from the reference source, checks that the edge table is exactly the one
implied by the reference's corner and edge numbering (marchingCubes.cpp:372-479)
and by the triangle table, and writes them as C headers:

    oracle/gg_mc_tables.h                    (oracle restatement)
    gragles_3d_b200/csrc/gg_mc_tables.inc    (CUDA path)

Run:  python oracle/gen_mc_tables.py [path/to/reference/src/marchingCubes.cpp]
(default: the reference beside this repository, or $GG_REFERENCE_SRC/marchingCubes.cpp)
"""
from __future__ import annotations

import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

# Cube corners as (dx, dy, dz) in cubeindex bit order (marchingCubes.cpp:376-385).
CORNERS = [(0, 0, 1), (1, 0, 1), (1, 0, 0), (0, 0, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0), (0, 1, 0)]
# Edge e joins corners EDGES[e] (the VertexInterp calls at marchingCubes.cpp:392-469).
EDGES = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]


def parse(path: str):
    src = open(path).read()
    m = re.search(r"int\s+edgeTable\s*\[256\]\s*=\s*\{(.*?)\};", src, re.S)
    edge = [int(t, 16) for t in re.findall(r"0x[0-9a-fA-F]+", m.group(1))]
    m = re.search(r"int\s+triTable\s*\[256\]\s*\[16\]\s*=\s*\{(.*?)\};", src, re.S)
    rows = re.findall(r"\{([^{}]*)\}", m.group(1))
    tri = [[int(t) for t in r.split(",") if t.strip()] for r in rows]
    assert len(edge) == 256 and len(tri) == 256 and all(len(r) == 16 for r in tri)
    return edge, tri


def check(edge, tri):
    for c in range(256):
        inside = [(c >> b) & 1 for b in range(8)]
        want = 0
        for e, (a, b) in enumerate(EDGES):
            if inside[a] != inside[b]:
                want |= 1 << e
        assert edge[c] == want, (c, edge[c], want)
        used = 0
        for t in tri[c]:
            if t < 0:
                break
            used |= 1 << t
        assert used == want, (c, used, want)
        n = next(i for i, t in enumerate(tri[c] + [-1]) if t < 0)
        assert n % 3 == 0 and all(t == -1 for t in tri[c][n:])


def emit(edge, tri, qualifier: str) -> str:
    out = ["/* Generated by oracle/gen_mc_tables.py -- the Lorensen-Cline / Bourke marching-cubes",
           " * tables in the reference's corner and edge numbering.  Do not edit. */",
           f"{qualifier} int gg_mc_edge_table[256] = {{"]
    for i in range(0, 256, 8):
        out.append("    " + ", ".join(f"0x{v:03x}" for v in edge[i:i + 8]) + ",")
    out.append("};")
    out.append(f"{qualifier} signed char gg_mc_tri_table[256][16] = {{")
    for r in tri:
        out.append("    {" + ", ".join(str(v) for v in r) + "},")
    out.append("};")
    return "\n".join(out) + "\n"


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    src = os.environ.get("GG_REFERENCE_SRC", os.path.join(here, "..", "..", "reference", "src"))
    path = sys.argv[1] if len(sys.argv) > 1 else os.path.join(src, "marchingCubes.cpp")
    edge, tri = parse(path)
    check(edge, tri)
    with open(os.path.join(HERE, "gg_mc_tables.h"), "w") as f:
        f.write(emit(edge, tri, "static const"))
    with open(os.path.join(ROOT, "gragles_3d_b200", "csrc", "gg_mc_tables.inc"), "w") as f:
        f.write(emit(edge, tri, "__constant__ const"))
    print("ok")


if __name__ == "__main__":
    main()
