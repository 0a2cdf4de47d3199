"""Regenerates tests/golden/ref_mc_cases.npz: the triangle list the
REFERENCE'S OWN CUDA sparse marching cubes (include/gpu/spcumc.cuh, compiled
into oracle/_ref by `make -C oracle ref REF=<checkout>`) emits for each of
the 256 corner configurations of one voxel.  Needs a GPU:

    python tests/golden/make_ref_mc_cases.py [--out PATH]

For case c (bit k set: corner k inside), the voxel at (0, 0, 0) gets corner
values -1 (inside, below iso 0) or +1, so every vertex sits at the midpoint
of its edge and names that edge.  The reference writes each table triangle
(e0, e1, e2) as vertices (e0, e2, e1) (src: spcumc.cuh generateTriangles),
so `tri_edges[c]` lists the edge triples (e0, e1, e2) in emission order,
padded with -1: the reference's marching-cubes case table, recovered from
its outputs.  `tris[c]` keeps the raw vertex triples and `verts[c]` the
vertices of each case.  cubvh_b200/csrc/make_mc_cases.py turns the table
into the library's constant table.
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

CORNER_OFF = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
EDGE_CORNERS = np.array([[0, 1], [1, 2], [2, 3], [3, 0], [4, 5], [5, 6], [6, 7], [7, 4], [0, 4], [1, 5], [2, 6],
                         [3, 7]])
EDGE_MID = (CORNER_OFF[EDGE_CORNERS[:, 0]] + CORNER_OFF[EDGE_CORNERS[:, 1]]) / 2.0


def edge_of(p):
    d = np.abs(EDGE_MID - p[None]).sum(1)
    e = int(np.argmin(d))
    assert d[e] == 0.0, p
    return e


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_mc_cases.npz"))
    a = ap.parse_args()
    table = -np.ones((256, 16), np.int8)
    out = {}
    for c in range(256):
        corners = np.array([[-1.0 if (c >> k) & 1 else 1.0 for k in range(8)]], np.float32)
        verts, tris = O.ref_sparse_mc(np.zeros((1, 3), np.int32), corners, 0.0)
        edges = [edge_of(v) for v in verts]
        row = []
        for v0, v1, v2 in tris:
            row += [edges[v0], edges[v2], edges[v1]]   # undo the reference's (e0, e2, e1) order
        table[c, :len(row)] = row
        out[f"verts_{c}"] = verts
        out[f"tris_{c}"] = tris
    np.savez_compressed(a.out, tri_edges=table, **out)
    print("wrote", a.out, "triangles per case:", (table >= 0).sum(1).reshape(16, 16) // 3)


if __name__ == "__main__":
    main()
