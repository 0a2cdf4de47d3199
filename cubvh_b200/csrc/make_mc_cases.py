"""Writes mc_cases.h (beside this file): the marching-cubes case table of the
sparse marching cubes kernels, from tests/golden/ref_mc_cases.npz, the
triangle lists the reference's own sparse marching cubes emits for the 256
corner configurations of one voxel (recorded by
tests/golden/make_ref_mc_cases.py).  The table is the one the reference's
triangle array is built from, so the library's triangles equal the
reference's index for index.

    python cubvh_b200/csrc/make_mc_cases.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "..", "..", "tests", "golden", "ref_mc_cases.npz")
OUT = os.path.join(HERE, "mc_cases.h")


def main():
    t = np.load(SRC)["tri_edges"].astype(int)
    assert t.shape == (256, 16)
    lines = ["// Generated by make_mc_cases.py from tests/golden/ref_mc_cases.npz: for each",
             "// corner configuration (bit k: corner k below iso), the triangles as edge",
             "// triples (e0, e1, e2), -1 after the last.  The reference's sparse marching",
             "// cubes emits each as vertices (e0, e2, e1).  Do not edit.",
             "#pragma once",
             "#include <cstdint>",
             "",
             "namespace cubvh {",
             "__constant__ int8_t c_mc_tri[256][16] = {"]
    for c in range(256):
        lines.append("    {" + ", ".join(str(v) for v in t[c]) + "},")
    lines += ["};", "}  // namespace cubvh", ""]
    with open(OUT, "w") as fh:
        fh.write("\n".join(lines))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
