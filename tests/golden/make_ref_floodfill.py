"""Regenerates tests/golden/ref_floodfill.npz: occupancy grids with the labels
that the REFERENCE'S OWN CUDA floodfill (include/gpu/floodfill.cuh, compiled
into oracle/_ref by `make -C oracle ref`) returns for them.  Needs a GPU and
the built oracle/_ref/libref_floodfill.so:

    python tests/golden/make_ref_floodfill.py [--out PATH]

The CPU tests pin the floodfill oracle (oracle.cpp `orc_floodfill`) to these
labels, so the fixtures hold the reference's outputs, not the oracle's.

Cases: random blocked fractions 0.25 / 0.45 / 0.60 / 0.72 with H, W, D equal
and unequal (the reference decodes a voxel's coordinates as x = l % W,
y = (l / W) % H, z = l / (W H)), a batch of 3 volumes, the reference's
small-grid schedule (3^3 volumes), a closed sphere shell, all-free and
all-blocked volumes, 1-voxel-thick lines along both ends of the layout, the
occupancy (udf < 2/64) of the 12-tori mesh on a 64^3 grid, and a serpentine
corridor (one component 528 voxels long, against the reference's limit of
106 hook passes at 32^3: its pointer jumping still converges).
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cubvh_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def snake(n: int) -> np.ndarray:
    """[1, n, n, n]: everything blocked except slice 0, where even rows are
    free corridors and odd rows are walls with one gap, alternating ends."""
    g = np.ones((1, n, n, n), bool)
    s = g[0, 0]
    for w in range(n):
        if w % 2 == 0:
            s[w, :] = False
        else:
            s[w, n - 1 if (w // 2) % 2 == 0 else 0] = False
    return g


def cases():
    rng = lambda s: np.random.default_rng(s)  # noqa: E731
    out = {}
    out["rand25"] = rng(11).random((1, 20, 24, 28)) < 0.25
    out["rand45"] = rng(12).random((1, 24, 24, 24)) < 0.45
    out["rand60"] = rng(13).random((1, 20, 24, 28)) < 0.60
    out["rand72"] = rng(14).random((1, 24, 24, 24)) < 0.72
    out["batch3"] = rng(15).random((3, 16, 12, 20)) < 0.5
    out["tiny"] = rng(16).random((2, 3, 3, 3)) < 0.4
    c = (np.arange(32) + 0.5) / 16.0 - 1.0
    r = np.sqrt(c[:, None, None] ** 2 + c[None, :, None] ** 2 + c[None, None, :] ** 2)
    out["shell"] = (np.abs(r - 0.6) < 0.08)[None]
    out["free"] = np.zeros((1, 8, 9, 10), bool)
    out["blocked"] = np.ones((1, 5, 5, 5), bool)
    out["line_d"] = rng(17).random((1, 1, 1, 64)) < 0.2
    out["line_h"] = rng(18).random((1, 64, 1, 1)) < 0.2
    v, f = W.random_tori(2)
    pts = W.dense_grid(64)
    udf = O.RefBVH(v, f).unsigned_distance(pts)[0]
    out["tori64"] = (udf.reshape(64, 64, 64) < 2.0 / 64)[None]
    out["snake32"] = snake(32)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_floodfill.npz"))
    args = ap.parse_args()
    res = {}
    for name, g in cases().items():
        res[name + "_grid"] = np.packbits(g.reshape(-1))
        res[name + "_shape"] = np.array(g.shape, np.int64)
        res[name + "_ref"] = O.ref_floodfill(g)
    np.savez_compressed(args.out, **res)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
