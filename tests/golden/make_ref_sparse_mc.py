"""Regenerates tests/golden/ref_sparse_mc.npz: sparse voxel sets with the
vertex and triangle arrays that the REFERENCE'S OWN CUDA sparse marching cubes
(include/gpu/spcumc.cuh, compiled into oracle/_ref by `make -C oracle ref`)
returns for them.  Needs a GPU and oracle/_ref/libref_sparse_mc.so:

    python tests/golden/make_ref_sparse_mc.py [--out PATH]

Cases (`cases()`, also used by the tests): a sphere's signed distance on the
voxels of a band around it (shared corners agree: a closed surface), random
corner values on a random voxel subset (shared corners disagree: the same
edge gets different positions from different voxels), and a random lattice
field on a full 12^3 block (ambiguous faces).
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

OFF = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])


def sphere_band(n=24, c=(12.2, 11.7, 12.5), r=7.3):
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
    cp = g[:, None, :] + OFF[None]
    f = (np.linalg.norm(cp - np.array(c), axis=-1) - r).astype(np.float32)
    keep = (f.min(1) < 1.5) & (f.max(1) > -1.5)
    return g[keep].astype(np.int32), f[keep]


def random_subset(seed=3, n=16, frac=0.4):
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
    g = g[rng.random(len(g)) < frac]
    rng.shuffle(g)
    return g.astype(np.int32), rng.uniform(-1, 1, (len(g), 8)).astype(np.float32)


def lattice_field(seed=5, n=12):
    rng = np.random.default_rng(seed)
    field = rng.uniform(-1, 1, (n + 1, n + 1, n + 1)).astype(np.float32)
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
    cp = g[:, None, :] + OFF[None]
    return g.astype(np.int32), field[cp[..., 0], cp[..., 1], cp[..., 2]]


def cases():
    return {"sphere": sphere_band() + (0.0,), "random": random_subset() + (0.1,), "lattice": lattice_field() + (0.0,)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_sparse_mc.npz"))
    args = ap.parse_args()
    res = {}
    for name, (coords, corners, iso) in cases().items():
        v, t = O.ref_sparse_mc(coords, corners, iso)
        res[name + "_verts"] = v
        res[name + "_tris"] = t
    np.savez_compressed(args.out, **res)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
