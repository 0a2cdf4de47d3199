"""Regenerates tests/golden/golden.npz: small seeded inputs with the FP64 CPU
oracle's results (oracle/), used as frozen regression fixtures.

    python tests/golden/make_golden.py

Cases: the 20-vertex / 36-face dodecahedron with 1000 N(0,1) points
(unsigned distance + uvw, both signs), 512 camera rays against a displaced
icosphere, a 24^3 random occupancy grid (floodfill), and the first 64 stab
offsets of the raystab sign rule.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cubvh_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    out = {}
    v, f = W.dodecahedron()
    pts = np.random.default_rng(2024).standard_normal((1000, 3)).astype(np.float32)
    d, fid, uvw, cp, nn = O.udf64(v, f, pts)
    sw, _, flw = O.sdf_watertight64(v, f, pts)
    sr, _, flr = O.sdf_raystab64(v, f, pts)
    out.update(dodeca_v=v, dodeca_f=f, dodeca_pts=pts, dodeca_dist=d, dodeca_fid=fid, dodeca_uvw=uvw,
               dodeca_nnear=nn, dodeca_sdf_w=sw, dodeca_sdf_r=sr)
    v2, f2 = W.displaced_icosphere(3, 7)
    ro, rd = W.camera_rays(2, 16, 50.0, 2.5, 7)
    t, rfid, rfl = O.ray64(v2, f2, ro, rd)
    out.update(ico_v=v2, ico_f=f2, rays_o=ro, rays_d=rd, ray_t=t, ray_fid=rfid)
    g = np.random.default_rng(5).random((24, 24, 24)) < 0.4
    out.update(ff_grid=g, ff_labels=O.floodfill(g))
    out.update(stab_offsets=O.stab_offsets(64))
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"))


if __name__ == "__main__":
    main()
