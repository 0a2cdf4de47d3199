"""Regenerates tests/golden/ref_bvh.npz: meshes and queries with the outputs
of the REFERENCE'S OWN BVH code (src/bvh.cu compiled unchanged into
oracle/_ref/libref_bvh.so by `make -C oracle ref REF=<checkout>`): its CUDA
kernels and its host build of the same traversals.

Two steps, because the reference checkout and the GPU live on different
machines:

    # where the reference checkout is: its test's dodecahedron -> inputs
    python tests/golden/make_ref_bvh.py inputs --reference <checkout>
    # on a GPU machine (oracle/_ref built): inputs -> outputs
    python tests/golden/make_ref_bvh.py outputs [--out PATH]

Cases (mesh: queries):
  dodeca  the reference test's own dodecahedron (test/unsigned_distance.py:
          9-76, its create_dodecahedron run as written, with trimesh's mesh
          constructor replaced by returning the arrays): 1000 N(0,1) points
          as that test draws them (seeded here), 512 rays from N(0,2) origins
          towards N(0,0.3) targets
  ico3    icosphere level 3, radius 0.8: 4096 points U[-1,1]^3, 512 rays
  disp4   displaced icosphere level 4: 2048 points U[-1,1]^3 + 2048 within
          0.02 of the surface; 2 x 16^2 camera rays
  tori3   3 random tori 48 x 12 with 10% of the faces removed (open): 4096
          points in the box, 512 rays
For every case: unsigned distance + uvw, signed distance (watertight and
raystab; raystab seeds query i with index i of the call), ray_trace, from the
reference's CUDA kernels (`gpu_*`) and from its host traversals (`host_*`);
for dodeca and tori3 also the reference's device stab directions of the
queries (`gpu_stab_dirs`, the raystab oracle's input).
"""
import argparse
import ast
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cubvh_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

INPUTS = os.path.join(HERE, "ref_bvh_inputs.npz")
OUT = os.path.join(HERE, "ref_bvh.npz")


def reference_dodecahedron(checkout):
    """Runs the reference test's create_dodecahedron (parsed out of its file)
    with a stand-in trimesh whose Trimesh returns (vertices, faces)."""
    path = os.path.join(checkout, "test", "unsigned_distance.py")
    tree = ast.parse(open(path).read())
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "create_dodecahedron")

    class _Trimesh:
        @staticmethod
        def Trimesh(vertices, faces):
            return vertices, faces

    ns = {"np": np, "trimesh": _Trimesh}
    exec(compile(ast.Module(body=[fn], type_ignores=[]), path, "exec"), ns)
    v, f = ns["create_dodecahedron"]()
    return np.asarray(v, np.float32), np.asarray(f, np.int64)


def _rays(n, seed, spread=2.0, aim=0.3):
    rng = np.random.default_rng(seed)
    o = (rng.standard_normal((n, 3)) * spread).astype(np.float32)
    d = (rng.standard_normal((n, 3)) * aim - o).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return o, d.astype(np.float32)


def cases(inputs):
    out = {}
    v, f = inputs["dodeca_v"], inputs["dodeca_f"]
    pts = np.random.default_rng(2024).standard_normal((1000, 3)).astype(np.float32)
    out["dodeca"] = (v, f, pts, *_rays(512, 11))
    v, f = W.icosphere(3, 0.8)
    out["ico3"] = (v, f, W.uniform_points(4096, 12), *_rays(512, 12))
    v, f = W.displaced_icosphere(4, 1)
    rng = np.random.default_rng(13)
    pts = np.concatenate([rng.uniform(-1, 1, (2048, 3)).astype(np.float32), W.surface_points(v, f, 2048, 0.02, rng)])
    ro, rd = W.camera_rays(2, 16, 50.0, 2.5, 13)
    out["disp4"] = (v, f, pts, ro, rd)
    v, f = W.random_tori(2, n_tori=3, n_major=48, n_minor=12)
    lo, hi = v.min(0), v.max(0)
    pts = np.random.default_rng(14).uniform(lo - 0.1, hi + 0.1, (4096, 3)).astype(np.float32)
    out["tori3"] = (v, f, pts, *_rays(512, 14, spread=1.0, aim=0.2))
    return out


def run_outputs(path):
    import torch
    inputs = np.load(INPUTS)
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev).cuda_stream
    res = {}
    for name, (v, f, pts, ro, rd) in cases(inputs).items():
        R = O.ReferenceBVH(v, f)
        res.update({f"{name}_v": v, f"{name}_f": f, f"{name}_pts": pts, f"{name}_ro": ro, f"{name}_rd": rd})
        P = torch.from_numpy(pts).to(dev)
        n = len(pts)
        for tag, mode in (("udf", None), ("sdfw", 0), ("sdfr", 1)):
            d = torch.empty(n, device=dev)
            fid = torch.empty(n, dtype=torch.int64, device=dev)
            u = torch.empty(n, 3, device=dev)
            if mode is None:
                R.unsigned_distance_gpu(P.data_ptr(), n, d.data_ptr(), fid.data_ptr(), u.data_ptr(), stream)
                hd, hf, hu = R.unsigned_distance(pts, return_uvw=True)
            else:
                R.signed_distance_gpu(P.data_ptr(), n, mode, d.data_ptr(), fid.data_ptr(), u.data_ptr(), stream)
                hd, hf, hu = R.signed_distance(pts, mode, return_uvw=True)
            torch.cuda.synchronize()
            res.update({f"{name}_gpu_{tag}_d": d.cpu().numpy(), f"{name}_gpu_{tag}_fid": fid.cpu().numpy(),
                        f"{name}_gpu_{tag}_uvw": u.cpu().numpy(), f"{name}_host_{tag}_d": hd,
                        f"{name}_host_{tag}_fid": hf, f"{name}_host_{tag}_uvw": hu})
        m = len(ro)
        Ro, Rd = torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev)
        pos = torch.empty(m, 3, device=dev)
        fid = torch.empty(m, dtype=torch.int64, device=dev)
        dep = torch.empty(m, device=dev)
        R.ray_trace_gpu(Ro.data_ptr(), Rd.data_ptr(), m, pos.data_ptr(), fid.data_ptr(), dep.data_ptr(), stream)
        torch.cuda.synchronize()
        hp, hf, hdep = R.ray_trace(ro, rd)
        res.update({f"{name}_gpu_ray_pos": pos.cpu().numpy(), f"{name}_gpu_ray_fid": fid.cpu().numpy(),
                    f"{name}_gpu_ray_depth": dep.cpu().numpy(), f"{name}_host_ray_pos": hp,
                    f"{name}_host_ray_fid": hf, f"{name}_host_ray_depth": hdep})
        # the reference's device stab directions of these queries (the raystab
        # oracle's input), for the closed and the open mesh case
        if name in ("dodeca", "tori3"):
            dirs = torch.empty(n, 32, 3, device=dev)
            O.ref_stab_dirs_gpu_ptr(0, n, dirs.data_ptr(), stream)
            torch.cuda.synchronize()
            res[f"{name}_gpu_stab_dirs"] = dirs.cpu().numpy()
    np.savez_compressed(path, **res)
    print("wrote", path)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("step", choices=["inputs", "outputs"])
    ap.add_argument("--reference", help="reference checkout (inputs step)")
    ap.add_argument("--out", default=OUT)
    a = ap.parse_args()
    if a.step == "inputs":
        v, f = reference_dodecahedron(a.reference)
        np.savez_compressed(INPUTS, dodeca_v=v, dodeca_f=f)
        print("wrote", INPUTS, v.shape, f.shape)
    else:
        run_outputs(a.out)


if __name__ == "__main__":
    main()
