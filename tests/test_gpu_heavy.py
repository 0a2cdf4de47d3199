"""Packets whose walk grows far past the launch's fair share (points near the
centre of a sphere, about equally far from every triangle, among cheap
queries elsewhere) are handed to the warp-per-query kernel; the results must
still equal the FP64 oracle's bit for bit, for the signed modes (which read
the winning slot), and in an arena (per-mesh roots)."""

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _centre_points(n, radius, seed):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return (d * radius * rng.uniform(0, 1, (n, 1)) ** (1 / 3)).astype(np.float32)


def _check_udf(oracle, v, f, pts, out):
    d, fid, uvw = (_np(x) for x in out)
    od, ofid, ouvw, _, _ = oracle.udf64(v, f, pts)
    assert np.array_equal(d, od.astype(np.float32)), f"{(d != od.astype(np.float32)).sum()} distances differ"
    assert np.array_equal(fid, ofid), f"{(fid != ofid).sum()} faces differ"
    assert np.array_equal(uvw, ouvw.astype(np.float32))


def test_heavy_udf_uvw(oracle, dev):
    v, f = W.icosphere(4, 0.8)
    pts = np.concatenate([_centre_points(3000, 0.05, 0), W.uniform_points(6000, 1)])
    out = cubvh.cuBVH(v, f).unsigned_distance(torch.from_numpy(pts).to(dev), return_uvw=True)
    _check_udf(oracle, v, f, pts, out)


@pytest.mark.parametrize("mode", ["watertight", "raystab"])
def test_heavy_signed(oracle, dev, stab_dirs, mode):
    v, f = W.displaced_icosphere(3, 1)
    pts = np.concatenate([_centre_points(2500, 0.1, 2), W.uniform_points(4000, 3)])
    d, fid, _ = cubvh.cuBVH(v, f).signed_distance(torch.from_numpy(pts).to(dev), mode=mode)
    if mode == "watertight":
        sd, ofid, _ = oracle.sdf_watertight64(v, f, pts)
    else:
        sd, ofid, _ = oracle.sdf_raystab64(v, f, pts, dirs=stab_dirs(len(pts)))
    assert np.array_equal(_np(fid), ofid)
    assert np.array_equal(_np(d), sd.astype(np.float32))
    assert (_np(d)[:2500] < 0).all()


def test_heavy_many(oracle, dev):
    """200k near-centre queries among 800k uniform ones."""
    v, f = W.icosphere(4, 0.8)
    pts = np.concatenate([W.uniform_points(800_000, 9), _centre_points(200_000, 0.03, 4)])
    d, fid, uvw = cubvh.cuBVH(v, f).unsigned_distance(torch.from_numpy(pts).to(dev), return_uvw=True)
    sub = np.arange(0, len(pts), 97)
    _check_udf(oracle, v, f, pts[sub], (d[sub], fid[sub], uvw[sub]))


def test_heavy_in_arena(oracle, dev, stab_dirs):
    meshes = [W.icosphere(4, 0.8), W.torus(0.5, 0.2, 48, 16), W.displaced_icosphere(3, 5)]
    meshes = [(np.asarray(v, np.float32), np.asarray(f, np.int64)) for v, f in meshes]
    qs = [_centre_points(2000, 0.05, 6), W.uniform_points(5000, 7), _centre_points(1500, 0.1, 8)]
    arena = cubvh.BVHArena(meshes)
    arena.set_queries([len(q) for q in qs], ["unsigned", "unsigned", "raystab"])
    d, fid, _ = arena.distance(torch.from_numpy(np.concatenate(qs)).to(dev))
    d, fid = _np(d), _np(fid)
    off = np.concatenate([[0], np.cumsum([len(q) for q in qs])])
    for m, ((v, f), q) in enumerate(zip(meshes, qs)):
        sl = slice(off[m], off[m + 1])
        if m == 2:
            sd, ofid, _ = oracle.sdf_raystab64(v, f, q, dirs=stab_dirs(len(q)))
            want = sd.astype(np.float32)
        else:
            od, ofid, _, _, _ = oracle.udf64(v, f, q)
            want = od.astype(np.float32)
        assert np.array_equal(fid[sl], ofid), f"mesh {m}: faces differ"
        assert np.array_equal(d[sl], want), f"mesh {m}: distances differ"
