"""Watertight signs through the per-triangle candidate lists: lists rebuilt
after a refit, and triangles whose lists overflow (more than 32 candidates)
falling back to the tree walk, all equal to the FP64 oracle."""

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _check(oracle, bvh, v, f, pts, dev):
    """Distances and face ids exact; signs exact except where the oracle flags
    the normal-sum dot product as zero to 1e-12 (the sign there depends on
    the summation order)."""
    d, fid, _ = bvh.signed_distance(torch.from_numpy(pts).to(dev), mode="watertight")
    sd, ofid, fl = oracle.sdf_watertight64(v, f, pts)
    d, want = _np(d), sd.astype(np.float32)
    assert np.array_equal(_np(fid), ofid)
    assert np.array_equal(np.abs(d), np.abs(want))
    ok = (fl & 1) == 0
    assert ok.mean() > 0.99
    assert np.array_equal(np.signbit(d[ok]), np.signbit(want[ok]))


def test_watertight_after_refit(oracle, dev):
    V, F = W.displaced_icosphere(3, 2)
    bvh = cubvh.cuBVH(V, F)
    rng = np.random.default_rng(9)
    pts = np.concatenate([W.uniform_points(3000, 5), W.surface_points(V, F, 3000, 0.01, rng)])
    _check(oracle, bvh, V, F, pts, dev)          # builds the lists
    # flatten the sphere into a thin disc: triangles of the two faces come
    # within the normal-sum radius of each other, so stale lists would miss them
    V2 = (V * np.array([1.0, 1.0, 0.0015], np.float32)).astype(np.float32)
    bvh.refit(torch.from_numpy(V2).to(dev))
    pts2 = np.concatenate([W.uniform_points(3000, 6) * np.array([1, 1, 0.01], np.float32),
                           W.surface_points(V2, F, 3000, 0.002, rng)]).astype(np.float32)
    _check(oracle, bvh, V2, F, pts2, dev)


def test_refit_to_degenerate_faces(oracle, dev):
    """A refit that collapses faces (an edge shrunk to a point, a vertex moved
    onto the opposite edge) recomputes their filter error factors: distances,
    face ids and uvw after the refit equal the oracle's, with the collapsed
    faces among the nearest."""
    V, F = W.displaced_icosphere(3, 2)
    bvh = cubvh.cuBVH(V, F)
    rng = np.random.default_rng(13)
    pts = W.uniform_points(4000, 7)
    bvh.unsigned_distance(torch.from_numpy(pts).to(dev))
    V2 = V.copy()
    sel = rng.choice(len(F), 40, replace=False)
    for k, t in enumerate(sel):
        a, b, c = F[t]
        if k % 2 == 0:
            V2[b] = V2[a]                      # edge a-b shrunk to a point
        else:
            V2[c] = 0.5 * (V2[a] + V2[b])      # c on the edge a-b
    bvh.refit(torch.from_numpy(V2).to(dev))
    around = V2[F[sel]].mean(1).repeat(50, 0) + rng.normal(0, 0.01, (2000, 3))
    near = np.concatenate([pts, around]).astype(np.float32)
    d, fid, uvw = bvh.unsigned_distance(torch.from_numpy(near).to(dev), return_uvw=True)
    od, ofid, ouvw, _, _ = oracle.udf64(V2, F, near)
    assert np.array_equal(_np(d), od.astype(np.float32))
    assert np.array_equal(_np(fid), ofid)
    assert np.array_equal(_np(uvw), ouvw.astype(np.float32))
    t = V2[F].astype(np.float64)
    zero = np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1) == 0
    assert zero.sum() >= 20 and zero[ofid].sum() > 0
    _check(oracle, bvh, V2, F, near, dev)


def _double_cone(n=40, r=0.5, h=0.6):
    a = np.linspace(0, 2 * np.pi, n, endpoint=False)
    ring = np.stack([r * np.cos(a), r * np.sin(a), np.zeros(n)], 1)
    v = np.concatenate([ring, [[0, 0, h], [0, 0, -h]]]).astype(np.float32)
    top, bot = n, n + 1
    f = []
    for i in range(n):
        j = (i + 1) % n
        f.append([i, j, top])
        f.append([j, i, bot])
    return v, np.array(f, np.int64)


def test_watertight_list_overflow(oracle, dev):
    # 40 triangles share each apex: their lists hold 40 > 32 candidates
    v, f = _double_cone()
    bvh = cubvh.cuBVH(v, f)
    rng = np.random.default_rng(11)
    apex = np.array([[0, 0, 0.6], [0, 0, -0.6]], np.float32)
    pts = np.concatenate([rng.uniform(-0.8, 0.8, (2000, 3)),
                          apex[rng.integers(0, 2, 2000)] + rng.normal(0, 0.01, (2000, 3))]).astype(np.float32)
    _check(oracle, bvh, v, f, pts, dev)


def test_watertight_overflow_repeated(oracle, dev):
    """Back-to-back calls whose scratch is reused: the overflow queue of one
    call holds only that call's queries (its length counter is its own, not
    shared with the distance pass's tail statistics), so repeated calls with
    few packets per warp (the distance pass's tail control on) and
    overflowing lists keep every sign.  A triangle soup with every face four
    times overflows every list."""
    v, f = W.icosphere(2, 0.5)
    f = np.concatenate([f, f, f, f[:7]])
    bvh = cubvh.cuBVH(v, f)
    for seed in range(4):
        rng = np.random.default_rng(40 + seed)
        pts = np.concatenate([rng.uniform(-0.7, 0.7, (3000, 3)),
                              W.surface_points(v, f, 3000, 0.02, rng)]).astype(np.float32)
        _check(oracle, bvh, v, f, pts, dev)
