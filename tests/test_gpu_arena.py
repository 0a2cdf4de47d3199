"""BVHArena: many meshes in one launch must give exactly what one cuBVH per
mesh gives (which the other tests pin to the oracle), including raystab
streams indexed per mesh, gradients, and CUDA-graph replay."""

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W
from cubvh_b200.autotune import autotune_leaf_sizes

pytestmark = pytest.mark.gpu


def _meshes():
    out = [W.displaced_icosphere(2, 1), W.icosphere(3, 0.6), W.torus(0.5, 0.2, 24, 8),
           W.displaced_icosphere(4, 2), W.dodecahedron(), W.random_tori(5, n_tori=2, n_major=32, n_minor=8)]
    return [(np.asarray(v, np.float32), np.asarray(f, np.int64)) for v, f in out]


def _queries(meshes, counts, seed=0):
    rng = np.random.default_rng(seed)
    qs = []
    for (v, f), c in zip(meshes, counts):
        lo, hi = v.min(0), v.max(0)
        ctr, half = (lo + hi) / 2, (hi - lo) / 2 * 1.1
        qs.append((ctr + rng.uniform(-1, 1, (c, 3)) * half).astype(np.float32))
    return qs


@pytest.mark.parametrize("uvw", [False, True])
def test_arena_matches_per_mesh(dev, uvw):
    meshes = _meshes()
    counts = [1000, 0, 33, 5000, 31, 4097]
    modes = ["unsigned", "raystab", "watertight", "raystab", "watertight", "unsigned"]
    qs = _queries(meshes, counts)
    arena = cubvh.BVHArena(meshes)
    arena.set_queries(counts, modes)
    pts = torch.from_numpy(np.concatenate(qs)).to(dev)
    d, fid, u = arena.distance(pts, return_uvw=uvw)
    off = np.concatenate([[0], np.cumsum(counts)])
    for m, ((v, f), q, mode) in enumerate(zip(meshes, qs, modes)):
        if counts[m] == 0:
            continue
        bvh = cubvh.cuBVH(v, f)
        p = torch.from_numpy(q).to(dev)
        if mode == "unsigned":
            rd, rf, ru = bvh.unsigned_distance(p, return_uvw=uvw)
        else:
            rd, rf, ru = bvh.signed_distance(p, return_uvw=uvw, mode=mode)
        sl = slice(off[m], off[m + 1])
        assert torch.equal(d[sl], rd), f"mesh {m} ({mode}) distances"
        assert torch.equal(fid[sl], rf), f"mesh {m} ({mode}) faces"
        if uvw:
            assert torch.equal(u[sl], ru)


def test_arena_backward_matches_per_mesh(dev):
    meshes = _meshes()[:4]
    counts = [700, 300, 64, 2000]
    modes = ["unsigned", "raystab", "watertight", "unsigned"]
    qs = _queries(meshes, counts, seed=1)
    arena = cubvh.BVHArena(meshes)
    arena.set_queries(counts, modes)
    pts = torch.from_numpy(np.concatenate(qs)).to(dev).requires_grad_()
    w = torch.rand(pts.shape[0], device=dev)
    d, _, _ = arena.distance(pts)
    (w * d).sum().backward()
    off = np.concatenate([[0], np.cumsum(counts)])
    for m, ((v, f), q, mode) in enumerate(zip(meshes, qs, modes)):
        p = torch.from_numpy(q).to(dev).requires_grad_()
        bvh = cubvh.cuBVH(v, f)
        r = bvh.unsigned_distance(p)[0] if mode == "unsigned" else bvh.signed_distance(p, mode=mode)[0]
        (w[off[m]:off[m + 1]] * r).sum().backward()
        assert torch.allclose(pts.grad[off[m]:off[m + 1]], p.grad, rtol=0, atol=1e-6)


def test_arena_graph_replay(dev):
    meshes = _meshes()[:3]
    counts = [2000, 1500, 900]
    modes = ["unsigned", "watertight", "raystab"]
    arena = cubvh.BVHArena(meshes)
    arena.set_queries(counts, modes)
    q1 = torch.from_numpy(np.concatenate(_queries(meshes, counts, 2))).to(dev)
    q2 = torch.from_numpy(np.concatenate(_queries(meshes, counts, 3))).to(dev)
    buf = q1.clone()
    replay, (d, fid, _) = arena.capture(buf)
    replay()
    torch.cuda.synchronize()
    d1, f1, _ = arena.distance(q1)
    assert torch.equal(d, d1) and torch.equal(fid, f1)
    buf.copy_(q2)
    replay()
    torch.cuda.synchronize()
    d2, f2, _ = arena.distance(q2)
    assert torch.equal(d, d2) and torch.equal(fid, f2)


def test_arena_errors(dev):
    arena = cubvh.BVHArena(_meshes()[:2])
    with pytest.raises(RuntimeError, match="set_queries"):
        arena.distance(torch.zeros(4, 3, device=dev))
    with pytest.raises(RuntimeError):
        arena.set_queries([1, 2, 3], ["unsigned"] * 3)
    arena.set_queries([4, 4], ["unsigned", "raystab"])
    with pytest.raises(RuntimeError, match=r"\[8, 3\]"):
        arena.distance(torch.zeros(5, 3, device=dev))


def test_autotuner_picks_leaf_sizes(dev):
    meshes = _meshes()
    qs = _queries(meshes, [4000] * len(meshes), 4)
    modes = ["unsigned", "raystab"] * 3
    leaves, report = autotune_leaf_sizes(meshes, qs, modes, sample=4000, repeats=1)
    assert len(leaves) == len(meshes) and set(leaves) <= {2, 3, 4}
    arena = cubvh.BVHArena(meshes, leaf_sizes=leaves)
    arena.set_queries([len(q) for q in qs], modes)
    d, fid, _ = arena.distance(torch.from_numpy(np.concatenate(qs)).to(dev))
    ref = cubvh.BVHArena(meshes)
    ref.set_queries([len(q) for q in qs], modes)
    d2, f2, _ = ref.distance(torch.from_numpy(np.concatenate(qs)).to(dev))
    assert torch.equal(d, d2) and torch.equal(fid, f2)     # leaf size never changes results


_FIRST_IN_PROCESS = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W
v, f = W.displaced_icosphere(3, 1)
rng = np.random.default_rng(3)
lo, hi = v.min(0), v.max(0)
q = ((lo + hi) / 2 + rng.uniform(-1, 1, (3000, 3)) * (hi - lo) / 2 * 1.1).astype(np.float32)
arena = cubvh.BVHArena([(v, f)])          # the process's first GPU work
arena.set_queries([3000], ["raystab"])
d, fid, _ = arena.distance(torch.from_numpy(q).cuda())
rd, rf, _ = cubvh.cuBVH(v, f).signed_distance(torch.from_numpy(q).cuda(), mode="raystab")
assert torch.equal(d, rd) and torch.equal(fid, rf), "arena raystab differs from cuBVH"
assert (d < 0).any() and (d > 0).any()
print("ok")
"""


def test_arena_raystab_first_in_process():
    """An arena's raystab pass in a process where no single-BVH query ran
    before: the stab-direction tables must be set by the arena itself."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FIRST_IN_PROCESS, root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
