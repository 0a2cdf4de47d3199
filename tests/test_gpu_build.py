"""BVH built on the GPU (cuBVH(..., device_build=True)): the same layout as
the host builder's (every face once, child boxes that contain their
content, breadth-first levels, at most 13 levels), and therefore the same
results for every query as a host-built BVH, which the other tests pin to
the FP64 oracle."""

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W
from test_host import decode, layout

pytestmark = pytest.mark.gpu


def _mesh(name):
    if name == "ico4":
        return W.icosphere(4, 0.8)
    if name == "disp4":
        return W.displaced_icosphere(4, 1)
    if name == "tori":
        return W.random_tori(2, n_tori=3, n_major=40, n_minor=10)
    if name == "dodeca":
        return W.dodecahedron()
    if name == "duplicates":  # many faces with one centroid: equal Morton codes
        v, f = W.icosphere(2, 0.5)
        return v, np.concatenate([f, f, f, f[:7]])
    if name == "flat":        # a planar grid: zero extent on one axis
        n = 40
        x, y = np.meshgrid(np.linspace(-1, 1, n), np.linspace(-1, 1, n), indexing="ij")
        v = np.stack([x.ravel(), y.ravel(), np.zeros(n * n)], 1).astype(np.float32)
        i = np.arange(n * n).reshape(n, n)
        a, b, c, d = i[:-1, :-1].ravel(), i[1:, :-1].ravel(), i[1:, 1:].ravel(), i[:-1, 1:].ravel()
        return v, np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)])
    if name == "degenerate":  # zero-area faces: a segment, a point, a sphere edge
        v, f = W.icosphere(2, 0.8)
        nv = len(v)
        extra = np.array([[0.2, 0.1, 0.85], [0.3, 0.1, 0.85], [0.4, 0.1, 0.85], [-0.3, -0.2, 0.9]], np.float32)
        return (np.concatenate([v, extra]).astype(np.float32),
                np.concatenate([f, [[nv, nv + 1, nv + 2], [nv + 3, nv + 3, nv + 3], [0, 0, 1]]]))
    if name == "slivers":
        from test_gpu_queries import sliver_mesh
        v, f, _, _ = sliver_mesh(2000, 71)
        return v, f
    raise KeyError(name)


MESHES = ["ico4", "disp4", "tori", "dodeca", "duplicates", "flat", "degenerate", "slivers"]


@pytest.mark.parametrize("mesh", MESHES)
def test_device_build_layout(dev, mesh):
    v, f = _mesh(mesh)
    v, f = np.asarray(v, np.float32), np.asarray(f, np.int64)
    nodes, tris, depth = layout(cubvh.cuBVH(v, f, device_build=True))
    assert 1 <= depth <= 13
    assert np.array_equal(np.sort(tris['id']), np.arange(len(f)))
    tv = v[f[tris['id']]]
    assert np.array_equal(tris['a'], tv[:, 0]) and np.array_equal(tris['b'], tv[:, 1])
    assert np.array_equal(tris['c'], tv[:, 2])
    tlo = np.minimum(np.minimum(tris['a'], tris['b']), tris['c'])
    thi = np.maximum(np.maximum(tris['a'], tris['b']), tris['c'])
    seen = np.zeros(len(tris), np.int32)

    def walk(i):
        n = nodes[i]
        lo, hi = decode(n)
        blo, bhi = np.full(3, np.inf, np.float32), np.full(3, -np.inf, np.float32)
        k = 0
        for j in range(8):
            m = n['meta'][j]
            if m == 0xFF:
                continue
            if m & 0x80:
                assert (m & 7) == k, "internal children are numbered in slot order"
                k += 1
                c = n['cb'] + (m & 7)
                assert c > i
                clo, chi = walk(c)
            else:
                s0 = n['tb'] + (m & 31)
                s1 = s0 + ((m >> 5) & 3) + 1
                seen[s0:s1] += 1
                clo, chi = tlo[s0:s1].min(0), thi[s0:s1].max(0)
            assert (lo[j] <= clo).all() and (hi[j] >= chi).all(), "child box does not contain its content"
            blo, bhi = np.minimum(blo, clo), np.maximum(bhi, chi)
        assert n['nint'] == k
        return blo, bhi

    walk(0)
    assert (seen == 1).all(), "every soup slot belongs to exactly one leaf"
    # the filter's error factors equal the host builder's, face by face
    _, htris, _ = layout(cubvh.cuBVH(v, f))
    hk, dk = np.empty(len(f), np.float32), np.empty(len(f), np.float32)
    hk[htris['id']], dk[tris['id']] = htris['k'], tris['k']
    assert np.array_equal(hk, dk)
    hk[htris['id']], dk[tris['id']] = htris['ke2'], tris['ke2']
    assert np.array_equal(hk, dk)


@pytest.mark.parametrize("mesh", MESHES)
def test_device_build_same_results(oracle, dev, mesh):
    v, f = _mesh(mesh)
    host = cubvh.cuBVH(v, f)
    gpu = cubvh.cuBVH(v, f, device_build=True)
    rng = np.random.default_rng(3)
    p = torch.from_numpy(rng.uniform(-1.2, 1.2, (20000, 3)).astype(np.float32)).to(dev)
    for a, b in zip(host.unsigned_distance(p, return_uvw=True), gpu.unsigned_distance(p, return_uvw=True)):
        assert torch.equal(a, b)
    for mode in ("watertight", "raystab"):
        a, b = host.signed_distance(p, mode=mode), gpu.signed_distance(p, mode=mode)
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    ro = torch.from_numpy(rng.uniform(-1.5, 1.5, (20000, 3)).astype(np.float32)).to(dev)
    rd = torch.nn.functional.normalize(torch.from_numpy(rng.standard_normal((20000, 3)).astype(np.float32)).to(dev), dim=1)
    for a, b in zip(host.ray_trace(ro, rd), gpu.ray_trace(ro, rd)):
        assert torch.equal(a, b)
    # and directly against the oracle
    od, ofid, _, _, _ = oracle.udf64(np.asarray(v, np.float32), np.asarray(f, np.int64), p[:3000].cpu().numpy())
    d, fid, _ = gpu.unsigned_distance(p[:3000])
    assert np.array_equal(d.cpu().numpy(), od.astype(np.float32)) and np.array_equal(fid.cpu().numpy(), ofid)


def test_device_build_state_dict_and_grad(dev):
    v, f = W.displaced_icosphere(3, 2)
    gpu = cubvh.cuBVH(v, f, device_build=True)
    host = cubvh.cuBVH(v, f)
    p = torch.from_numpy(W.uniform_points(5000, 4)).to(dev)
    back = cubvh.cuBVH.from_state_dict(gpu.state_dict())
    assert torch.equal(back.unsigned_distance(p)[0], gpu.unsigned_distance(p)[0])
    grads = []
    for b in (host, gpu):
        pts = p.clone().requires_grad_()
        vv = torch.from_numpy(np.asarray(v, np.float32)).to(dev).requires_grad_()
        d, _, _ = b.unsigned_distance(pts, vertices=vv)
        d.sum().backward()
        grads.append((pts.grad, vv.grad))
    assert torch.equal(grads[0][0], grads[1][0])
    # vertex gradients are sums of float atomics, in an order that follows the
    # tree's soup order: equal up to float rounding
    assert torch.allclose(grads[0][1], grads[1][1], rtol=1e-5, atol=1e-5)


def test_device_build_errors(dev):
    v, f = W.icosphere(2, 0.5)
    bad = np.asarray(f, np.int64).copy()
    bad[5, 1] = len(v)
    with pytest.raises(RuntimeError, match="vertex index"):
        cubvh.cuBVH(v, bad, device_build=True)
    vn = np.asarray(v, np.float32).copy()
    vn[3, 0] = np.nan
    with pytest.raises(RuntimeError, match="finite"):
        cubvh.cuBVH(vn, f, device_build=True)


def test_device_built_arena(dev):
    """All meshes built on the GPU in one pass: every query of every mesh
    equals the host-built arena's result, including raystab and per-mesh
    leaf sizes, one-face and four-face meshes, and the backward."""
    meshes = [W.displaced_icosphere(2, 1), W.icosphere(3, 0.6), W.torus(0.5, 0.2, 24, 8),
              W.displaced_icosphere(4, 2), W.dodecahedron(), W.random_tori(5, n_tori=2, n_major=32, n_minor=8)]
    meshes = [(np.asarray(v, np.float32), np.asarray(f, np.int64)) for v, f in meshes]
    v0, f0 = meshes[1]
    meshes.append((v0, f0[:1]))          # a one-face mesh
    meshes.append((v0, f0[:4]))          # a single-leaf mesh
    counts = [1000, 300, 33, 5000, 31, 4097, 50, 70]
    modes = ["unsigned", "raystab", "watertight", "raystab", "watertight", "unsigned", "unsigned", "unsigned"]
    leaves = [4, 2, 3, 4, 1, 3, 4, 2]
    rng = np.random.default_rng(7)
    qs = []
    for (v, f), c in zip(meshes, counts):
        lo, hi = v.min(0), v.max(0)
        qs.append(((lo + hi) / 2 + rng.uniform(-1, 1, (c, 3)) * (hi - lo) / 2 * 1.1).astype(np.float32))
    pts = torch.from_numpy(np.concatenate(qs)).to(dev)
    res = []
    for device_build in (False, True):
        ar = cubvh.BVHArena(meshes, leaf_sizes=leaves, device_build=device_build)
        ar.set_queries(counts, modes)
        p = pts.clone().requires_grad_()
        d, fid, uvw = ar.distance(p, return_uvw=True)
        d.sum().backward()
        res.append((d.detach(), fid, uvw, p.grad, ar.info()))
    (d0, f0_, u0, g0, i0), (d1, f1, u1, g1, i1) = res
    assert torch.equal(d0, d1) and torch.equal(f0_, f1) and torch.equal(u0, u1) and torch.equal(g0, g1)
    assert i0["faces"] == i1["faces"] and i1["meshes"] == len(meshes)
