"""Gradients of the distance queries.

CPU: the analytic gradient, built from the oracle's face / barycentrics /
closest point,
    d d/dp = (p - c)/d,   d d/dv_k = -lambda_k (p - c)/d,
is pinned against FP64 central finite differences (h = 1e-4) of the exact
point-triangle distance (the face held fixed; points near a tie are skipped,
where the distance to the nearest face is not differentiable).

GPU: the backward kernel equals that analytic reference (float32 round-off),
refit moves the BVH exactly like a rebuild, and the autograd path drives an
optimiser.
"""

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W


def analytic(oracle, V, F, pts, w):
    d, fid, uvw, cp, nn = oracle.udf64(V, F, pts)
    r = pts.astype(np.float64) - cp
    gp = w[:, None] * r / d[:, None]
    gv = np.zeros((len(V), 3))
    for k in range(3):
        np.add.at(gv, F[fid, k], -(uvw[:, k] * w)[:, None] * r / d[:, None])
    return d, fid, nn, gp, gv


def test_analytic_gradient_matches_fd(oracle):
    V, F = W.displaced_icosphere(2, 3)
    rng = np.random.default_rng(0)
    pts = np.concatenate([rng.uniform(-1, 1, (150, 3)), W.surface_points(V, F, 150, 0.05, rng)]).astype(np.float32)
    w = rng.random(len(pts))
    d, fid, nn, gp, _ = analytic(oracle, V, F, pts, w)
    keep = (nn == 1) & (d > 1e-3)
    tri = V[F[fid]].astype(np.float64)
    h = 1e-4
    # points
    for k in range(3):
        e = np.zeros(3); e[k] = h
        dp, _ = oracle.tri_dist64d(tri, pts + e)
        dm, _ = oracle.tri_dist64d(tri, pts - e)
        fd = w * (dp - dm) / (2 * h)
        assert np.abs(fd - gp[:, k])[keep].max() < 1e-6
    # vertices of each point's face
    _, lam = oracle.tri_dist64d(tri, pts)
    r = pts - np.einsum("nk,nkj->nj", lam, tri)
    for vk in range(3):
        for k in range(3):
            t2 = tri.copy(); t2[:, vk, k] += h
            dp, _ = oracle.tri_dist64d(t2, pts)
            t2[:, vk, k] -= 2 * h
            dm, _ = oracle.tri_dist64d(t2, pts)
            fd = (dp - dm) / (2 * h)
            an = -lam[:, vk] * r[:, k] / d
            assert np.abs(fd - an)[keep].max() < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("signed", [False, True])
def test_backward_matches_analytic(oracle, dev, signed):
    V, F = W.displaced_icosphere(3, 5)
    rng = np.random.default_rng(1)
    pts = np.concatenate([rng.uniform(-1, 1, (3000, 3)), W.surface_points(V, F, 3000, 0.05, rng)]).astype(np.float32)
    w = rng.random(len(pts)).astype(np.float32)
    bvh = cubvh.cuBVH(V, F)
    p = torch.from_numpy(pts).to(dev).requires_grad_()
    v = torch.from_numpy(V).to(dev).requires_grad_()
    if signed:
        d, fid, _ = bvh.signed_distance(p, mode="watertight", vertices=v)
    else:
        d, fid, _ = bvh.unsigned_distance(p, vertices=v)
    (torch.from_numpy(w).to(dev) * d).sum().backward()
    od, ofid, nn, gp, gv = analytic(oracle, V, F, pts, w.astype(np.float64))
    assert np.array_equal(fid.cpu().numpy(), ofid)
    s = np.sign(d.detach().cpu().numpy()).astype(np.float64) if signed else 1.0
    gp = gp * (s[:, None] if signed else 1.0)
    got_p = p.grad.cpu().numpy().astype(np.float64)
    assert np.abs(got_p - gp).max() < 1e-6 * (1 + np.abs(gp).max())
    # vertex gradients: sum of the same terms (signed: per-point sign)
    if signed:
        _, _, uvw, cp, _ = oracle.udf64(V, F, pts)
        r = pts.astype(np.float64) - cp
        gv = np.zeros((len(V), 3))
        for k in range(3):
            np.add.at(gv, F[ofid, k], -(uvw[:, k] * w * s)[:, None] * r / od[:, None])
    got_v = v.grad.cpu().numpy().astype(np.float64)
    assert np.abs(got_v - gv).max() < 1e-5 * (1 + np.abs(gv).max())


@pytest.mark.gpu
def test_refit_equals_rebuild(oracle, dev):
    V, F = W.displaced_icosphere(3, 2)
    bvh = cubvh.cuBVH(V, F)
    rng = np.random.default_rng(7)
    V2 = (V * 1.15 + rng.normal(0, 0.01, V.shape)).astype(np.float32)
    bvh.refit(torch.from_numpy(V2).to(dev))
    pts = W.uniform_points(5000, 3)
    d, fid, uvw = bvh.unsigned_distance(torch.from_numpy(pts).to(dev), return_uvw=True)
    od, ofid, ouvw, _, _ = oracle.udf64(V2, F, pts)
    assert np.array_equal(d.cpu().numpy(), od.astype(np.float32))
    assert np.array_equal(fid.cpu().numpy(), ofid)
    assert np.array_equal(uvw.cpu().numpy(), ouvw.astype(np.float32))
    ro, rd = W.camera_rays(1, 32, 50.0, 2.5, 3)
    _, rf, t = bvh.ray_trace(torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev))
    ot, orf, _ = oracle.ray64(V2, F, ro, rd)
    assert np.array_equal(t.cpu().numpy(), ot.astype(np.float32)) and np.array_equal(rf.cpu().numpy(), orf)


@pytest.mark.gpu
def test_adam_fit_decreases_loss(dev):
    target_v, target_f = W.displaced_icosphere(4, 1)
    rng = np.random.default_rng(3)
    samples = torch.from_numpy(W.surface_points(target_v, target_f, 20000, 0.0, rng)).to(dev)
    v0, f0 = W.icosphere(3, 0.5)
    bvh = cubvh.cuBVH(v0, f0)
    v = torch.from_numpy(v0).to(dev).requires_grad_()
    opt = torch.optim.Adam([v], lr=5e-3)
    losses = []
    for _ in range(30):
        opt.zero_grad()
        d, _, _ = bvh.unsigned_distance(samples, vertices=v)
        loss = d.mean()
        loss.backward()
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < 0.5 * losses[0]


@pytest.mark.gpu
def test_points_only_grad(dev):
    v, f = W.icosphere(2, 0.8)
    bvh = cubvh.cuBVH(v, f)
    p = torch.tensor([[1.5, 0.0, 0.0], [0.0, 0.0, 0.1]], device=dev, requires_grad=True)
    d, _, _ = bvh.unsigned_distance(p)
    d.sum().backward()
    g = p.grad.cpu().numpy()
    assert np.allclose(np.linalg.norm(g, axis=1), 1.0, atol=1e-5)
    # unit gradients: outward from the sphere, and (inside, below the pole) away
    # from the nearest face above, whose plane is slightly tilted
    assert g[0, 0] > 0.99 and g[1, 2] < -0.95
