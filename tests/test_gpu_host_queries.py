"""Host-buffer queries (`out=`, C ABI cubvh_ray_trace_host /
cubvh_signed_distance_host): the same results as the device-tensor calls,
bit for bit, in one chunk and across several chunks (raystab included: its
stab rays follow the query index within the whole call)."""

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W

CHUNK = 1 << 21   # queries per chunk of the host pipeline


def _host_like(shape, dtype, pinned):
    return torch.empty(shape, dtype=dtype, pin_memory=pinned)


def _rays_equal(bvh, ro, rd, dev, pinned=True):
    n = ro.shape[0]
    want = bvh.ray_trace(ro.to(dev), rd.to(dev))
    out = (_host_like((n, 3), torch.float32, pinned), _host_like((n,), torch.int64, pinned),
           _host_like((n,), torch.float32, pinned))
    got = bvh.ray_trace(ro, rd, out=out)
    for a, b in zip(got, want):
        assert torch.equal(a, b.cpu())


def _dist_equal(bvh, pts, dev, mode, uvw=False, pinned=True):
    n = pts.shape[0]
    out = [_host_like((n,), torch.float32, pinned), _host_like((n,), torch.int64, pinned)]
    if uvw:
        out.append(_host_like((n, 3), torch.float32, pinned))
    if mode is None:
        want = bvh.unsigned_distance(pts.to(dev), return_uvw=uvw)
        got = bvh.unsigned_distance(pts, return_uvw=uvw, out=out)
    else:
        want = bvh.signed_distance(pts.to(dev), return_uvw=uvw, mode=mode)
        got = bvh.signed_distance(pts, return_uvw=uvw, mode=mode, out=out)
    for a, b in zip(got, want):
        if b is None:
            assert a is None
        else:
            assert torch.equal(a, b.cpu())


@pytest.mark.gpu
@pytest.mark.parametrize("pinned", [True, False])
def test_host_queries_one_chunk(dev, pinned):
    v, f = W.displaced_icosphere(4, 1)
    bvh = cubvh.cuBVH(v, f)
    ro, rd = W.camera_rays(2, 64, 50.0, 2.5, 1)
    _rays_equal(bvh, torch.from_numpy(ro), torch.from_numpy(rd), dev, pinned)
    pts = torch.from_numpy(W.uniform_points(5000, 3))
    _dist_equal(bvh, pts, dev, None, uvw=True, pinned=pinned)
    _dist_equal(bvh, pts, dev, "watertight", pinned=pinned)
    _dist_equal(bvh, pts, dev, "raystab", pinned=pinned)


@pytest.mark.gpu
def test_host_queries_several_chunks(dev):
    # five chunks, the last one partial: more chunks than the pipe's four
    # staging sets, so sets are reused
    n = 4 * CHUNK + 123_457
    v, f = W.icosphere(3, 0.8)
    bvh = cubvh.cuBVH(v, f)
    rng = np.random.default_rng(17)
    pts = torch.from_numpy(rng.uniform(-1, 1, (n, 3)).astype(np.float32))
    _dist_equal(bvh, pts, dev, None)
    _dist_equal(bvh, pts, dev, "raystab")
    _dist_equal(bvh, pts, dev, "watertight")
    ro = torch.from_numpy(np.repeat(np.array([[0.0, 0.0, 2.5]], np.float32), n, 0))
    d = rng.standard_normal((n, 3)).astype(np.float32)
    d[:, 2] = -np.abs(d[:, 2]) - 1.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    _rays_equal(bvh, ro, torch.from_numpy(d), dev)


def test_host_queries_argument_checks():
    """Host-buffer calls check their out= tensors before touching the GPU."""
    v, f = W.icosphere(2, 0.8)
    bvh = cubvh.cuBVH(v, f)
    pts = torch.zeros(10, 3)
    with pytest.raises(ValueError):
        bvh.unsigned_distance(pts, out=(torch.empty(10, dtype=torch.float64), torch.empty(10, dtype=torch.int64)))
    with pytest.raises(ValueError):
        bvh.unsigned_distance(pts, out=(torch.empty(9), torch.empty(10, dtype=torch.int64)))
    with pytest.raises(ValueError):
        bvh.unsigned_distance(pts, return_uvw=True, out=(torch.empty(10), torch.empty(10, dtype=torch.int64)))
    with pytest.raises(ValueError):
        bvh.ray_trace(pts, pts, out=(torch.empty(10, 3), torch.empty(10, dtype=torch.int32), torch.empty(10)))
    with pytest.raises(ValueError):
        bvh.signed_distance(pts, vertices=torch.zeros(4, 3), out=(torch.empty(10), torch.empty(10, dtype=torch.int64)))


@pytest.mark.gpu
def test_host_queries_non_blocking_two_streams(dev):
    """non_blocking calls on two streams overlap (separate internal streams
    per caller stream) and give the blocking results once synchronized."""
    v, f = W.displaced_icosphere(4, 1)
    bvh = cubvh.cuBVH(v, f)
    ro, rd = (torch.from_numpy(x).pin_memory() for x in W.camera_rays(4, 512, 50.0, 2.5, 1))
    pts = torch.from_numpy(W.uniform_points(3 * CHUNK // 2, 5)).pin_memory()
    n, m = ro.shape[0], pts.shape[0]
    want_r = bvh.ray_trace(ro.to(dev), rd.to(dev))
    want_s = bvh.signed_distance(pts.to(dev), mode="watertight")
    out_r = (torch.empty((n, 3), pin_memory=True), torch.empty(n, dtype=torch.int64, pin_memory=True),
             torch.empty(n, pin_memory=True))
    out_s = (torch.empty(m, pin_memory=True), torch.empty(m, dtype=torch.int64, pin_memory=True))
    s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    for _ in range(2):
        for t in out_r + out_s:
            t.zero_()
        with torch.cuda.stream(s1):
            bvh.ray_trace(ro, rd, out=out_r, non_blocking=True)
        with torch.cuda.stream(s2):
            bvh.signed_distance(pts, mode="watertight", out=out_s, non_blocking=True)
        s1.synchronize(); s2.synchronize()
        for a, b in zip(out_r, want_r):
            assert torch.equal(a, b.cpu())
        for a, b in zip(out_s, want_s):
            assert torch.equal(a, b.cpu())
    with pytest.raises(ValueError):
        bvh.ray_trace(ro.double(), rd, out=out_r, non_blocking=True)


@pytest.mark.gpu
def test_host_queries_priority_streams(dev):
    """A compute-heavy call on a low-priority stream and a copy-heavy one on a
    high-priority stream (the C1 end-to-end arrangement: the distance kernels
    of the first yield SMs to the second's chunk kernels) give the blocking
    results, several chunks each."""
    v, f = W.displaced_icosphere(5, 2)
    bvh = cubvh.cuBVH(v, f)
    ro, rd = (torch.from_numpy(x).pin_memory() for x in W.camera_rays(2, 1448, 50.0, 2.5, 3))  # ~4.2M rays
    pts = torch.from_numpy(W.uniform_points(5 * CHUNK // 2, 8)).pin_memory()
    n, m = ro.shape[0], pts.shape[0]
    want_r = bvh.ray_trace(ro.to(dev), rd.to(dev))
    want_s = bvh.signed_distance(pts.to(dev), mode="watertight")
    want_u = bvh.unsigned_distance(pts.to(dev), return_uvw=True)
    out_r = (torch.empty((n, 3), pin_memory=True), torch.empty(n, dtype=torch.int64, pin_memory=True),
             torch.empty(n, pin_memory=True))
    out_s = (torch.empty(m, pin_memory=True), torch.empty(m, dtype=torch.int64, pin_memory=True))
    out_u = (torch.empty(m, pin_memory=True), torch.empty(m, dtype=torch.int64, pin_memory=True),
             torch.empty((m, 3), pin_memory=True))
    lo = torch.cuda.Stream(dev, priority=0)
    lo2 = torch.cuda.Stream(dev, priority=0)
    hi = torch.cuda.Stream(dev, priority=-1)
    for _ in range(2):
        for t in out_r + out_s + out_u:
            t.zero_()
        with torch.cuda.stream(lo):
            bvh.signed_distance(pts, mode="watertight", out=out_s, non_blocking=True)
        with torch.cuda.stream(lo2):
            bvh.unsigned_distance(pts, return_uvw=True, out=out_u, non_blocking=True)
        with torch.cuda.stream(hi):
            bvh.ray_trace(ro, rd, out=out_r, non_blocking=True)
        for s in (lo, lo2, hi):
            s.synchronize()
        for a, b in zip(out_r, want_r):
            assert torch.equal(a, b.cpu())
        for a, b in zip(out_s, want_s):
            assert torch.equal(a, b.cpu())
        for a, b in zip(out_u, want_u):
            assert torch.equal(a, b.cpu())
