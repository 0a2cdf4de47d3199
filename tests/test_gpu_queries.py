"""GPU parity of the query kernels against the FP64 CPU oracle.

The kernels decide every distance, closest point, uvw, hit and sign in double
with the oracle's operation order, so on the same float inputs the float32
outputs must equal the oracle's double results rounded to float32 (bit for
bit), and face_id must equal the oracle's lowest-index minimiser.  The
required tolerance (1e-6 relative / 1e-7 absolute) is checked
as well and the maximum error reported.
"""

import numpy as np
import pytest
import torch

import cubvh_b200 as cubvh
from cubvh_b200 import workloads as W

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-7


def _np(t):
    return t.detach().cpu().numpy()


def assert_close(got, want, what):
    err = np.abs(got.astype(np.float64) - want)
    bound = ATOL + RTOL * np.abs(want)
    bad = err > bound
    assert not bad.any(), f"{what}: {bad.sum()} outside tolerance, max err {err.max():.3g}"
    return float(err.max()) if err.size else 0.0


def check_udf(oracle, v, f, pts, out, with_uvw=True):
    d, fid, uvw = out
    od, ofid, ouvw, _, nn = oracle.udf64(v, f, pts)
    d, fid = _np(d), _np(fid)
    assert_close(d, od, "distance")
    assert np.array_equal(d, od.astype(np.float32)), f"distance bits differ at {np.nonzero(d != od.astype(np.float32))[0][:8]}"
    bad = fid != ofid
    assert not bad.any(), f"face_id differs at {bad.sum()} points (ties there: {nn[bad][:8]})"
    if with_uvw:
        uvw = _np(uvw)
        assert_close(uvw, ouvw, "uvw")
        assert np.array_equal(uvw, ouvw.astype(np.float32))


@pytest.mark.parametrize("level,n", [(2, 4000), (4, 20000)])
def test_udf_icosphere(oracle, dev, level, n):
    v, f = W.icosphere(level, 0.8)
    bvh = cubvh.cuBVH(v, f)
    pts = W.uniform_points(n, level)
    out = bvh.unsigned_distance(torch.from_numpy(pts).to(dev), return_uvw=True)
    check_udf(oracle, v, f, pts, out)


def test_udf_dodecahedron_randn(oracle, dev):
    # the reference's unsigned_distance test setup: dodecahedron, randn points
    v, f = W.dodecahedron()
    bvh = cubvh.cuBVH(v, f)
    pts = np.random.default_rng(11).standard_normal((5000, 3)).astype(np.float32)
    out = bvh.unsigned_distance(torch.from_numpy(pts).to(dev), return_uvw=True)
    check_udf(oracle, v, f, pts, out)
    # closest point rebuilt from uvw + face_id (reference test, atol 1e-5)
    d, fid, uvw = (_np(x) for x in out)
    cp = np.einsum("nk,nkj->nj", uvw.astype(np.float64), v[f[fid]].astype(np.float64))
    assert np.abs(np.linalg.norm(pts - cp, axis=1) - d).max() < 1e-5


def test_udf_displaced_near_surface(oracle, dev):
    v, f = W.displaced_icosphere(5, 1)
    bvh = cubvh.cuBVH(v, f)
    rng = np.random.default_rng(5)
    pts = np.concatenate([W.surface_points(v, f, 6000, 0.02, rng), W.surface_points(v, f, 2000, 1e-4, rng),
                          rng.uniform(-1, 1, (4000, 3)).astype(np.float32)])
    out = bvh.unsigned_distance(torch.from_numpy(pts).to(dev), return_uvw=True)
    check_udf(oracle, v, f, pts, out)


def test_udf_tori_open_mesh(oracle, dev):
    v, f = W.random_tori(2, n_tori=3, n_major=64, n_minor=16)
    bvh = cubvh.cuBVH(v, f)
    g = W.dense_grid(24)
    out = bvh.unsigned_distance(torch.from_numpy(g).to(dev), return_uvw=False)
    check_udf(oracle, v, f, g, out, with_uvw=False)


def test_udf_far_points_and_shapes(oracle, dev):
    v, f = W.icosphere(2, 0.8)
    bvh = cubvh.cuBVH(v, f)
    pts = torch.tensor([[2000.0, 0, 0], [0, 0, 999.0], [0.1, 0.2, 0.3]], device=dev)
    d, fid, uvw = bvh.unsigned_distance(pts, return_uvw=True)
    assert d[0].item() == 0.0 and fid[0].item() == 0     # beyond MAX_DIST: distance 0, face 0
    od, ofid, ouvw, _, _ = oracle.udf64(v, f, _np(pts))
    assert np.array_equal(_np(d), od.astype(np.float32)) and np.array_equal(_np(fid), ofid)
    assert np.array_equal(_np(uvw), ouvw.astype(np.float32))
    # prefix shapes, CPU float64 input, empty input
    p = torch.from_numpy(W.uniform_points(60, 1)).double().view(3, 4, 5, 3)
    d, fid, uvw = bvh.unsigned_distance(p, return_uvw=True)
    assert d.shape == (3, 4, 5) and fid.shape == (3, 4, 5) and uvw.shape == (3, 4, 5, 3)
    assert d.dtype == torch.float32 and fid.dtype == torch.int64 and d.is_cuda
    d, fid, uvw = bvh.unsigned_distance(torch.zeros(0, 3, device=dev))
    assert d.shape == (0,) and uvw is None


def check_rays(oracle, v, f, ro, rd, out):
    pos, fid, depth = (_np(x) for x in out)
    ot, ofid, fl = oracle.ray64(v, f, ro, rd)
    assert_close(depth, ot, "depth")
    assert np.array_equal(depth, ot.astype(np.float32))
    assert np.array_equal(fid, ofid), f"{(fid != ofid).sum()} ray faces differ"
    opos = (ro.astype(np.float64) + ot[:, None] * rd.astype(np.float64)).astype(np.float32)
    assert np.array_equal(pos, opos)
    return fl


def test_ray_trace_camera(oracle, dev):
    v, f = W.displaced_icosphere(4, 1)
    bvh = cubvh.cuBVH(v, f)
    ro, rd = W.camera_rays(2, 64, 50.0, 2.5, 1)
    out = bvh.ray_trace(torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev))
    check_rays(oracle, v, f, ro, rd, out)
    hit = _np(out[1]) >= 0
    assert 0.1 < hit.mean() < 0.9


def test_ray_trace_inside_and_random(oracle, dev):
    v, f = W.random_tori(2, n_tori=3, n_major=48, n_minor=12)
    bvh = cubvh.cuBVH(v, f)
    rng = np.random.default_rng(9)
    ro = rng.uniform(-1, 1, (6000, 3)).astype(np.float32)
    rd = rng.standard_normal((6000, 3)).astype(np.float32)
    rd[:100, 0] = 0.0          # axis-parallel components
    rd[100:150, :2] = 0.0
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    out = bvh.ray_trace(torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev))
    check_rays(oracle, v, f, ro, rd, out)
    assert out[0].shape == (6000, 3)


def test_ray_trace_in_face_planes(oracle, dev):
    """Rays with a zero direction component whose origin lies exactly on a
    face plane of an axis-aligned cube (and so on a child box plane): they run
    along the box face and hit the edges of the triangles there."""
    v = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float32)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    f = np.array([t for a, b, c, d in quads for t in ((a, b, c), (a, c, d))], np.int64)
    ro, rd = [], []
    for ax in range(3):
        u, w = (ax + 1) % 3, (ax + 2) % 3
        for side in (-1.0, 1.0):
            for x in np.linspace(-1.5, 1.5, 13):
                for dirn in ((0.0, 1.0), (0.6, 0.8), (-0.28, 0.96)):
                    o = np.zeros(3); o[ax] = side; o[u] = x; o[w] = -3.0
                    d = np.zeros(3); d[u], d[w] = dirn
                    ro.append(o); rd.append(d)
    ro, rd = np.array(ro, np.float32), np.array(rd, np.float32)
    bvh = cubvh.cuBVH(v, f)
    out = bvh.ray_trace(torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev))
    check_rays(oracle, v, f, ro, rd, out)
    assert (_np(out[1]) >= 0).mean() > 0.3


def test_ray_trace_order_independent(oracle, dev):
    """Results do not depend on how the rays are split into calls (one call of
    6000 rays against six of 1000: packets and work distribution differ) and
    equal the oracle's, also for 2160 rays along cube face planes."""
    v, f = W.random_tori(2, n_tori=3, n_major=48, n_minor=12)
    bvh = cubvh.cuBVH(v, f)
    rng = np.random.default_rng(21)
    ro = rng.uniform(-1, 1, (6000, 3)).astype(np.float32)
    rd = rng.standard_normal((6000, 3)).astype(np.float32)
    rd[:300, 2] = 0.0
    rd /= np.linalg.norm(rd, axis=1, keepdims=True)
    ro_t, rd_t = torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev)
    whole = bvh.ray_trace(ro_t, rd_t)
    parts = [bvh.ray_trace(ro_t[i:i + 1000], rd_t[i:i + 1000]) for i in range(0, 6000, 1000)]
    for k in range(3):
        assert torch.equal(whole[k], torch.cat([p[k] for p in parts]))
    check_rays(oracle, v, f, ro, rd, whole)
    cv = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float32)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    cf = np.array([t for a, b, c, d in quads for t in ((a, b, c), (a, c, d))], np.int64)
    o2, d2 = [], []
    for ax in range(3):
        u, w = (ax + 1) % 3, (ax + 2) % 3
        for side in (-1.0, 1.0):
            for x in np.linspace(-1.5, 1.5, 90):
                for dirn in ((0.0, 1.0), (0.6, 0.8), (-0.28, 0.96), (0.28, -0.96)):
                    o = np.zeros(3); o[ax] = side; o[u] = x; o[w] = -3.0 * np.sign(dirn[1])
                    d = np.zeros(3); d[u], d[w] = dirn
                    o2.append(o); d2.append(d)
    o2, d2 = np.array(o2, np.float32), np.array(d2, np.float32)
    assert len(o2) >= 2048
    out = cubvh.cuBVH(cv, cf).ray_trace(torch.from_numpy(o2).to(dev), torch.from_numpy(d2).to(dev))
    check_rays(oracle, cv, cf, o2, d2, out)


def check_sdf(got, sd_o, fid_o, what):
    d, fid, _ = (_np(x) if x is not None else None for x in got)
    assert np.array_equal(fid, fid_o), f"{what}: face ids differ at {(fid != fid_o).sum()} points"
    want = sd_o.astype(np.float32)
    bad = d != want
    assert not bad.any(), f"{what}: {bad.sum()} values differ, e.g. {d[bad][:5]} vs {want[bad][:5]}"
    assert np.array_equal(np.signbit(d), np.signbit(want))


def test_sdf_watertight(oracle, dev):
    v, f = W.displaced_icosphere(4, 1)
    bvh = cubvh.cuBVH(v, f)
    rng = np.random.default_rng(2)
    pts = np.concatenate([rng.uniform(-1, 1, (3000, 3)).astype(np.float32),
                          W.surface_points(v, f, 3000, 0.02, rng)])
    got = bvh.signed_distance(torch.from_numpy(pts).to(dev), return_uvw=True, mode="watertight")
    sd, fid, fl = oracle.sdf_watertight64(v, f, pts)
    check_sdf(got, sd, fid, "watertight")
    r = np.linalg.norm(pts, axis=1)
    inner = r < 0.5
    assert (_np(got[0])[inner] < 0).all()


@pytest.mark.parametrize("mesh", ["sphere", "tori"])
def test_sdf_raystab(oracle, dev, stab_dirs, mesh):
    if mesh == "sphere":
        v, f = W.displaced_icosphere(3, 1)
    else:
        v, f = W.random_tori(2, n_tori=2, n_major=32, n_minor=8)
    bvh = cubvh.cuBVH(v, f)
    rng = np.random.default_rng(4)
    pts = np.concatenate([rng.uniform(-1, 1, (1500, 3)).astype(np.float32),
                          W.surface_points(v, f, 1500, 0.02, rng)])
    got = bvh.signed_distance(torch.from_numpy(pts).to(dev), mode="raystab")
    sd, fid, fl = oracle.sdf_raystab64(v, f, pts, dirs=stab_dirs(len(pts)))
    check_sdf(got, sd, fid, "raystab")
    assert got[2] is None


def test_sdf_bad_mode(dev):
    v, f = W.icosphere(1)
    bvh = cubvh.cuBVH(v, f)
    with pytest.raises(KeyError):
        bvh.signed_distance(torch.zeros(4, 3, device=dev), mode="pathescape")


def test_state_dict_roundtrip(oracle, dev):
    v, f = W.displaced_icosphere(3, 1)
    bvh = cubvh.cuBVH(v, f)
    pts = torch.from_numpy(W.uniform_points(3000, 3)).to(dev)
    d0, f0, u0 = bvh.unsigned_distance(pts, return_uvw=True)
    sd = bvh.state_dict()
    bvh2 = cubvh.cuBVH.from_state_dict({k: val.clone() for k, val in sd.items()})
    d1, f1, u1 = bvh2.unsigned_distance(pts, return_uvw=True)
    assert torch.equal(d0, d1) and torch.equal(f0, f1) and torch.equal(u0, u1)


def test_load_reference_records(oracle, dev):
    # records in the reference's byte format (as its state_dict() writes them)
    v, f = W.displaced_icosphere(3, 1)
    nodes, tris = oracle.RefBVH(v, f).state_dict_arrays()
    bvh = cubvh.cuBVH.from_state_dict({"nodes": torch.from_numpy(nodes), "triangles": torch.from_numpy(tris)})
    pts = W.uniform_points(3000, 8)
    out = bvh.unsigned_distance(torch.from_numpy(pts).to(dev), return_uvw=True)
    check_udf(oracle, v, f, pts, out)


def test_reference_mirror_agreement(oracle, dev):
    """Our exact results next to the FP32 restatement of the reference: the
    distances agree to FP32 rounding and faces differ only at ties."""
    v, f = W.icosphere(4, 0.8)
    bvh = cubvh.cuBVH(v, f)
    pts = W.uniform_points(20000, 0)
    d, fid, _ = (_np(x) if x is not None else None for x in bvh.unsigned_distance(torch.from_numpy(pts).to(dev)))
    rd, rfid, _ = oracle.RefBVH(v, f).unsigned_distance(pts)
    assert np.abs(d.astype(np.float64) - rd).max() < 2e-7
    diff = fid != rfid
    if diff.any():
        a, _ = oracle.face_dist64(v, f, pts[diff], fid[diff])
        b, _ = oracle.face_dist64(v, f, pts[diff], rfid[diff])
        assert np.abs(a - b).max() <= 1e-7


def test_queries_in_cuda_graph(dev):
    """A device-resident query recorded in a CUDA graph (its scratch then
    comes from the graph's memory nodes) replays to the direct call's
    results; direct calls between synchronisations reuse the library pool."""
    v, f = W.displaced_icosphere(3, 1)
    bvh = cubvh.cuBVH(v, f)
    pts = torch.from_numpy(W.uniform_points(6000, 11)).to(dev)
    want = bvh.signed_distance(pts, mode="watertight")
    want_r = bvh.ray_trace(torch.zeros(500, 3, device=dev), torch.nn.functional.normalize(pts[:500], dim=1))
    torch.cuda.synchronize()
    s = torch.cuda.Stream(dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        got = bvh.signed_distance(pts, mode="watertight")
        got_r = bvh.ray_trace(torch.zeros(500, 3, device=dev), torch.nn.functional.normalize(pts[:500], dim=1))
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(got[0], want[0]) and torch.equal(got[1], want[1])
        assert all(torch.equal(a, b) for a, b in zip(got_r, want_r))
    for _ in range(3):   # synchronising callers: same results from the pool's scratch
        d, fid, _ = bvh.signed_distance(pts, mode="watertight")
        torch.cuda.synchronize()
        assert torch.equal(d, want[0]) and torch.equal(fid, want[1])


def test_non_finite_queries_leave_the_others_unchanged(dev):
    """NaN and infinite query points / rays in a batch: the calls succeed, and
    every finite query's result equals its result in the same batch with the
    bad entries replaced by finite ones (a packet's shared walk never lets one
    lane's values change another's; raystab stab rays follow the query index,
    which both batches share)."""
    v, f = W.displaced_icosphere(4, 1)
    bvh = cubvh.cuBVH(v, f)
    rng = np.random.default_rng(21)
    n = 4096
    good = rng.uniform(-1.2, 1.2, (n, 3)).astype(np.float32)
    bad_idx = rng.choice(n, 64, replace=False)
    bad = good.copy()
    vals = np.array([np.nan, np.inf, -np.inf, 1e30], np.float32)
    bad[bad_idx, rng.integers(0, 3, 64)] = vals[rng.integers(0, 4, 64)]
    keep = np.ones(n, bool)
    keep[bad_idx] = False
    P = lambda a: torch.from_numpy(a).to(dev)
    for mode in (None, "watertight", "raystab"):
        if mode is None:
            a, b = bvh.unsigned_distance(P(bad), return_uvw=True), bvh.unsigned_distance(P(good), return_uvw=True)
        else:
            a, b = bvh.signed_distance(P(bad), mode=mode), bvh.signed_distance(P(good), mode=mode)
        for x, y in zip(a, b):
            if x is None:
                continue
            assert torch.equal(x[torch.from_numpy(keep).to(dev)], y[torch.from_numpy(keep).to(dev)]), mode
    ro, rd = W.camera_rays(1, 64, 50.0, 2.5, 4)
    rbad = rd.copy()
    ridx = rng.choice(len(rd), 64, replace=False)
    rbad[ridx, rng.integers(0, 3, 64)] = vals[rng.integers(0, 4, 64)]
    rkeep = np.ones(len(rd), bool)
    rkeep[ridx] = False
    a = bvh.ray_trace(P(ro), P(rbad))
    b = bvh.ray_trace(P(ro), P(rd))
    for x, y in zip(a, b):
        m = torch.from_numpy(rkeep).to(dev)
        assert torch.equal(x[m], y[m])


def test_degenerate_triangles(oracle, dev, stab_dirs):
    """Zero-area faces (a segment, a point, a sphere edge, the segment again
    with its vertices reordered) added to a closed sphere, outside it and near
    it: every mode still equals the oracle bit for bit, including the queries
    whose closest face is a degenerate one, and no ray reports a hit on one."""
    v, f = W.icosphere(3, 0.8)
    nv, nf = len(v), len(f)
    extra = np.array([[0.2, 0.1, 0.85], [0.3, 0.1, 0.85], [0.4, 0.1, 0.85],
                      [-0.3, -0.2, 0.9]], np.float32)
    v = np.concatenate([v, extra]).astype(np.float32)
    f = np.concatenate([f, [[nv, nv + 1, nv + 2], [nv + 3, nv + 3, nv + 3],
                            [0, 0, 1], [nv, nv + 2, nv + 1]]]).astype(np.int64)
    rng = np.random.default_rng(31)
    pts = np.concatenate([rng.uniform(-1, 1, (3000, 3)),
                          np.repeat(extra, 100, 0) + rng.normal(0, 0.03, (400, 3)),
                          extra]).astype(np.float32)
    bvh = cubvh.cuBVH(v, f)
    P = torch.from_numpy(pts).to(dev)
    out = bvh.unsigned_distance(P, return_uvw=True)
    check_udf(oracle, v, f, pts, out)
    assert (_np(out[1]) >= nf).sum() > 100
    got = bvh.signed_distance(P, return_uvw=True, mode="watertight")
    sd, fid, _ = oracle.sdf_watertight64(v, f, pts)
    check_sdf(got, sd, fid, "watertight")
    got = bvh.signed_distance(P, mode="raystab")
    sd, fid, _ = oracle.sdf_raystab64(v, f, pts, dirs=stab_dirs(len(pts)))
    check_sdf(got, sd, fid, "raystab")
    ro = rng.normal(0, 2, (2000, 3)).astype(np.float32)
    tgt = np.concatenate([np.repeat(extra, 400, 0), rng.uniform(-0.5, 0.5, (400, 3))])
    rd = tgt + rng.normal(0, 0.01, tgt.shape) - ro
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    out = bvh.ray_trace(torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev))
    check_rays(oracle, v, f, ro, rd, out)
    assert not (_np(out[1]) >= nf).any()


def sliver_mesh(n, seed):
    """n disjoint slivers: needles with the small angle at a, caps with an
    angle near 180 degrees at a, and needles with the small angle at b; the
    sine of that angle is 1/g with g log-uniform in [1, 1e7]."""
    rng = np.random.default_rng(seed)
    g = 10 ** rng.uniform(0, 7, n)
    cen = rng.uniform(-0.8, 0.8, (n, 3))
    R = np.linalg.qr(rng.normal(size=(n, 3, 3)))[0]
    L = rng.uniform(0.02, 0.1, n)
    th, z, kind = 1.0 / g, 0 * L, rng.integers(0, 3, n)
    b0 = np.stack([L, z, z], 1)
    c = np.where(kind[:, None] == 0, np.stack([L * np.cos(th), L * np.sin(th), z], 1),
                 np.where(kind[:, None] == 1, np.stack([-L * np.cos(th), L * np.sin(th), z], 1),
                          np.stack([z, L * th, z], 1)))
    tri = np.stack([cen, cen + np.einsum("nij,nj->ni", R, b0), cen + np.einsum("nij,nj->ni", R, c)], 1)
    v = tri.reshape(-1, 3).astype(np.float32)
    f = np.arange(3 * n, dtype=np.int64).reshape(n, 3)
    t = v[f].astype(np.float64)
    w = rng.dirichlet([1, 1, 1], n)
    inside = np.einsum("nk,nkj->nj", w, t)
    nrm = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True) + 1e-300
    h = 10 ** rng.uniform(-4, 0, n) * rng.choice([-1, 1], n)
    lat = rng.normal(0, 1e-3, (n, 3)) * (rng.random(n) < 0.5)[:, None]
    pts = np.concatenate([inside + h[:, None] * nrm + lat, rng.uniform(-1, 1, (n, 3))]).astype(np.float32)
    return v, f, pts, rng


def test_sliver_triangles(oracle, dev, stab_dirs):
    """Slivers, whose float plane normal is inaccurate (up to g = 1e7 times
    the rounding of a well-shaped triangle), with points above their
    interiors at heights 1e-4 .. 1 and off to the side: UDF + uvw, both signs
    and rays equal the oracle bit for bit."""
    v, f, pts, rng = sliver_mesh(3000, 51)
    bvh = cubvh.cuBVH(v, f)
    P = torch.from_numpy(pts).to(dev)
    check_udf(oracle, v, f, pts, bvh.unsigned_distance(P, return_uvw=True))
    got = bvh.signed_distance(P, return_uvw=True, mode="watertight")
    sd, fid, _ = oracle.sdf_watertight64(v, f, pts)
    check_sdf(got, sd, fid, "watertight")
    got = bvh.signed_distance(P, mode="raystab")
    sd, fid, _ = oracle.sdf_raystab64(v, f, pts, dirs=stab_dirs(len(pts)))
    check_sdf(got, sd, fid, "raystab")
    ro = rng.uniform(-1.5, 1.5, (6000, 3)).astype(np.float32)
    rd = pts[rng.integers(0, 3000, 6000)] - ro
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    out = bvh.ray_trace(torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev))
    check_rays(oracle, v, f, ro, rd, out)
    assert (_np(out[1]) >= 0).mean() > 0.05


@pytest.mark.parametrize("scale,shift", [(1e-3, 0.0), (1e3, 0.0), (1.0, 3000.0), (0.05, -700.0)])
def test_scaled_and_translated_meshes(oracle, dev, stab_dirs, scale, shift):
    """A displaced sphere shrunk, enlarged and moved far from the origin
    (coordinates whose float spacing is up to 2.4e-4): node quantisation,
    the FP32 filters' error bounds (relative to |p - a|) and the fixed
    constants of the reference's semantics (1e-3 normal radius, 1000-unit
    stab rays) all meet the oracle bit for bit."""
    v, f = W.displaced_icosphere(3, 1)
    v = (v.astype(np.float64) * scale + np.array([shift, -0.5 * shift, 0.25 * shift])).astype(np.float32)
    rng = np.random.default_rng(61)
    lo, hi = v.min(0).astype(np.float64), v.max(0).astype(np.float64)
    c, h = (lo + hi) / 2, (hi - lo) / 2
    pts = np.concatenate([c + rng.uniform(-1.3, 1.3, (3000, 3)) * h,
                          W.surface_points(v, f, 2000, 0.02 * scale, rng)]).astype(np.float32)
    bvh = cubvh.cuBVH(v, f)
    P = torch.from_numpy(pts).to(dev)
    check_udf(oracle, v, f, pts, bvh.unsigned_distance(P, return_uvw=True))
    got = bvh.signed_distance(P, return_uvw=True, mode="watertight")
    sd, fid, _ = oracle.sdf_watertight64(v, f, pts)
    check_sdf(got, sd, fid, "watertight")
    got = bvh.signed_distance(P, mode="raystab")
    sd, fid, _ = oracle.sdf_raystab64(v, f, pts, dirs=stab_dirs(len(pts)))
    check_sdf(got, sd, fid, "raystab")
    ro = (c + rng.uniform(-2, 2, (4000, 3)) * h).astype(np.float32)
    rd = (c + rng.uniform(-0.5, 0.5, (4000, 3)) * h) - ro
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    out = bvh.ray_trace(torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev))
    check_rays(oracle, v, f, ro, rd, out)
    assert (_np(out[1]) >= 0).mean() > 0.2


def test_exact_ties_at_vertices_edges_and_centroids(oracle, dev, stab_dirs):
    """Queries exactly at the mesh vertices (distance 0 to every incident
    face), on shared edges, at face centroids, and rays aimed at vertices
    and edge points: every exact tie goes to the lowest face index, as in
    the oracle, and all outputs equal it bit for bit."""
    v, f = W.random_tori(2, n_tori=2, n_major=32, n_minor=10)
    v, f = np.asarray(v, np.float32), np.asarray(f, np.int64)
    rng = np.random.default_rng(77)
    e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
    mid = (0.5 * (v[e[:, 0]].astype(np.float64) + v[e[:, 1]])).astype(np.float32)
    cen = v[f].astype(np.float64).mean(1).astype(np.float32)
    used = v[np.unique(f)]                     # vertices of at least one face
    pts = np.concatenate([used, mid[rng.permutation(len(mid))[:3000]], cen[:2000]])
    bvh = cubvh.cuBVH(v, f)
    P = torch.from_numpy(pts).to(dev)
    out = bvh.unsigned_distance(P, return_uvw=True)
    check_udf(oracle, v, f, pts, out)
    d = _np(out[0])
    assert (d[:len(used)] == 0).all()
    _, _, _, _, nn = oracle.udf64(v, f, pts)
    assert (nn[:len(used)] >= 2).mean() > 0.9  # vertices: ties among the incident faces
    got = bvh.signed_distance(P, return_uvw=True, mode="watertight")
    sd, fid, _ = oracle.sdf_watertight64(v, f, pts)
    check_sdf(got, sd, fid, "watertight")
    got = bvh.signed_distance(P, mode="raystab")
    sd, fid, _ = oracle.sdf_raystab64(v, f, pts, dirs=stab_dirs(len(pts)))
    check_sdf(got, sd, fid, "raystab")
    tgt = np.concatenate([used[rng.integers(0, len(used), 3000)], mid[rng.integers(0, len(mid), 3000)]]).astype(np.float64)
    ro = rng.uniform(-2, 2, (6000, 3))
    rd = tgt - ro
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    ro = ro.astype(np.float32)
    out = bvh.ray_trace(torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev))
    fl = check_rays(oracle, v, f, ro, rd, out)
    assert (_np(out[1]) >= 0).mean() > 0.8 and (fl & 2).sum() > 10   # with exact ties in t


def test_ray_trace_window_order(oracle, dev):
    """Rays are traced in packets of nearby rays (a sort of each 8,192-ray
    window by box entry point), incoherent packets ray by ray: camera rays, rays
    from inside, rays that miss the box, axis-parallel and non-finite rays,
    and a last window that is only partly filled.  Results equal the oracle's
    and those of the same rays traced in calls of 30,000 (other windows,
    packets and packet kinds)."""
    v, f = W.displaced_icosphere(4, 1)
    bvh = cubvh.cuBVH(v, f)
    ro_c, rd_c = W.camera_rays(4, 128, 50.0, 2.5, 7)
    rng = np.random.default_rng(81)
    m = 20000 + 123
    ro_r = rng.uniform(-1.5, 1.5, (m, 3)).astype(np.float32)
    rd_r = rng.standard_normal((m, 3)).astype(np.float32)
    rd_r[:500, 0] = 0.0
    rd_r[500:600, 1:] = 0.0
    rd_r /= np.linalg.norm(rd_r, axis=1, keepdims=True)
    ro_r[600:700] += np.float32(10.0)           # far outside, pointing anywhere: mostly misses
    ro = np.concatenate([ro_c, ro_r]).astype(np.float32)
    rd = np.concatenate([rd_c, rd_r]).astype(np.float32)
    n = len(ro)
    assert n > 8192 and n % 8192 != 0
    ro_t, rd_t = torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev)
    whole = bvh.ray_trace(ro_t, rd_t)
    parts = [bvh.ray_trace(ro_t[i:i + 30000], rd_t[i:i + 30000]) for i in range(0, n, 30000)]
    for k in range(3):
        assert torch.equal(whole[k], torch.cat([p[k] for p in parts]))
    check_rays(oracle, v, f, ro, rd, whole)
    hit = _np(whole[1]) >= 0
    assert 0.2 < hit.mean() < 0.9
    bad = rd.copy()
    bad[rng.choice(n, 64, replace=False), 0] = np.nan
    bad[rng.choice(n, 64, replace=False), 2] = np.inf
    keep = np.isfinite(bad).all(1)
    got = bvh.ray_trace(ro_t, torch.from_numpy(bad).to(dev))
    m_t = torch.from_numpy(keep).to(dev)
    for x, y in zip(got, whole):
        assert torch.equal(x[m_t], y[m_t])


def test_ray_trace_axis_parallel_grid(oracle, dev):
    """A 256 x 256 grid of rays along +z and along -x (the rays of a
    voxeliser or a parity test: zero direction components, one direction
    for all), traced in packets: results equal the oracle's."""
    v, f = W.displaced_icosphere(4, 1)
    bvh = cubvh.cuBVH(v, f)
    g = np.linspace(-1.1, 1.1, 256)
    x, y = np.meshgrid(g, g, indexing="ij")
    ro_z = np.stack([x.ravel(), y.ravel(), np.full(x.size, -2.0)], 1)
    ro_x = np.stack([np.full(x.size, 2.0), x.ravel(), y.ravel()], 1)
    ro = np.concatenate([ro_z, ro_x]).astype(np.float32)
    rd = np.concatenate([np.tile([0.0, 0.0, 1.0], (x.size, 1)), np.tile([-1.0, 0.0, 0.0], (x.size, 1))]).astype(np.float32)
    out = bvh.ray_trace(torch.from_numpy(ro).to(dev), torch.from_numpy(rd).to(dev))
    check_rays(oracle, v, f, ro, rd, out)
    assert 0.2 < (_np(out[1]) >= 0).mean() < 0.9
