"""Pins of the CPU oracle (no GPU): published PCG32 known answers, analytic
distances / hits / signs on simple solids, floodfill against an independent
breadth-first search, and the FP32 mirror of the reference against FP64."""

from collections import deque

import numpy as np
import pytest

from cubvh_b200 import workloads as W


def cube_mesh(h=1.0):
    v = np.array([[x, y, z] for x in (-h, h) for y in (-h, h) for z in (-h, h)], np.float32)
    # two triangles per face, outward winding
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    f = []
    for a, b, c, d in quads:
        f += [(a, b, c), (a, c, d)]
    return v, np.array(f, np.int64)


def cube_truth(p, h=1.0):
    """Exact distance to the surface of [-h, h]^3 and the closest point."""
    p = np.asarray(p, np.float64)
    out = np.abs(p) > h
    if out.any(axis=-1).item() if p.ndim == 1 else False:
        pass
    q = np.clip(p, -h, h)
    d_out = np.linalg.norm(p - q)
    if d_out > 0:
        return d_out, q
    # inside: nearest face
    k = np.argmax(np.abs(p))
    q = p.copy()
    q[k] = np.sign(p[k]) * h if p[k] != 0 else h
    return h - abs(p[k]), q


def test_pcg32_known_answer(oracle):
    # pcg32_srandom(42, 54): first six outputs of the published PCG32 demo
    want = [0xa15c02b7, 0x7b47f409, 0xba1d3330, 0x83d2f293, 0xbfa4784b, 0xcbed606e]
    assert list(oracle.pcg32_seq(42, 54, 6)) == want


def test_stab_directions(oracle):
    d = oracle.stab_dirs(64, 0)
    assert d.shape == (64, 32, 3)
    n = np.linalg.norm(d.astype(np.float64), axis=-1)
    assert np.abs(n - 1).max() < 1e-6
    # the Fibonacci lattice: cos(theta) = 1 - 2 * frac((k + 1.33) / 33.66 + offset.x)
    off = oracle.stab_offsets(64)
    k = np.arange(32, dtype=np.float32)
    a = (k + np.float32(1.33)) / (np.float32(31) + np.float32(2) * np.float32(1.33)) + off[:, :1]
    a = a - np.floor(a)
    assert np.array_equal(d[..., 2], np.float32(-2) * a + np.float32(1))
    # a direction table given to the raystab oracle replaces the host rule
    v, f = cube_mesh()
    pts = np.array([[0.1, 0.2, 0.3], [3.0, 0.0, 0.0]], np.float32)
    s0, _, _ = oracle.sdf_raystab64(v, f, pts)
    s1, _, _ = oracle.sdf_raystab64(v, f, pts, dirs=oracle.stab_dirs(2, 0))
    assert np.array_equal(s0, s1) and s0[0] < 0 < s0[1]
    # per-query offsets differ (jump-ahead by 2 per query)
    assert len(np.unique(off[:4, 0])) == 4


def test_udf64_cube_analytic(oracle):
    v, f = cube_mesh()
    rng = np.random.default_rng(7)
    pts = np.concatenate([rng.uniform(-3, 3, (300, 3)), rng.uniform(-0.99, 0.99, (100, 3)),
                          [[2, 0, 0], [2, 2, 0], [2, 2, 2], [0.5, 0, 0], [0, 0, 0.25]]]).astype(np.float32)
    dist, fid, uvw, cp, nn = oracle.udf64(v, f, pts)
    for i, p in enumerate(pts):
        dt, qt = cube_truth(p)
        assert abs(dist[i] - dt) <= 1e-12 * max(1.0, dt), (p, dist[i], dt)
        # closest point rebuilt from uvw on the returned face
        tri = v[f[fid[i]]].astype(np.float64)
        q = uvw[i] @ tri
        assert np.abs(q - cp[i]).max() < 1e-12
        assert abs(np.linalg.norm(p.astype(np.float64) - q) - dt) < 1e-12
        assert abs(uvw[i].sum() - 1) < 1e-12 and (uvw[i] >= -1e-15).all()
    assert dist[-5] == 1.0 and dist[-2] == 0.5
    assert abs(dist[-4] - np.sqrt(2)) < 1e-15 and abs(dist[-3] - np.sqrt(3)) < 1e-15


def test_udf64_max_dist_rule(oracle):
    v, f = cube_mesh()
    pts = np.array([[5000, 0, 0], [0, 0, 999.5]], np.float32)
    dist, fid, uvw, _, _ = oracle.udf64(v, f, pts)
    assert dist[0] == 0.0 and fid[0] == 0          # beyond 1000: distance 0, face 0
    assert abs(dist[1] - 998.5) < 1e-9


def test_ray64_cube_analytic(oracle):
    v, f = cube_mesh()
    ro = np.array([[0.1, 0.2, 5], [3, 3, 3], [0.3, -0.2, 0.1], [5, 0.5, 0.5], [0, 0, 5]], np.float32)
    rd = np.array([[0, 0, -1], [1, 0, 0], [0, 0, 1], [-1, 0, 0], [0, 0, 1]], np.float32)
    t, fid, fl = oracle.ray64(v, f, ro, rd)
    assert t[0] == 4.0 and fid[0] >= 0
    assert t[1] == 1000.0 and fid[1] == -1
    assert abs(t[2] - 0.9) < 1e-7 and fid[2] >= 0          # from inside, exits through z = +1
    assert t[3] == 4.0
    assert t[4] == 1000.0 and fid[4] == -1                  # pointing away


def test_tetrahedron_distance(oracle):
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    f = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]] * 3, np.int64)  # > 8 faces
    pts = np.array([[1, 1, 1], [-1, -1, -1], [0.1, 0.1, 0.1], [2, 0, 0], [0.5, 0.5, -1]], np.float32)
    dist, _, _, _, _ = oracle.udf64(v, f, pts)
    # (1,1,1): plane x+y+z=1; (-1,-1,-1): vertex 0; (t,t,t) inside: the
    # coordinate planes at distance t (t = float32(0.1)); (2,0,0): vertex 1;
    # (.5,.5,-1): the z = 0 face
    want = [2 / np.sqrt(3), np.sqrt(3), float(np.float32(0.1)), 1.0, 1.0]
    assert np.allclose(dist, want, atol=1e-12, rtol=0)


def test_sign_rules_on_cube(oracle):
    v, f = cube_mesh()
    rng = np.random.default_rng(3)
    inside = rng.uniform(-0.9, 0.9, (200, 3)).astype(np.float32)
    outside = (rng.uniform(1.1, 2.0, (200, 3)) * rng.choice([-1, 1], (200, 3))).astype(np.float32)
    pts = np.concatenate([inside, outside])
    sw, _, flw = oracle.sdf_watertight64(v, f, pts)
    assert (sw[:200] < 0).all() and (sw[200:] > 0).all()
    sr, _, flr = oracle.sdf_raystab64(v, f, pts)
    assert (sr[:200] < 0).all() and (sr[200:] > 0).all()
    ud, _, _, _, _ = oracle.udf64(v, f, pts)
    assert np.array_equal(np.abs(sw), ud) and np.array_equal(np.abs(sr), ud)


def test_raystab_open_box_is_outside(oracle):
    v, f = cube_mesh()
    keep = np.ones(len(f), bool)
    keep[2:4] = False          # remove the x = +1 face: rays escape through it
    pts = np.array([[0, 0, 0], [0.5, 0.2, -0.1]], np.float32)
    f2 = np.concatenate([f[keep], f[keep][:2]])   # keep > 8 faces
    sr, _, _ = oracle.sdf_raystab64(v, f2, pts)
    assert (sr > 0).all()


def bfs_labels(grid):
    """Independent floodfill: BFS in the reference's [D][H][W] reading."""
    B, H, W, D = grid.shape
    lab = np.full(grid.shape, -1, np.int64)
    flat = grid.reshape(B, -1)
    out = lab.reshape(B, -1)
    nvol = H * W * D
    for b in range(B):
        seen = np.zeros(nvol, bool)
        for s in range(nvol):
            if flat[b, s] or seen[s]:
                continue
            comp = [s]
            seen[s] = True
            q = deque([s])
            while q:
                l = q.popleft()
                x, y, z = l % W, (l // W) % H, l // (W * H)
                for ok, n in ((x > 0, l - 1), (x < W - 1, l + 1), (y > 0, l - W), (y < H - 1, l + W),
                              (z > 0, l - W * H), (z < D - 1, l + W * H)):
                    if ok and not flat[b, n] and not seen[n]:
                        seen[n] = True
                        comp.append(n)
                        q.append(n)
            m = min(comp)
            out[b, comp] = b * nvol + m
    return lab.astype(np.int32)


@pytest.mark.parametrize("shape,p", [((1, 6, 6, 6), 0.4), ((2, 5, 7, 3), 0.35), ((1, 9, 4, 11), 0.5),
                                     ((3, 4, 4, 4), 0.2), ((1, 1, 1, 40), 0.3)])
def test_floodfill_oracle_vs_bfs(oracle, shape, p):
    rng = np.random.default_rng(sum(shape))
    g = rng.random(shape) < p
    assert np.array_equal(oracle.floodfill(g), bfs_labels(g))


def test_floodfill_known_answers(oracle):
    g = np.zeros((3, 3, 3), bool)
    assert (oracle.floodfill(g) == 0).all()
    g[1, 1, 1] = True
    lab = oracle.floodfill(g)
    assert lab[1, 1, 1] == -1 and (lab[g == 0] == 0).all()
    # a wall splits the volume: z = l // (W*H) plane index 1 occupied
    g = np.zeros((4, 4, 4), bool)
    g.reshape(-1)[16:32] = True
    lab = oracle.floodfill(g).reshape(-1)
    assert (lab[:16] == 0).all() and (lab[16:32] == -1).all() and (lab[32:] == 32).all()


def test_ref32_mirror_tracks_fp64(oracle):
    v, f = W.icosphere(4, 0.8)
    ref = oracle.RefBVH(v, f)
    assert ref.n_nodes == 1365                    # BVH4, leaf <= 8 on 5120 faces
    pts = W.uniform_points(2000, 0)
    d32, fid32, uvw32 = ref.unsigned_distance(pts, return_uvw=True)
    d64, _, _, _, _ = oracle.udf64(v, f, pts)
    assert np.abs(d32 - d64).max() < 2e-7
    # the mirror's face is always a (near-)minimiser
    df, _ = oracle.face_dist64(v, f, pts, fid32)
    assert (df - d64).max() < 2e-7
    nodes, tris = ref.state_dict_arrays()
    assert nodes.shape == (1365, 9) and tris.shape == (5120, 12)


def test_udf_to_sdf_known_answer():
    """Hollow box: a 6^3 shell of occupied voxels (udf 0) around a 4^3
    cavity (udf 1) inside an 10^3 grid whose outside voxels have udf 1: the
    cavity is cut off from voxel (0,0,0), so it is inside and negative."""
    from oracle import oracle as O
    u = np.ones((10, 10, 10), np.float32)
    u[2:8, 2:8, 2:8] = 0.0
    u[3:7, 3:7, 3:7] = 1.0
    eps = np.float32(0.25)
    s = O.udf_to_sdf(u, eps)
    assert s[0, 0, 0] == np.float32(0.75) and s[9, 9, 9] == np.float32(0.75)
    assert (s[3:7, 3:7, 3:7] == np.float32(-0.75)).all()
    assert (s[2, 2:8, 2:8] == np.float32(-0.25)).all()      # shell: udf - eps < 0 stays as is
    # voxel (0,0,0) occupied: its label is -1, so every occupied voxel is "outside"
    u2 = u.copy(); u2[0, 0, 0] = 0.0
    s2 = O.udf_to_sdf(u2, eps)
    assert (s2[3:7, 3:7, 3:7] == np.float32(-0.75)).all() and s2[9, 9, 9] == np.float32(-0.75)
