"""Seeded synthetic meshes and queries for the cubvh query workloads.

No dataset is involved: every mesh and query set is generated here from a
numpy ``default_rng`` seed.  The shapes follow the five workloads this
package is measured on:

* ``udf_icosphere``   - icosphere level 4 (2562 v / 5120 f), radius 0.8;
  1,048,576 points uniform in [-1, 1]^3 (seed 0); unsigned distance with uvw.
* ``rays_displaced``  - displaced icosphere level 6 (40962 v / 81920 f, seed 1);
  8 pinhole cameras 2048x2048, fov 50 deg, on a sphere of radius 2.5 looking at
  the origin (33,554,432 rays) and 8,388,608 signed-distance points (half
  uniform in [-1, 1]^3, half within +-0.02 of the surface).
* ``dense_tori``      - 12 random tori (seed 2), 10% of faces removed in
  contiguous patches; unsigned distance on the 512^3 linspace(-1, 1) grid and
  floodfill of ``udf < 2/512``.
* ``grad_displaced``  - the displaced icosphere with 4,194,304 points (half
  uniform, half within +-0.05 of the surface) and weights U(0, 1) (seed 3).
* ``batch_256``       - 256 meshes (seed 4): displaced icospheres of levels 2-7
  or tori, face counts log-uniform in 320..~330k, each with log-uniform
  10k..2M points in its bounding box dilated by 10%.

"256x64 tessellation" for a torus is read as 256 * 64 = 16,384 triangles
(256 segments around the ring x 32 around the tube, two triangles per quad),
which is what gives the ~180k-face total of the dense-grid workload.
"""

from __future__ import annotations

import functools
import math

import numpy as np

__all__ = [
    "icosphere", "displaced_icosphere", "torus", "random_tori", "dodecahedron",
    "uniform_points", "surface_points", "camera_rays", "dense_grid",
    "udf_icosphere", "rays_displaced", "dense_tori", "grad_displaced", "batch_256",
]


# --------------------------------------------------------------------------
# meshes
# --------------------------------------------------------------------------
def icosphere(level: int, radius: float = 1.0):
    """Subdivided icosahedron: 10*4^level + 2 vertices, 20*4^level faces."""
    v, f = _unit_icosphere(level)
    return (v * radius).astype(np.float32), f.copy()


@functools.lru_cache(maxsize=None)
def _unit_icosphere(level: int):
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([
        [-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
        [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
        [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([
        [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
        [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
        [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
        [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
        e.sort(axis=1)
        key = e[:, 0] * (len(v) + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // (len(v) + 1)
        b = uniq % (len(v) + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1).T + len(v)   # midpoints of edges (01, 12, 20)
        v = np.concatenate([v, mid], axis=0)
        f0, f1, f2 = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([
            np.stack([f0, m01, m20], 1), np.stack([f1, m12, m01], 1),
            np.stack([f2, m20, m12], 1), np.stack([m01, m12, m20], 1)], axis=0)
    v.setflags(write=False)
    f = f.astype(np.int64)
    f.setflags(write=False)
    return v, f


def displaced_icosphere(level: int, seed: int, radius: float = 0.7, amp: float = 0.08,
                        noise: float = 0.02):
    """radius * (1 + amp*sin(5x)sin(4y)sin(3z) + noise*N(0,1)) along each unit direction."""
    v, f = icosphere(level, 1.0)
    v = v.astype(np.float64)
    rng = np.random.default_rng(seed)
    s = 1.0 + amp * np.sin(5 * v[:, 0]) * np.sin(4 * v[:, 1]) * np.sin(3 * v[:, 2]) \
        + noise * rng.standard_normal(len(v))
    return (v * (radius * s)[:, None]).astype(np.float32), f


def torus(R: float, r: float, n_major: int, n_minor: int):
    """Closed torus in the xy-plane, two triangles per (major, minor) quad."""
    u = np.arange(n_major) * (2 * np.pi / n_major)
    w = np.arange(n_minor) * (2 * np.pi / n_minor)
    uu, ww = np.meshgrid(u, w, indexing="ij")
    x = (R + r * np.cos(ww)) * np.cos(uu)
    y = (R + r * np.cos(ww)) * np.sin(uu)
    z = r * np.sin(ww)
    v = np.stack([x, y, z], -1).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(n_major), np.arange(n_minor), indexing="ij")
    i1, j1 = (i + 1) % n_major, (j + 1) % n_minor
    a, b = i * n_minor + j, i1 * n_minor + j
    c, d = i1 * n_minor + j1, i * n_minor + j1
    f = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3),
                        np.stack([a, c, d], -1).reshape(-1, 3)], 0)
    return v.astype(np.float64), f.astype(np.int64)


def _random_rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def random_tori(seed: int = 2, n_tori: int = 12, n_major: int = 256, n_minor: int = 32,
                delete_frac: float = 0.10):
    """n_tori random tori (R~U(.15,.4), r~U(.03,.1), random rotation, centre in
    [-.5,.5]^3) with ``delete_frac`` of all faces removed in contiguous
    rectangular patches of the (major, minor) parameter grid."""
    rng = np.random.default_rng(seed)
    vs, fs, off = [], [], 0
    per = 2 * n_major * n_minor
    keep_all = []
    for _ in range(n_tori):
        R = rng.uniform(0.15, 0.4)
        r = rng.uniform(0.03, 0.1)
        v, f = torus(R, r, n_major, n_minor)
        v = v @ _random_rotation(rng).T + rng.uniform(-0.5, 0.5, 3)
        keep = np.ones(per, dtype=bool)
        quad = np.ones((n_major, n_minor), dtype=bool)
        target = int(round(delete_frac * per))
        while (~keep).sum() < target:
            i0, j0 = rng.integers(n_major), rng.integers(n_minor)
            h, w = rng.integers(4, 24), rng.integers(3, 12)
            ii = (i0 + np.arange(h)) % n_major
            jj = (j0 + np.arange(w)) % n_minor
            quad[np.ix_(ii, jj)] = False
            keep = np.concatenate([quad.reshape(-1), quad.reshape(-1)])
        vs.append(v)
        fs.append(f + off)
        keep_all.append(keep)
        off += len(v)
    v = np.concatenate(vs, 0).astype(np.float32)
    f = np.concatenate(fs, 0)[np.concatenate(keep_all)]
    return v, f


def dodecahedron(radius: float = 1.0):
    """A regular dodecahedron inscribed in a sphere of ``radius`` (20 vertices,
    36 faces: each pentagon fanned into 3 triangles), the same solid the
    reference's test scripts query.  Built as the dual of the icosahedron:
    vertices are the normalised centroids of the 20 icosahedron faces, and the
    5 faces around each icosahedron vertex form one pentagon."""
    iv, ifc = icosphere(0, 1.0)
    iv = iv.astype(np.float64)
    v = iv[ifc].mean(1)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    faces = []
    for i in range(len(iv)):
        ring = np.nonzero((ifc == i).any(1))[0]
        n = iv[i]
        c = v[ring].mean(0)
        e1 = v[ring[0]] - c
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(n, e1)
        ang = np.arctan2((v[ring] - c) @ e2, (v[ring] - c) @ e1)
        ring = ring[np.argsort(ang)]
        for k in range(1, 4):
            faces.append([ring[0], ring[k], ring[k + 1]])
    return (v * radius).astype(np.float32), np.array(faces, dtype=np.int64)


# --------------------------------------------------------------------------
# queries
# --------------------------------------------------------------------------
def uniform_points(n: int, seed: int, lo=-1.0, hi=1.0):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, (n, 3)).astype(np.float32)


def surface_points(v, f, n: int, band: float, rng):
    """Random points on random faces (area-weighted), offset along the face
    normal by U(-band, band)."""
    v = v.astype(np.float64)
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    nrm = np.cross(b - a, c - a)
    area = np.linalg.norm(nrm, axis=1)
    face = rng.choice(len(f), size=n, p=area / area.sum())
    r1, r2 = rng.random(n), rng.random(n)
    s = np.sqrt(r1)
    w0, w1, w2 = 1 - s, s * (1 - r2), s * r2
    p = w0[:, None] * a[face] + w1[:, None] * b[face] + w2[:, None] * c[face]
    un = nrm[face] / area[face, None]
    return (p + un * rng.uniform(-band, band, (n, 1))).astype(np.float32)


def camera_rays(n_poses: int, res: int, fov_deg: float, radius: float, seed: int):
    """Pinhole cameras on a sphere looking at the origin.  Returns float32
    origins and unit directions, each [n_poses*res*res, 3]."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((n_poses, 3))
    c /= np.linalg.norm(c, axis=1, keepdims=True)
    c *= radius
    focal = (res / 2) / math.tan(math.radians(fov_deg) / 2)
    j, i = np.meshgrid(np.arange(res, dtype=np.float64), np.arange(res, dtype=np.float64),
                       indexing="xy")
    dx = (j + 0.5 - res / 2) / focal
    dy = -(i + 0.5 - res / 2) / focal
    cam_dirs = np.stack([dx, dy, -np.ones_like(dx)], -1).reshape(-1, 3)
    os_, ds = [], []
    for k in range(n_poses):
        fwd = -c[k] / np.linalg.norm(c[k])
        up = np.array([0.0, 1.0, 0.0]) if abs(fwd[1]) < 0.99 else np.array([1.0, 0.0, 0.0])
        right = np.cross(fwd, up)
        right /= np.linalg.norm(right)
        up2 = np.cross(right, fwd)
        rot = np.stack([right, up2, -fwd], 1)      # camera -> world columns
        d = cam_dirs @ rot.T
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        ds.append(d.astype(np.float32))
        os_.append(np.broadcast_to(c[k].astype(np.float32), d.shape))
    return np.ascontiguousarray(np.concatenate(os_, 0)), np.concatenate(ds, 0)


def dense_grid(res: int):
    """[res^3, 3] float32 points of linspace(-1, 1) with meshgrid indexing 'ij'."""
    x = np.linspace(-1, 1, res, dtype=np.float32)
    g = np.stack(np.meshgrid(x, x, x, indexing="ij"), -1)
    return g.reshape(-1, 3)


# --------------------------------------------------------------------------
# named workloads (full sizes; ``scale`` shrinks query counts for tests)
# --------------------------------------------------------------------------
def udf_icosphere(n_points: int = 1 << 20):
    v, f = icosphere(4, 0.8)
    return dict(vertices=v, faces=f, points=uniform_points(n_points, 0))


def rays_displaced(res: int = 2048, n_poses: int = 8, n_sdf: int = 8 << 20):
    v, f = displaced_icosphere(6, 1)
    ro, rd = camera_rays(n_poses, res, 50.0, 2.5, 1)
    rng = np.random.default_rng(1)
    half = n_sdf // 2
    pts = np.concatenate([rng.uniform(-1, 1, (half, 3)).astype(np.float32),
                          surface_points(v, f, n_sdf - half, 0.02, rng)], 0)
    return dict(vertices=v, faces=f, rays_o=ro, rays_d=rd, points=pts)


def incoherent_rays(n: int, seed: int = 5):
    """n float32 rays without coherence between neighbours: the first half
    start uniformly in [-1, 1]^3 with uniformly random unit directions, the
    second half start on the sphere of radius 3 and point at uniform random
    points of [-0.8, 0.8]^3."""
    rng = np.random.default_rng(seed)
    h = n // 2
    o1 = rng.uniform(-1, 1, (h, 3))
    d1 = rng.standard_normal((h, 3))
    s = rng.standard_normal((n - h, 3))
    o2 = 3 * s / np.linalg.norm(s, axis=1, keepdims=True)
    d2 = rng.uniform(-0.8, 0.8, (n - h, 3)) - o2
    o = np.concatenate([o1, o2]).astype(np.float32)
    d = np.concatenate([d1, d2])
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return o, d


def dense_tori(res: int = 512):
    v, f = random_tori(2)
    return dict(vertices=v, faces=f, grid_res=res)


def grad_displaced(n_points: int = 4 << 20):
    v, f = displaced_icosphere(6, 1)
    rng = np.random.default_rng(3)
    half = n_points // 2
    pts = np.concatenate([rng.uniform(-1, 1, (half, 3)).astype(np.float32),
                          surface_points(v, f, n_points - half, 0.05, rng)], 0)
    w = rng.random(n_points).astype(np.float32)
    return dict(vertices=v, faces=f, points=pts, weights=w)


def batch_256(n_meshes: int = 256, min_q: int = 10_000, max_q: int = 2_000_000,
              seed: int = 4):
    """List of dicts (vertices, faces, points) for the batched workload."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n_meshes):
        target = math.exp(rng.uniform(math.log(320), math.log(330_000)))
        if rng.random() < 0.5:
            level = int(np.clip(round(math.log(target / 20, 4)), 2, 7))
            v, f = displaced_icosphere(level, seed * 1000 + m)
        else:
            k = int(np.clip(round(math.sqrt(target / 8)), 8, 128))
            R, r = rng.uniform(0.3, 0.6), rng.uniform(0.08, 0.25)
            v, f = torus(R, r, 4 * k, k)
            v = (v @ _random_rotation(rng).T).astype(np.float32)
        nq = int(math.exp(rng.uniform(math.log(min_q), math.log(max_q))))
        lo, hi = v.min(0), v.max(0)
        ctr, half = (lo + hi) / 2, (hi - lo) / 2 * 1.1
        pts = (ctr + rng.uniform(-1, 1, (nq, 3)) * half).astype(np.float32)
        out.append(dict(vertices=np.ascontiguousarray(v, dtype=np.float32), faces=f, points=pts))
    return out
