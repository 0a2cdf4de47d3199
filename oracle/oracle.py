"""ctypes front end of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke(), the
CPU-baseline leg and the reference arm of bench.py, never by the cubvh_b200
package.  See the header
of oracle.cpp for what is restated from which reference file, and for the
pinning status (floodfill and the sparse-marching-cubes vertices: pinned to
the reference's own CUDA code, compiled into oracle/_ref; distance, ray and
sign queries: unpinned against the reference's outputs, whose BVH code
cannot be built in this image).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liborc.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile liborc.so with the committed Makefile (g++, OpenMP)."""
    if force or not os.path.exists(_LIB_PATH) or \
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "oracle.cpp")):
        subprocess.run(["make", "-s", "-C", _HERE, "liborc.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_ref_build.restype = ctypes.c_void_p
        _lib.orc_ref_num_nodes.restype = ctypes.c_int64
        _lib.orc_get_threads.restype = ctypes.c_int
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


I64 = ctypes.c_int64
F64 = ctypes.c_double


def set_threads(n: int):
    lib().orc_set_threads(ctypes.c_int(n))


def threads() -> int:
    return int(lib().orc_get_threads())


# ---------------------------------------------------------------- FP64 oracle
def udf64(V, F, pts, tie_eps=1e-7):
    """-> dist, fid (lowest index among exact minima), uvw, cp, n_near."""
    V, F, pts = _f32(V), _i64(F), _f32(pts)
    n = len(pts)
    dist = np.empty(n, np.float64); fid = np.empty(n, np.int64)
    uvw = np.empty((n, 3), np.float64); cp = np.empty((n, 3), np.float64)
    nn = np.empty(n, np.int32)
    lib().orc_udf64(_p(V), I64(len(V)), _p(F), I64(len(F)), _p(pts), I64(n), F64(tie_eps),
                    _p(dist), _p(fid), _p(uvw), _p(cp), _p(nn))
    return dist, fid, uvw, cp, nn


def face_dist64(V, F, pts, fids):
    V, F, pts, fids = _f32(V), _i64(F), _f32(pts), _i64(fids)
    n = len(pts)
    dist = np.empty(n, np.float64); uvw = np.empty((n, 3), np.float64)
    lib().orc_face_dist64(_p(V), _p(F), _p(pts), _p(fids), I64(n), _p(dist), _p(uvw))
    return dist, uvw


def tri_dist64d(tri, pts):
    """Distance from double points [n, 3] to double triangles [n, 3, 3]."""
    tri = np.ascontiguousarray(tri, dtype=np.float64).reshape(-1, 9)
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    n = len(pts)
    d = np.empty(n, np.float64); b = np.empty((n, 3), np.float64)
    lib().orc_tri_dist64d(_p(tri), _p(pts), I64(n), _p(d), _p(b))
    return d, b


def ray64(V, F, ro, rd, tmax=1000.0, eps_b=1e-9, eps_g=1e-9, tie_eps=1e-7):
    """-> t (tmax on miss), fid (-1 on miss), flags (bit0 ambiguous, bit1 tie)."""
    V, F, ro, rd = _f32(V), _i64(F), _f32(ro), _f32(rd)
    n = len(ro)
    t = np.empty(n, np.float64); fid = np.empty(n, np.int64); fl = np.empty(n, np.int32)
    lib().orc_ray64(_p(V), _p(F), I64(len(F)), _p(ro), _p(rd), I64(n), F64(tmax), F64(eps_b),
                    F64(eps_g), F64(tie_eps), _p(t), _p(fid), _p(fl))
    return t, fid, fl


def sdf_watertight64(V, F, pts):
    V, F, pts = _f32(V), _i64(F), _f32(pts)
    n = len(pts)
    sd = np.empty(n, np.float64); fid = np.empty(n, np.int64); fl = np.empty(n, np.int32)
    lib().orc_sdf_watertight64(_p(V), _p(F), I64(len(F)), _p(pts), I64(n), _p(sd), _p(fid), _p(fl))
    return sd, fid, fl


def sdf_raystab64(V, F, pts, i0=0, eps_b=1e-9, eps_g=1e-9, dirs=None):
    """Raystab signed distance in double.  dirs: float32 [n, 32, 3] stab
    directions of the n points (e.g. the reference's CUDA directions from
    ref_stab_dirs_gpu_ptr), or None for the host rule (stab_dirs)."""
    V, F, pts = _f32(V), _i64(F), _f32(pts)
    n = len(pts)
    if dirs is not None:
        dirs = _f32(dirs)
        if dirs.shape != (n, 32, 3):
            raise ValueError("dirs must be [n, 32, 3]")
    sd = np.empty(n, np.float64); fid = np.empty(n, np.int64); fl = np.empty(n, np.int32)
    lib().orc_sdf_raystab64(_p(V), _p(F), I64(len(F)), _p(pts), I64(n), I64(i0), F64(eps_b),
                            F64(eps_g), _p(dirs), _p(sd), _p(fid), _p(fl))
    return sd, fid, fl


def pcg32_seq(initstate, initseq, n):
    out = np.empty(n, np.uint32)
    lib().orc_pcg32_seq(ctypes.c_uint64(initstate), ctypes.c_uint64(initseq), ctypes.c_int(n), _p(out))
    return out


def stab_offsets(n, i0=0):
    out = np.empty((n, 2), np.float32)
    lib().orc_stab_offsets(I64(n), I64(i0), _p(out))
    return out


def stab_dirs(n, i0=0):
    """Stab directions [n, 32, 3] of points i0 .. i0+n-1 with the host's
    sin / cos (the reference's host build gives the same bits)."""
    out = np.empty((n, 32, 3), np.float32)
    lib().orc_stab_dirs(I64(n), I64(i0), _p(out))
    return out


def floodfill(grid):
    """grid: bool/uint8 [B,H,W,D] or [H,W,D] -> int32 labels (reference semantics)."""
    g = np.ascontiguousarray(grid, dtype=np.uint8)
    squeeze = g.ndim == 3
    if squeeze:
        g = g[None]
    B, H, W, D = g.shape
    out = np.empty(g.shape, np.int32)
    rc = lib().orc_floodfill(_p(g), ctypes.c_int(B), ctypes.c_int(H), ctypes.c_int(W),
                             ctypes.c_int(D), _p(out))
    if rc != 0:
        raise ValueError("grid too large for int32 labels")
    return out[0] if squeeze else out


_REF_FF_PATH = os.path.join(_HERE, "_ref", "libref_floodfill.so")
_ref_ff = None


def ref_floodfill_available() -> bool:
    """True when the reference's own CUDA floodfill has been compiled into
    oracle/_ref (oracle/Makefile target `ref`; needs the reference tree)."""
    return os.path.exists(_REF_FF_PATH)


def ref_floodfill(grid):
    """The reference's own CUDA floodfill (include/gpu/floodfill.cuh
    `_floodfill_batch`) on a host grid: bool/uint8 [B,H,W,D] or [H,W,D] ->
    int32 labels.  Needs a GPU; its iteration count is the reference's
    (at most min(ceil(|(H,W,D)|) + 50, 10 max(H,W,D)) hook passes)."""
    global _ref_ff
    if _ref_ff is None:
        if not ref_floodfill_available():
            raise FileNotFoundError(_REF_FF_PATH + " not built (make -C oracle ref)")
        _ref_ff = ctypes.CDLL(_REF_FF_PATH)
        _ref_ff.ref_floodfill.restype = ctypes.c_int
    g = np.ascontiguousarray(np.asarray(grid) != 0, dtype=np.uint8)
    squeeze = g.ndim == 3
    if squeeze:
        g = g[None]
    B, H, W, D = g.shape
    out = np.empty(g.shape, np.int32)
    rc = _ref_ff.ref_floodfill(_p(g), ctypes.c_int(B), ctypes.c_int(H), ctypes.c_int(W),
                               ctypes.c_int(D), _p(out))
    if rc != 0:
        raise RuntimeError("reference floodfill failed (code %d)" % rc)
    return out[0] if squeeze else out


# ------------------------------------------------------ sparse marching cubes
_SMC_CORNER_OFF = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                            [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], np.int64)
_SMC_EDGE_CORNERS = np.array([[0, 1], [1, 2], [2, 3], [3, 0], [4, 5], [5, 6],
                              [6, 7], [7, 4], [0, 4], [1, 5], [2, 6], [3, 7]], np.int64)


def sparse_mc_vertices(coords, corners, iso, return_ids=False):
    """The reference's sparse-marching-cubes vertex array
    (include/gpu/spcumc.cuh generateVertices and the sort / unique that
    follows): for every voxel (in order) and every edge (in edge order) with
    one corner below iso, t = clamp((iso - va) / (vb - va), 0, 1) (0.5 when
    |vb - va| < 1e-30) in float32 and the point pA + t (pB - pA); vertices
    with the same edge key (lower corner, axis) merged keeping the first,
    sorted by key (x, y, z, axis).  The corner offsets are 0 or 1, so t (pB -
    pA) is exact and one float64 sum rounded to float32 equals the device's
    fused multiply-add.  Returns float32 [M, 3]; with return_ids also the
    (voxel, edge, merged vertex id) of every cut voxel edge."""
    coords = np.asarray(coords, np.int64)
    v = np.asarray(corners, np.float32)
    iso = np.float32(iso)
    inside = v < iso
    a, b = _SMC_EDGE_CORNERS[:, 0], _SMC_EDGE_CORNERS[:, 1]
    cut = inside[:, a] != inside[:, b]                      # [N, 12]
    vi, ei = np.nonzero(cut)                                # voxel-major, edges ascending
    if len(vi) == 0:
        z = np.zeros((0, 3), np.float32)
        return (z, vi, ei, vi) if return_ids else z
    ca, cb = a[ei], b[ei]
    va, vb = v[vi, ca], v[vi, cb]
    den = (vb - va).astype(np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = ((iso - va).astype(np.float32) / den).astype(np.float32)
    t = np.minimum(np.maximum(t, np.float32(0)), np.float32(1))
    t = np.where(np.abs(den) < np.float32(1e-30), np.float32(0.5), t).astype(np.float32)
    pa = coords[vi] + _SMC_CORNER_OFF[ca]
    pb = coords[vi] + _SMC_CORNER_OFF[cb]
    pos = (pa.astype(np.float64) + t.astype(np.float64)[:, None] * (pb - pa).astype(np.float64)).astype(np.float32)
    lo = np.minimum(pa, pb)
    axis = np.where(pa[:, 0] != pb[:, 0], 0, np.where(pa[:, 1] != pb[:, 1], 1, 2))
    order = np.lexsort((np.arange(len(vi)), axis, lo[:, 2], lo[:, 1], lo[:, 0]))
    keys = np.stack([lo[order, 0], lo[order, 1], lo[order, 2], axis[order]], 1)
    head = np.ones(len(order), bool)
    head[1:] = np.any(keys[1:] != keys[:-1], axis=1)
    if not return_ids:
        return pos[order[head]]
    ids = np.empty(len(order), np.int64)
    ids[order] = np.cumsum(head) - 1
    return pos[order[head]], vi, ei, ids


def sparse_mc_triangles(coords, corners, iso, table):
    """The reference's sparse-marching-cubes triangle array
    (include/gpu/spcumc.cuh classifyVoxels / generateTriangles and the remap
    to merged vertices): voxel by voxel, for its corner configuration c (bit
    k: corner k below iso) the case table's triangles table[c] = (e0, e1,
    e2, ...), -1 after the last, each written as the merged vertices of
    edges (e0, e2, e1).  table: int [256, 16] (the reference's case table,
    e.g. tests/golden/ref_mc_cases.npz `tri_edges`).  Returns int32 [T, 3]."""
    coords = np.asarray(coords)
    v = np.asarray(corners, np.float32)
    table = np.asarray(table)
    _, vi, ei, ids = sparse_mc_vertices(coords, v, iso, return_ids=True)
    vid = {}
    for a, e, i in zip(vi.tolist(), ei.tolist(), ids.tolist()):
        vid[(a, e)] = i
    cube = ((v < np.float32(iso)) * (1 << np.arange(8))).sum(1)
    out = []
    for n, c in enumerate(cube.tolist()):
        row = table[c]
        for t in range(5):
            if row[3 * t] < 0:
                break
            e0, e1, e2 = int(row[3 * t]), int(row[3 * t + 1]), int(row[3 * t + 2])
            out.append((vid[(n, e0)], vid[(n, e2)], vid[(n, e1)]))
    return np.array(out, np.int32).reshape(-1, 3)


_REF_SMC_PATH = os.path.join(_HERE, "_ref", "libref_sparse_mc.so")
_ref_smc = None


def ref_sparse_mc_available() -> bool:
    """True when the reference's own CUDA sparse marching cubes has been
    compiled into oracle/_ref (oracle/Makefile target `ref`)."""
    return os.path.exists(_REF_SMC_PATH)


def ref_sparse_mc(coords, corners, iso, ensure_consistency=False):
    """The reference's own CUDA sparse marching cubes
    (include/gpu/spcumc.cuh `_sparse_marching_cubes`) on host arrays:
    -> vertices float32 [M, 3], triangles int32 [T, 3].  Needs a GPU."""
    global _ref_smc
    if _ref_smc is None:
        if not ref_sparse_mc_available():
            raise FileNotFoundError(_REF_SMC_PATH + " not built (make -C oracle ref)")
        _ref_smc = ctypes.CDLL(_REF_SMC_PATH)
        _ref_smc.ref_sparse_mc.restype = ctypes.c_int
        _ref_smc.ref_sparse_mc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_float,
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_int)]
        _ref_smc.ref_sparse_mc_free.argtypes = [ctypes.c_void_p]
    c = np.ascontiguousarray(coords, np.int32)
    v = np.ascontiguousarray(corners, np.float32)
    pv, pt = ctypes.c_void_p(), ctypes.c_void_p()
    nv, nt = ctypes.c_int(), ctypes.c_int()
    rc = _ref_smc.ref_sparse_mc(_p(c), _p(v), len(c), float(iso), 1 if ensure_consistency else 0,
                                ctypes.byref(pv), ctypes.byref(nv), ctypes.byref(pt), ctypes.byref(nt))
    try:
        if rc != 0:
            raise RuntimeError("reference sparse marching cubes failed (code %d)" % rc)
        verts = np.ctypeslib.as_array(ctypes.cast(pv, ctypes.POINTER(ctypes.c_float)), (max(nv.value, 1) * 3,))
        tris = np.ctypeslib.as_array(ctypes.cast(pt, ctypes.POINTER(ctypes.c_int32)), (max(nt.value, 1) * 3,))
        return (verts[:3 * nv.value].reshape(-1, 3).copy(), tris[:3 * nt.value].reshape(-1, 3).copy())
    finally:
        if pv.value:
            _ref_smc.ref_sparse_mc_free(pv)
        if pt.value:
            _ref_smc.ref_sparse_mc_free(pt)


def udf_to_sdf(udf, eps):
    """The reference's occupancy -> SDF recipe (test/benchmark_watertight.py:
    98-143, readme.md:95-102) on float32 numpy grids [B,H,W,D] or [H,W,D]:
    occ = udf < eps, labels = floodfill(occ), the component of voxel (0,0,0)
    of each volume is outside, sdf = udf - eps negated on the other voxels
    where it is > 0."""
    u = np.asarray(udf, np.float32)
    squeeze = u.ndim == 3
    if squeeze:
        u = u[None]
    lab = floodfill(u < np.float32(eps))
    s = u - np.float32(eps)
    out = s.copy()
    for b in range(u.shape[0]):
        inner = (lab[b] != lab[b, 0, 0, 0]) & (s[b] > 0)
        out[b][inner] = -s[b][inner]
    return out[0] if squeeze else out


# ------------------------------------------------- FP32 mirror of the reference
class RefBVH:
    """FP32 restatement of the reference's BVH4 build + traversals (CPU)."""

    def __init__(self, V, F, n_per_leaf=8):
        V, F = _f32(V), _i64(F)
        self._h = ctypes.c_void_p(lib().orc_ref_build(_p(V), I64(len(V)), _p(F), I64(len(F)),
                                                      ctypes.c_int(n_per_leaf)))
        self.n_faces = len(F)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.orc_ref_free(h)
            self._h = None

    @property
    def n_nodes(self):
        return int(lib().orc_ref_num_nodes(self._h))

    def state_dict_arrays(self):
        nodes = np.empty((self.n_nodes, 9), np.int32)
        tris = np.empty((self.n_faces, 12), np.int32)
        lib().orc_ref_state(self._h, _p(nodes), _p(tris))
        return nodes, tris

    def unsigned_distance(self, pts, return_uvw=False, count=False):
        pts = _f32(pts); n = len(pts)
        d = np.empty(n, np.float32); fid = np.empty(n, np.int64)
        uvw = np.empty((n, 3), np.float32) if return_uvw else None
        c = np.zeros(2, np.int64) if count else None
        lib().orc_ref_udf(self._h, _p(pts), I64(n), _p(d), _p(fid), _p(uvw), _p(c))
        return (d, fid, uvw, c) if count else (d, fid, uvw)

    def ray_trace(self, ro, rd, count=False):
        ro, rd = _f32(ro), _f32(rd); n = len(ro)
        pos = np.empty((n, 3), np.float32); fid = np.empty(n, np.int64); dep = np.empty(n, np.float32)
        c = np.zeros(2, np.int64) if count else None
        lib().orc_ref_ray(self._h, _p(ro), _p(rd), I64(n), _p(pos), _p(fid), _p(dep), _p(c))
        return (pos, fid, dep, c) if count else (pos, fid, dep)

    def signed_distance(self, pts, mode=0, return_uvw=False, count=False):
        pts = _f32(pts); n = len(pts)
        d = np.empty(n, np.float32); fid = np.empty(n, np.int64)
        uvw = np.empty((n, 3), np.float32) if return_uvw else None
        c = np.zeros(2, np.int64) if count else None
        lib().orc_ref_sdf(self._h, _p(pts), I64(n), ctypes.c_int(mode), _p(d), _p(fid), _p(uvw), _p(c))
        return (d, fid, uvw, c) if count else (d, fid, uvw)


# ------------------------------------------- the reference's own BVH (oracle/_ref)
_REF_BVH_PATH = os.path.join(_HERE, "_ref", "libref_bvh.so")
_ref_bvh = None


def ref_bvh_available() -> bool:
    """True when the reference's own BVH code (src/bvh.cu, compiled unchanged
    against the Eigen stand-in) is in oracle/_ref (oracle/Makefile target
    `ref`)."""
    return os.path.exists(_REF_BVH_PATH)


def _ref_bvh_lib():
    global _ref_bvh
    if _ref_bvh is None:
        if not ref_bvh_available():
            raise FileNotFoundError(_REF_BVH_PATH + " not built (make -C oracle ref REF=<reference checkout>)")
        L = ctypes.CDLL(_REF_BVH_PATH)
        vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        L.ref_bvh_create.restype = vp
        L.ref_bvh_create.argtypes = [vp, i64, vp, i64]
        L.ref_bvh_destroy.argtypes = [vp]
        L.ref_bvh_num_nodes.restype = i64
        L.ref_bvh_num_nodes.argtypes = [vp]
        L.ref_bvh_export.argtypes = [vp, vp, vp]
        L.ref_bvh_last_error.restype = ctypes.c_char_p
        L.ref_bvh_unsigned_distance_gpu.argtypes = [vp, vp, i64, vp, vp, vp, vp]
        L.ref_bvh_signed_distance_gpu.argtypes = [vp, vp, i64, i32, vp, vp, vp, vp]
        L.ref_bvh_ray_trace_gpu.argtypes = [vp, vp, vp, i64, vp, vp, vp, vp]
        L.ref_stab_directions_gpu.argtypes = [i64, i64, vp, vp]
        L.ref_stab_directions_host.argtypes = [i64, i64, vp]
        L.ref_bvh_unsigned_distance_host.argtypes = [vp, vp, i64, i64, vp, vp, vp, i32]
        L.ref_bvh_signed_distance_host.argtypes = [vp, vp, i64, i64, i32, i64, vp, vp, vp, i32]
        L.ref_bvh_ray_trace_host.argtypes = [vp, vp, vp, i64, i64, vp, vp, vp, i32]
        for fn in ("unsigned_distance_gpu", "signed_distance_gpu", "ray_trace_gpu", "unsigned_distance_host",
                   "signed_distance_host", "ray_trace_host"):
            getattr(L, "ref_bvh_" + fn).restype = i32
        L.ref_stab_directions_gpu.restype = i32
        _ref_bvh = L
    return _ref_bvh


def ref_stab_dirs_host(n, i0=0):
    """Stab directions [n, 32, 3] of queries i0 .. i0+n-1 from the reference's
    own code built for the host (host sincosf)."""
    out = np.empty((n, 32, 3), np.float32)
    _ref_bvh_lib().ref_stab_directions_host(I64(i0), I64(n), _p(out))
    return out


def ref_stab_dirs_gpu_ptr(first, n, out_ptr, stream_ptr=0):
    """Stab directions [n, 32, 3] float32 written to device memory out_ptr, as
    the reference's raystab kernel computes them for its threads first ..
    first+n-1 (CUDA sincosf).  Asynchronous on stream_ptr."""
    L = _ref_bvh_lib()
    if L.ref_stab_directions_gpu(I64(first), I64(n), ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream_ptr)) != 0:
        raise RuntimeError("reference stab directions: " + L.ref_bvh_last_error().decode())


class ReferenceBVH:
    """The reference's own BVH4 (src/bvh.cu), built from vertices / faces as
    cuBVHImpl does (src/api_gpu.cu:21-40, leaf size 8).

    Host methods run the reference's __host__ traversals per query on the
    host cores (OpenMP) and return numpy arrays; `stride` takes every
    stride-th query.  *_gpu methods run the reference's CUDA launchers on
    device pointers (ints, e.g. torch's data_ptr()) on the given stream."""

    def __init__(self, V, F):
        V, F = _f32(V), _i64(F)
        if F.size and (F.min() < 0 or F.max() >= len(V)):
            raise ValueError("face index out of range")
        L = _ref_bvh_lib()
        h = L.ref_bvh_create(_p(V), I64(len(V)), _p(F), I64(len(F)))
        if not h:
            raise RuntimeError("reference BVH build: " + L.ref_bvh_last_error().decode())
        self._h = ctypes.c_void_p(h)
        self.n_faces = len(F)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _ref_bvh is not None:
            _ref_bvh.ref_bvh_destroy(h)
            self._h = None

    @property
    def n_nodes(self):
        return int(_ref_bvh_lib().ref_bvh_num_nodes(self._h))

    def state_dict_arrays(self):
        nodes = np.empty((self.n_nodes, 9), np.int32)
        tris = np.empty((self.n_faces, 12), np.int32)
        _ref_bvh_lib().ref_bvh_export(self._h, _p(nodes), _p(tris))
        return nodes, tris

    # ---- host traversals
    def unsigned_distance(self, pts, return_uvw=False, stride=1, threads=0):
        pts = _f32(pts)
        m = (len(pts) + stride - 1) // stride
        d = np.empty(m, np.float32); fid = np.empty(m, np.int64)
        uvw = np.empty((m, 3), np.float32) if return_uvw else None
        _ref_bvh_lib().ref_bvh_unsigned_distance_host(self._h, _p(pts), I64(len(pts)), I64(stride), _p(d), _p(fid),
                                                      _p(uvw), ctypes.c_int(threads))
        return d, fid, uvw

    def signed_distance(self, pts, mode=0, return_uvw=False, first_index=0, stride=1, threads=0):
        pts = _f32(pts)
        m = (len(pts) + stride - 1) // stride
        d = np.empty(m, np.float32); fid = np.empty(m, np.int64)
        uvw = np.empty((m, 3), np.float32) if return_uvw else None
        _ref_bvh_lib().ref_bvh_signed_distance_host(self._h, _p(pts), I64(len(pts)), I64(stride), ctypes.c_int(mode),
                                                    I64(first_index), _p(d), _p(fid), _p(uvw), ctypes.c_int(threads))
        return d, fid, uvw

    def ray_trace(self, ro, rd, stride=1, threads=0):
        ro, rd = _f32(ro), _f32(rd)
        m = (len(ro) + stride - 1) // stride
        pos = np.empty((m, 3), np.float32); fid = np.empty(m, np.int64); dep = np.empty(m, np.float32)
        _ref_bvh_lib().ref_bvh_ray_trace_host(self._h, _p(ro), _p(rd), I64(len(ro)), I64(stride), _p(pos), _p(fid),
                                              _p(dep), ctypes.c_int(threads))
        return pos, fid, dep

    # ---- the reference's CUDA launchers (device pointers)
    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError("reference %s: %s" % (what, _ref_bvh_lib().ref_bvh_last_error().decode()))

    def unsigned_distance_gpu(self, pts, n, dist, fid, uvw=0, stream=0):
        vp = ctypes.c_void_p
        self._check(_ref_bvh_lib().ref_bvh_unsigned_distance_gpu(self._h, vp(pts), I64(n), vp(dist), vp(fid),
                                                                  vp(uvw), vp(stream)), "unsigned_distance")

    def signed_distance_gpu(self, pts, n, mode, dist, fid, uvw=0, stream=0):
        vp = ctypes.c_void_p
        self._check(_ref_bvh_lib().ref_bvh_signed_distance_gpu(self._h, vp(pts), I64(n), ctypes.c_int(mode),
                                                                vp(dist), vp(fid), vp(uvw), vp(stream)),
                    "signed_distance")

    def ray_trace_gpu(self, ro, rd, n, pos, fid, depth, stream=0):
        vp = ctypes.c_void_p
        self._check(_ref_bvh_lib().ref_bvh_ray_trace_gpu(self._h, vp(ro), vp(rd), I64(n), vp(pos), vp(fid),
                                                         vp(depth), vp(stream)), "ray_trace")
